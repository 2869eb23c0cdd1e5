// Allocation-free association entry point.
//
// moea_associate_static runs the full-scan association (the same kernels as
// moea_associate in MOEA_ASSOC_SCAN mode) with its scratch in file-scope
// device arrays instead of a workspace.  It is for callers that hold no
// workspace and must not allocate on the call: a strategy invoked inside a
// generation that only receives borrowed device views (an environment
// selector or problem plugin), where cudaMalloc/cudaFree would synchronise the
// device in the middle of the generation's stream-ordered work, and processes
// that cap device memory after start-up.
//
// Scratch per device, statically sized: kStaticMaxPoints packed minima
// (8 bytes each, 512 KiB), one count word and one delta word.  The packed
// minima are reset by a kernel on every call; the count and delta are fully
// written by kernels before they are read, so nothing relies on the zero
// initialisation of the arrays.
//
// The scratch is shared by every call on a device: two calls whose work
// overlaps on the GPU (different streams, or different host threads without
// ordering) race on it and may return each other's results.  The first call on
// a device resolves the scratch addresses with cudaGetSymbolAddress (a
// runtime call that is not stream-ordered); make that first call before any
// stream capture that includes this entry point begins.
#include <atomic>
#include <mutex>

#include "internal.cuh"

namespace moea {

int run_associate_scan_scratch(const float* x, const float* refs, int M, const int* d_n, int n_cap,
                               int H, int* idx, float* dist, unsigned long long* best, float* delta,
                               int device, cudaStream_t stream);

namespace {

constexpr int kStaticMaxPoints = 65536;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_best[kStaticMaxPoints];
static __device__ __align__(256) int g_count[1];
static __device__ __align__(256) float g_delta[1];

struct StaticScratch {
    unsigned long long* best = nullptr;
    int* count = nullptr;
    float* delta = nullptr;
};

StaticScratch g_scratch[kMaxDevices];
std::atomic<bool> g_ready[kMaxDevices];
std::mutex g_setup;

__global__ void set_count_kernel(int* count, int n) { *count = n; }

// Scratch addresses on the current device, resolved once per device.
int scratch_for_current_device(StaticScratch& out, int& device)
{
    MOEA_CUDA_TRY(cudaGetDevice(&device));
    if (device < 0 || device >= kMaxDevices)
        return set_error(MOEA_ERR_UNSUPPORTED, "associate_static: device %d out of range", device);
    if (!g_ready[device].load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> lock(g_setup);
        if (!g_ready[device].load(std::memory_order_relaxed)) {
            StaticScratch s;
            cudaError_t e = cudaGetSymbolAddress((void**)&s.best, g_best);
            if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&s.count, g_count);
            if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&s.delta, g_delta);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return set_error(MOEA_ERR_CUDA, "associate_static: cudaGetSymbolAddress failed: %s",
                                 cudaGetErrorString(e));
            }
            g_scratch[device] = s;
            g_ready[device].store(true, std::memory_order_release);
        }
    }
    out = g_scratch[device];
    return MOEA_OK;
}

}  // namespace
}  // namespace moea

using namespace moea;

extern "C" moea_status moea_associate_static(const float* d_x, const float* d_refs, int M, int n, int H,
                                             int* d_idx, float* d_dist, void* stream)
{
    if (!d_x || !d_refs || !d_idx || !d_dist || n < 0 || M < 1 || M > kMaxObjectives || H < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "associate_static: bad arguments");
    if (n > kStaticMaxPoints)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "associate_static: n=%d exceeds the static scratch (%d points)",
                         n, kStaticMaxPoints);
    if (n == 0) return MOEA_OK;
    StaticScratch s;
    int device = 0;
    MOEA_TRY(scratch_for_current_device(s, device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    set_count_kernel<<<1, 1, 0, st>>>(s.count, n);
    MOEA_CUDA_TRY(cudaGetLastError());
    return run_associate_scan_scratch(d_x, d_refs, M, s.count, n, H, d_idx, d_dist, s.best, s.delta, device,
                                      st);
}
