// Inverted generational distance in FP64 on the GPU.
//
// Reference: tests/evaluation/metrics/igd.py:23-47 (igd) and :8-20
// (nondominated_mask).  The approximation keeps its rows whose objectives are
// all finite and, optionally, of those the non-dominated ones; the IGD is the
// mean over the reference points of the Euclidean distance to the nearest
// kept row.  Distances are direct FP64 differences (the reference's
// torch.cdist may expand |a-b|^2 into a matrix product for large inputs), and
// the mean is a fixed-order FP64 block sum.
//
// The non-dominated filter reuses the non-dominated sort: rows with a
// non-finite objective get a violation of 1, so they never dominate a finite
// row and never enter front 0, and front 0 of the remaining rows is exactly
// the set the reference keeps (identical rows do not dominate each other).
#include <cmath>

#include "internal.cuh"

namespace moea {

int run_ndsort(Workspace& ws, const SplitPop& pop, int M, int target, int* out_fronts, cudaStream_t stream);

namespace {

constexpr int kIgdThreads = 256;
constexpr int kIgdTile = 256;

__global__ void igd_mark(const float* __restrict__ objs, int n, int M, float* __restrict__ cv,
                         int* __restrict__ finite_count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool ok = false;
    if (i < n) {
        ok = true;
        for (int m = 0; m < M; ++m) ok &= isfinite(objs[(size_t)m * n + i]);
        cv[i] = ok ? 0.0f : 1.0f;
    }
    const unsigned b = __ballot_sync(0xFFFFFFFFu, ok);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(finite_count, __popc(b));
}

// keep[i]: the row takes part in the distances
__global__ void igd_keep(const float* __restrict__ cv, const int* __restrict__ fronts, int n, int filter,
                         int* __restrict__ keep)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keep[i] = (cv[i] == 0.0f) && (!filter || fronts[i] == 0);
}

// One thread per reference point; the kept rows pass through shared memory
// in tiles of kIgdTile rows, converted to FP64.
__global__ void __launch_bounds__(kIgdThreads)
igd_min_dist(const double* __restrict__ ref, int r, const float* __restrict__ objs, const int* __restrict__ keep,
             int n, int M, double* __restrict__ out)
{
    extern __shared__ double s_pts[];  // [M][kIgdTile], then kIgdTile keep flags
    int* s_keep = reinterpret_cast<int*>(s_pts + (size_t)M * kIgdTile);
    const int k = blockIdx.x * kIgdThreads + threadIdx.x;
    double q[16];
    for (int m = 0; m < M; ++m) q[m] = (k < r) ? ref[(size_t)k * M + m] : 0.0;
    double best = INFINITY;
    for (int t0 = 0; t0 < n; t0 += kIgdTile) {
        const int cnt = min(kIgdTile, n - t0);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += kIgdThreads) {
            s_keep[t] = keep[t0 + t];
            for (int m = 0; m < M; ++m) s_pts[(size_t)m * kIgdTile + t] = (double)objs[(size_t)m * n + t0 + t];
        }
        __syncthreads();
        for (int t = 0; t < cnt; ++t) {
            if (!s_keep[t]) continue;
            double d2 = 0.0;
            for (int m = 0; m < M; ++m) {
                const double d = q[m] - s_pts[(size_t)m * kIgdTile + t];
                d2 = fma(d, d, d2);
            }
            best = fmin(best, d2);
        }
    }
    if (k < r) out[k] = sqrt(best);
}

// mean of out[0..r) in FP64: strided partial sums, then a fixed tree
__global__ void __launch_bounds__(1024) igd_mean(const double* __restrict__ v, int r, double* __restrict__ mean)
{
    __shared__ double s[1024];
    double a = 0.0;
    for (int i = threadIdx.x; i < r; i += blockDim.x) a += v[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *mean = s[0] / (double)r;
}

}  // namespace

int run_igd(Workspace& ws, const float* objs, int n, int M, const double* ref, int r, int filter,
            double* d_min_dist, double* h_igd, cudaStream_t stream)
{
    if (n < 1 || n > ws.n_max || M < 1 || M > ws.m_max || M > 16 || r < 1 || !ref || !d_min_dist || !h_igd)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "igd: bad arguments (n=%d M=%d r=%d)", n, M, r);
    float* cv = ws.nds_objs;   // scratch: violations of the rows
    int* count = ws.sizes + 6;
    MOEA_CUDA_TRY(cudaMemsetAsync(count, 0, sizeof(int), stream));
    const int G = ceil_div(n, 256);
    igd_mark<<<G, 256, 0, stream>>>(objs, n, M, cv, count);
    MOEA_CUDA_TRY(cudaGetLastError());
    int finite = 0;
    MOEA_CUDA_TRY(cudaMemcpyAsync(&finite, count, sizeof(int), cudaMemcpyDeviceToHost, stream));
    MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
    if (finite == 0) return set_error(MOEA_ERR_INVALID_ARGUMENT, "approximation contains no finite objective rows");
    if (filter) MOEA_TRY(run_ndsort(ws, merged_view(objs, cv, n), M, 1, ws.fronts, stream));
    igd_keep<<<G, 256, 0, stream>>>(cv, ws.fronts, n, filter, ws.flags);
    const size_t smem = (size_t)M * kIgdTile * sizeof(double) + kIgdTile * sizeof(int);
    igd_min_dist<<<ceil_div(r, kIgdThreads), kIgdThreads, smem, stream>>>(ref, r, objs, ws.flags, n, M, d_min_dist);
    igd_mean<<<1, 1024, 0, stream>>>(d_min_dist, r, ws.scalar_d);
    MOEA_CUDA_TRY(cudaGetLastError());
    MOEA_CUDA_TRY(cudaMemcpyAsync(h_igd, ws.scalar_d, sizeof(double), cudaMemcpyDeviceToHost, stream));
    MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
    return MOEA_OK;
}

}  // namespace moea

using namespace moea;

extern "C" moea_status moea_igd(moea_workspace* w, const float* d_objs, int n, int M, const double* d_ref, int r,
                                int filter_nondominated, double* d_min_dist, double* h_igd, void* stream)
{
    if (!w || !d_objs) return set_error(MOEA_ERR_INVALID_ARGUMENT, "igd: NULL argument");
    return run_igd(w->ws, d_objs, n, M, d_ref, r, filter_nondominated, d_min_dist, h_igd,
                   static_cast<cudaStream_t>(stream));
}
