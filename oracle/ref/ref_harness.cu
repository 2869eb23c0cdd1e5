// TEST INFRASTRUCTURE ONLY -- C entry points over CUDA-MOEA's own stage
// functions, compiled from the reference sources where they lie (see
// oracle/ref/Makefile).  The GPU tests call these to pin the oracle and the
// product against the reference's outputs on identical inputs.  Random draws
// are passed in (the reference's cuRAND launchers are not called: their grid
// mapping depends on the GPU model).
//
// Stage functions used (python/csrc/native/src/...):
//   run_ndsort / run_ndsort_init   selection/nsga3/kernels/non_dominated_sort.cu:1337, :1407
//   execute_normalization          selection/nsga3/kernels/normalization.cu:1593
//   execute_association            selection/nsga3/kernels/association.cu:586
//   execute_niching                selection/nsga3/kernels/niching.cu:250
//   compute_fv / compute_cv        problem/dtlz/dtlz_kernels.cu:748, :1094
//   rvea::translate_fv / execute_partition / compute_apd / compute_gamma / run_elitism_selection
//   nsga3::quantize_cv             selection/nsga3/kernels/cv_quantization.cu:65-95
//   rvea::adapt_refvecs            reference/rvea_reference_adaptation.cu:279-317
//   rvea::merge_* / update_iter_vars selection/rvea/kernels/rvea_population_update.cu:209-300
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "cuda_moea/core/cuda/cuda_globals.cuh"
#include "cuda_moea/core/cuda/cuda_manager.cuh"
#include "cuda_moea/problem/dtlz/evaluation_workspace.cuh"
#include "cuda_moea/reference/rvea_reference_adaptation.cuh"
#include "cuda_moea/selection/nsga3/kernels/cv_quantization.cuh"
#include "cuda_moea/selection/nsga3/kernels/association.cuh"
#include "cuda_moea/selection/nsga3/kernels/niching.cuh"
#include "cuda_moea/selection/nsga3/kernels/non_dominated_sort.cuh"
#include "cuda_moea/selection/nsga3/kernels/normalization.cuh"
#include "cuda_moea/selection/rvea/kernels/angle_penalized_distance.cuh"
#include "cuda_moea/selection/rvea/kernels/elitism_selection.cuh"
#include "cuda_moea/selection/rvea/kernels/objective_translation.cuh"
#include "cuda_moea/selection/rvea/kernels/reference_partition.cuh"
#include "cuda_moea/selection/rvea/kernels/rvea_population_update.cuh"
#include "cuda_moea/problem/dtlz/population_adapter.cuh"

void compute_fv(float* d_pop, float* d_fit_trans, float* d_fit, int N, int D, int M,
                cudaStream_t fit_stream, MOPType dtlz_type);
void compute_cv(const float* d_fit, float* d_cv, int N, int M, cudaStream_t stream,
                MOPType c_dtlz_type);
void compute_csdp_cv(const float* d_pop, float* d_cv, int N, cudaStream_t stream);

namespace {

struct Scratch {
    std::vector<void*> ptrs;
    template <class T>
    T* get(size_t n)
    {
        void* p = nullptr;
        cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1));
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    ~Scratch()
    {
        cudaDeviceSynchronize();
        for (void* p : ptrs) cudaFree(p);
    }
};

cudaMemPool_t default_pool()
{
    cudaMemPool_t pool;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetDefaultMemPool(&pool, dev);
    return pool;
}

int status() { return cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 1; }

// Timing mode (bench.py's reference arm): with a positive repeat count, a
// stage call is made once for its outputs and then `repeat` more times between
// two events on the legacy stream, with its scratch already allocated; the
// mean is kept for ref_last_ms().  Host waits inside the reference's stage
// (its front loop reads sizes back) count, as they do in its generation.
int g_repeat = 0;
float g_ms = 0.0f;

template <class F>
void run_timed(F&& f)
{
    f();
    g_ms = 0.0f;
    if (g_repeat <= 0) return;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a, nullptr);
    for (int i = 0; i < g_repeat; ++i) f();
    cudaEventRecord(b, nullptr);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&g_ms, a, b);
    g_ms /= (float)g_repeat;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
}

}  // namespace

extern "C" {

void ref_set_repeat(int repeat) { g_repeat = repeat; }
float ref_last_ms(void) { return g_ms; }

// Non-dominated sort of n_mix = 2N merged points (run_ndsort) or, when
// n_mix == N, of a parent population (run_ndsort_init).  The pair buffer is
// sized for every pair (sparse ratio 1.0) so the reference never overflows.
int ref_ndsort(const float* d_cv, const float* d_objs, int M, int n_mix, int N, int* d_fronts,
               int* h_max_front)
{
    Scratch s;
    cudaStream_t stream = nullptr;
    const long long cap = compute_max_dompairs(n_mix, 1.0f);
    int* pairs = s.get<int>(2 * (size_t)cap);
    int* dominatee = s.get<int>(n_mix);
    long long* dom_cnt = s.get<long long>(1);
    int* asgn = s.get<int>(1);
    int* new_front = s.get<int>(1);
    int mf;
    if (n_mix == N) {
        cudaStreamSync streams{};
        streams.exec_stream = stream;
        mf = run_ndsort_init(streams, const_cast<float*>(d_cv), const_cast<float*>(d_objs), d_fronts,
                             pairs, dominatee, dom_cnt, asgn, new_front, cap, M, N, default_pool());
    } else {
        const int tiles = (n_mix + 31) / 32;
        uint32_t* mask = s.get<uint32_t>((size_t)n_mix * tiles);
        bool prop_free = false;
        run_timed([&] {
            mf = run_ndsort(const_cast<float*>(d_cv), const_cast<float*>(d_objs), d_fronts, pairs, mask,
                            dominatee, dom_cnt, asgn, new_front, cap, prop_free, 0, 100, M, N, stream,
                            default_pool());
        });
    }
    *h_max_front = mf;
    return status();
}

// In-place normalisation of (M, n) objectives; writes the reciprocal intercepts.
int ref_normalize(float* d_f, const float* d_ideal, int M, int n, float* d_rcp)
{
    Scratch s;
    const int blocks = (n + 1023) / 1024 + 1;
    std::vector<float> ones(M, 1.0f);
    float* d_ones = s.get<float>(M);
    cudaMemcpy(d_ones, ones.data(), sizeof(float) * M, cudaMemcpyHostToDevice);
    float* b0 = s.get<float>((size_t)blocks * M);
    int* b1 = s.get<int>((size_t)blocks * M);
    int* b2 = s.get<int>(M);
    float* b3 = s.get<float>(M * M);
    int* b4 = s.get<int>(1);
    float* b5 = s.get<float>(M * M);
    float* b6 = s.get<float>(M);
    float* b7 = s.get<float>(M * M);
    int* b8 = s.get<int>(1);
    float* b9 = s.get<float>(M);
    float* b10 = s.get<float>(M);
    float* b11 = s.get<float>(M);
    // in timing mode the repeats normalise the already normalised values again
    run_timed([&] {
        execute_normalization(d_f, d_ideal, b0, b1, b2, b3, d_rcp, b4, b5, b6, b7, b8, b9, d_ones, b10, b11, M,
                              n, default_pool(), nullptr);
    });
    return status();
}

int ref_associate(const float* d_x, const float* d_refs, int M, int n, int H, int* d_idx, float* d_dist)
{
    Scratch s;
    const int nbr = (H + 255) / 256;
    float* bmax = s.get<float>((size_t)nbr * n);
    int* barg = s.get<int>((size_t)nbr * n);
    run_timed([&] {
        execute_association(const_cast<float*>(d_x), const_cast<float*>(d_refs), bmax, barg, d_dist, d_idx, H,
                            M, n, nullptr);
    });
    return status();
}

int ref_niching(uint64_t seed, uint64_t* h_offset, const int* d_gidx, const float* d_dist,
                const int* d_idx, const int* h_sizes, int H, int N, int* d_selected)
{
    Scratch s;
    NumNDSData sz;
    sz.N_prior = h_sizes[0];
    sz.N_last = h_sizes[1];
    sz.N_rem = h_sizes[2];
    sz.N_nds = h_sizes[3];
    const size_t nl = sz.N_last > 0 ? sz.N_last : 1;
    ull off = *h_offset;
    int* c0 = s.get<int>(H);
    ull* k0 = s.get<ull>(nl);
    ull* k1 = s.get<ull>(nl);
    int* i0 = s.get<int>(nl);
    int* i1 = s.get<int>(nl);
    int* i2 = s.get<int>(nl);
    int* i3 = s.get<int>(nl);
    int* i4 = s.get<int>(nl);
    uint* u0 = s.get<uint>(nl);
    ull first_off = 0;
    bool first = true;
    run_timed([&] {
        execute_niching(seed, off, d_gidx, d_dist, d_idx, c0, k0, k1, i0, i1, i2, i3, i4, u0, d_selected, sz, H,
                        N, default_pool(), nullptr, false);
        if (first) first_off = off;
        first = false;
    });
    *h_offset = first_off;
    return status();
}

// Built-in problem: objectives (M,N) and violation (N).
int ref_problem(int kind, const float* d_x, int N, int D, int M, float* d_objs, float* d_cv)
{
    Scratch s;
    float* trans = s.get<float>((size_t)N * M);
    static const int base[16] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 1, 3, 2, 8, 1, 4, 15};
    run_timed([&] { compute_fv(const_cast<float*>(d_x), trans, d_objs, N, D, M, nullptr, (MOPType)base[kind]); });
    cudaMemset(d_cv, 0, sizeof(float) * N);
    if (kind == 15) compute_csdp_cv(d_x, d_cv, N, nullptr);
    else if (kind >= 9) compute_cv(d_objs, d_cv, N, M, nullptr, (MOPType)kind);
    return status();
}

int ref_rvea_translate(const float* d_objs, int M, int n, float* d_out, float* d_zmin)
{
    rvea::translate_fv(d_objs, d_out, d_zmin, M, n, nullptr);
    return status();
}

int ref_rvea_partition(const float* d_t, const float* d_refs, int M, int n, int K, int n_active,
                       int n_parent, float* d_theta, int* d_idx)
{
    Scratch s;
    const int nbr = (K + 255) / 256;
    rvea::execute_partition(d_t, d_refs, s.get<float>((size_t)nbr * n), s.get<int>((size_t)nbr * n),
                            d_theta, d_idx, K, M, n, n_active, n_parent, nullptr);
    return status();
}

int ref_rvea_gamma(const float* d_refs, int M, int K, float* d_gamma)
{
    Scratch s;
    const int nbr = (K + 255) / 256;
    rvea::compute_gamma(d_refs, s.get<float>((size_t)nbr * K), d_gamma, M, K, nullptr);
    return status();
}

int ref_rvea_apd(const float* d_t, const float* d_theta, const float* d_gamma, const int* d_idx, int M,
                 int n, int K, int gen, int max_gen, float alpha, float* d_apd)
{
    Scratch s;
    rvea::compute_apd(d_t, d_theta, d_gamma, d_idx, d_apd, s.get<float>(n), n, M, K, gen, max_gen, alpha,
                      nullptr);
    return status();
}

// Elitism; writes the selected indices (unordered) and the active count.
int ref_rvea_elitism(const int* d_idx, const float* d_cv, const float* d_apd, int N, int n_mix, int K,
                     int* d_selected, int* h_active)
{
    Scratch s;
    int active = N;
    cudaMemPool_t pool = default_pool();
    rvea::run_elitism_selection(d_idx, d_cv, d_apd, s.get<ull>(n_mix), s.get<ull>(n_mix),
                                s.get<int>(n_mix), s.get<int>(n_mix), s.get<int>(n_mix), s.get<int>(n_mix),
                                s.get<int>(n_mix), s.get<int>(n_mix), s.get<int>(1), d_selected, N, n_mix,
                                K, active, pool, nullptr);
    *h_active = active;
    return status();
}

// RVEA survivor update as RVEAEnvironmentSelector::select does it
// (rvea_environment_selector.cu:187-290): merge parents and offspring, then
// gather the `active` selected rows (d_sel, sorted in place) and write the
// dead-slot sentinels into rows [active, N).
int ref_rvea_update(const float* d_par_x, const float* d_off_x, const float* d_par_f, const float* d_off_f,
                    const float* d_par_cv, const float* d_off_cv, int* d_sel, int active, int N, int D, int M,
                    float* d_next_x, float* d_next_f, float* d_next_cv)
{
    Scratch s;
    PopData par(N, D), off(N, D), mix(2 * N, D), next(N, D);
    par.d_pop = const_cast<float*>(d_par_x);
    off.d_pop = const_cast<float*>(d_off_x);
    mix.d_pop = s.get<float>((size_t)2 * N * D);
    next.d_pop = d_next_x;
    float* mix_f = s.get<float>((size_t)2 * N * M);
    float* mix_cv = s.get<float>((size_t)2 * N);
    rvea::merge_pop(par, off, mix, D, N, nullptr);
    rvea::merge_cv(d_par_cv, d_off_cv, mix_cv, N, nullptr);
    rvea::merge_fv(d_par_f, d_off_f, mix_f, M, N, nullptr);
    rvea::update_iter_vars(mix, mix_cv, mix_f, d_sel, next, d_next_cv, d_next_f, D, M, active, N, nullptr);
    const int rc = status();
    par.d_pop = off.d_pop = mix.d_pop = next.d_pop = nullptr;
    return rc;
}

// Optional CV quantisation of n violations (validated parameters only).
int ref_quantize_cv(const float* d_cv, float* d_out, int n, float eps_feas, float clip_upper,
                    float log_alpha, int bins)
{
    if (!nsga3::validate_cv_quant_params(bins, clip_upper, log_alpha, eps_feas)) return 2;
    nsga3::quantize_cv(d_cv, d_out, n, eps_feas, clip_upper, log_alpha, bins, nullptr);
    return status();
}

// Direction adaptation V = normalise(V0 * (zmax - zmin)) over the first
// n_active columns of d_objs (M, n_stride), called the way
// AdaptiveRVEADirections::update calls it (reference_directions.cu:132-162:
// fr = 1 and a zero trigger, so every call adapts).
int ref_rvea_adapt(const float* d_v0, const float* d_objs, int M, int K, int n_active, int n_stride,
                   float* d_v)
{
    Scratch s;
    float trigger = 0.0f;
    rvea::adapt_refvecs(d_v0, d_objs, d_v, s.get<float>(M), s.get<float>(M), 0, 1, 1.0f, trigger, M, K,
                        n_active, n_stride, nullptr);
    return status();
}

}  // extern "C"
