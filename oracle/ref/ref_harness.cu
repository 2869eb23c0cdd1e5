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
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "cuda_moea/core/cuda/cuda_globals.cuh"
#include "cuda_moea/core/cuda/cuda_manager.cuh"
#include "cuda_moea/problem/dtlz/evaluation_workspace.cuh"
#include "cuda_moea/selection/nsga3/kernels/association.cuh"
#include "cuda_moea/selection/nsga3/kernels/niching.cuh"
#include "cuda_moea/selection/nsga3/kernels/non_dominated_sort.cuh"
#include "cuda_moea/selection/nsga3/kernels/normalization.cuh"
#include "cuda_moea/selection/rvea/kernels/angle_penalized_distance.cuh"
#include "cuda_moea/selection/rvea/kernels/elitism_selection.cuh"
#include "cuda_moea/selection/rvea/kernels/objective_translation.cuh"
#include "cuda_moea/selection/rvea/kernels/reference_partition.cuh"

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

}  // namespace

extern "C" {

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
        mf = run_ndsort(const_cast<float*>(d_cv), const_cast<float*>(d_objs), d_fronts, pairs, mask,
                        dominatee, dom_cnt, asgn, new_front, cap, prop_free, 0, 100, M, N, stream,
                        default_pool());
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
    execute_normalization(d_f, d_ideal, s.get<float>((size_t)blocks * M), s.get<int>((size_t)blocks * M),
                          s.get<int>(M), s.get<float>(M * M), d_rcp, s.get<int>(1), s.get<float>(M * M),
                          s.get<float>(M), s.get<float>(M * M), s.get<int>(1), s.get<float>(M), d_ones,
                          s.get<float>(M), s.get<float>(M), M, n, default_pool(), nullptr);
    return status();
}

int ref_associate(const float* d_x, const float* d_refs, int M, int n, int H, int* d_idx, float* d_dist)
{
    Scratch s;
    const int nbr = (H + 255) / 256;
    execute_association(const_cast<float*>(d_x), const_cast<float*>(d_refs),
                        s.get<float>((size_t)nbr * n), s.get<int>((size_t)nbr * n), d_dist, d_idx, H, M,
                        n, nullptr);
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
    execute_niching(seed, off, d_gidx, d_dist, d_idx, s.get<int>(H), s.get<ull>(nl), s.get<ull>(nl),
                    s.get<int>(nl), s.get<int>(nl), s.get<int>(nl), s.get<int>(nl), s.get<int>(nl),
                    s.get<uint>(nl), d_selected, sz, H, N, default_pool(), nullptr, false);
    *h_offset = off;
    return status();
}

// Built-in problem: objectives (M,N) and violation (N).
int ref_problem(int kind, const float* d_x, int N, int D, int M, float* d_objs, float* d_cv)
{
    Scratch s;
    float* trans = s.get<float>((size_t)N * M);
    static const int base[16] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 1, 3, 2, 8, 1, 4, 15};
    compute_fv(const_cast<float*>(d_x), trans, d_objs, N, D, M, nullptr, (MOPType)base[kind]);
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

}  // extern "C"
