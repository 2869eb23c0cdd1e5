// RVEA environmental selection and direction adaptation for sm_100a.
//
// Reference (paths relative to python/csrc/native/src/):
//   translation   selection/rvea/kernels/objective_translation.cu:15-167
//   partition     selection/rvea/kernels/reference_partition.cu:48-439
//   APD, gamma    selection/rvea/kernels/angle_penalized_distance.cu:45-417
//   elitism       selection/rvea/kernels/elitism_selection.cu:68-419
//   update        selection/rvea/kernels/rvea_population_update.cu:185-293
//   adaptation    reference/rvea_reference_adaptation.cu:20-317
//   front 0       selection/rvea/kernels/front_zero.cu:200-293
// The reference reads the winner count back to the host every generation
// (elitism_selection.cu:256-257); here the count stays on the device and the
// truncation, the active count and the sentinel rows are decided there.
#include <algorithm>

#include <cub/cub.cuh>

#include <math_constants.h>

#include "internal.cuh"

namespace moea {

int run_problem(int kind, const float* x, int N, int D, int M, float* objs, float* cv,
                cudaStream_t s);

namespace {

constexpr float kMetricMax = 1e30f;
constexpr float kSentinel = 1e15f;

__global__ void __launch_bounds__(512) zmin_kernel(SplitPop pop, float* __restrict__ zmin)
{
    const int m = blockIdx.x;
    float v = CUDART_INF_F;
    for (int i = threadIdx.x; i < pop.n; i += blockDim.x) v = fminf(v, pop.obj(m, i));
    __shared__ float sh[16];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_down_sync(0xFFFFFFFFu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = CUDART_INF_F;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fminf(r, sh[w]);
        zmin[m] = r;
    }
}

__global__ void translate_kernel(SplitPop pop, int M, const float* __restrict__ zmin,
                                 float* __restrict__ t, int t_stride)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pop.n) return;
    for (int m = 0; m < M; ++m) t[(size_t)m * t_stride + i] = fmaxf(pop.obj(m, i) - zmin[m], 1e-32f);
}

// A warp per point: lane l takes the directions l, l+32, ... with the same
// FMA order over m as a sequential scan, keeps the first maximum it meets,
// and the warp reduces to the largest cosine with the smallest direction
// index on ties, which is the sequential scan's `if (c > best)` result.
template <int M>
__global__ void __launch_bounds__(256)
partition_kernel(const float* __restrict__ t, int t_stride, int n, const float* __restrict__ refs,
                 int K, const int* __restrict__ d_active, int n_active_host, int n_parent,
                 float* __restrict__ theta, int* __restrict__ idx)
{
    const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;  // uniform over the warp
    float x[M];
    float sqr = 0.f;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const float v = t[(size_t)m * t_stride + i];
        x[m] = v;
        sqr = fmaf(v, v, sqr);
    }
    const float inv_norm = rsqrtf(sqr + 1e-12f);
    float best = -CUDART_INF_F;
    int bj = -1;
    for (int j = lane; j < K; j += 32) {
        float dot = 0.f;
#pragma unroll
        for (int m = 0; m < M; ++m) dot = fmaf(x[m], __ldg(refs + (size_t)m * K + j), dot);
        const float c = dot * inv_norm;
        if (c > best) { best = c; bj = j; }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float ob = __shfl_xor_sync(0xFFFFFFFFu, best, o);
        const int oj = __shfl_xor_sync(0xFFFFFFFFu, bj, o);
        if (ob > best || (ob == best && oj >= 0 && (bj < 0 || oj < bj))) {
            best = ob;
            bj = oj;
        }
    }
    if (lane != 0) return;
    theta[i] = (best > -CUDART_INF_F) ? acosf(fminf(fmaxf(best, 0.f), 1.f)) : CUDART_INF_F;
    const int n_active = d_active ? *d_active : n_active_host;
    idx[i] = (i >= n_active && i < n_parent) ? K : bj;
}

// gamma_j: the angle to the nearest other direction.  The directions are
// staged in shared memory tiles (every thread reads every direction).
template <int M>
__global__ void gamma_kernel(const float* __restrict__ refs, int K, float* __restrict__ gamma)
{
    constexpr int kTile = 512;
    __shared__ float s_t[M][kTile];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    float q[M];
#pragma unroll
    for (int m = 0; m < M; ++m) q[m] = j < K ? refs[(size_t)m * K + j] : 0.f;
    float mx = -CUDART_INF_F;
    for (int k0 = 0; k0 < K; k0 += kTile) {
        const int cnt = min(kTile, K - k0);
        __syncthreads();
        for (int u = threadIdx.x; u < cnt; u += blockDim.x)
#pragma unroll
            for (int m = 0; m < M; ++m) s_t[m][u] = refs[(size_t)m * K + k0 + u];
        __syncthreads();
        for (int u = 0; u < cnt; ++u) {
            if (k0 + u == j) continue;
            float dot = 0.f;
#pragma unroll
            for (int m = 0; m < M; ++m) dot = fmaf(q[m], s_t[m][u], dot);
            mx = fmaxf(mx, dot);
        }
    }
    if (j >= K) return;
    if (K == 1) { gamma[j] = CUDART_PI_F; return; }
    gamma[j] = (mx > -CUDART_INF_F) ? acosf(fminf(fmaxf(mx, 0.f), 1.f)) : CUDART_PI_F;
}

template <int M>
__global__ void apd_kernel(const float* __restrict__ t, int t_stride, int n,
                           const float* __restrict__ theta, const float* __restrict__ gamma,
                           const int* __restrict__ idx, int K, const float* __restrict__ ps_table,
                           const int* __restrict__ d_gen, float ps_host, float* __restrict__ apd)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float penalty_scale = ps_table ? ps_table[*d_gen] : ps_host;
    float norm_sq = 0.f;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const float v = t[(size_t)m * t_stride + i];
        norm_sq = fmaf(v, v, norm_sq);
    }
    const float norm = sqrtf(norm_sq);
    if (norm > 1e-12f) {
        const int r = idx[i];
        if (r < 0 || r >= K) { apd[i] = kMetricMax; return; }
        const float theta_safe = fminf(fmaxf(theta[i], 0.f), CUDART_PI_F);
        const float gamma_safe = fmaxf(gamma[r], 1e-6f);
        const float a = (1.f + penalty_scale * theta_safe / gamma_safe) * norm;
        apd[i] = (!isfinite(a) || a < 0.f) ? kMetricMax : a;
    } else {
        apd[i] = 0.f;
    }
}

__device__ __forceinline__ uint32_t metric_bits(float cv, float apd, uint32_t& flag)
{
    const bool feas = cv <= 1e-8f;
    float m = feas ? apd : cv;
    if (!(isfinite(m) && m >= 0.f)) m = kMetricMax;
    flag = feas ? 0u : 1u;
    return __float_as_uint(m) & 0x7FFFFFFFu;
}

__global__ void elite_keys(const int* __restrict__ idx, SplitPop pop, const float* __restrict__ apd,
                           uint64_t* __restrict__ key, int* __restrict__ val)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pop.n) return;
    uint32_t flag;
    const uint32_t mb = metric_bits(pop.cvv(i), apd[i], flag);
    key[i] = ((uint64_t)(uint32_t)idx[i] << 32) | ((uint64_t)flag << 31) | mb;
    val[i] = i;
}

__global__ void elite_heads(const uint64_t* __restrict__ key, int n, int* __restrict__ head)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    head[t] = (t == 0 || (uint32_t)(key[t] >> 32) != (uint32_t)(key[t - 1] >> 32)) ? t : 0;
}

__global__ void elite_winners(const uint64_t* __restrict__ key, const int* __restrict__ val,
                              const int* __restrict__ run_start, int n, int K,
                              int* __restrict__ win_flag, int* __restrict__ win_count)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    bool w = false;
    if (t < n) {
        const int ref = (int)(uint32_t)(key[t] >> 32);
        w = (t == run_start[t]) && ref >= 0 && ref < K;
        win_flag[val[t]] = w ? 1 : 0;
    }
    const unsigned m = __ballot_sync(0xFFFFFFFFu, w);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(win_count, __popc(m));
}

__global__ void elite_trunc_keys(const int* __restrict__ win_flag, SplitPop pop,
                                 const float* __restrict__ apd, uint64_t* __restrict__ key,
                                 int* __restrict__ val)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pop.n) return;
    if (win_flag[i]) {
        uint32_t flag;
        const uint32_t mb = metric_bits(pop.cvv(i), apd[i], flag);
        key[i] = ((uint64_t)flag << 63) | ((uint64_t)mb << 32) | (uint32_t)i;
    } else {
        key[i] = ~0ull;
    }
    val[i] = i;
}

// selected = first N of the first sort when there is no winner, else the
// first min(W, N) winners in truncation order; active = that count.
__global__ void elite_select(const int* __restrict__ first_vals, const int* __restrict__ trunc_vals,
                             const int* __restrict__ win_count, int N, int* __restrict__ selected,
                             int* __restrict__ active, int* __restrict__ flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int W = *win_count;
    const int a = (W > 0) ? min(W, N) : N;
    if (i == 0) *active = a;
    if (i < a) {
        const int s = (W > 0) ? trunc_vals[i] : first_vals[i];
        selected[i] = s;
        flags[s] = 1;
    }
}

// Next population: active rows gathered, the rest sentinel rows.
// Next parents: survivor rows of the variables (one row per block iteration,
// float4 when D is a multiple of 4), then objectives and violations; rows at
// or beyond `active` get the sentinels.
// Next parents: survivor rows of the variables, rows at or beyond `active`
// the NaN sentinels, then objectives and violations (sentinels past
// `active`).  The rows are cut into work items of kUpdateChunk variables, so
// a large D spreads over every SM whatever the active count.  Dead rows at or
// beyond *nan_rows already hold the sentinels and are skipped (all dead rows
// are written when nan_rows is null).
constexpr int kUpdateChunk = 8192;

__global__ void rvea_update(SplitPop pop, const float* __restrict__ vars_a,
                            const float* __restrict__ vars_b, const int* __restrict__ survivors,
                            const int* __restrict__ d_active, const int* __restrict__ nan_rows, int N, int D,
                            int M, float* __restrict__ vars, float* __restrict__ objs, float* __restrict__ cv)
{
    const int active = *d_active;
    const int fill_end = nan_rows ? min(N, *nan_rows) : N;
    const int per_row = (D + kUpdateChunk - 1) / kUpdateChunk;
    const long long items = (long long)N * per_row;
    const bool vec = (D & 3) == 0;
    for (long long w = blockIdx.x; w < items; w += gridDim.x) {
        const int r = (int)(w / per_row);
        const int d0 = (int)(w - (long long)r * per_row) * kUpdateChunk;
        const int d1 = min(D, d0 + kUpdateChunk);
        float* dst = vars + (size_t)r * D;
        if (r < active) {
            const int s = survivors[r];
            const float* src = (s < pop.n_a) ? vars_a + (size_t)s * D : vars_b + (size_t)(s - pop.n_a) * D;
            if (vec) {
                copy_units4(reinterpret_cast<float4*>(dst + d0), reinterpret_cast<const float4*>(src + d0),
                            (d1 - d0) >> 2, threadIdx.x, blockDim.x);
            } else {
                for (int d = d0 + threadIdx.x; d < d1; d += blockDim.x) dst[d] = __ldg(src + d);
            }
        } else if (r < fill_end) {
            if (vec) {
                const float4 nan4 = make_float4(CUDART_NAN_F, CUDART_NAN_F, CUDART_NAN_F, CUDART_NAN_F);
                for (int u = (d0 >> 2) + threadIdx.x; u < (d1 >> 2); u += blockDim.x)
                    reinterpret_cast<float4*>(dst)[u] = nan4;
            } else {
                for (int d = d0 + threadIdx.x; d < d1; d += blockDim.x) dst[d] = CUDART_NAN_F;
            }
        }
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N; e += gridDim.x * blockDim.x) {
        const int r = (int)e;
        if (r < active) {
            const int s = survivors[r];
            for (int m = 0; m < M; ++m) objs[(size_t)m * N + r] = pop.obj(m, s);
            cv[r] = pop.cvv(s);
        } else {
            for (int m = 0; m < M; ++m) objs[(size_t)m * N + r] = kSentinel;
            cv[r] = kSentinel;
        }
    }
}

// After an update: every row from the active count on holds the sentinels.
__global__ void rvea_mark_nan_rows(int* __restrict__ nan_rows, const int* __restrict__ d_active)
{
    *nan_rows = *d_active;
}

__global__ void fill_int_kernel(int* __restrict__ p, int count, int value)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) p[i] = value;
}

__global__ void zrange_kernel(const float* __restrict__ objs, int stride, const int* __restrict__ d_n,
                              int n_host, float* __restrict__ range)
{
    const int m = blockIdx.x;
    const int n = d_n ? *d_n : n_host;
    float lo = CUDART_INF_F, hi = -CUDART_INF_F;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float v = objs[(size_t)m * stride + i];
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
    }
    __shared__ float sl[32], sh[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_down_sync(0xFFFFFFFFu, lo, o));
        hi = fmaxf(hi, __shfl_down_sync(0xFFFFFFFFu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) { sl[threadIdx.x >> 5] = lo; sh[threadIdx.x >> 5] = hi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { lo = fminf(lo, sl[w]); hi = fmaxf(hi, sh[w]); }
        float r = hi - lo;
        if (!isfinite(r) || r < 1e-12f) r = 1e-12f;
        range[m] = r;
    }
}

template <int M>
__global__ void adapt_kernel(const float* __restrict__ v0, const float* __restrict__ range, int K,
                             float* __restrict__ v)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= K) return;
    float base[M], sc[M], bs = 0.f, ss = 0.f;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        float b = v0[(size_t)m * K + j];
        if (!isfinite(b)) b = 0.f;
        base[m] = b;
        bs = fmaf(b, b, bs);
        float s = b * range[m];
        if (!isfinite(s)) s = 0.f;
        sc[m] = s;
        ss = fmaf(s, s, ss);
    }
    const bool us = isfinite(ss) && (ss > 1e-12f);
    const bool ub = isfinite(bs) && (bs > 1e-12f);
    const float is = us ? rsqrtf(ss) : 0.f;
    const float ib = ub ? rsqrtf(bs) : 0.f;
#pragma unroll
    for (int m = 0; m < M; ++m)
        v[(size_t)m * K + j] = us ? sc[m] * is : (ub ? base[m] * ib : (m == 0 ? 1.f : 0.f));
}

// ---- the selection of a small merged population in three launches --------
//
// For 2N <= kRveaBlockPoints merged points and K <= kRveaBlockDirs directions
// the staged translate (two launches), partition, APD and elitism (about ten
// launches with two library sorts and a scan) become three launches:
//   rvea_translate_block  one CTA: zmin and the translated objectives;
//   partition_apd_kernel  a warp per point: the partition of partition_kernel
//                         and, on lane 0, the APD of apd_kernel;
//   rvea_elite_block      one CTA: each direction's winner, the survivors in
//                         ascending order and the active count.
// Every value comes from the same expressions in the same order as the staged
// kernels, and the elitism keeps the same survivors:
//   - the winner of direction j is the point with the smallest
//     (flag, metric, index) among those partitioned to j: the head of j's run
//     in the staged stable sort by (j, flag, metric), found here with a
//     shared-memory atomicMin on the packed key;
//   - with W winners, 0 < W <= N keeps them all; W > N keeps the N smallest
//     winners by (flag, metric, index), and W = 0 keeps the N smallest points
//     by (direction, flag, metric, index), both by counting ranks (rare cases,
//     where the staged path sorts);
//   - the active count is min(W, N), or N when W = 0.
constexpr int kRveaBlockThreads = 1024;
constexpr int kRveaBlockPoints = 4096;
constexpr int kRveaBlockDirs = 4096;

template <int M>
__global__ void __launch_bounds__(kRveaBlockThreads, 1)
rvea_translate_block(SplitPop pop, float* __restrict__ t, int t_stride, float* __restrict__ zmin)
{
    __shared__ float s_zw[M][32];
    __shared__ float s_z[M];
    const int n = pop.n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nthreads = blockDim.x, nwarps = nthreads >> 5;
    // zmin: fminf is order independent on the GPU, so this equals zmin_kernel
    float z[M];
#pragma unroll
    for (int m = 0; m < M; ++m) z[m] = CUDART_INF_F;
    for (int i = tid; i < n; i += nthreads)
#pragma unroll
        for (int m = 0; m < M; ++m) z[m] = fminf(z[m], pop.obj(m, i));
#pragma unroll
    for (int m = 0; m < M; ++m) {
        float v = z[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_down_sync(0xFFFFFFFFu, v, o));
        if (lane == 0) s_zw[m][warp] = v;
    }
    __syncthreads();
    if (tid < M) {
        float r = CUDART_INF_F;
        for (int w = 0; w < nwarps; ++w) r = fminf(r, s_zw[tid][w]);
        s_z[tid] = r;
        zmin[tid] = r;
    }
    __syncthreads();
    for (int i = tid; i < n; i += nthreads)
#pragma unroll
        for (int m = 0; m < M; ++m) t[(size_t)m * t_stride + i] = fmaxf(pop.obj(m, i) - s_z[m], 1e-32f);
}

// partition_kernel with apd_kernel on the warp's lane 0.
template <int M>
__global__ void __launch_bounds__(256)
partition_apd_kernel(const float* __restrict__ t, int t_stride, int n, const float* __restrict__ refs, int K,
                     const int* __restrict__ d_active, int n_parent, const float* __restrict__ gamma,
                     const float* __restrict__ ps_table, const int* __restrict__ d_gen, float ps_host,
                     float* __restrict__ theta, int* __restrict__ idx, float* __restrict__ apd)
{
    const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;  // uniform over the warp
    float x[M];
    float sqr = 0.f;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        const float v = t[(size_t)m * t_stride + i];
        x[m] = v;
        sqr = fmaf(v, v, sqr);
    }
    const float inv_norm = rsqrtf(sqr + 1e-12f);
    float best = -CUDART_INF_F;
    int bj = -1;
    for (int j = lane; j < K; j += 32) {
        float dot = 0.f;
#pragma unroll
        for (int m = 0; m < M; ++m) dot = fmaf(x[m], __ldg(refs + (size_t)m * K + j), dot);
        const float c = dot * inv_norm;
        if (c > best) { best = c; bj = j; }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float ob = __shfl_xor_sync(0xFFFFFFFFu, best, o);
        const int oj = __shfl_xor_sync(0xFFFFFFFFu, bj, o);
        if (ob > best || (ob == best && oj >= 0 && (bj < 0 || oj < bj))) {
            best = ob;
            bj = oj;
        }
    }
    if (lane != 0) return;
    const float th = (best > -CUDART_INF_F) ? acosf(fminf(fmaxf(best, 0.f), 1.f)) : CUDART_INF_F;
    theta[i] = th;
    const int r = (i >= *d_active && i < n_parent) ? K : bj;
    idx[i] = r;
    // apd_kernel: its norm is the same FMA sum over the translated values
    const float penalty_scale = ps_table ? ps_table[*d_gen] : ps_host;
    const float norm = sqrtf(sqr);
    float a;
    if (norm > 1e-12f) {
        if (r < 0 || r >= K) {
            a = kMetricMax;
        } else {
            const float theta_safe = fminf(fmaxf(th, 0.f), CUDART_PI_F);
            const float gamma_safe = fmaxf(gamma[r], 1e-6f);
            const float v = (1.f + penalty_scale * theta_safe / gamma_safe) * norm;
            a = (!isfinite(v) || v < 0.f) ? kMetricMax : v;
        }
    } else {
        a = 0.f;
    }
    apd[i] = a;
}

__global__ void __launch_bounds__(kRveaBlockThreads, 1)
rvea_elite_block(SplitPop pop, const int* __restrict__ idx, const float* __restrict__ apd, int K, int N,
                 int* __restrict__ d_active, int* __restrict__ survivors)
{
    extern __shared__ unsigned long long s_key[];  // max(K, n): winners, then the W = 0 keys
    __shared__ unsigned char s_flag[kRveaBlockPoints];
    __shared__ int s_red[32];
    __shared__ int s_w;
    const int n = pop.n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nthreads = blockDim.x, nwarps = nthreads >> 5;
    for (int j = tid; j < K; j += nthreads) s_key[j] = ~0ull;
    for (int i = tid; i < n; i += nthreads) s_flag[i] = 0;
    __syncthreads();
    for (int i = tid; i < n; i += nthreads) {
        const int r = idx[i];
        if (r >= 0 && r < K) {
            uint32_t flag;
            const uint32_t mb = metric_bits(pop.cvv(i), apd[i], flag);
            atomicMin(&s_key[r], ((unsigned long long)flag << 63) | ((unsigned long long)mb << 32) | (uint32_t)i);
        }
    }
    __syncthreads();
    int wl = 0;
    for (int j = tid; j < K; j += nthreads) wl += s_key[j] != ~0ull ? 1 : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wl += __shfl_down_sync(0xFFFFFFFFu, wl, o);
    if (lane == 0) s_red[warp] = wl;
    __syncthreads();
    if (tid == 0) {
        int w = 0;
        for (int k = 0; k < nwarps; ++k) w += s_red[k];
        s_w = w;
    }
    __syncthreads();
    const int W = s_w;
    const int active = W > 0 ? min(W, N) : N;
    if (W > 0 && W <= N) {
        for (int j = tid; j < K; j += nthreads)
            if (s_key[j] != ~0ull) s_flag[(uint32_t)s_key[j]] = 1;
    } else if (W > N) {
        // the N smallest winners (keys are distinct: they hold the index)
        for (int j = tid; j < K; j += nthreads) {
            const unsigned long long kj = s_key[j];
            if (kj == ~0ull) continue;
            int rank = 0;
            for (int j2 = 0; j2 < K; ++j2) rank += s_key[j2] < kj ? 1 : 0;
            if (rank < N) s_flag[(uint32_t)kj] = 1;
        }
    } else {
        // no winner: the N smallest points by (direction, flag, metric), then index
        for (int i = tid; i < n; i += nthreads) {
            uint32_t flag;
            const uint32_t mb = metric_bits(pop.cvv(i), apd[i], flag);
            s_key[i] = ((unsigned long long)(uint32_t)idx[i] << 32) | ((unsigned long long)flag << 31) | mb;
        }
        __syncthreads();
        for (int i = tid; i < n; i += nthreads) {
            const unsigned long long ki = s_key[i];
            int rank = 0;
            for (int i2 = 0; i2 < n; ++i2) {
                const unsigned long long k2 = s_key[i2];
                rank += (k2 < ki || (k2 == ki && i2 < i)) ? 1 : 0;
            }
            if (rank < N) s_flag[i] = 1;
        }
    }
    __syncthreads();
    // the ascending survivor list: each thread counts a run of consecutive
    // flags, a block scan gives the run's offset
    const int per = (n + nthreads - 1) / nthreads;
    const int b0 = tid * per, b1 = min(n, b0 + per);
    int c = 0;
    for (int i = b0; i < b1; ++i) c += s_flag[i];
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_red[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int v = lane < nwarps ? s_red[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xFFFFFFFFu, v, o);
            if (lane >= o) v += u;
        }
        s_red[lane] = v;  // inclusive over the warps
    }
    __syncthreads();
    int pos = incl - c + (warp > 0 ? s_red[warp - 1] : 0);
    for (int i = b0; i < b1; ++i)
        if (s_flag[i]) survivors[pos++] = i;
    if (tid == 0) *d_active = active;
}

#define MOEA_DISPATCH_M(M, CALL)                                                      \
    switch (M) {                                                                      \
    case 1: { constexpr int MM = 1; CALL; } break;                                   \
    case 2: { constexpr int MM = 2; CALL; } break;                                   \
    case 3: { constexpr int MM = 3; CALL; } break;                                   \
    case 4: { constexpr int MM = 4; CALL; } break;                                   \
    case 5: { constexpr int MM = 5; CALL; } break;                                   \
    case 6: { constexpr int MM = 6; CALL; } break;                                   \
    case 7: { constexpr int MM = 7; CALL; } break;                                   \
    case 8: { constexpr int MM = 8; CALL; } break;                                   \
    case 9: { constexpr int MM = 9; CALL; } break;                                   \
    case 10: { constexpr int MM = 10; CALL; } break;                                 \
    case 11: { constexpr int MM = 11; CALL; } break;                                 \
    case 12: { constexpr int MM = 12; CALL; } break;                                 \
    case 13: { constexpr int MM = 13; CALL; } break;                                 \
    case 14: { constexpr int MM = 14; CALL; } break;                                 \
    case 15: { constexpr int MM = 15; CALL; } break;                                 \
    case 16: { constexpr int MM = 16; CALL; } break;                                 \
    default: return set_error(MOEA_ERR_UNSUPPORTED, "objectives=%d", (M));           \
    }

}  // namespace

int run_rvea_translate(const SplitPop& pop, int M, float* t, int t_stride, float* zmin,
                       cudaStream_t s)
{
    zmin_kernel<<<M, 512, 0, s>>>(pop, zmin);
    translate_kernel<<<ceil_div(pop.n, 256), 256, 0, s>>>(pop, M, zmin, t, t_stride);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_rvea_partition(const float* t, int t_stride, int n, const float* refs, int M, int K,
                       const int* d_active, int n_active, int n_parent, float* theta, int* idx,
                       cudaStream_t s)
{
    MOEA_DISPATCH_M(M, (partition_kernel<MM><<<ceil_div(n, 8), 256, 0, s>>>(
                           t, t_stride, n, refs, K, d_active, n_active, n_parent, theta, idx)));
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_rvea_gamma(const float* refs, int M, int K, float* gamma, cudaStream_t s)
{
    MOEA_DISPATCH_M(M, (gamma_kernel<MM><<<ceil_div(K, 128), 128, 0, s>>>(refs, K, gamma)));
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_rvea_apd(const float* t, int t_stride, int n, const float* theta, const float* gamma,
                 const int* idx, int M, int K, const float* ps_table, const int* d_gen,
                 float ps_host, float* apd, cudaStream_t s)
{
    MOEA_DISPATCH_M(M, (apd_kernel<MM><<<ceil_div(n, 256), 256, 0, s>>>(
                           t, t_stride, n, theta, gamma, idx, K, ps_table, d_gen, ps_host, apd)));
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

// Whether the three-launch selection applies, and its launches.  Writes the
// same t / zmin / theta / idx / apd values, survivors and active count as the
// staged translate, partition, APD and elitism.
bool rvea_block_eligible(int n, int M, int K)
{
    return n >= 1 && n <= kRveaBlockPoints && K >= 1 && K <= kRveaBlockDirs && M >= 1 && M <= 16;
}

int run_rvea_select_block(const SplitPop& pop, const float* refs, int M, int K, const float* gamma, int* d_active,
                          int N, const float* ps_table, const int* d_gen, float ps_host, float* t, int t_stride,
                          float* zmin, float* theta, int* idx, float* apd, int* survivors, cudaStream_t s)
{
    const int n = pop.n;
    MOEA_DISPATCH_M(M, (rvea_translate_block<MM><<<1, kRveaBlockThreads, 0, s>>>(pop, t, t_stride, zmin)));
    MOEA_DISPATCH_M(M, (partition_apd_kernel<MM><<<ceil_div(n, 8), 256, 0, s>>>(
                           t, t_stride, n, refs, K, d_active, N, gamma, ps_table, d_gen, ps_host, theta, idx, apd)));
    const size_t smem = sizeof(unsigned long long) * (size_t)(K > n ? K : n);
    rvea_elite_block<<<1, kRveaBlockThreads, smem, s>>>(pop, idx, apd, K, N, d_active, survivors);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

float rvea_penalty_scale(int M, int gen, int max_gen, float alpha)
{
    const float iter_total = std::fmax(static_cast<float>(max_gen), 1.0f);
    const float progress = std::fmin(std::fmax(static_cast<float>(gen) / iter_total, 0.0f), 1.0f);
    return static_cast<float>(M) * std::pow(progress, alpha);
}

// Elitism on the split population; writes the ascending survivor set into
// survivors (first *d_active entries) and the active count to d_active.
int run_rvea_elitism(Workspace& ws, const int* idx, const SplitPop& pop, const float* apd, int N,
                     int K, int* survivors, int* d_active, cudaStream_t s)
{
    const int n = pop.n;
    const int T = 256, G = ceil_div(n, T);
    size_t tmp = ws.cub_bytes;
    int* win_count = ws.counters + 7;
    MOEA_CUDA_TRY(cudaMemsetAsync(win_count, 0, sizeof(int), s));
    elite_keys<<<G, T, 0, s>>>(idx, pop, apd, ws.key64[0], ws.sel_vals[0]);
    MOEA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp, tmp, ws.key64[0], ws.key64[1],
                                                  ws.sel_vals[0], ws.rank, n, 0, 64, s));
    elite_heads<<<G, T, 0, s>>>(ws.key64[1], n, ws.head);
    MOEA_CUDA_TRY(cub::DeviceScan::InclusiveScan(ws.cub_tmp, tmp, ws.head, ws.run_start, cub::Max(),
                                                 n, s));
    elite_winners<<<G, T, 0, s>>>(ws.key64[1], ws.rank, ws.run_start, n, K, ws.blocker, win_count);
    elite_trunc_keys<<<G, T, 0, s>>>(ws.blocker, pop, apd, ws.key64[0], ws.sel_vals[0]);
    MOEA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp, tmp, ws.key64[0], ws.key64[1],
                                                  ws.sel_vals[0], ws.sel_vals[1], n, 0, 64, s));
    MOEA_CUDA_TRY(cudaMemsetAsync(ws.flags, 0, sizeof(int) * (size_t)n, s));
    elite_select<<<ceil_div(N, T), T, 0, s>>>(ws.rank, ws.sel_vals[1], win_count, N, ws.selected,
                                             d_active, ws.flags);
    MOEA_CUDA_TRY(cudaGetLastError());
    // ascending order of the selected set: compaction of the flags
    return run_flag_compaction(ws, n, survivors, s);
}

int run_rvea_update(const SplitPop& pop, const float* vars_a, const float* vars_b,
                    const int* survivors, const int* d_active, int N, int D, int M, float* vars,
                    float* objs, float* cv, cudaStream_t s, int* nan_rows)
{
    const long long items = (long long)N * ((D + kUpdateChunk - 1) / kUpdateChunk);
    const int blocks = (int)std::max(1ll, std::min(items, (long long)148 * 16));
    rvea_update<<<blocks, 256, 0, s>>>(pop, vars_a, vars_b, survivors, d_active, nan_rows, N, D, M, vars, objs, cv);
    if (nan_rows) rvea_mark_nan_rows<<<1, 1, 0, s>>>(nan_rows, d_active);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_fill_int(int* p, int count, int value, cudaStream_t s)
{
    fill_int_kernel<<<(count + 255) / 256, 256, 0, s>>>(p, count, value);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_rvea_adapt(const float* v0, const float* objs, int stride, const int* d_active,
                   int n_active, int M, int K, float* range_tmp, float* v, cudaStream_t s)
{
    zrange_kernel<<<M, 512, 0, s>>>(objs, stride, d_active, n_active, range_tmp);
    MOEA_DISPATCH_M(M, (adapt_kernel<MM><<<ceil_div(K, 256), 256, 0, s>>>(v0, range_tmp, K, v)));
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

}  // namespace moea

using namespace moea;

extern "C" {

moea_status moea_rvea_translate(moea_workspace* w, const float* d_objs, int M, int n, float* d_out,
                                float* d_zmin, void* stream)
{
    if (!d_objs || !d_out || !d_zmin || n < 1 || M < 1 || M > kMaxObjectives)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "rvea_translate: bad arguments");
    (void)w;
    return run_rvea_translate(merged_view(d_objs, d_objs, n), M, d_out, n, d_zmin, (cudaStream_t)stream);
}

moea_status moea_rvea_partition(moea_workspace* w, const float* d_t, const float* d_refs, int M,
                                int n, int K, int n_active, int n_parent, float* d_theta,
                                int* d_idx, void* stream)
{
    (void)w;
    if (!d_t || !d_refs || !d_theta || !d_idx || n < 1 || K < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "rvea_partition: bad arguments");
    return run_rvea_partition(d_t, n, n, d_refs, M, K, nullptr, n_active, n_parent, d_theta, d_idx,
                              (cudaStream_t)stream);
}

moea_status moea_rvea_gamma(moea_workspace* w, const float* d_refs, int M, int K, float* d_gamma,
                            void* stream)
{
    (void)w;
    if (!d_refs || !d_gamma || K < 1) return set_error(MOEA_ERR_INVALID_ARGUMENT, "rvea_gamma: bad arguments");
    return run_rvea_gamma(d_refs, M, K, d_gamma, (cudaStream_t)stream);
}

moea_status moea_rvea_apd(moea_workspace* w, const float* d_t, const float* d_theta,
                          const float* d_gamma, const int* d_idx, int M, int n, int K, int gen,
                          int max_gen, float alpha, float* d_apd, void* stream)
{
    (void)w;
    if (!d_t || !d_theta || !d_gamma || !d_idx || !d_apd || n < 1 || K < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "rvea_apd: bad arguments");
    return run_rvea_apd(d_t, n, n, d_theta, d_gamma, d_idx, M, K, nullptr, nullptr,
                        rvea_penalty_scale(M, gen, max_gen, alpha), d_apd, (cudaStream_t)stream);
}

moea_status moea_rvea_elitism(moea_workspace* w, const int* d_idx, const float* d_cv,
                              const float* d_apd, int N, int n_mix, int K, int* d_selected,
                              int* h_active, void* stream)
{
    if (!w || !d_idx || !d_cv || !d_apd || !d_selected || !h_active || N < 1 || n_mix < 1 ||
        n_mix > w->ws.n_max)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "rvea_elitism: bad arguments");
    Workspace& ws = w->ws;
    const cudaStream_t s = (cudaStream_t)stream;
    SplitPop pop{d_cv, d_cv, d_cv, d_cv, n_mix, n_mix, n_mix, n_mix};
    int* d_active = ws.counters + 8;
    MOEA_TRY(run_rvea_elitism(ws, d_idx, pop, d_apd, N, K, d_selected, d_active, s));
    MOEA_CUDA_TRY(cudaMemcpyAsync(h_active, d_active, sizeof(int), cudaMemcpyDeviceToHost, s));
    MOEA_CUDA_TRY(cudaStreamSynchronize(s));
    return MOEA_OK;
}

moea_status moea_rvea_adapt(moea_workspace* w, const float* d_v0, const float* d_objs, int M, int K,
                            int n_active, int n_stride, float* d_v, void* stream)
{
    if (!w || !d_v0 || !d_objs || !d_v || K < 1 || n_active < 1 || n_stride < n_active)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "rvea_adapt: bad arguments");
    return run_rvea_adapt(d_v0, d_objs, n_stride, nullptr, n_active, M, K, w->ws.ideal_tmp, d_v,
                          (cudaStream_t)stream);
}

}  // extern "C"
