// NSGA-III selection stages after the non-dominated sort, for sm_100a.
//
// Reference stages (paths relative to python/csrc/native/src/selection/nsga3/):
//   extraction      kernels/non_dominated_sort.cu:1580-1781
//   ideal point     kernels/ideal_point.cu:13-165
//   normalisation   kernels/normalization.cu:370-856, 1217-1394, 1593-1636
//   association     kernels/association.cu:86-188, 397-447, 586-608
//   niching         kernels/niching.cu:21-400 + core/cuda/cuda_ref_segment_ops.cu
//   survivor update kernels/nsga3_population_update.cu:119-281
// Every stage is stream-ordered and reads its sizes from device memory, so a
// whole generation runs without a host round trip.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include <cooperative_groups.h>

#include "internal.cuh"
#include "dirtree.h"

namespace cg = cooperative_groups;

namespace moea {
namespace {

constexpr int kChunk = 1024;

// ---------------------------------------------------------------------------
// ordered two-class compaction (ascending index order inside each class)
// ---------------------------------------------------------------------------

// class of element i: 0 = first group, 1 = second group, -1 = dropped
struct FrontClass {
    const int* fronts;
    const int* max_front;
    __device__ __forceinline__ int operator()(int i) const
    {
        const int f = fronts[i], mf = *max_front;
        return (f >= 0 && f < mf) ? 0 : (f == mf ? 1 : -1);
    }
};
struct FlagClass {
    const int* flags;
    __device__ __forceinline__ int operator()(int i) const { return flags[i] ? 0 : -1; }
};

__device__ __forceinline__ int block_sum_1024(int v, int* sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    int t = 0;
    if (threadIdx.x < 32) {
        t = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xFFFFFFFFu, t, o);
        if (lane == 0) sh[32] = t;
    }
    __syncthreads();
    const int r = sh[32];
    __syncthreads();
    return r;
}

template <class C>
__global__ void __launch_bounds__(kChunk) compact_count(C cls, int n, int* counts, int nchunks)
{
    __shared__ int sh[33];
    const int i = blockIdx.x * kChunk + threadIdx.x;
    const int c = (i < n) ? cls(i) : -1;
    const int a = block_sum_1024(c == 0, sh);
    const int b = block_sum_1024(c == 1, sh);
    if (threadIdx.x == 0) {
        counts[blockIdx.x] = a;
        counts[nchunks + blockIdx.x] = b;
    }
}

template <class C>
__global__ void __launch_bounds__(kChunk)
compact_write(C cls, int n, const int* counts, int nchunks, int N, int* out, int* sizes)
{
    __shared__ int sh[33];
    __shared__ int wa[32], wb[32];
    // offsets of this chunk and totals
    int pa = 0, pb = 0, ta = 0, tb = 0;
    for (int c = threadIdx.x; c < nchunks; c += blockDim.x) {
        const int a = counts[c], b = counts[nchunks + c];
        ta += a; tb += b;
        if (c < (int)blockIdx.x) { pa += a; pb += b; }
    }
    pa = block_sum_1024(pa, sh);
    pb = block_sum_1024(pb, sh);
    ta = block_sum_1024(ta, sh);
    tb = block_sum_1024(tb, sh);
    const int i = blockIdx.x * kChunk + threadIdx.x;
    const int c = (i < n) ? cls(i) : -1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned ma = __ballot_sync(0xFFFFFFFFu, c == 0);
    const unsigned mb = __ballot_sync(0xFFFFFFFFu, c == 1);
    if (lane == 0) { wa[warp] = __popc(ma); wb[warp] = __popc(mb); }
    __syncthreads();
    int oa = 0, ob = 0;
    for (int w = 0; w < warp; ++w) { oa += wa[w]; ob += wb[w]; }
    const unsigned lt = (1u << lane) - 1u;
    if (c == 0) out[pa + oa + __popc(ma & lt)] = i;
    if (c == 1) out[ta + pb + ob + __popc(mb & lt)] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0 && sizes) {
        sizes[0] = ta;
        sizes[1] = tb;
        sizes[2] = N - ta;
        sizes[3] = ta + tb;
    }
}

template <class C>
int run_compaction(C cls, int n, int* counts, int N, int* out, int* sizes, cudaStream_t stream)
{
    const int nchunks = ceil_div(n, kChunk);
    compact_count<C><<<nchunks, kChunk, 0, stream>>>(cls, n, counts, nchunks);
    compact_write<C><<<nchunks, kChunk, 0, stream>>>(cls, n, counts, nchunks, N, out, sizes);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

// ---------------------------------------------------------------------------
// ideal point
// ---------------------------------------------------------------------------

// Running minimum of each objective (ideal_point.cu:97-165): one 8-CTA
// cluster per objective, each CTA over a contiguous eighth of the points;
// CTA 0 combines the eight minima from the cluster's shared memory.
constexpr int kIdealCtas = 8, kIdealThreads = 256;
__global__ void __cluster_dims__(kIdealCtas, 1, 1) __launch_bounds__(kIdealThreads)
ideal_kernel(const float* __restrict__ objs, int stride, int n, const float* prev, float* out)
{
    cg::cluster_group cluster = cg::this_cluster();
    const int r = (int)cluster.block_rank();
    const int m = blockIdx.x / kIdealCtas;
    const int per = (n + kIdealCtas - 1) / kIdealCtas;
    const int lo = r * per, hi = min(n, lo + per);
    float v = INFINITY;
    for (int i = lo + threadIdx.x; i < hi; i += kIdealThreads) v = fminf(v, objs[(size_t)m * stride + i]);
    __shared__ float sh[kIdealThreads / 32];
    __shared__ float s_min;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_down_sync(0xFFFFFFFFu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = INFINITY;
        for (int w = 0; w < kIdealThreads / 32; ++w) b = fminf(b, sh[w]);
        s_min = b;
    }
    cluster.sync();  // every CTA's minimum is published
    if (r == 0 && threadIdx.x == 0) {
        float acc = s_min;
        for (int c = 1; c < kIdealCtas; ++c) acc = fminf(acc, *cluster.map_shared_rank(&s_min, c));
        out[m] = prev ? fminf(prev[m], acc) : acc;
    }
    cluster.sync();  // CTA 0 has read every CTA's minimum
}

// ---------------------------------------------------------------------------
// normalisation
// ---------------------------------------------------------------------------

constexpr int kNormThreads = 256;

__device__ __forceinline__ bool asf_better(float v, int i, float cur, int cur_i)
{
    return v < cur || (v == cur && i < cur_i);
}

// Gathers and translates the nds objectives, and reduces per block the ASF
// argmin of every axis and the per-objective maximum (fallback intercepts).
template <int M>
__global__ void __launch_bounds__(kNormThreads)
norm_gather(SplitPop pop, const int* __restrict__ gidx, const int* __restrict__ sizes,
            const float* __restrict__ ideal, float* __restrict__ nds, int nds_stride,
            float* __restrict__ part_val, int* __restrict__ part_idx, float* __restrict__ part_max,
            int gather)
{
    const int n = sizes[3];
    const int i = blockIdx.x * kNormThreads + threadIdx.x;
    float v[M];
    if (i < n) {
#pragma unroll
        for (int m = 0; m < M; ++m) {
            float t = gather ? pop.obj(m, gidx[i]) : nds[(size_t)m * nds_stride + i];
            t = t - ideal[m];
            if (isfinite(t)) t = fmaxf(t, 0.0f);
            v[m] = t;
            nds[(size_t)m * nds_stride + i] = t;
        }
    }
    __shared__ float s_val[kNormThreads / 32][M];
    __shared__ int s_idx[kNormThreads / 32][M];
    __shared__ float s_max[kNormThreads / 32][M];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < M; ++j) {
        float a = INFINITY;
        int ai = -1;
        float mx = -INFINITY;
        if (i < n) {
            float s = -INFINITY;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const float t = isnan(v[m]) ? INFINITY : v[m];
                s = fmaxf(s, t * ((m == j) ? 1.0f : 1e6f));
            }
            if (asf_better(s, i, a, ai)) { a = s; ai = i; }
            mx = isnan(v[j]) ? -INFINITY : v[j];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_down_sync(0xFFFFFFFFu, a, o);
            const int oi = __shfl_down_sync(0xFFFFFFFFu, ai, o);
            if (asf_better(ov, oi, a, ai)) { a = ov; ai = oi; }
            mx = fmaxf(mx, __shfl_down_sync(0xFFFFFFFFu, mx, o));
        }
        if (lane == 0) { s_val[warp][j] = a; s_idx[warp][j] = ai; s_max[warp][j] = mx; }
    }
    __syncthreads();
    if (threadIdx.x < M) {
        const int j = threadIdx.x;
        float a = INFINITY;
        int ai = -1;
        float mx = -INFINITY;
        for (int w = 0; w < kNormThreads / 32; ++w) {
            if (asf_better(s_val[w][j], s_idx[w][j], a, ai)) { a = s_val[w][j]; ai = s_idx[w][j]; }
            mx = fmaxf(mx, s_max[w][j]);
        }
        part_val[blockIdx.x * M + j] = a;
        part_idx[blockIdx.x * M + j] = ai;
        part_max[blockIdx.x * M + j] = mx;
    }
}

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Reciprocal intercepts from the extreme points s_ext (and the per-objective
// maxima s_max for the fallback), by all threads of a block; the Jacobi
// sweeps run in warp 0 with lane r holding row r.
template <int M>
__device__ __forceinline__ void norm_solve(const float* __restrict__ nds, int nds_stride,
                                           const int* s_ext, const float* s_max,
                                           float* __restrict__ rcp_out, int* __restrict__ extreme_out,
                                           int* __restrict__ ill_out)
{
    __shared__ double sA[M][M];
    __shared__ double sV[M][M];
    __shared__ double s_sigma[M];
    __shared__ int s_bad;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < M * M; t += blockDim.x) {
        const int r = t / M, m = t % M;  // row r = extreme point of axis r
        const int e = s_ext[r];
        const float val = (e >= 0) ? nds[(size_t)m * nds_stride + e] : INFINITY;
        if (!isfinite(val)) atomicExch(&s_bad, 1);
        sA[r][m] = (double)val;
        sV[r][m] = (r == m) ? 1.0 : 0.0;
    }
    __syncthreads();
    // Sweeps in round-robin order (circle method over P = M rounded up to
    // even columns, column P - 1 a bye when M is odd): in round r column
    // P - 1 meets column r and, for k >= 1, (r + k) mod (P - 1) meets
    // (r - k) mod (P - 1).  The pairs of a round share no column, so warp k
    // rotates pair k; every pair comes once per sweep.
    __shared__ int s_stop, s_rot;
    constexpr int P = (M + 1) & ~1;
    constexpr int kPairs = P / 2;
    int bad = s_bad;
    if (!bad) {
        for (int sweep = 0; sweep < 60; ++sweep) {
            // A rotation leaves its two columns with the eigenvalues of their
            // 2x2 Gram matrix, so the smallest column norm never grows and the
            // largest never shrinks: once the current norms fail the
            // conditioning test below, the converged ones fail it too, and
            // the fallback (which ignores the rotations) is the result.
            // Degenerate extreme points (repeated rows) stop here instead of
            // rotating rounding noise for all 60 sweeps.
            if (warp == 0) {
                double cmax = 0.0, cmin = INFINITY;
                for (int i = 0; i < M; ++i) {
                    const double x = (lane < M) ? sA[lane][i] : 0.0;
                    const double sg = sqrt(warp_sum_d(x * x));
                    cmax = fmax(cmax, sg);
                    cmin = fmin(cmin, sg);
                }
                if (lane == 0) {
                    s_stop = (cmin < 1e-10 || cmax / cmin > 1e6) ? 1 : 0;
                    s_rot = 0;
                }
            }
            __syncthreads();
            if (s_stop) {  // uniform over the block
                bad = 1;
                break;
            }
            for (int r = 0; r < P - 1; ++r) {
                if (warp < kPairs) {
                    int i = (warp == 0) ? r : (r + warp) % (P - 1);
                    int j = (warp == 0) ? P - 1 : (r - warp + (P - 1)) % (P - 1);
                    if (i > j) {
                        const int tmp = i;
                        i = j;
                        j = tmp;
                    }
                    if (j < M) {  // j == M is the bye
                        const double x = (lane < M) ? sA[lane][i] : 0.0;
                        const double y = (lane < M) ? sA[lane][j] : 0.0;
                        const double al = warp_sum_d(x * x);
                        const double be = warp_sum_d(y * y);
                        const double ga = warp_sum_d(x * y);
                        if (!(ga == 0.0 || fabs(ga) <= 1e-15 * sqrt(al * be))) {
                            const double zeta = (be - al) / (2.0 * ga);
                            const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                            const double c = 1.0 / sqrt(1.0 + t * t);
                            const double s = c * t;
                            if (lane < M) {
                                sA[lane][i] = c * x - s * y;
                                sA[lane][j] = s * x + c * y;
                                const double vx = sV[lane][i], vy = sV[lane][j];
                                sV[lane][i] = c * vx - s * vy;
                                sV[lane][j] = s * vx + c * vy;
                            }
                            if (lane == 0) s_rot = 1;
                        }
                    }
                }
                __syncthreads();
            }
            const int rotated = s_rot;
            __syncthreads();  // every thread read s_rot before warp 0 clears it
            if (!rotated) break;
        }
    }
    if (warp == 0) {
        {
            double smax = 0.0, smin = INFINITY;
            for (int i = 0; i < M && !bad; ++i) {
                const double x = (lane < M) ? sA[lane][i] : 0.0;
                const double sg = sqrt(warp_sum_d(x * x));
                if (lane == 0) s_sigma[i] = sg;
                if (!isfinite(sg)) bad = 1;
                smax = fmax(smax, sg);
                smin = fmin(smin, sg);
            }
            if (smin < 1e-10 || smax / smin > 1e6) bad = 1;
        }
        __syncwarp();
        float r = 1.0f;
        if (lane < M) {
            if (!bad) {
                double acc = 0.0;
                for (int i = 0; i < M; ++i) {
                    double ut1 = 0.0;
                    for (int k = 0; k < M; ++k) ut1 += sA[k][i];
                    const double sg = s_sigma[i];
                    const double coef = (sg > 1e-5) ? ut1 / (sg * sg) : 0.0;
                    acc += sV[lane][i] * coef;
                }
                r = (float)acc;
            } else {
                const float mx = s_max[lane];
                r = (mx > 1e-10f) ? 1.0f / fmaxf(mx, 1e-6f) : 1.0f;
            }
            if (!isfinite(r) || r <= 0.0f) r = 1.0f;
            rcp_out[lane] = r;
            if (extreme_out) extreme_out[lane] = s_ext[lane];
        }
        if (lane == 0 && ill_out) *ill_out = bad;
    }
}

// Intercepts from the extreme points: one-sided Jacobi SVD in FP64 of the
// matrix whose row r is extreme point r, pseudo-inverse applied to the ones
// vector with singular values <= 1e-5 dropped, and the reference's
// ill-conditioning tests and row-maximum fallback
// (normalization.cu:739-856, 1302-1394).  Run by one block of 256 threads.
template <int M>
__global__ void __launch_bounds__(kNormThreads)
norm_finalize(const float* __restrict__ nds, int nds_stride, const float* __restrict__ part_val,
              const int* __restrict__ part_idx, const float* __restrict__ part_max, int nblocks,
              float* __restrict__ rcp_out, int* __restrict__ extreme_out, int* __restrict__ ill_out)
{
    __shared__ int s_ext[M];
    __shared__ float s_max[M];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = warp; j < M; j += kNormThreads / 32) {
        float a = INFINITY;
        int ai = -1;
        float mx = -INFINITY;
        for (int b = lane; b < nblocks; b += 32) {
            float v = part_val[b * M + j];
            v = isnan(v) ? INFINITY : v;
            if (asf_better(v, part_idx[b * M + j], a, ai)) { a = v; ai = part_idx[b * M + j]; }
            mx = fmaxf(mx, part_max[b * M + j]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_down_sync(0xFFFFFFFFu, a, o);
            const int oi = __shfl_down_sync(0xFFFFFFFFu, ai, o);
            if (asf_better(ov, oi, a, ai)) { a = ov; ai = oi; }
            mx = fmaxf(mx, __shfl_down_sync(0xFFFFFFFFu, mx, o));
        }
        if (lane == 0) { s_ext[j] = ai; s_max[j] = mx; }
    }
    __syncthreads();
    norm_solve<M>(nds, nds_stride, s_ext, s_max, rcp_out, extreme_out, ill_out);
}

__global__ void norm_scale(float* __restrict__ nds, int stride, const int* __restrict__ d_n, int M,
                           const float* __restrict__ rcp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *d_n) return;
    for (int m = 0; m < M; ++m) nds[(size_t)m * stride + i] = nds[(size_t)m * stride + i] * rcp[m];
}

template <int M>
int launch_norm(Workspace& ws, const SplitPop& pop, const int* gidx, const int* sizes,
                const float* ideal, int gather, int n_cap, int* ill_out, cudaStream_t stream)
{
    const int nb = ceil_div(n_cap, kNormThreads);
    float* pv = ws.norm_part;
    float* pm = ws.norm_part + (size_t)nb * M;
    norm_gather<M><<<nb, kNormThreads, 0, stream>>>(pop, gidx, sizes, ideal, ws.nds_objs, ws.n_max,
                                                    pv, ws.norm_part_idx, pm, gather);
    norm_finalize<M><<<1, kNormThreads, 0, stream>>>(ws.nds_objs, ws.n_max, pv, ws.norm_part_idx, pm,
                                                     nb, ws.rcp_b, ws.extreme, ill_out);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int dispatch_norm(Workspace& ws, const SplitPop& pop, const int* gidx, const int* sizes,
                  const float* ideal, int M, int gather, int n_cap, int* ill_out,
                  cudaStream_t stream)
{
    switch (M) {
#define MOEA_NORM_CASE(K) case K: return launch_norm<K>(ws, pop, gidx, sizes, ideal, gather, n_cap, ill_out, stream);
    MOEA_NORM_CASE(1) MOEA_NORM_CASE(2) MOEA_NORM_CASE(3) MOEA_NORM_CASE(4)
    MOEA_NORM_CASE(5) MOEA_NORM_CASE(6) MOEA_NORM_CASE(7) MOEA_NORM_CASE(8)
    MOEA_NORM_CASE(9) MOEA_NORM_CASE(10) MOEA_NORM_CASE(11) MOEA_NORM_CASE(12)
    MOEA_NORM_CASE(13) MOEA_NORM_CASE(14) MOEA_NORM_CASE(15) MOEA_NORM_CASE(16)
#undef MOEA_NORM_CASE
    default: return set_error(MOEA_ERR_UNSUPPORTED, "normalize: M=%d", M);
    }
}

// ---------------------------------------------------------------------------
// association
// ---------------------------------------------------------------------------
//
// For unit directions r_j the perpendicular distance satisfies
// d2_j = |x|^2 - (x.r_j)^2 up to rounding, so the reference argmin is found
// among the directions whose dot^2 lies within a rounding margin of the
// largest dot^2.  Each thread keeps a running max of dot^2 and evaluates the
// reference's FP32 formula (association.cu:139-170: fmaf dot, contracted
// residual, fmaf sum of squares) only for those candidates.  Ties keep the
// smaller index within a thread (ascending j, strict <) and across direction
// splits through a packed (d2 bits, j) atomicMin, so the result equals the
// reference argmin exactly.  Margin: |d2_fp32(j) - (|x|^2 - dot_j^2)| is bounded
// by about (4M+5) eps |x|^2; the kernel uses (16M+64) eps |x|^2.

constexpr int kAssocThreads = 256;
constexpr int kAssocTile = 1024;

template <int M>
struct DirTile {
    static constexpr int kLen = (M <= 4) ? kAssocTile : 512;  // directions per smem tile
};

// delta = max_j | |r_j|^2 - 1 | in FP64, rounded up to FP32 (one block).
__global__ void dir_delta_kernel(const float* __restrict__ refs, int M, int H, float* __restrict__ out)
{
    __shared__ double s_max[32];
    double d = 0.0;
    for (int j = threadIdx.x; j < H; j += blockDim.x) {
        double rr = 0.0;
        for (int m = 0; m < M; ++m) {
            const double v = refs[(size_t)m * H + j];
            rr += v * v;
        }
        const double e = fabs(rr - 1.0);
        d = (e == e) ? fmax(d, e) : INFINITY;
    }
    for (int o = 16; o; o >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = d;
    __syncthreads();
    if (threadIdx.x < 32) {
        d = threadIdx.x < (blockDim.x >> 5) ? s_max[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
        if (threadIdx.x == 0) out[0] = __double2float_ru(fmin(d, 1e30));
    }
}

// One block of points (bx) against one range of directions (by).  With
// best_out the packed (d2, index) minimum is merged atomically across ranges;
// without it the block covers every direction and writes idx/dist directly.
template <int M>
__device__ __forceinline__ void assoc_scan_block(int bx, int by, const float* __restrict__ x, int x_stride,
                                                 const float* __restrict__ scale,
                                                 const float* __restrict__ refs, int H, int n, int split_len,
                                                 float delta, unsigned long long* __restrict__ best_out,
                                                 int* __restrict__ idx_out, float* __restrict__ dist_out)
{
    constexpr int TL = DirTile<M>::kLen;
    __shared__ __align__(16) float s_dir[TL * ((M <= 4) ? 4 : M)];
    const int i = bx * kAssocThreads + threadIdx.x;
    const int j_begin = by * split_len;
    const int j_end = min(H, j_begin + split_len);
    if (bx * kAssocThreads >= n || j_begin >= j_end) return;
    const bool valid = i < n;
    float xr[M];
    float xx = 0.0f;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        float v = valid ? x[(size_t)m * x_stride + i] : 0.0f;
        if (scale) v = v * scale[m];
        xr[m] = v;
        xx = fmaf(v, v, xx);
    }
    const float margin = assoc_margin(M, xx, delta);
    // coarse pre-pass over a strided subset to start with a tight threshold
    float maxd = -INFINITY;
    for (int j = j_begin; j < j_end; j += 61) {
        float dot = 0.0f;
#pragma unroll
        for (int m = 0; m < M; ++m) dot = fmaf(xr[m], __ldg(refs + (size_t)m * H + j), dot);
        maxd = fmaxf(maxd, dot * dot);
    }
    float thr = maxd - margin;
    if (!(thr == thr)) thr = -INFINITY;
    float best = INFINITY;
    int bj = -1;
    for (int t0 = j_begin; t0 < j_end; t0 += TL) {
        const int cnt = min(TL, j_end - t0);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += kAssocThreads) {
            if (M <= 4) {
                float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
                d.x = refs[t0 + t];
                if (M > 1) d.y = refs[(size_t)H + t0 + t];
                if (M > 2) d.z = refs[(size_t)2 * H + t0 + t];
                if (M > 3) d.w = refs[(size_t)3 * H + t0 + t];
                reinterpret_cast<float4*>(s_dir)[t] = d;
            } else {
#pragma unroll
                for (int m = 0; m < M; ++m) s_dir[(size_t)m * TL + t] = refs[(size_t)m * H + t0 + t];
            }
        }
        __syncthreads();
        if (!valid) continue;
#pragma unroll 4
        for (int t = 0; t < cnt; ++t) {
            float r[M];
            if (M <= 4) {
                const float4 d = reinterpret_cast<const float4*>(s_dir)[t];
                r[0] = d.x;
                if (M > 1) r[1 % M] = d.y;
                if (M > 2) r[2 % M] = d.z;
                if (M > 3) r[3 % M] = d.w;
            } else {
#pragma unroll
                for (int m = 0; m < M; ++m) r[m] = s_dir[(size_t)m * TL + t];
            }
            float dot = 0.0f;
#pragma unroll
            for (int m = 0; m < M; ++m) dot = fmaf(xr[m], r[m], dot);
            const float dd = dot * dot;
            if (dd >= thr) {
                float d2 = 0.0f;
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    const float res = fmaf(-dot, r[m], xr[m]);
                    d2 = fmaf(res, res, d2);
                }
                if (d2 < best) { best = d2; bj = t0 + t; }
                if (dd > maxd) {
                    maxd = dd;
                    const float nt = maxd - margin;
                    thr = (nt == nt) ? nt : -INFINITY;
                }
            }
        }
    }
    if (best_out) {
        if (valid && best < INFINITY) {
            const unsigned long long packed =
                ((unsigned long long)__float_as_uint(best) << 32) | (unsigned)bj;
            atomicMin(best_out + i, packed);
        }
    } else if (valid) {
        const bool found = best < INFINITY;
        idx_out[i] = found ? bj : -1;
        dist_out[i] = found ? sqrtf(best) : INFINITY;
    }
}

template <int M>
__global__ void __launch_bounds__(kAssocThreads)
assoc_plain(const float* __restrict__ x, int x_stride, const float* __restrict__ scale,
            const float* __restrict__ refs, int H, const int* __restrict__ d_n, int split_len,
            const float* __restrict__ d_delta, unsigned long long* __restrict__ best_out)
{
    assoc_scan_block<M>(blockIdx.x, blockIdx.y, x, x_stride, scale, refs, H, *d_n, split_len, *d_delta, best_out,
                        nullptr, nullptr);
}

__global__ void assoc_reset(unsigned long long* best, int n_cap)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_cap) best[i] = ~0ull;
}

__global__ void assoc_finish(const unsigned long long* __restrict__ best, const int* __restrict__ d_n,
                             int* __restrict__ idx, float* __restrict__ dist)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *d_n) return;
    const unsigned long long b = best[i];
    if (b == ~0ull) {
        idx[i] = -1;
        dist[i] = INFINITY;
    } else {
        idx[i] = (int)(unsigned)(b & 0xFFFFFFFFull);
        dist[i] = sqrtf(__uint_as_float((unsigned)(b >> 32)));
    }
}

template <int M>
void launch_assoc(const float* x, int x_stride, const float* scale, const float* refs, int H,
                  const int* d_n, int n_cap, const float* d_delta, unsigned long long* best, int sms,
                  cudaStream_t stream)
{
    const int pb = ceil_div(n_cap, kAssocThreads);
    int splits = ceil_div(8LL * sms, pb);
    const int max_splits = ceil_div(H, kAssocTile);
    if (splits > max_splits) splits = max_splits;
    if (splits < 1) splits = 1;
    const int split_len = ceil_div(H, splits);
    assoc_plain<M><<<dim3(pb, splits), kAssocThreads, 0, stream>>>(x, x_stride, scale, refs, H, d_n,
                                                                   split_len, d_delta, best);
}

// ---- cone-tree search ------------------------------------------------------
//
// One warp per point.  The directions sit in the leaves of a 32-ary cone tree
// (at most 32 per leaf, children of a node contiguous).  The warp keeps the
// same running state as the scan kernel -- the largest dot^2 seen (maxd), the
// threshold thr = maxd - margin, and the best packed (d2 bits, index) -- and
// visits children best first (largest projection on the cone axis).  A
// subtree is skipped when a bound on the FP32 dot^2 of every member lies
// below thr: such members are never candidates in the scan kernel either,
// and skipping them cannot change maxd.  Ties are resolved by the packed
// minimum on the original index, so the result equals the reference argmin.
//
// Bound for a cone with axis c and half angle rho: the angle between x and a
// member lies in [theta - rho, theta + rho] (theta = angle(x, c)), so
// |cos| <= max(|cos(max(0, theta - rho))|, |cos(min(pi, theta + rho))|).
// cos(theta) is estimated as (c . x) / |x| with error below dc = (4M + 16)
// 2^-24; sin(theta) is bounded above from the estimate's interval; the FP32
// dot of a member is within (M + 1) 2^-24 |x| |r| of the exact one (covered
// by the 2 dc slack) and |r|^2 <= 1 + delta.

constexpr int kTreeWarps = 8;
constexpr int kTreeMaxDepth = kDirTreeMaxDepth;
// Above this many objectives the cones prune little: the tensor-core search
// (large problems) or one thread per point over all directions is cheaper
// than one warp per point over the tree.
constexpr int kTreeMaxObjectives = 5;

struct TreeArgs {
    const float* dirs;    // (M, H) in tree order
    const int* order;     // tree position -> direction index
    const float* center;  // (M, nodes)
    const float* cos_r;
    const float* sin_r;
    const int2* link;
    int H, nodes;
    float delta;
};

template <int M>
__device__ __forceinline__ void assoc_tree_block(int block, const float* __restrict__ x, int x_stride,
                                                 const float* __restrict__ scale, const TreeArgs& t,
                                                 const int* __restrict__ d_n, int* __restrict__ idx_out,
                                                 float* __restrict__ dist_out)
{
    __shared__ float s_bound[kTreeWarps][kTreeMaxDepth][32];
    __shared__ float s_proj[kTreeWarps][kTreeMaxDepth][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = block * kTreeWarps + warp;
    if (i >= *d_n) return;
    float xr[M];
    float xx = 0.0f;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        float v = x[(size_t)m * x_stride + i];
        if (scale) v = v * scale[m];
        xr[m] = v;
        xx = fmaf(v, v, xx);
    }
    const float kEps = 5.9604645e-08f;  // 2^-24
    const float margin = assoc_margin(M, xx, t.delta);
    const bool prune = margin < INFINITY && xx > 0.0f;
    const float rnorm = prune ? 1.0f / sqrtf(xx) : 0.0f;
    const float dc = (4.0f * M + 16.0f) * kEps;
    const float dd_scale = (1.0f + t.delta) * (1.0f + 9.5367432e-07f);  // (1 + delta)(1 + 2^-20)
    float maxd = -INFINITY, thr = -INFINITY;
    unsigned long long best = ~0ull;

    // bounds of children first..first+count-1 (one per lane) at stack level `level`
    auto test = [&](int first, int count, int level) -> unsigned {
        float bound = INFINITY, proj = 0.0f;
        if (lane < count && prune) {
            const int k = first + lane;
            float p = 0.0f;
#pragma unroll
            for (int m = 0; m < M; ++m) p = fmaf(__ldg(t.center + (size_t)m * t.nodes + k), xr[m], p);
            const float ce = p * rnorm;
            proj = ce;
            const float cr = __ldg(t.cos_r + k);
            if (cr > 0.0f) {
                const float sr = __ldg(t.sin_r + k);
                const float hi = fminf(1.0f, ce + dc), lo = fmaxf(-1.0f, ce - dc);
                const float mc = (lo <= 0.0f && hi >= 0.0f) ? 0.0f : fminf(lo * lo, hi * hi);
                const float sh = fminf(1.0f, sqrtf(fmaxf(0.0f, 1.0f - mc) + 4.0f * kEps));
                const float a = (hi >= cr) ? 1.0f : fmaf(hi, cr, sh * sr);
                const float b = (lo <= -cr) ? -1.0f : fmaf(lo, cr, -(sh * sr));
                const float cm = fminf(1.0f, fmaxf(fabsf(a), fabsf(b))) + 2.0f * dc;
                bound = xx * (cm * cm * dd_scale);
            }
        }
        s_bound[warp][level][lane] = bound;
        s_proj[warp][level][lane] = proj;
        __syncwarp();
        return __ballot_sync(0xffffffffu, lane < count && bound >= thr);
    };

    // exact FP32 evaluation of the directions of one leaf (one per lane)
    auto visit = [&](int start, int count) {
        const bool v = lane < count;
        float r[M];
        float dot = 0.0f;
        if (v) {
#pragma unroll
            for (int m = 0; m < M; ++m) {
                r[m] = __ldg(t.dirs + (size_t)m * t.H + start + lane);
                dot = fmaf(xr[m], r[m], dot);
            }
        }
        const float dd = dot * dot;
        float g = v ? dd : -INFINITY;
#pragma unroll
        for (int o = 16; o; o >>= 1) g = fmaxf(g, __shfl_xor_sync(0xffffffffu, g, o));
        if (g > maxd) {
            maxd = g;
            const float nt = maxd - margin;
            thr = (nt == nt) ? nt : -INFINITY;
        }
        if (v && dd >= thr) {
            float d2 = 0.0f;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const float res = fmaf(-dot, r[m], xr[m]);
                d2 = fmaf(res, res, d2);
            }
            if (d2 < INFINITY) {
                const unsigned long long packed = ((unsigned long long)__float_as_uint(d2) << 32) |
                                                  (unsigned)__ldg(t.order + start + lane);
                best = packed < best ? packed : best;
            }
        }
    };

    const int2 root = __ldg(t.link);
    if (root.y <= 0) {
        visit(root.x, -root.y);
    } else {
        int first_s[kTreeMaxDepth];
        unsigned mask_s[kTreeMaxDepth];
        int sp = 0;
        first_s[0] = root.x;
        mask_s[0] = test(root.x, root.y, 0);
        while (sp >= 0) {
            const bool mine = (mask_s[sp] >> lane) & 1u;
            const unsigned m = __ballot_sync(0xffffffffu, mine && s_bound[warp][sp][lane] >= thr);
            if (!m) {
                --sp;
                continue;
            }
            float pv = ((m >> lane) & 1u) ? s_proj[warp][sp][lane] : -INFINITY;
            int pl = lane;
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const float ov = __shfl_xor_sync(0xffffffffu, pv, o);
                const int ol = __shfl_xor_sync(0xffffffffu, pl, o);
                if (ov > pv || (ov == pv && ol < pl)) {
                    pv = ov;
                    pl = ol;
                }
            }
            mask_s[sp] = m & ~(1u << pl);
            const int2 ln = __ldg(t.link + first_s[sp] + pl);
            if (ln.y <= 0) {
                visit(ln.x, -ln.y);
            } else {
                ++sp;  // the host guarantees depth <= kTreeMaxDepth
                first_s[sp] = ln.x;
                mask_s[sp] = test(ln.x, ln.y, sp);
            }
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const unsigned long long ob = __shfl_xor_sync(0xffffffffu, best, o);
        best = ob < best ? ob : best;
    }
    if (lane == 0) {
        if (best == ~0ull) {
            idx_out[i] = -1;
            dist_out[i] = INFINITY;
        } else {
            idx_out[i] = (int)(unsigned)(best & 0xFFFFFFFFull);
            dist_out[i] = sqrtf(__uint_as_float((unsigned)(best >> 32)));
        }
    }
}

template <int M>
__global__ void __launch_bounds__(kTreeWarps * 32)
assoc_tree(const float* __restrict__ x, int x_stride, const float* __restrict__ scale, TreeArgs t,
           const int* __restrict__ d_n, int* __restrict__ idx_out, float* __restrict__ dist_out)
{
    assoc_tree_block<M>(blockIdx.x, x, x_stride, scale, t, d_n, idx_out, dist_out);
}

// ---------------------------------------------------------------------------
// niching
// ---------------------------------------------------------------------------

__global__ void nich_prior(const int* __restrict__ nds_gidx, const int* __restrict__ idx,
                           const int* __restrict__ sizes, int H, int* __restrict__ rho,
                           int* __restrict__ selected)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sizes[0]) return;
    selected[i] = nds_gidx[i];
    const int r = idx[i];
    if (r >= 0 && r < H) atomicAdd(rho + r, 1);
}

__global__ void nich_keys1(const int* __restrict__ idx, const float* __restrict__ dist,
                           const int* __restrict__ sizes, int n_cap, uint64_t* __restrict__ key,
                           int* __restrict__ val)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_cap) return;
    const int np = sizes[0], nl = sizes[1];
    if (t < nl) {
        key[t] = ((uint64_t)(uint32_t)idx[np + t] << 32) | __float_as_uint(dist[np + t]);
    } else {
        key[t] = ~0ull;
    }
    val[t] = t;
}

__global__ void nich_heads(const uint64_t* __restrict__ key, int n_cap, int* __restrict__ head)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_cap) return;
    const bool h = (t == 0) || ((uint32_t)(key[t] >> 32) != (uint32_t)(key[t - 1] >> 32));
    head[t] = h ? t : 0;
}

// stage 2: rank keys (niching.cu:114-139); stage 3: niching keys (:157-178)
__global__ void nich_keys23(uint64_t* __restrict__ key, const int* __restrict__ run_start,
                            const int* __restrict__ sizes, const int* __restrict__ rho, int H,
                            uint64_t seed, const unsigned long long* __restrict__ offset, int stage)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nl = sizes[1];
    if (t >= nl) return;
    const uint32_t ref = (uint32_t)(key[t] >> 32);
    const int r_i = (int)ref;
    const int rho_r = (r_i >= 0 && r_i < H) ? rho[r_i] : 0;
    const int rank = t - run_start[t];
    if (stage == 2) {
        const uint32_t rnd = splitmix_u32(*offset + (uint64_t)t, seed);
        const uint32_t low = (rho_r == 0 && rank == 0) ? 0u : (rnd | 1u);
        key[t] = ((uint64_t)ref << 32) | low;
    } else {
        const uint32_t rnd = splitmix_u32(*offset + (uint64_t)nl + (uint64_t)t, seed);
        key[t] = ((uint64_t)(uint32_t)(rho_r + rank) << 32) | rnd;
    }
}

__global__ void nich_select(const int* __restrict__ vals, const int* __restrict__ nds_gidx,
                            const int* __restrict__ sizes, int* __restrict__ selected,
                            unsigned long long* __restrict__ offset)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int np = sizes[0], nl = sizes[1], nrem = sizes[2];
    if (i < nrem && i < nl) selected[np + i] = nds_gidx[np + vals[i]];
    if (i == 0) *offset += 2ull * (unsigned long long)nl;
}

// ---------------------------------------------------------------------------
// survivors
// ---------------------------------------------------------------------------

__global__ void flags_set(const int* __restrict__ sel, int count, int* __restrict__ flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) flags[sel[i]] = 1;
}

__global__ void gather_fronts(const int* __restrict__ surv, int N, const int* __restrict__ fronts,
                              int* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = fronts[surv[i]];
}

int sm_count(int device)
{
    static int cached[64] = {0};
    if (device >= 0 && device < 64 && cached[device]) return cached[device];
    int s = 148;
    cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, device);
    if (device >= 0 && device < 64) cached[device] = s;
    return s;
}

// ---------------------------------------------------------------------------
// fused batch: selection stages of every instance, one launch per stage
// ---------------------------------------------------------------------------

// Block sorts of the last front's members with 2, 4 or 8 items per thread:
// the smallest that holds the front (the sort's work grows with the items).
template <int ITEMS>
using FusedSortK64 = cub::BlockRadixSort<uint64_t, kFusedThreads, ITEMS, int>;
using FusedScanInt = cub::BlockScan<int, kFusedThreads>;
union FusedSelStorage {
    typename FusedSortK64<2>::TempStorage sort2;
    typename FusedSortK64<4>::TempStorage sort4;
    typename FusedSortK64<kFusedItems>::TempStorage sort8;
    typename FusedScanInt::TempStorage scan;
};

// Extraction of [prior; last] in ascending index order, running ideal point
// over the offspring, translation and intercepts of one instance per CTA:
// run_extract, run_ideal and run_normalize_split of the single-instance path.
template <int M>
__global__ void __launch_bounds__(kFusedThreads)
fused_prep(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    __shared__ typename FusedScanInt::TempStorage scan_tmp;
    __shared__ float s_red[32];
    __shared__ float s_val[kFusedThreads / 32][M];
    __shared__ int s_idx[kFusedThreads / 32][M];
    __shared__ float s_mx[kFusedThreads / 32][M];
    __shared__ int s_ext[M];
    __shared__ float s_max[M];
    __shared__ int s_tot;
    const BatchInst& I = insts[ids[blockIdx.x]];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int n = I.n, N = I.N;
    const SplitPop pop{I.objsP, I.objsO, I.cvP, I.cvO, N, N, N, n};

    // ordered two-class compaction: class 0 = fronts below the last, 1 = the last
    const int mf = I.counters[2];
    int cls[kFusedItems];
    int ca = 0, cb = 0;
#pragma unroll
    for (int j = 0; j < kFusedItems; ++j) {
        const int i = t * kFusedItems + j;
        int c = -1;
        if (i < n) {
            const int f = I.fronts[i];
            c = (f >= 0 && f < mf) ? 0 : (f == mf ? 1 : -1);
        }
        cls[j] = c;
        ca += c == 0;
        cb += c == 1;
    }
    int packed = ca | (cb << 16), total;
    FusedScanInt(scan_tmp).ExclusiveSum(packed, packed, total);
    const int ta = total & 0xFFFF, tb = total >> 16;
    int pa = packed & 0xFFFF, pb = ta + (packed >> 16);
#pragma unroll
    for (int j = 0; j < kFusedItems; ++j) {
        const int i = t * kFusedItems + j;
        if (cls[j] == 0) I.nds_gidx[pa++] = i;
        else if (cls[j] == 1) I.nds_gidx[pb++] = i;
    }
    if (t == 0) {
        I.sizes[0] = ta;
        I.sizes[1] = tb;
        I.sizes[2] = N - ta;
        I.sizes[3] = ta + tb;
        s_tot = ta + tb;
    }
    // ideal point: fminf orders -0 below +0, so any reduction order gives
    // the single-instance kernel's result
    for (int m = 0; m < M; ++m) {
        float v = INFINITY;
        if (t < 512)
            for (int i = t; i < N; i += 512) v = fminf(v, I.objsO[(size_t)m * N + i]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_down_sync(0xFFFFFFFFu, v, o));
        if (lane == 0 && warp < 16) s_red[warp] = v;
        __syncthreads();
        if (t == 0) {
            float r = INFINITY;
            for (int w = 0; w < 16; ++w) r = fminf(r, s_red[w]);
            I.ideal[m] = fminf(I.ideal[m], r);
        }
        __syncthreads();
    }
    // translated nds objectives, ASF argmin per axis, per-objective maximum
    const int n_nds = s_tot;
    float ideal[M];
#pragma unroll
    for (int m = 0; m < M; ++m) ideal[m] = I.ideal[m];
    float a[M], mx[M];
    int ai[M];
#pragma unroll
    for (int j = 0; j < M; ++j) { a[j] = INFINITY; ai[j] = -1; mx[j] = -INFINITY; }
    for (int i = t; i < n_nds; i += kFusedThreads) {
        const int g = I.nds_gidx[i];
        float v[M];
#pragma unroll
        for (int m = 0; m < M; ++m) {
            float x = pop.obj(m, g) - ideal[m];
            if (isfinite(x)) x = fmaxf(x, 0.0f);
            v[m] = x;
            I.nds_objs[(size_t)m * I.n_max + i] = x;
        }
#pragma unroll
        for (int j = 0; j < M; ++j) {
            float sv = -INFINITY;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const float x = isnan(v[m]) ? INFINITY : v[m];
                sv = fmaxf(sv, x * ((m == j) ? 1.0f : 1e6f));
            }
            if (asf_better(sv, i, a[j], ai[j])) { a[j] = sv; ai[j] = i; }
            mx[j] = fmaxf(mx[j], isnan(v[j]) ? -INFINITY : v[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < M; ++j) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_down_sync(0xFFFFFFFFu, a[j], o);
            const int oi = __shfl_down_sync(0xFFFFFFFFu, ai[j], o);
            if (asf_better(ov, oi, a[j], ai[j])) { a[j] = ov; ai[j] = oi; }
            mx[j] = fmaxf(mx[j], __shfl_down_sync(0xFFFFFFFFu, mx[j], o));
        }
        if (lane == 0) { s_val[warp][j] = a[j]; s_idx[warp][j] = ai[j]; s_mx[warp][j] = mx[j]; }
    }
    __syncthreads();
    if (t < M) {
        float b = INFINITY, bm = -INFINITY;
        int bi = -1;
        for (int w = 0; w < kFusedThreads / 32; ++w) {
            if (asf_better(s_val[w][t], s_idx[w][t], b, bi)) { b = s_val[w][t]; bi = s_idx[w][t]; }
            bm = fmaxf(bm, s_mx[w][t]);
        }
        s_ext[t] = bi;
        s_max[t] = bm;
    }
    __syncthreads();
    norm_solve<M>(I.nds_objs, I.n_max, s_ext, s_max, I.rcp_b, I.extreme, nullptr);
}

template <int M>
__global__ void __launch_bounds__(kAssocThreads)
fused_scan(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    assoc_scan_block<M>(blockIdx.x, 0, I.nds_objs, I.n_max, I.rcp_b, I.t_dirs_orig, I.H, I.sizes[3], I.H,
                        I.t_delta, nullptr, I.assoc_idx, I.assoc_dist);
}

// The same scan with the directions split into `splits` ranges (blockIdx.z),
// merged through the packed (d2 bits, index) minimum as in the staged path;
// fused_scan_reset before it, fused_scan_finish after.  An instance's scan
// then runs on `splits` times the CTAs: within one fused generation the
// instances of a group run side by side and each stage lasts as long as its
// slowest instance, so the long scans of the many-direction instances are
// split rather than run by one thread per point over every direction.
template <int M>
__global__ void __launch_bounds__(kAssocThreads)
fused_scan_split(const BatchInst* __restrict__ insts, const int* __restrict__ ids, int splits)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    assoc_scan_block<M>(blockIdx.x, blockIdx.z, I.nds_objs, I.n_max, I.rcp_b, I.t_dirs_orig, I.H, I.sizes[3],
                        (I.H + splits - 1) / splits, I.t_delta, I.assoc_best, nullptr, nullptr);
}

__global__ void fused_scan_reset(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < I.sizes[3]) I.assoc_best[i] = ~0ull;
}

__global__ void fused_scan_finish(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= I.sizes[3]) return;
    const unsigned long long b = I.assoc_best[i];
    if (b == ~0ull) {
        I.assoc_idx[i] = -1;
        I.assoc_dist[i] = INFINITY;
    } else {
        I.assoc_idx[i] = (int)(unsigned)(b & 0xFFFFFFFFull);
        I.assoc_dist[i] = sqrtf(__uint_as_float((unsigned)(b >> 32)));
    }
}

template <int M>
__global__ void __launch_bounds__(kTreeWarps * 32)
fused_assoc(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const TreeArgs t{I.t_dirs, I.t_order, I.t_center, I.t_cos, I.t_sin, I.t_link, I.H, I.t_nodes, I.t_delta};
    assoc_tree_block<M>(blockIdx.x, I.nds_objs, I.n_max, I.rcp_b, t, I.sizes + 3, I.assoc_idx, I.assoc_dist);
}

// Run starts of the sorted keys (by direction index, the high word) into
// rs[] for this thread's items at positions < n; the keys are staged in
// `stage`, which holds n entries.
template <int ITEMS>
__device__ __forceinline__ void fused_run_starts(const uint64_t (&keys)[ITEMS], uint64_t* stage, int n,
                                                 FusedScanInt::TempStorage& tmp, int (&rs)[ITEMS])
{
    const int t = threadIdx.x;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j)
        if (t * ITEMS + j < n) stage[t * ITEMS + j] = keys[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int pos = t * ITEMS + j;
        const bool h = pos < n &&
                       (pos == 0 || (uint32_t)(keys[j] >> 32) != (uint32_t)(stage[pos - 1] >> 32));
        rs[j] = h ? pos : 0;
    }
    FusedScanInt(tmp).InclusiveScan(rs, rs, cub::Max());
    __syncthreads();
}

// The three niching stages of a last front of nl > kFusedThreads members as
// stable block sorts with ITEMS keys per thread (ITEMS * kFusedThreads >= nl).
template <int ITEMS>
__device__ __forceinline__ void fused_niching_sorted(const BatchInst& I, FusedSelStorage& tmp, int np, int nl,
                                                     int nrem, int H, unsigned long long off)
{
    using Sort = FusedSortK64<ITEMS>;
    typename Sort::TempStorage& sort_tmp = *reinterpret_cast<typename Sort::TempStorage*>(&tmp);
    const int t = threadIdx.x;
    // The high words are direction indices (< H) or niche counts plus ranks
    // (< n); padding keys are all ones.  Bits above the largest of them are
    // zero in every real key, so the sorts stop below them.
    const unsigned hi_max = (unsigned)max(H, I.n);
    const int end_bit = 32 + (32 - __clz(hi_max)) + 1;
    uint64_t keys[ITEMS];
    int vals[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int p = t * ITEMS + j;
        keys[j] = (p < nl) ? (((uint64_t)(uint32_t)I.assoc_idx[np + p] << 32) |
                              __float_as_uint(I.assoc_dist[np + p]))
                           : ~0ull;
        vals[j] = p;
    }
    __syncthreads();  // rho complete
    for (int stage = 1; stage <= 3; ++stage) {
        Sort(sort_tmp).Sort(keys, vals, 0, end_bit);
        __syncthreads();
        if (stage == 3) break;
        int rs[ITEMS];
        fused_run_starts<ITEMS>(keys, I.key64, I.n, tmp.scan, rs);
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const int p = t * ITEMS + j;
            if (p >= nl) continue;
            const uint32_t ref = (uint32_t)(keys[j] >> 32);
            const int r_i = (int)ref;
            const int rho_r = (r_i >= 0 && r_i < H) ? I.rho[r_i] : 0;
            const int rank = p - rs[j];
            if (stage == 1) {
                const uint32_t rnd = splitmix_u32(off + (uint64_t)p, I.nich_seed);
                const uint32_t low = (rho_r == 0 && rank == 0) ? 0u : (rnd | 1u);
                keys[j] = ((uint64_t)ref << 32) | low;
            } else {
                const uint32_t rnd = splitmix_u32(off + (uint64_t)nl + (uint64_t)p, I.nich_seed);
                keys[j] = ((uint64_t)(uint32_t)(rho_r + rank) << 32) | rnd;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int i = t * ITEMS + j;
        if (i < nrem && i < nl) I.selected[np + i] = I.nds_gidx[np + vals[j]];
    }
}

// Niche selection of one instance per CTA: run_niching with block sorts.
__global__ void __launch_bounds__(kFusedThreads)
fused_niching(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    extern __shared__ __align__(16) unsigned char fused_smem[];
    FusedSelStorage& tmp = *reinterpret_cast<FusedSelStorage*>(fused_smem);
    const BatchInst& I = insts[ids[blockIdx.x]];
    const int t = threadIdx.x;
    const int np = I.sizes[0], nl = I.sizes[1], nrem = I.sizes[2], H = I.H;
    const unsigned long long off = *I.offset;
    for (int r = t; r < H; r += kFusedThreads) I.rho[r] = 0;
    __syncthreads();
    for (int i = t; i < np; i += kFusedThreads) {
        I.selected[i] = I.nds_gidx[i];
        const int r = I.assoc_idx[i];
        if (r >= 0 && r < H) atomicAdd(I.rho + r, 1);
    }
    if (nl <= kFusedThreads) {
        // Small fronts: each stage is a stable sort by (key, position), done by
        // counting for every member the members before it, instead of block
        // sorts sized for kFusedMaxPoints.  Same orders, same random words.
        uint64_t* s_key = reinterpret_cast<uint64_t*>(fused_smem);   // [2][kFusedThreads]
        int* s_val = reinterpret_cast<int*>(s_key + 2 * kFusedThreads);  // [2][kFusedThreads]
        int* s_wmax = s_val + 2 * kFusedThreads;                        // [kFusedThreads / 32]
        int cur = 0;
        if (t < nl) {
            s_key[t] = ((uint64_t)(uint32_t)I.assoc_idx[np + t] << 32) | __float_as_uint(I.assoc_dist[np + t]);
            s_val[t] = t;
        }
        __syncthreads();  // rho complete, stage-1 keys in place
        for (int stage = 1; stage <= 3; ++stage) {
            const uint64_t* kc = s_key + cur * kFusedThreads;
            if (t < nl) {
                const uint64_t k = kc[t];
                int r = 0;
                for (int u = 0; u < nl; ++u) {
                    const uint64_t ku = kc[u];
                    r += (ku < k || (ku == k && u < t)) ? 1 : 0;
                }
                s_key[(cur ^ 1) * kFusedThreads + r] = k;
                s_val[(cur ^ 1) * kFusedThreads + r] = s_val[cur * kFusedThreads + t];
            }
            __syncthreads();
            cur ^= 1;
            if (stage == 3) break;
            // start of each direction's run: max-scan of the run heads
            const uint64_t* kn = s_key + cur * kFusedThreads;
            const int lane = t & 31, warp = t >> 5;
            int head = -1;
            if (t < nl && (t == 0 || (uint32_t)(kn[t] >> 32) != (uint32_t)(kn[t - 1] >> 32))) head = t;
            int incl = head;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= o) incl = max(incl, y);
            }
            if (lane == 31) s_wmax[warp] = incl;
            __syncthreads();
            int rs = incl;
            for (int w = 0; w < warp; ++w) rs = max(rs, s_wmax[w]);
            if (t < nl) {
                const uint32_t ref = (uint32_t)(kn[t] >> 32);
                const int r_i = (int)ref;
                const int rho_r = (r_i >= 0 && r_i < H) ? I.rho[r_i] : 0;
                const int rank = t - rs;
                uint64_t nk;
                if (stage == 1) {
                    const uint32_t rnd = splitmix_u32(off + (uint64_t)t, I.nich_seed);
                    const uint32_t low = (rho_r == 0 && rank == 0) ? 0u : (rnd | 1u);
                    nk = ((uint64_t)ref << 32) | low;
                } else {
                    const uint32_t rnd = splitmix_u32(off + (uint64_t)nl + (uint64_t)t, I.nich_seed);
                    nk = ((uint64_t)(uint32_t)(rho_r + rank) << 32) | rnd;
                }
                s_key[cur * kFusedThreads + t] = nk;  // own slot only; heads were read above
            }
            __syncthreads();
        }
        if (t < nrem && t < nl) I.selected[np + t] = I.nds_gidx[np + s_val[cur * kFusedThreads + t]];
    } else if (nl <= 2 * kFusedThreads) {
        fused_niching_sorted<2>(I, tmp, np, nl, nrem, H, off);
    } else if (nl <= 4 * kFusedThreads) {
        fused_niching_sorted<4>(I, tmp, np, nl, nrem, H, off);
    } else {
        fused_niching_sorted<kFusedItems>(I, tmp, np, nl, nrem, H, off);
    }
    if (t == 0) *I.offset = off + 2ull * (unsigned long long)nl;
}

// Survivors in ascending mixed index (run_order_selection) of one instance per CTA.
__global__ void __launch_bounds__(kFusedThreads)
fused_order(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    __shared__ typename FusedScanInt::TempStorage scan_tmp;
    __shared__ unsigned char s_flag[kFusedMaxPoints];
    const BatchInst& I = insts[ids[blockIdx.x]];
    const int t = threadIdx.x, n = I.n, N = I.N;
    for (int i = t; i < kFusedMaxPoints; i += kFusedThreads) s_flag[i] = 0;
    __syncthreads();
    for (int i = t; i < N; i += kFusedThreads) s_flag[I.selected[i]] = 1;
    __syncthreads();
    int c = 0;
#pragma unroll
    for (int j = 0; j < kFusedItems; ++j) {
        const int i = t * kFusedItems + j;
        c += (i < n && s_flag[i]) ? 1 : 0;
    }
    FusedScanInt(scan_tmp).ExclusiveSum(c, c);
#pragma unroll
    for (int j = 0; j < kFusedItems; ++j) {
        const int i = t * kFusedItems + j;
        if (i < n && s_flag[i]) I.survivors[c++] = i;
    }
}

// Next parents from the survivors (gather_next), then the generation counter.
__global__ void fused_gather(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int N = I.N, D = I.D, M = I.M;
    const SplitPop pop{I.objsP, I.objsO, I.cvP, I.cvO, N, N, N, I.n};
    const long long total = (long long)N * D;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e / D), d = (int)(e % D);
        const int s = I.survivors[r];
        I.varsX[e] = (s < N) ? I.varsP[(size_t)s * D + d] : I.varsO[(size_t)(s - N) * D + d];
    }
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
        const int s = I.survivors[r];
        for (int m = 0; m < M; ++m) I.objsX[(size_t)m * N + r] = pop.obj(m, s);
        I.cvX[r] = pop.cvv(s);
        I.rankX[r] = I.fronts[s];
    }
}

__global__ void fused_bump(const BatchInst* __restrict__ insts, const int* __restrict__ ids, int count)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) *insts[ids[k]].d_gen += 1;
}

}  // namespace

int run_extract(Workspace& ws, const int* fronts, int n, const int* d_max_front, int N,
                int* nds_gidx, int* sizes, cudaStream_t stream)
{
    return run_compaction(FrontClass{fronts, d_max_front}, n, ws.chunk_counts, N, nds_gidx, sizes,
                          stream);
}

int run_ideal(const float* objs, int stride, int M, int n, const float* prev, float* ideal_out,
              cudaStream_t stream)
{
    ideal_kernel<<<M * kIdealCtas, kIdealThreads, 0, stream>>>(objs, stride, n, prev, ideal_out);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_normalize_split(Workspace& ws, const SplitPop& pop, const int* nds_gidx, const int* sizes,
                        const float* ideal, int M, cudaStream_t stream)
{
    return dispatch_norm(ws, pop, nds_gidx, sizes, ideal, M, 1, pop.n, nullptr, stream);
}

// Normalisation of a contiguous (M, n) array in place (stage entry point).
int run_normalize_inplace(Workspace& ws, float* objs, const float* ideal, int M, int n,
                          float* rcp_out, int* extreme_out, cudaStream_t stream)
{
    if (n > ws.n_max || M > ws.m_max || M < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "normalize: n=%d M=%d exceed the workspace", n, M);
    // copy into the workspace layout (stride n_max), normalise, copy back scaled
    for (int m = 0; m < M; ++m)
        MOEA_CUDA_TRY(cudaMemcpyAsync(ws.nds_objs + (size_t)m * ws.n_max, objs + (size_t)m * n,
                                      sizeof(float) * n, cudaMemcpyDeviceToDevice, stream));
    int hs[4] = {0, n, 0, n};
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.sizes, hs, sizeof(hs), cudaMemcpyHostToDevice, stream));
    SplitPop none{};
    MOEA_TRY(dispatch_norm(ws, none, nullptr, ws.sizes, ideal, M, 0, n, nullptr, stream));
    norm_scale<<<ceil_div(n, 256), 256, 0, stream>>>(ws.nds_objs, ws.n_max, ws.sizes + 3, M, ws.rcp_b);
    for (int m = 0; m < M; ++m)
        MOEA_CUDA_TRY(cudaMemcpyAsync(objs + (size_t)m * n, ws.nds_objs + (size_t)m * ws.n_max,
                                      sizeof(float) * n, cudaMemcpyDeviceToDevice, stream));
    MOEA_CUDA_TRY(cudaMemcpyAsync(rcp_out, ws.rcp_b, sizeof(float) * M, cudaMemcpyDeviceToDevice, stream));
    if (extreme_out)
        MOEA_CUDA_TRY(cudaMemcpyAsync(extreme_out, ws.extreme, sizeof(int) * M,
                                      cudaMemcpyDeviceToDevice, stream));
    return MOEA_OK;
}

bool direction_tree_ready(const Workspace& ws, const float* d_refs, int M, int H)
{
    return ws.tree_src == d_refs && d_refs && ws.tree_M == M && ws.tree_H == H && ws.tree_nodes > 0;
}

int prepare_direction_tree(Workspace& ws, const float* d_refs, const float* h_refs, int M, int H,
                           cudaStream_t stream)
{
    if (!d_refs || M < 1 || M > kMaxObjectives || H < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "direction tree: bad arguments");
    std::vector<float> host;
    if (!h_refs) {
        host.resize((size_t)M * H);
        MOEA_CUDA_TRY(cudaMemcpyAsync(host.data(), d_refs, sizeof(float) * host.size(),
                                      cudaMemcpyDeviceToHost, stream));
        MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
        h_refs = host.data();
    }
    DirectionTreeHost t;
    MOEA_TRY(build_direction_tree(h_refs, M, H, t));
    ws.tree_src = nullptr;
    const size_t nd = (size_t)M * H, nn = (size_t)t.nodes;
    if (nd > ws.tree_cap_dirs) {
        cudaFree(ws.tree_dirs);
        cudaFree(ws.tree_order);
        ws.tree_dirs = nullptr;
        ws.tree_order = nullptr;
        ws.tree_cap_dirs = 0;
        MOEA_CUDA_TRY(cudaMalloc((void**)&ws.tree_dirs, sizeof(float) * nd));
        MOEA_CUDA_TRY(cudaMalloc((void**)&ws.tree_order, sizeof(int) * nd));
        ws.tree_cap_dirs = nd;
    }
    // one allocation for the nodes: center (M*nodes), cos (nodes), sin (nodes),
    // then link (nodes int2) at an even float offset
    const size_t link_off = ((size_t)(M + 2) * nn + 1) & ~(size_t)1;
    const size_t node_words = link_off + 2 * nn;
    if (node_words > ws.tree_cap_nodes) {
        cudaFree(ws.tree_center);
        ws.tree_center = nullptr;
        ws.tree_cap_nodes = 0;
        MOEA_CUDA_TRY(cudaMalloc((void**)&ws.tree_center, sizeof(float) * node_words));
        ws.tree_cap_nodes = node_words;
    }
    ws.tree_cos = ws.tree_center + (size_t)M * nn;
    ws.tree_sin = ws.tree_cos + nn;
    ws.tree_link = reinterpret_cast<int2*>(ws.tree_center + link_off);
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.tree_dirs, t.dirs.data(), sizeof(float) * nd, cudaMemcpyHostToDevice, stream));
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.tree_order, t.order.data(), sizeof(int) * H, cudaMemcpyHostToDevice, stream));
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.tree_center, t.center.data(), sizeof(float) * M * nn, cudaMemcpyHostToDevice, stream));
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.tree_cos, t.cos_r.data(), sizeof(float) * nn, cudaMemcpyHostToDevice, stream));
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.tree_sin, t.sin_r.data(), sizeof(float) * nn, cudaMemcpyHostToDevice, stream));
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.tree_link, t.link.data(), sizeof(int) * 2 * nn, cudaMemcpyHostToDevice, stream));
    MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
    ws.tree_src = d_refs;
    ws.tree_M = M;
    ws.tree_H = H;
    ws.tree_nodes = t.nodes;
    ws.tree_depth = t.max_depth;
    ws.tree_delta = t.delta;
    return MOEA_OK;
}

bool tensor_preferred(int M, int n_cap, int H)
{
    return M > kTreeMaxObjectives && (long long)n_cap * H >= kTensorMinPairs;
}

int run_dir_delta(const float* refs, int M, int H, float* out, cudaStream_t stream)
{
    dir_delta_kernel<<<1, 1024, 0, stream>>>(refs, M, H, out);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_assoc_reset(unsigned long long* best, int n_cap, cudaStream_t stream)
{
    assoc_reset<<<ceil_div(n_cap, 256), 256, 0, stream>>>(best, n_cap);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_assoc_finish(const unsigned long long* best, const int* d_n, int n_cap, int* idx, float* dist,
                     cudaStream_t stream)
{
    assoc_finish<<<ceil_div(n_cap, 256), 256, 0, stream>>>(best, d_n, idx, dist);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_associate(Workspace& ws, const float* x, int x_stride, const float* scale,
                  const float* refs, int M, const int* d_n, int n_cap, int H, int* idx,
                  float* dist, int mode, cudaStream_t stream)
{
    if (n_cap <= 0) return MOEA_OK;
    if (H <= 0) return set_error(MOEA_ERR_INVALID_ARGUMENT, "associate: no directions");
    if (mode != MOEA_ASSOC_TREE && mode != MOEA_ASSOC_SCAN && mode != MOEA_ASSOC_TENSOR)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "associate: mode %d", mode);
    if (mode == MOEA_ASSOC_TENSOR) {
        if (!tensor_directions_ready(ws, refs, M, H))
            return set_error(MOEA_ERR_STATE, "associate: no tensor operand prepared for these directions");
        return run_associate_tensor(ws, x, x_stride, scale, refs, M, d_n, n_cap, H, idx, dist, stream);
    }
    if (mode == MOEA_ASSOC_TREE) {
        if (!direction_tree_ready(ws, refs, M, H))
            return set_error(MOEA_ERR_STATE, "associate: no cone tree prepared for these directions");
        if (ws.tree_depth <= kTreeMaxDepth && M <= kTreeMaxObjectives) {
            const TreeArgs t{ws.tree_dirs, ws.tree_order, ws.tree_center, ws.tree_cos, ws.tree_sin,
                             ws.tree_link, H, ws.tree_nodes, ws.tree_delta};
            const int blocks = ceil_div(n_cap, kTreeWarps);
            switch (M) {
#define MOEA_TREE_CASE(K) case K: assoc_tree<K><<<blocks, kTreeWarps * 32, 0, stream>>>(x, x_stride, scale, t, d_n, idx, dist); break;
            MOEA_TREE_CASE(1) MOEA_TREE_CASE(2) MOEA_TREE_CASE(3) MOEA_TREE_CASE(4)
            MOEA_TREE_CASE(5) MOEA_TREE_CASE(6) MOEA_TREE_CASE(7) MOEA_TREE_CASE(8)
            MOEA_TREE_CASE(9) MOEA_TREE_CASE(10) MOEA_TREE_CASE(11) MOEA_TREE_CASE(12)
            MOEA_TREE_CASE(13) MOEA_TREE_CASE(14) MOEA_TREE_CASE(15) MOEA_TREE_CASE(16)
#undef MOEA_TREE_CASE
            default: return set_error(MOEA_ERR_UNSUPPORTED, "associate: M=%d", M);
            }
            MOEA_CUDA_TRY(cudaGetLastError());
            return MOEA_OK;
        }
        // many objectives: the tensor-core search where it was prepared (the
        // cones prune little), else -- and for a tree deeper than the
        // kernel's stack -- the scan
        if (tensor_preferred(M, n_cap, H) && tensor_directions_ready(ws, refs, M, H))
            return run_associate_tensor(ws, x, x_stride, scale, refs, M, d_n, n_cap, H, idx, dist, stream);
    }
    dir_delta_kernel<<<1, 1024, 0, stream>>>(refs, M, H, ws.dir_delta);
    assoc_reset<<<ceil_div(n_cap, 256), 256, 0, stream>>>(ws.assoc_best, n_cap);
    const int sms = sm_count(ws.device);
    switch (M) {
#define MOEA_ASSOC_CASE(K) case K: launch_assoc<K>(x, x_stride, scale, refs, H, d_n, n_cap, ws.dir_delta, ws.assoc_best, sms, stream); break;
    MOEA_ASSOC_CASE(1) MOEA_ASSOC_CASE(2) MOEA_ASSOC_CASE(3) MOEA_ASSOC_CASE(4)
    MOEA_ASSOC_CASE(5) MOEA_ASSOC_CASE(6) MOEA_ASSOC_CASE(7) MOEA_ASSOC_CASE(8)
    MOEA_ASSOC_CASE(9) MOEA_ASSOC_CASE(10) MOEA_ASSOC_CASE(11) MOEA_ASSOC_CASE(12)
    MOEA_ASSOC_CASE(13) MOEA_ASSOC_CASE(14) MOEA_ASSOC_CASE(15) MOEA_ASSOC_CASE(16)
#undef MOEA_ASSOC_CASE
    default: return set_error(MOEA_ERR_UNSUPPORTED, "associate: M=%d", M);
    }
    MOEA_CUDA_TRY(cudaGetLastError());
    assoc_finish<<<ceil_div(n_cap, 256), 256, 0, stream>>>(ws.assoc_best, d_n, idx, dist);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

// The full-scan association with caller-provided scratch instead of a
// workspace: best (n_cap packed minima), delta (1 float), d_n (device count).
// Used by the allocation-free entry point (noalloc.cu).
int run_associate_scan_scratch(const float* x, const float* refs, int M, const int* d_n, int n_cap,
                               int H, int* idx, float* dist, unsigned long long* best, float* delta,
                               int device, cudaStream_t stream)
{
    dir_delta_kernel<<<1, 1024, 0, stream>>>(refs, M, H, delta);
    assoc_reset<<<ceil_div(n_cap, 256), 256, 0, stream>>>(best, n_cap);
    const int sms = sm_count(device);
    switch (M) {
#define MOEA_SCRATCH_CASE(K) case K: launch_assoc<K>(x, n_cap, nullptr, refs, H, d_n, n_cap, delta, best, sms, stream); break;
    MOEA_SCRATCH_CASE(1) MOEA_SCRATCH_CASE(2) MOEA_SCRATCH_CASE(3) MOEA_SCRATCH_CASE(4)
    MOEA_SCRATCH_CASE(5) MOEA_SCRATCH_CASE(6) MOEA_SCRATCH_CASE(7) MOEA_SCRATCH_CASE(8)
    MOEA_SCRATCH_CASE(9) MOEA_SCRATCH_CASE(10) MOEA_SCRATCH_CASE(11) MOEA_SCRATCH_CASE(12)
    MOEA_SCRATCH_CASE(13) MOEA_SCRATCH_CASE(14) MOEA_SCRATCH_CASE(15) MOEA_SCRATCH_CASE(16)
#undef MOEA_SCRATCH_CASE
    default: return set_error(MOEA_ERR_UNSUPPORTED, "associate: M=%d", M);
    }
    MOEA_CUDA_TRY(cudaGetLastError());
    assoc_finish<<<ceil_div(n_cap, 256), 256, 0, stream>>>(best, d_n, idx, dist);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_niching(Workspace& ws, uint64_t seed, const int* nds_gidx, const float* dist,
                const int* idx, const int* sizes, int H, int N, int* selected,
                cudaStream_t stream)
{
    const int n_cap = ws.n_max < 2 * N ? ws.n_max : 2 * N;
    const int T = 256, G = ceil_div(n_cap, T);
    MOEA_CUDA_TRY(cudaMemsetAsync(ws.rho, 0, sizeof(int) * (size_t)H, stream));
    nich_prior<<<G, T, 0, stream>>>(nds_gidx, idx, sizes, H, ws.rho, selected);
    // the last front in one cluster's shared memory, sorted over its nl members
    if (n_cap <= niching_cluster_capacity() && niching_cluster_ready()) {
        MOEA_CUDA_TRY(cudaGetLastError());
        return launch_niching_cluster(idx, dist, sizes, ws.rho, H, seed, ws.offset_dev, nds_gidx, selected,
                                      ws.counters + 6, stream);
    }
    nich_keys1<<<G, T, 0, stream>>>(idx, dist, sizes, n_cap, ws.key64[0], ws.sel_vals[0]);
    size_t tmp = ws.cub_bytes;
    // Bits that order the keys: the high word holds a direction index below
    // H (0xFFFFFFFF for none) in stages 1-2 and rho + rank <= 2N in stage 3;
    // padding keys are all ones, the maximum of any bit range, and an index
    // 0xFFFFFFFF truncated to the range still sorts after every valid index.
    auto bits_for = [](long long v) { int b = 1; while ((1ll << b) <= v) ++b; return b; };
    const int end12 = std::min(64, 32 + bits_for((long long)H + 1));
    const int end3 = std::min(64, 32 + bits_for(2ll * N + 1));
    for (int stage = 1; stage <= 3; ++stage) {
        MOEA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp, tmp, ws.key64[0], ws.key64[1],
                                                      ws.sel_vals[0], ws.sel_vals[1], n_cap, 0,
                                                      stage == 3 ? end3 : end12, stream));
        std::swap(ws.key64[0], ws.key64[1]);
        std::swap(ws.sel_vals[0], ws.sel_vals[1]);
        if (stage == 3) break;
        nich_heads<<<G, T, 0, stream>>>(ws.key64[0], n_cap, ws.head);
        MOEA_CUDA_TRY(cub::DeviceScan::InclusiveScan(ws.cub_tmp, tmp, ws.head, ws.run_start,
                                                     cub::Max(), n_cap, stream));
        nich_keys23<<<G, T, 0, stream>>>(ws.key64[0], ws.run_start, sizes, ws.rho, H, seed,
                                         ws.offset_dev, stage + 1);
    }
    nich_select<<<G, T, 0, stream>>>(ws.sel_vals[0], nds_gidx, sizes, selected, ws.offset_dev);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_flag_compaction(Workspace& ws, int n, int* out, cudaStream_t stream)
{
    return run_compaction(FlagClass{ws.flags}, n, ws.chunk_counts, 0, out, nullptr, stream);
}

int run_order_selection(Workspace& ws, const int* selected, int count, int n_mix,
                        int* out_sorted, cudaStream_t stream)
{
    MOEA_CUDA_TRY(cudaMemsetAsync(ws.flags, 0, sizeof(int) * (size_t)n_mix, stream));
    flags_set<<<ceil_div(count, 256), 256, 0, stream>>>(selected, count, ws.flags);
    return run_compaction(FlagClass{ws.flags}, n_mix, ws.chunk_counts, 0, out_sorted, nullptr,
                          stream);
}

// One NSGA-III environmental selection on the split population.
int run_nsga3_select(Workspace& ws, const SplitPop& pop, int M, int N, const float* refs, int H,
                     uint64_t seed, float* ideal_last, int* survivors, int* survivor_fronts,
                     int assoc_mode, cudaStream_t stream, const SplitPop* sort_pop)
{
    const int n_mix = pop.n;
    // the sort may see quantised violations (cv_quantization.cu), the rest the raw ones
    MOEA_TRY(run_ndsort(ws, sort_pop ? *sort_pop : pop, M, N, ws.fronts, stream));
    MOEA_TRY(run_extract(ws, ws.fronts, n_mix, ws.counters + 2, N, ws.nds_gidx, ws.sizes, stream));
    // ideal point: running minimum over the offspring objectives (ideal_point.cu:97-165)
    MOEA_TRY(run_ideal(pop.objs_b, pop.stride_b, M, n_mix - pop.n_a, ideal_last, ideal_last, stream));
    stage_mark("select.extract_ideal", stream);
    MOEA_TRY(run_normalize_split(ws, pop, ws.nds_gidx, ws.sizes, ideal_last, M, stream));
    stage_mark("select.normalize", stream);
    MOEA_TRY(run_associate(ws, ws.nds_objs, ws.n_max, ws.rcp_b, refs, M, ws.sizes + 3, n_mix, H,
                           ws.assoc_idx, ws.assoc_dist, assoc_mode, stream));
    stage_mark("select.associate", stream);
    MOEA_TRY(run_niching(ws, seed, ws.nds_gidx, ws.assoc_dist, ws.assoc_idx, ws.sizes, H, N,
                         ws.selected, stream));
    stage_mark("select.niching", stream);
    MOEA_TRY(run_order_selection(ws, ws.selected, N, n_mix, survivors, stream));
    if (survivor_fronts) {
        gather_fronts<<<ceil_div(N, 256), 256, 0, stream>>>(survivors, N, ws.fronts, survivor_fronts);
        MOEA_CUDA_TRY(cudaGetLastError());
    }
    return MOEA_OK;
}

// ---------------------------------------------------------------------------
// CV quantisation (cv_quantization.cu:11-95)
// ---------------------------------------------------------------------------

__global__ void cv_quant_kernel(const float* __restrict__ cv, float* __restrict__ out, int n,
                                float eps, float clip, float inv_clip_log, float log_alpha,
                                float inv_clip, int bins)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float raw = cv[i];
    const float u = fminf(fmaxf(raw, 0.0f), clip);
    const float x = (log_alpha > 0.0f) ? log1pf(log_alpha * u) * inv_clip_log : u * inv_clip;
    int bin = 1 + __float2int_rd(x * __int2float_rn(bins));
    bin = max(1, min(bins, bin));
    const bool infeas = (eps == 0.0f) ? (raw != 0.0f) : (raw > eps);
    out[i] = infeas ? __int2float_rn(bin) : 0.0f;
}

int run_quantize_cv(const float* cv, float* out, int n, float eps, float clip, float log_alpha,
                    int bins, cudaStream_t stream)
{
    if (n <= 0) return MOEA_OK;
    const float inv_clip = 1.0f / clip;
    const float inv_clip_log = (log_alpha > 0.0f) ? 1.0f / log1pf(log_alpha * clip) : 0.0f;
    cv_quant_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(cv, out, n, eps, clip, inv_clip_log,
                                                          log_alpha, inv_clip, bins);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int fused_select_configure()
{
    MOEA_CUDA_TRY(cudaFuncSetAttribute(fused_niching, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(FusedSelStorage)));
    return MOEA_OK;
}

// Association of a bucket of M > kTreeMaxObjectives instances: one thread
// per point over every direction, or, above kFusedScanSplitLen directions,
// the direction-split scan (at most kFusedScanMaxSplits ranges).
constexpr int kFusedScanSplitLen = 1024;
constexpr int kFusedScanMaxSplits = 8;

template <int M>
void fused_scan_launch(const BatchInst* d_inst, const FusedBucket& b, cudaStream_t s)
{
    const int splits = std::min(kFusedScanMaxSplits, std::max(1, ceil_div(b.max_H, kFusedScanSplitLen)));
    const dim3 grid(ceil_div(b.max_n, kAssocThreads), b.count);
    if (splits == 1) {
        fused_scan<M><<<grid, kAssocThreads, 0, s>>>(d_inst, b.d_ids);
        return;
    }
    fused_scan_reset<<<grid, kAssocThreads, 0, s>>>(d_inst, b.d_ids);
    fused_scan_split<M><<<dim3(grid.x, grid.y, splits), kAssocThreads, 0, s>>>(d_inst, b.d_ids, splits);
    fused_scan_finish<<<grid, kAssocThreads, 0, s>>>(d_inst, b.d_ids);
}

int fused_select(const BatchInst* d_inst, const FusedGroup& g, cudaStream_t s)
{
    const int sort_smem = (int)sizeof(FusedSelStorage);
    for (const FusedBucket& b : g.buckets) {
        switch (b.M) {
#define MOEA_FP_CASE(K)                                                                              \
        case K:                                                                                      \
            fused_prep<K><<<b.count, kFusedThreads, 0, s>>>(d_inst, b.d_ids);                        \
            if (K <= kTreeMaxObjectives)                                                             \
                fused_assoc<K><<<dim3(ceil_div(b.max_n, kTreeWarps), b.count), kTreeWarps * 32, 0,    \
                                 s>>>(d_inst, b.d_ids);                                              \
            else                                                                                     \
                fused_scan_launch<K>(d_inst, b, s);                                                  \
            break;
        MOEA_FP_CASE(1) MOEA_FP_CASE(2) MOEA_FP_CASE(3) MOEA_FP_CASE(4)
        MOEA_FP_CASE(5) MOEA_FP_CASE(6) MOEA_FP_CASE(7) MOEA_FP_CASE(8)
        MOEA_FP_CASE(9) MOEA_FP_CASE(10) MOEA_FP_CASE(11) MOEA_FP_CASE(12)
        MOEA_FP_CASE(13) MOEA_FP_CASE(14) MOEA_FP_CASE(15) MOEA_FP_CASE(16)
#undef MOEA_FP_CASE
        default: return set_error(MOEA_ERR_UNSUPPORTED, "fused select: M=%d", b.M);
        }
    }
    MOEA_CUDA_TRY(cudaGetLastError());
    fused_niching<<<g.count, kFusedThreads, sort_smem, s>>>(d_inst, g.d_ids);
    fused_order<<<g.count, kFusedThreads, 0, s>>>(d_inst, g.d_ids);
    const long long per = (long long)g.max_N * g.max_D;
    const unsigned gx = (unsigned)std::min<long long>(64, (per + 255) / 256);
    fused_gather<<<dim3(gx, g.count), 256, 0, s>>>(d_inst, g.d_ids);
    fused_bump<<<ceil_div(g.count, 256), 256, 0, s>>>(d_inst, g.d_ids, g.count);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

}  // namespace moea
