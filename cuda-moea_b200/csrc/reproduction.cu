// Mating selection, SBX and polynomial mutation for sm_100a.
//
// Reference operators (paths relative to python/csrc/native/src/reproduction/):
//   tournament / random mating   mating_selection.cu:11-108
//   SBX                          sbx_crossover.cu:12-190
//   polynomial mutation          polynomial_mutation.cu:12-124
// The reference fills global buffers with cuRAND draws (three launches for SBX,
// one for PM, one for mating) whose element-to-thread mapping depends on the
// GPU model.  Here every draw is a Philox4x32-10 block computed in registers
// from (seed, element, generation, tag): no random buffers, the same numbers on
// every GPU, and the streams can be regenerated on the host for checking.  The
// `*_explicit` kernels take the draws as arrays instead, which is how the
// stage parity tests feed identical numbers to the oracle.
#include "internal.cuh"

namespace moea {
namespace {

// Winner of a binary tournament (mating_selection.cu:11-35): feasible first,
// then smaller violation (ties to a), then rank (ties to a).
__device__ __forceinline__ int tournament_pick(int a, int b, const float* __restrict__ cv,
                                               const int* __restrict__ rank)
{
    const float ca = cv[a], cb = cv[b];
    if (ca == 0.0f && cb != 0.0f) return a;
    if (ca != 0.0f && cb == 0.0f) return b;
    if (ca != 0.0f && cb != 0.0f) return ca <= cb ? a : b;
    return rank[a] <= rank[b] ? a : b;
}

// Annealed distribution index; the product and sum are kept separate so the
// value is the one the reference computes on the host (sbx_crossover.cu:12-18).
__device__ __forceinline__ float annealed_eta(float begin, float end, int gen, int total)
{
    float p = 1.0f;
    if (total > 0) {
        p = __fdiv_rn((float)gen, (float)total);
        p = fminf(fmaxf(p, 0.0f), 1.0f);
    }
    return __fadd_rn(begin, __fmul_rn(__fsub_rn(end, begin), p));
}

// SBX on one variable pair (sbx_crossover.cu:44-70).  Returns false when the
// pair is copied unchanged.
__device__ __forceinline__ void sbx_pair(float x1, float x2, float u1, float u2, int sign,
                                         float copy, float eta, float prob, float copy_prob,
                                         float lo, float hi, float& c1, float& c2)
{
    if (u2 >= prob || copy < copy_prob) {
        c1 = x1;
        c2 = x2;
        return;
    }
    const float power = 1.0f / (1.0f + eta);
    // one powf on the selected base (the same value as calling it in either
    // branch, without a warp running both when its lanes disagree)
    const float base = u1 < 0.5f ? 2.0f * u1 : 1.0f / (2.0f - 2.0f * u1);
    float beta = powf(base, power);
    beta *= 2 * sign - 1;
    const float midpoint = 0.5f * (x1 + x2);
    const float delta = 0.5f * beta * (x1 - x2);
    c1 = fminf(fmaxf(midpoint + delta, lo), hi);
    c2 = fminf(fmaxf(midpoint - delta, lo), hi);
}

// Deb's bounded polynomial mutation of one value (polynomial_mutation.cu:30-59).
__device__ __forceinline__ float pm_value(float value, float u1, float u2, float eta, float prob,
                                          int D, float lo, float hi)
{
    if (u1 >= prob / static_cast<float>(D)) return value;
    const float range = hi - lo;
    const float normalized = (value - lo) / range;
    const float exponent = eta + 1.0f;
    float delta;
    if (u2 <= 0.5f) {
        const float xy = 1.0f - normalized;
        const float value_mut = 2.0f * u2 + (1.0f - 2.0f * u2) * powf(xy, exponent);
        delta = powf(value_mut, 1.0f / exponent) - 1.0f;
    } else {
        const float xy = normalized;
        const float value_mut = 2.0f * (1.0f - u2) + 2.0f * (u2 - 0.5f) * powf(xy, exponent);
        delta = 1.0f - powf(value_mut, 1.0f / exponent);
    }
    return fminf(fmaxf(value + delta * range, lo), hi);
}

__global__ void tournament_explicit(const int2* __restrict__ cand, const int* __restrict__ rank,
                                    const float* __restrict__ cv, int n, int* __restrict__ winners)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 c = cand[i];
    winners[i] = tournament_pick(c.x, c.y, cv, rank);
}

__global__ void sbx_explicit(const float* __restrict__ parents, const int* __restrict__ pidx,
                             const float* __restrict__ bounds, const float2* __restrict__ u,
                             const int* __restrict__ sign, const float* __restrict__ copy,
                             float* __restrict__ off, float eta, float prob, float copy_prob,
                             int pairs, int D)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)pairs * D) return;
    const int p = (int)(e / D), d = (int)(e % D);
    const int ca = 2 * p, cb = ca + 1;
    const float x1 = parents[(size_t)pidx[ca] * D + d];
    const float x2 = parents[(size_t)pidx[cb] * D + d];
    const float2 r = u[e];
    float c1, c2;
    sbx_pair(x1, x2, r.x, r.y, sign[e], copy[e], eta, prob, copy_prob, bounds[2 * d],
             bounds[2 * d + 1], c1, c2);
    off[(size_t)ca * D + d] = c1;
    off[(size_t)cb * D + d] = c2;
}

__global__ void copy_last_child(const float* __restrict__ parents, const int* __restrict__ pidx,
                                float* __restrict__ off, int child, int D)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d < D) off[(size_t)child * D + d] = parents[(size_t)pidx[child] * D + d];
}

__global__ void pm_explicit(float* __restrict__ off, const float* __restrict__ bounds,
                            const float2* __restrict__ u, float eta, float prob, long long count,
                            int D)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int d = (int)(i % D);
    const float2 r = u[i];
    off[i] = pm_value(off[i], r.x, r.y, eta, prob, D, bounds[2 * d], bounds[2 * d + 1]);
}

// Mating with Philox draws: child i draws block (i, generation, kTagMating).
__device__ __forceinline__ void mating_child(int i, const float* __restrict__ cv,
                                             const int* __restrict__ rank, int active, uint64_t seed,
                                             uint32_t gen, int* __restrict__ pidx)
{
    uint32_t r[4];
    rng_block(seed, (uint64_t)i, gen, kTagMating, r);
    const int a = (int)(r[0] % (uint32_t)active);
    if (rank == nullptr) {
        pidx[i] = a;
        return;
    }
    const int b = (int)(r[1] % (uint32_t)active);
    pidx[i] = tournament_pick(a, b, cv, rank);
}

__global__ void mating_philox(const float* __restrict__ cv, const int* __restrict__ rank,
                              const int* __restrict__ d_active, int active_host, int n_off,
                              uint64_t seed, const int* __restrict__ d_gen, uint32_t gen_host,
                              int* __restrict__ pidx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_off) return;
    const int active = d_active ? *d_active : active_host;
    const uint32_t gen = d_gen ? (uint32_t)*d_gen : gen_host;
    mating_child(i, cv, rank, active, seed, gen, pidx);
}

// ---- variation with Philox draws ------------------------------------------
//
// Draw layout (this project's own stream; the same in the fused pass, the
// crossover-only pass followed by the mutation-only pass, and the batched
// form):
//
//  crossover of pair p, variables 4j .. 4j+3: block b = p * ceil(D/4) + j of
//    tag kTagCrossover; word i gives variable 4j+i its spread draw
//    u1 = unit(w) and its sign (w & 1).  Only when sbx_prob < 1 the block b
//    of tag kTagCrossTest gives the crossover test u2 (word i), and only when
//    copy_prob > 0 the block b of tag kTagCopy gives the copy draw.  Skipping
//    those draws changes nothing: u2 < 1 <= sbx_prob always passes and
//    copy < copy_prob <= 0 never holds.
//  mutation of child c: its mutated variables are drawn as geometric gaps,
//    which gives every variable an independent chance limit = pm_prob / D (in
//    FP32, the reference's test, polynomial_mutation.cu:34).  Draw k of child
//    c is block k * n_off + c of tag kTagMutation: gap = floor(ln u / ln(1 -
//    limit)) in FP64 with u = ((w0 >> 8) + 1) 2^-24, the site is the last
//    site + 1 + gap, and unit(w1) is the site's amplitude draw.
//
// One block per four variables (instead of one per variable) and no per
// variable mutation test: at large D the variation is then bound by its
// powf and its HBM stream, not by Philox rounds.

__device__ __forceinline__ void crossover_group(int t, int p, int j, const float* __restrict__ parents,
                                                const int* __restrict__ pidx, const float* __restrict__ bounds,
                                                float* __restrict__ off, int pairs, int D, bool vec, float eta_c,
                                                float sbx_prob, float copy_prob, uint64_t seed, uint32_t gen)
{
    const int ca = 2 * p, cb = ca + 1;
    const int d0 = 4 * j;
    const int cnt = min(4, D - d0);
    const float* xa = parents + (size_t)pidx[ca] * D + d0;
    if (p >= pairs) {  // odd population: the last child copies its parent
        for (int i = 0; i < cnt; ++i) off[(size_t)ca * D + d0 + i] = xa[i];
        return;
    }
    const float* xb = parents + (size_t)pidx[cb] * D + d0;
    float a[4], bv[4], lo[4], hi[4];
    if (vec) {
        const float4 a4 = __ldg(reinterpret_cast<const float4*>(xa));
        const float4 b4 = __ldg(reinterpret_cast<const float4*>(xb));
        const float4 l01 = __ldg(reinterpret_cast<const float4*>(bounds + 2 * d0));
        const float4 l23 = __ldg(reinterpret_cast<const float4*>(bounds + 2 * d0 + 4));
        a[0] = a4.x; a[1] = a4.y; a[2] = a4.z; a[3] = a4.w;
        bv[0] = b4.x; bv[1] = b4.y; bv[2] = b4.z; bv[3] = b4.w;
        lo[0] = l01.x; hi[0] = l01.y; lo[1] = l01.z; hi[1] = l01.w;
        lo[2] = l23.x; hi[2] = l23.y; lo[3] = l23.z; hi[3] = l23.w;
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const bool in = i < cnt;
            a[i] = in ? xa[i] : 0.0f;
            bv[i] = in ? xb[i] : 0.0f;
            lo[i] = in ? bounds[2 * (d0 + i)] : 0.0f;
            hi[i] = in ? bounds[2 * (d0 + i) + 1] : 0.0f;
        }
    }
    uint32_t r[4], rt[4] = {0u, 0u, 0u, 0u}, rc[4] = {0u, 0u, 0u, 0u};
    rng_block(seed, (uint64_t)t, gen, kTagCrossover, r);
    if (sbx_prob < 1.0f) rng_block(seed, (uint64_t)t, gen, kTagCrossTest, rt);
    if (copy_prob > 0.0f) rng_block(seed, (uint64_t)t, gen, kTagCopy, rc);
    float c1[4], c2[4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
        sbx_pair(a[i], bv[i], u32_to_unit(r[i]), u32_to_unit(rt[i]), (int)(r[i] & 1u), u32_to_unit(rc[i]), eta_c,
                 sbx_prob, copy_prob, lo[i], hi[i], c1[i], c2[i]);
    float* oa = off + (size_t)ca * D + d0;
    float* ob = off + (size_t)cb * D + d0;
    if (vec) {
        *reinterpret_cast<float4*>(oa) = make_float4(c1[0], c1[1], c1[2], c1[3]);
        *reinterpret_cast<float4*>(ob) = make_float4(c2[0], c2[1], c2[2], c2[3]);
    } else {
        for (int i = 0; i < cnt; ++i) {
            oa[i] = c1[i];
            ob[i] = c2[i];
        }
    }
}

__global__ void crossover_philox(const float* __restrict__ parents, const int* __restrict__ pidx,
                                 const float* __restrict__ bounds, float* __restrict__ off, int n_off, int D,
                                 bool vec, float sbx_eta0, float sbx_eta1, float sbx_prob, float copy_prob,
                                 int total, uint64_t seed, const int* __restrict__ d_gen, uint32_t gen_host)
{
    const int pairs = n_off / 2;
    const int D4 = (D + 3) >> 2;
    const long long count = (long long)(pairs + (n_off & 1)) * D4;
    const uint32_t gen = d_gen ? (uint32_t)*d_gen : gen_host;
    const float eta_c = annealed_eta(sbx_eta0, sbx_eta1, (int)gen, total);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(t / D4);
        crossover_group((int)t, p, (int)(t - (long long)p * D4), parents, pidx, bounds, off, pairs, D, vec, eta_c,
                        sbx_prob, copy_prob, seed, gen);
    }
}

// Polynomial mutation of child c in place at its geometric sites (layout
// above), by the four lanes sub = 0..3 of a lane group: draws k = 4i + sub
// are evaluated side by side, their gaps summed with shuffles, and every lane
// mutates its own site (sites are distinct).  Each draw moves the site by at
// least one, so a child takes at most D/4 + 1 rounds.  All four lanes of the
// group call this together (c and `active` uniform within the group).
__device__ __forceinline__ void mutate_child4(int c, bool active, int sub, float* __restrict__ off,
                                              const float* __restrict__ bounds, int n_off, int D, float eta_m,
                                              float pm_prob, uint64_t seed, uint32_t gen)
{
    const float limit = pm_prob / static_cast<float>(D);
    const double log_keep = limit >= 1.0f ? 0.0 : log1p(-(double)limit);
    const unsigned group = 0xFu << (threadIdx.x & 28u);
    float* row = off + (size_t)c * D;
    long long site = -1;  // the group's last site
    bool live = active && limit > 0.0f;
    for (long long k0 = 0; __any_sync(group, live); k0 += 4) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
        long long step = 1;
        if (live) {
            rng_block(seed, (uint64_t)(k0 + sub) * (uint64_t)n_off + (uint64_t)c, gen, kTagMutation, w);
            if (log_keep < 0.0) {
                const double u = (double)((w[0] >> 8) + 1u) * (1.0 / 16777216.0);
                const double g = floor(log(u) / log_keep);
                step += g < (double)D ? (long long)g : (long long)D;
            }
        }
        // inclusive sum of the steps over the group's lanes 0..sub
        long long acc = step;
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            const long long v = __shfl_up_sync(group, acc, o, 4);
            if (sub >= o) acc += v;
        }
        const long long my_site = site + acc;
        if (live && my_site < D) {
            const int d = (int)my_site;
            // test draw 0 < limit: the site mutates (pm_value's own test passes)
            row[d] = pm_value(row[d], 0.0f, u32_to_unit(w[1]), eta_m, pm_prob, D, bounds[2 * d], bounds[2 * d + 1]);
        }
        site = __shfl_sync(group, my_site, 3, 4);
        live = live && site < D;
    }
}

__global__ void mutation_philox(float* __restrict__ off, const float* __restrict__ bounds, int n_off, int D,
                                float pm_eta0, float pm_eta1, float pm_prob, int total, uint64_t seed,
                                const int* __restrict__ d_gen, uint32_t gen_host)
{
    const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 2);
    const uint32_t gen = d_gen ? (uint32_t)*d_gen : gen_host;
    const float eta_m = annealed_eta(pm_eta0, pm_eta1, (int)gen, total);
    mutate_child4(c < n_off ? c : 0, c < n_off, (int)(threadIdx.x & 3u), off, bounds, n_off, D, eta_m, pm_prob,
                  seed, gen);
}

// ---- fused batch: mating, crossover and mutation of every instance (blockIdx.y) ----
__global__ void fused_mating(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= I.N) return;
    mating_child(i, I.cvP, I.tournament ? I.rankP : nullptr, I.N, I.seed, (uint32_t)*I.d_gen, I.pidx);
}

__global__ void fused_crossover(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int pairs = I.N / 2;
    const int D4 = (I.D + 3) >> 2;
    const int count = (pairs + (I.N & 1)) * D4;  // fused instances hold at most 4096 x 263 variables
    const uint32_t gen = (uint32_t)*I.d_gen;
    const float eta_c = annealed_eta(I.sbx_eta0, I.sbx_eta1, (int)gen, I.T);
    const bool vec = (I.D & 3) == 0 && ((uintptr_t)I.varsP & 15) == 0 && ((uintptr_t)I.varsO & 15) == 0 &&
                     ((uintptr_t)I.bounds & 15) == 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const int p = t / D4;
        crossover_group(t, p, t - p * D4, I.varsP, I.pidx, I.bounds, I.varsO, pairs, I.D, vec, eta_c, I.sbx_prob,
                        I.sbx_copy, I.seed, gen);
    }
}

__global__ void fused_mutation(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    if (!I.mutate) return;  // uniform over the block
    const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 2);
    const uint32_t gen = (uint32_t)*I.d_gen;
    const float eta_m = annealed_eta(I.pm_eta0, I.pm_eta1, (int)gen, I.T);
    mutate_child4(c < I.N ? c : 0, c < I.N, (int)(threadIdx.x & 3u), I.varsO, I.bounds, I.N, I.D, eta_m, I.pm_prob,
                  I.seed, gen);
}

__global__ void rng_blocks_kernel(uint64_t seed, uint32_t gen, uint32_t tag, long long count,
                                  uint4* out)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    uint32_t r[4];
    rng_block(seed, (uint64_t)e, gen, tag, r);
    out[e] = make_uint4(r[0], r[1], r[2], r[3]);
}

// x = lb + u (ub - lb) (population.cu:12-24, 97-115) with Philox draws.
__global__ void init_uniform(float* __restrict__ vars, const float* __restrict__ bounds,
                             long long count, int D, uint64_t seed)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    uint32_t r[4];
    rng_block(seed, (uint64_t)(e >> 2), 0u, kTagInit, r);
    const float u = u32_to_unit(r[e & 3]);
    const int d = (int)(e % D);
    const float lower = bounds[2 * d], upper = bounds[2 * d + 1];
    vars[e] = lower + u * (upper - lower);
}

inline int grid_for(long long count, int threads, int cap = 148 * 32)
{
    long long g = (count + threads - 1) / threads;
    if (g > cap) g = cap;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

int run_mating(const float* cv, const int* rank, const int* d_active, int active, int n_off,
               uint64_t seed, const int* d_gen, uint32_t gen, int* pidx, cudaStream_t stream)
{
    mating_philox<<<ceil_div(n_off, 256), 256, 0, stream>>>(cv, rank, d_active, active, n_off, seed,
                                                            d_gen, gen, pidx);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_variation_pass(int passes, const float* parents, const int* pidx, const float* bounds, float* off,
                       int n_off, int D, float sbx_eta0, float sbx_eta1, float sbx_prob, float copy_prob,
                       int mutate, float pm_eta0, float pm_eta1, float pm_prob, int total,
                       uint64_t seed, const int* d_gen, uint32_t gen, cudaStream_t stream)
{
    if (passes & kPassCrossover) {
        const long long count = (long long)(n_off / 2 + (n_off & 1)) * ((D + 3) / 4);
        // 16-byte loads and stores when every row and the bounds are aligned
        const bool vec = (D & 3) == 0 && ((uintptr_t)parents & 15) == 0 && ((uintptr_t)off & 15) == 0 &&
                         ((uintptr_t)bounds & 15) == 0;
        crossover_philox<<<grid_for(count, 256), 256, 0, stream>>>(parents, pidx, bounds, off, n_off, D, vec,
                                                                   sbx_eta0, sbx_eta1, sbx_prob, copy_prob, total,
                                                                   seed, d_gen, gen);
        MOEA_CUDA_TRY(cudaGetLastError());
    }
    if ((passes & kPassMutation) && mutate && n_off > 0) {
        mutation_philox<<<ceil_div(4 * n_off, 128), 128, 0, stream>>>(off, bounds, n_off, D, pm_eta0, pm_eta1,
                                                                      pm_prob, total, seed, d_gen, gen);
        MOEA_CUDA_TRY(cudaGetLastError());
    }
    return MOEA_OK;
}

int run_variation(const float* parents, const int* pidx, const float* bounds, float* off,
                  int n_off, int D, float sbx_eta0, float sbx_eta1, float sbx_prob, float copy_prob,
                  int mutate, float pm_eta0, float pm_eta1, float pm_prob, int total,
                  uint64_t seed, const int* d_gen, uint32_t gen, cudaStream_t stream)
{
    return run_variation_pass(kPassBoth, parents, pidx, bounds, off, n_off, D, sbx_eta0, sbx_eta1, sbx_prob,
                              copy_prob, mutate, pm_eta0, pm_eta1, pm_prob, total, seed, d_gen, gen, stream);
}

int fused_reproduce(const BatchInst* d_inst, const FusedGroup& g, cudaStream_t s)
{
    fused_mating<<<dim3(ceil_div(g.max_N, 256), g.count), 256, 0, s>>>(d_inst, g.d_ids);
    const long long per = (long long)(g.max_N / 2 + 1) * ((g.max_D + 3) / 4);
    fused_crossover<<<dim3((unsigned)grid_for(per, 256, 64), g.count), 256, 0, s>>>(d_inst, g.d_ids);
    fused_mutation<<<dim3(ceil_div(4 * g.max_N, 128), g.count), 128, 0, s>>>(d_inst, g.d_ids);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

int run_init_uniform(float* vars, const float* bounds, int N, int D, uint64_t seed,
                     cudaStream_t stream)
{
    const long long count = (long long)N * D;
    init_uniform<<<(int)((count + 255) / 256), 256, 0, stream>>>(vars, bounds, count, D, seed);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

}  // namespace moea

using namespace moea;

extern "C" {

moea_status moea_tournament(const int* d_cand, const int* d_rank, const float* d_cv, int n,
                            int* d_winners, void* stream)
{
    if (!d_cand || !d_rank || !d_cv || !d_winners || n < 0)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "tournament: bad arguments");
    if (n == 0) return MOEA_OK;
    tournament_explicit<<<ceil_div(n, 256), 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const int2*>(d_cand), d_rank, d_cv, n, d_winners);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

moea_status moea_sbx(const float* d_parents, const int* d_pidx, const float* d_bounds,
                     const float* d_u, const int* d_sign, const float* d_copy, float* d_off,
                     float eta, float prob, float copy_prob, int n_off, int D, void* stream)
{
    if (!d_parents || !d_pidx || !d_bounds || !d_u || !d_sign || !d_copy || !d_off || n_off < 0 ||
        D < 1 || !(eta > 0.0f) || prob < 0.0f || prob > 1.0f || copy_prob < 0.0f || copy_prob > 1.0f)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "sbx: bad arguments");
    const cudaStream_t s = (cudaStream_t)stream;
    const int pairs = n_off / 2;
    const long long count = (long long)pairs * D;
    if (count > 0)
        sbx_explicit<<<(int)((count + 255) / 256), 256, 0, s>>>(
            d_parents, d_pidx, d_bounds, reinterpret_cast<const float2*>(d_u), d_sign, d_copy,
            d_off, eta, prob, copy_prob, pairs, D);
    if (n_off & 1)
        copy_last_child<<<ceil_div(D, 256), 256, 0, s>>>(d_parents, d_pidx, d_off, n_off - 1, D);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

moea_status moea_pm(float* d_off, const float* d_bounds, const float* d_u, float eta, float prob,
                    int n, int D, void* stream)
{
    if (!d_off || !d_bounds || !d_u || n < 0 || D < 1 || !(eta > 0.0f) || prob < 0.0f || prob > 1.0f)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "pm: bad arguments");
    const long long count = (long long)n * D;
    if (count > 0)
        pm_explicit<<<(int)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
            d_off, d_bounds, reinterpret_cast<const float2*>(d_u), eta, prob, count, D);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

moea_status moea_reproduce(const float* d_parents, const float* d_parent_cv, const int* d_rank,
                           int active, const float* d_bounds, float* d_off, int* d_parent_idx,
                           int n_parents, int n_off, int D, int mating, float sbx_eta,
                           float sbx_prob, float sbx_copy_prob, int mutate, float pm_eta,
                           float pm_prob, uint64_t seed, uint32_t generation, void* stream)
{
    if (!d_parents || !d_bounds || !d_off || !d_parent_idx || n_off < 1 || D < 1 ||
        active < 1 || active > n_parents || (mating == MOEA_MATING_TOURNAMENT && (!d_rank || !d_parent_cv)))
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "reproduce: bad arguments");
    const cudaStream_t s = (cudaStream_t)stream;
    MOEA_TRY(run_mating(d_parent_cv, mating == MOEA_MATING_TOURNAMENT ? d_rank : nullptr, nullptr,
                        active, n_off, seed, nullptr, generation, d_parent_idx, s));
    return run_variation(d_parents, d_parent_idx, d_bounds, d_off, n_off, D, sbx_eta, sbx_eta,
                         sbx_prob, sbx_copy_prob, mutate, pm_eta, pm_eta, pm_prob, 0, seed, nullptr,
                         generation, s);
}

moea_status moea_initialize_population(uint64_t seed, uint32_t epoch, const float* d_bounds, int N, int D,
                                      float* d_vars, void* stream)
{
    if (!d_bounds || !d_vars || N < 1 || D < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "initialize_population: bad arguments");
    return run_init_uniform(d_vars, d_bounds, N, D, derive_seed(seed) ^ ((uint64_t)epoch << 48),
                            (cudaStream_t)stream);
}

moea_status moea_rng_blocks(uint64_t seed, uint32_t generation, uint32_t tag, int64_t count,
                            uint32_t* d_out, void* stream)
{
    if (!d_out || count < 0) return set_error(MOEA_ERR_INVALID_ARGUMENT, "rng_blocks: bad arguments");
    if (count == 0) return MOEA_OK;
    rng_blocks_kernel<<<(int)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        seed, generation, tag, count, reinterpret_cast<uint4*>(d_out));
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

}  // extern "C"
