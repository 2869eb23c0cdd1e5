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
    float beta = u1 < 0.5f ? powf(2.0f * u1, power) : powf(1.0f / (2.0f - 2.0f * u1), power);
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

// 24-bit uniform from the low bytes of three draws (bits the SBX draws of
// the same block leave unused).
__device__ __forceinline__ float low_bytes_unit(uint32_t a, uint32_t b, uint32_t c)
{
    return (float)(((a & 0xFFu) << 16) | ((b & 0xFFu) << 8) | (c & 0xFFu)) * (1.0f / 16777216.0f);
}

// SBX + PM for pair element e = p*D + d.  One Philox block (tag crossover)
// gives the SBX draws (u1 and the sign from word 0, u2 from word 1, the copy
// draw from word 2) and both children's mutation test draws (word 3, and the
// unused low bytes of words 1-3).  A second block (tag mutation) is computed
// only where a child mutates, with probability pm_prob/D per child: at large
// D almost every element costs one block instead of two.
//
// kCross / kMutate select the passes: both (the fused variation), crossover
// alone (children written unmutated) or mutation alone (children read from
// off and mutated in place).  The draws are the same in every form, so
// crossover followed by mutation equals the fused pass bit for bit.
template <bool kCross, bool kMutate>
__device__ __forceinline__ void variation_element(long long e, int p, int d,
                                                  const float* __restrict__ parents,
                                                  const int* __restrict__ pidx,
                                                  const float* __restrict__ bounds,
                                                  float* __restrict__ off, int pairs, int D,
                                                  float eta_c, float sbx_prob, float copy_prob,
                                                  int mutate, float eta_m, float pm_prob,
                                                  uint64_t seed, uint32_t gen)
{
    const float lo = bounds[2 * d], hi = bounds[2 * d + 1];
    const int ca = 2 * p, cb = ca + 1;
    uint32_t r[4];
    rng_block(seed, (uint64_t)e, gen, kTagCrossover, r);
    float c1, c2 = 0.0f;
    if (kCross) {
        if (p < pairs) {
            const float x1 = parents[(size_t)pidx[ca] * D + d];
            const float x2 = parents[(size_t)pidx[cb] * D + d];
            sbx_pair(x1, x2, u32_to_unit(r[0]), u32_to_unit(r[1]), (int)(r[0] & 1u),
                     u32_to_unit(r[2]), eta_c, sbx_prob, copy_prob, lo, hi, c1, c2);
        } else {
            c1 = parents[(size_t)pidx[ca] * D + d];  // odd population: last child copies its parent
        }
    } else {
        c1 = off[(size_t)ca * D + d];
        if (p < pairs) c2 = off[(size_t)cb * D + d];
    }
    bool changed = kCross;
    if (kMutate && mutate) {
        // the reference's test, polynomial_mutation.cu:34
        const float limit = pm_prob / static_cast<float>(D);
        const float ta = u32_to_unit(r[3]);
        const float tb = low_bytes_unit(r[1], r[2], r[3]);
        const bool ma = ta < limit, mb = p < pairs && tb < limit;
        if (ma || mb) {
            uint32_t m[4];
            rng_block(seed, (uint64_t)e, gen, kTagMutation, m);
            if (ma) c1 = pm_value(c1, ta, u32_to_unit(m[0]), eta_m, pm_prob, D, lo, hi);
            if (mb) c2 = pm_value(c2, tb, u32_to_unit(m[1]), eta_m, pm_prob, D, lo, hi);
            changed = true;
        }
    }
    if (!changed) return;  // mutation pass: untouched children stay as they are
    off[(size_t)ca * D + d] = c1;
    if (p < pairs) off[(size_t)cb * D + d] = c2;
}

template <bool kCross, bool kMutate>
__global__ void variation_philox(const float* __restrict__ parents, const int* __restrict__ pidx,
                                 const float* __restrict__ bounds, float* __restrict__ off,
                                 int n_off, int D, float sbx_eta0, float sbx_eta1, float sbx_prob,
                                 float copy_prob, int mutate, float pm_eta0, float pm_eta1,
                                 float pm_prob, int total, uint64_t seed,
                                 const int* __restrict__ d_gen, uint32_t gen_host)
{
    const int pairs = n_off / 2;
    const long long count = (long long)(pairs + (n_off & 1)) * D;
    const uint32_t gen = d_gen ? (uint32_t)*d_gen : gen_host;
    const float eta_c = annealed_eta(sbx_eta0, sbx_eta1, (int)gen, total);
    const float eta_m = annealed_eta(pm_eta0, pm_eta1, (int)gen, total);
    if (count <= 0x7FFFFFFFll) {  // 32-bit row/column split
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < (int)count; e += gridDim.x * blockDim.x) {
            const int p = e / D;
            variation_element<kCross, kMutate>(e, p, e - p * D, parents, pidx, bounds, off, pairs, D, eta_c,
                                               sbx_prob, copy_prob, mutate, eta_m, pm_prob, seed, gen);
        }
        return;
    }
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        variation_element<kCross, kMutate>(e, (int)(e / D), (int)(e % D), parents, pidx, bounds, off, pairs, D,
                                           eta_c, sbx_prob, copy_prob, mutate, eta_m, pm_prob, seed, gen);
}

// ---- fused batch: mating then variation of every instance (blockIdx.y) ----
__global__ void fused_mating(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= I.N) return;
    mating_child(i, I.cvP, I.tournament ? I.rankP : nullptr, I.N, I.seed, (uint32_t)*I.d_gen, I.pidx);
}

__global__ void fused_variation(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int pairs = I.N / 2;
    const long long count = (long long)(pairs + (I.N & 1)) * I.D;
    const uint32_t gen = (uint32_t)*I.d_gen;
    const float eta_c = annealed_eta(I.sbx_eta0, I.sbx_eta1, (int)gen, I.T);
    const float eta_m = annealed_eta(I.pm_eta0, I.pm_eta1, (int)gen, I.T);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < (int)count; e += gridDim.x * blockDim.x) {
        const int p = e / I.D;  // fused instances hold at most 4096 x 263 elements
        variation_element<true, true>(e, p, e - p * I.D, I.varsP, I.pidx, I.bounds, I.varsO, pairs, I.D, eta_c,
                                      I.sbx_prob, I.sbx_copy, I.mutate, eta_m, I.pm_prob, I.seed, gen);
    }
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
    const long long count = (long long)(n_off / 2 + (n_off & 1)) * D;
    const int grid = grid_for(count, 256);
    if (passes == kPassBoth)
        variation_philox<true, true><<<grid, 256, 0, stream>>>(
            parents, pidx, bounds, off, n_off, D, sbx_eta0, sbx_eta1, sbx_prob, copy_prob, mutate,
            pm_eta0, pm_eta1, pm_prob, total, seed, d_gen, gen);
    else if (passes == kPassCrossover)
        variation_philox<true, false><<<grid, 256, 0, stream>>>(
            parents, pidx, bounds, off, n_off, D, sbx_eta0, sbx_eta1, sbx_prob, copy_prob, 0,
            pm_eta0, pm_eta1, pm_prob, total, seed, d_gen, gen);
    else
        variation_philox<false, true><<<grid, 256, 0, stream>>>(
            parents, pidx, bounds, off, n_off, D, sbx_eta0, sbx_eta1, sbx_prob, copy_prob, 1,
            pm_eta0, pm_eta1, pm_prob, total, seed, d_gen, gen);
    MOEA_CUDA_TRY(cudaGetLastError());
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
    const long long per = (long long)(g.max_N / 2 + 1) * g.max_D;
    fused_variation<<<dim3((unsigned)grid_for(per, 256, 64), g.count), 256, 0, s>>>(d_inst, g.d_ids);
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
