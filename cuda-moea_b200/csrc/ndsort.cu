// Constraint-dominance non-dominated sorting for sm_100a.
//
// Replaces run_ndsort / run_ndsort_init and the COO / CSR / bitmask paths of
// CUDA-MOEA (nat/src/selection/nsga3/kernels/non_dominated_sort.cu:158-1574).
// Same result (front index per point, -1 past the stop rule, index of the last
// front), different mechanism:
//
//  1. Lexicographic sort of the points by (class, f0 | cv, f1, ..., f_{M-1})
//     with stable LSD radix passes.  Class 0 = feasible, 1 = feasible with a NaN
//     objective, 2 = infeasible, 3 = infeasible with NaN violation.  In this
//     order every dominator of a point lies strictly before it, and a feasible
//     dominator already satisfies f0 <= q0.
//  2. For every sorted position q, dup[q] is the first position that cannot
//     dominate q: the start of q's run of identical objective vectors (class 0),
//     0 (class 1: nothing dominates it), the start of q's run of equal violation
//     (class 2) or the number of feasible points (class 3).  Then
//       infeasible q:  p dominates q  <=>  p < dup[q]
//       feasible q:    p dominates q  <=>  p < dup[q] and f_m(p) <= f_m(q), m >= 1
//     which is the reference relation (non_dominated_sort.cu:190-239) with one
//     integer and M-1 float comparisons per pair on the lower triangle only.
//  3. For every word of 32 sorted positions and every objective m >= 1 the
//     positions are sorted by f_m once, with the prefix sets of that order.
//     A tile kernel then evaluates the test for one dominatee per lane: the
//     dominators of a word with f_m(p) <= f_m(q) are one prefix set, found
//     by a binary search, and the row word is the AND of those sets with the
//     dup mask.  It stores for every q the bit row of its dominators.
//  4. One cooperative persistent kernel peels the fronts: q joins front k when
//     no still-unassigned point is left in its row.  Each point remembers one
//     unassigned dominator ("blocker"); while that blocker is unassigned the
//     point is skipped without touching memory, so every row is scanned at most
//     once over the whole sort.  Fronts are separated by a bounded grid barrier
//     and the loop stops once `target` points are assigned, like the
//     reference's front propagation loops (:792-843, :1070-1279).
#include <cub/cub.cuh>

#include "internal.cuh"

namespace moea {
namespace {

constexpr int kQB = 128;      // sorted positions (dominatees) per tile CTA
constexpr int kTileThreads = 256;
constexpr int kPeelThreads = 1024;
constexpr uint32_t kInfeasibleBit = 0x80000000u;

// ---------------------------------------------------------------------------
// 1. classification and lexicographic sort
// ---------------------------------------------------------------------------

__global__ void nds_classify(SplitPop pop, int M, uint64_t* __restrict__ key0,
                             int* __restrict__ perm, int* __restrict__ feasible_count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool feasible_class = false;
    if (i < pop.n) {
        const float cv = pop.cvv(i);
        uint32_t cls, val = 0;
        if (cv == 0.0f) {
            bool nan = false;
            for (int m = 0; m < M; ++m) nan |= isnan(pop.obj(m, i));
            cls = nan ? 1u : 0u;
            if (!nan) val = float_order_key(pop.obj(0, i));
        } else {
            cls = isnan(cv) ? 3u : 2u;
            if (cls == 2u) val = float_order_key(cv);
        }
        key0[i] = ((uint64_t)cls << 32) | val;
        perm[i] = i;
        feasible_class = cls <= 1u;
    }
    const unsigned fm = __ballot_sync(0xFFFFFFFFu, feasible_class);
    if ((threadIdx.x & 31) == 0 && fm) atomicAdd(feasible_count, __popc(fm));
}

// Key of LSD pass m (m >= 1) for the current order.
__global__ void nds_gather_key(SplitPop pop, int m, const uint64_t* __restrict__ key0,
                               const int* __restrict__ perm, uint32_t* __restrict__ key)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= pop.n) return;
    const int pt = perm[pos];
    key[pos] = ((key0[pt] >> 32) == 0) ? float_order_key(pop.obj(m, pt)) : 0u;
}

__global__ void nds_gather_key0(int n, const uint64_t* __restrict__ key0,
                                const int* __restrict__ perm, uint64_t* __restrict__ key)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos < n) key[pos] = key0[perm[pos]];
}

// Sorted copy of objectives 1..M-1 and run heads for the dup computation.
__global__ void nds_sorted_soa(SplitPop pop, int M, const uint64_t* __restrict__ key0,
                               const int* __restrict__ perm, float* __restrict__ sf,
                               int sf_stride, int* __restrict__ head)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= pop.n) return;
    const int pt = perm[pos];
    const uint64_t k0 = key0[pt];
    const uint32_t cls = (uint32_t)(k0 >> 32);
    for (int m = 1; m < M; ++m) sf[(size_t)(m - 1) * sf_stride + pos] = pop.obj(m, pt);
    bool is_head = true;
    if (pos > 0) {
        const int pp = perm[pos - 1];
        const uint64_t k1 = key0[pp];
        if (k1 == k0) {
            if (cls == 0u) {
                bool same = true;
                for (int m = 1; m < M; ++m)
                    same &= float_order_key(pop.obj(m, pt)) == float_order_key(pop.obj(m, pp));
                is_head = !same;
            } else {
                is_head = false;
            }
        }
    }
    head[pos] = is_head ? pos : 0;
}

__global__ void nds_finalize_rows(int n, const uint64_t* __restrict__ key0,
                                  const int* __restrict__ perm, const int* __restrict__ run_start,
                                  const int* __restrict__ feasible_count, int* __restrict__ qinfo,
                                  int* __restrict__ blocker, int* __restrict__ front_sorted)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const uint32_t cls = (uint32_t)(key0[perm[pos]] >> 32);
    uint32_t d;
    switch (cls) {
    case 0u: d = (uint32_t)run_start[pos]; break;
    case 1u: d = 0u; break;
    case 2u: d = (uint32_t)run_start[pos] | kInfeasibleBit; break;
    default: d = (uint32_t)(*feasible_count) | kInfeasibleBit; break;
    }
    qinfo[pos] = (int)d;
    blocker[pos] = -1;
    front_sorted[pos] = -1;
}

// ---------------------------------------------------------------------------
// 2. dominance rows
// ---------------------------------------------------------------------------

// Order key of an objective value for the dominance test; NaN maps above
// every other key so that a NaN dominator never satisfies key(p) <= key(q).
__device__ __forceinline__ uint32_t dom_key(float f)
{
    return isnan(f) ? 0xFFFFFFFFu : float_order_key(f);
}

// Per word of 32 sorted positions and per objective m >= 1: the 32 order
// keys in ascending order (keys[m][32 w + k]) and the prefix sets
// bits[m][33 w + k] = positions (bit j = position 32 w + j) of the k smallest
// keys, k = 0..32.  For a value v, the positions of the word whose objective
// is <= v are bits[m][33 w + c] with c = #{keys <= key(v)}: ties at the
// boundary all lie inside the prefix, whatever their order.  Positions >= n
// get the NaN key.  One warp per (word, objective): bitonic sort of
// (key, lane) pairs, then an inclusive OR-scan of the lane bits.
__global__ void nds_chunks(const float* __restrict__ sf, int sf_stride, int n, int W, int MF,
                           uint32_t* __restrict__ ckeys, uint32_t* __restrict__ cbits)
{
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (gw >= W * MF) return;
    const int m = gw / W, w = gw - m * W;
    const int p = w * 32 + lane;
    const uint32_t key = (p < n) ? dom_key(sf[(size_t)m * sf_stride + p]) : 0xFFFFFFFFu;
    unsigned long long kv = ((unsigned long long)key << 32) | (unsigned)lane;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, kv, j);
            const bool take_min = ((lane & j) == 0) == ((lane & k) == 0);
            kv = take_min ? (o < kv ? o : kv) : (o > kv ? o : kv);
        }
    }
    uint32_t pre = 1u << (unsigned)(kv & 31ull);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, pre, o);
        if (lane >= o) pre |= t;
    }
    ckeys[(size_t)m * W * 32 + (size_t)w * 32 + lane] = (uint32_t)(kv >> 32);
    uint32_t* b = cbits + (size_t)m * W * 33 + (size_t)w * 33;
    b[lane + 1] = pre;
    if (lane == 0) b[0] = 0u;
}

// Dominator words per tile CTA (32 positions each), sized so that the staged
// word tables and the transposed output fit in 48 KB of shared memory.
template <int M>
struct TileCfg {
    static constexpr int kPW = (M <= 4) ? 32 : ((M <= 8) ? 16 : 8);
    static constexpr int kMF = (M > 1) ? M - 1 : 1;   // objectives 1..M-1
};

// One CTA covers kQB dominatees q (one per lane of warps 0-3, again of warps
// 4-7) against kPW words of dominator positions p (the first half of the
// words for warps 0-3, the second half for warps 4-7).  The word tables of
// nds_chunks are staged in shared memory; for each word and objective a lane
// finds the count of dominator keys <= its own key with a six-probe search
// and ANDs the prefix set of that count into its row word, so a word of 32
// pairs costs about 13 integer operations per objective instead of 32
// comparisons.  Words are transposed through shared memory and written as
// coalesced row segments.  The epilogue raises blocker[q] to the highest
// dominator position seen, so that after the kernel blocker[q] == -1 exactly
// for the points that nothing dominates (front 0).
template <int M>
__global__ void __launch_bounds__(kTileThreads)
nds_tiles(const float* __restrict__ sf, int sf_stride, const int* __restrict__ qinfo,
          const uint32_t* __restrict__ ckeys, const uint32_t* __restrict__ cbits, int n, int W,
          int Wc, uint32_t* __restrict__ rows, int* __restrict__ blocker)
{
    constexpr int PW = TileCfg<M>::kPW;
    constexpr int MF = TileCfg<M>::kMF;
    const int q0 = blockIdx.y * kQB;
    if (q0 >= n) return;
    const int qend = min(q0 + kQB, n);
    // dominators of the block lie at positions < qend - 1
    const int nwords = (qend - 1 + 31) >> 5;
    const int w0 = blockIdx.x * PW;
    if (w0 >= nwords) return;
    const int wcount = min(PW, nwords - w0);

    __shared__ uint32_t s_key[MF][PW * 32];
    __shared__ uint32_t s_bits[MF][PW * 33];
    __shared__ uint32_t so[kQB][PW + 1];
    if (M > 1) {
        for (int t = threadIdx.x; t < wcount * 32; t += kTileThreads) {
#pragma unroll
            for (int m = 0; m < MF; ++m) s_key[m][t] = ckeys[(size_t)m * Wc * 32 + (size_t)w0 * 32 + t];
        }
        for (int t = threadIdx.x; t < wcount * 33; t += kTileThreads) {
#pragma unroll
            for (int m = 0; m < MF; ++m) s_bits[m][t] = cbits[(size_t)m * Wc * 33 + (size_t)w0 * 33 + t];
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ql = (warp & 3) * 32 + lane;
    const int q = q0 + ql;
    uint32_t qk[MF];
    int dup = 0;
    bool inf = false;
#pragma unroll
    for (int m = 0; m < MF; ++m) qk[m] = 0u;
    if (q < n) {
        if (M > 1) {
#pragma unroll
            for (int m = 0; m < MF; ++m) qk[m] = dom_key(sf[(size_t)m * sf_stride + q]);
        }
        const uint32_t info = (uint32_t)qinfo[q];
        inf = (info & kInfeasibleBit) != 0u;
        dup = (int)(info & ~kInfeasibleBit);
    }
    __syncthreads();

    constexpr int kHalf = PW / 2;
    const int wb = (warp >> 2) * kHalf;
    for (int wl = wb; wl < wb + kHalf; ++wl) {
        uint32_t bits = 0u;
        if (wl < wcount) {
            // positions p < dup[q] of this word
            const int rem = dup - (w0 + wl) * 32;
            const uint32_t mask = rem >= 32 ? 0xFFFFFFFFu : (rem <= 0 ? 0u : ((1u << rem) - 1u));
            const bool need = mask != 0u && !inf;
            if (M > 1 && __any_sync(0xFFFFFFFFu, need)) {
                uint32_t cmp = 0xFFFFFFFFu;
#pragma unroll
                for (int m = 0; m < MF; ++m) {
                    const uint32_t* sk = &s_key[m][wl * 32];
                    const uint32_t v = qk[m];
                    int k = 0;
                    k += (sk[k + 15] <= v) ? 16 : 0;
                    k += (sk[k + 7] <= v) ? 8 : 0;
                    k += (sk[k + 3] <= v) ? 4 : 0;
                    k += (sk[k + 1] <= v) ? 2 : 0;
                    k += (sk[k] <= v) ? 1 : 0;
                    k += (sk[k] <= v) ? 1 : 0;   // reaches 32 only from k == 31
                    cmp &= s_bits[m][wl * 33 + k];
                }
                bits = inf ? mask : (mask & cmp);
            } else {
                bits = (inf || M == 1) ? mask : 0u;
            }
        }
        so[ql][wl] = bits;
    }
    __syncthreads();
    for (int r = warp; r < kQB; r += kTileThreads / 32) {
        const int pos = q0 + r;
        if (pos >= n) break;
        const uint32_t word = (lane < wcount) ? so[r][lane] : 0u;
        if (lane < wcount) rows[(size_t)pos * W + w0 + lane] = word;
        const unsigned nz = __ballot_sync(0xFFFFFFFFu, word != 0u);
        if (nz && lane == 31 - __clz(nz))
            atomicMax(blocker + pos, (w0 + lane) * 32 + (31 - __clz(word)));
    }
}

// ---------------------------------------------------------------------------
// 3. front peeling
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier over co-resident CTAs.  Waits at most ~2 s, then records
// kDevBarrierTimeout in the status word and returns false.  The last CTA to
// arrive copies the front-list length (counters[1]) into counters[9] before
// releasing the others, so every CTA reads the same length after the barrier
// even when a fast CTA has already started appending the next front.
__device__ bool grid_barrier(int* counters, unsigned nblocks)
{
    __shared__ int s_ok;
    __syncthreads();
    if (nblocks == 1) {  // single-CTA peel: a block barrier suffices
        if (threadIdx.x == 0) counters[9] = atomicAdd(counters + 1, 0);
        __syncthreads();
        return true;
    }
    if (threadIdx.x == 0) {
        volatile int* vgen = counters + 5;
        volatile int* vstatus = counters + 6;
        const int g = *vgen;
        __threadfence();
        int ok = 1;
        if (atomicAdd(counters + 4, 1) == (int)nblocks - 1) {
            counters[9] = atomicAdd(counters + 1, 0);
            atomicExch(counters + 4, 0);
            __threadfence();
            atomicAdd(counters + 5, 1);
        } else {
            const unsigned long long t0 = global_ns();
            while (*vgen == g) {
                if (*vstatus != 0) { ok = 0; break; }
                if (global_ns() - t0 > 2000000000ull) {
                    atomicExch(counters + 6, kDevBarrierTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__global__ void __launch_bounds__(kPeelThreads)
nds_peel(const uint32_t* __restrict__ rows, int W, int n, int target, const int* __restrict__ qinfo,
         int* __restrict__ blocker, int* __restrict__ front_sorted, int* __restrict__ list,
         int* counters)
{
    extern __shared__ uint32_t U[];  // unassigned positions, one bit each
    __shared__ int s_len;
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        const int lo = w * 32;
        U[w] = (lo + 32 <= n) ? 0xFFFFFFFFu : (lo >= n ? 0u : ((1u << (n - lo)) - 1u));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int gwarp = blockIdx.x * wpb + warp;
    const int twarps = gridDim.x * wpb;
    const int ngroups = (n + 31) >> 5;
    int len_prev = 0, total = 0, k = 0;
    __syncthreads();

    for (;;) {
        for (int g = gwarp; g < ngroups; g += twarps) {
            const int q = g * 32 + lane;
            const bool alive = q < n && ((U[q >> 5] >> (q & 31)) & 1u);
            // blocker[q] is an unassigned dominator of q, or -1 when nothing dominates q
            bool is_free = false, need = false;
            int start_w = -1;
            if (alive) {
                const int b = blocker[q];
                if (b < 0) {
                    is_free = true;
                } else if (!((U[b >> 5] >> (b & 31)) & 1u)) {
                    // blocker assigned: probe its word and the one below; bits
                    // above it were already free of unassigned dominators
                    const uint32_t* row = rows + (size_t)q * W;
                    int w = b >> 5;
                    uint32_t bits = __ldg(row + w) & U[w];
                    if (!bits && w > 0) {
                        --w;
                        bits = __ldg(row + w) & U[w];
                    }
                    if (bits) {
                        blocker[q] = w * 32 + (31 - __clz(bits));
                    } else if (w == 0) {
                        is_free = true;
                    } else {
                        need = true;
                        start_w = w - 1;
                    }
                }
            }
            // rows not resolved by the probe: the whole warp scans each of
            // them downwards, 8 coalesced words per lane in flight
            unsigned needm = __ballot_sync(0xFFFFFFFFu, need);
            while (needm) {
                const int L = __ffs(needm) - 1;
                needm &= needm - 1;
                const int qL = g * 32 + L;
                const uint32_t* row = rows + (size_t)qL * W;
                const int sw = __shfl_sync(0xFFFFFFFFu, start_w, L);
                int found = -1;
                for (int w0 = sw; w0 >= 0 && found < 0; w0 -= 256) {
                    uint32_t acc[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int w = w0 - lane - 32 * i;
                        acc[i] = (w >= 0) ? (__ldg(row + w) & U[w]) : 0u;
                    }
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const unsigned nz = __ballot_sync(0xFFFFFFFFu, acc[i] != 0u);
                        if (nz) {
                            const int src = __ffs(nz) - 1;
                            const uint32_t bb = __shfl_sync(0xFFFFFFFFu, acc[i], src);
                            found = (w0 - src - 32 * i) * 32 + (31 - __clz(bb));
                            break;
                        }
                    }
                }
                if (lane == L) {
                    if (found >= 0) blocker[q] = found;
                    else is_free = true;
                }
            }
            const unsigned fm = __ballot_sync(0xFFFFFFFFu, is_free);
            if (fm) {
                int base = 0;
                if (lane == 0) base = atomicAdd(counters + 1, __popc(fm));
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (is_free) {
                    list[base + __popc(fm & ((1u << lane) - 1u))] = q;
                    front_sorted[q] = k;
                }
            }
        }
        if (!grid_barrier(counters, gridDim.x)) return;
        if (threadIdx.x == 0) s_len = *((volatile int*)counters + 9);
        __syncthreads();
        const int len = s_len;
        const int ck = len - len_prev;
        for (int i = threadIdx.x; i < ck; i += blockDim.x) {
            const int q = __ldcg(list + len_prev + i);
            atomicAnd(&U[q >> 5], ~(1u << (q & 31)));
        }
        __syncthreads();
        total += ck;
        len_prev = len;
        if (total >= target || ck == 0) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                counters[2] = k;
                counters[3] = total;
                if (ck == 0 && total < target) atomicExch(counters + 6, kDevPeelInconsistent);
            }
            return;
        }
        ++k;
    }
}

__global__ void nds_scatter_fronts(int n, const int* __restrict__ perm,
                                   const int* __restrict__ front_sorted, int* __restrict__ fronts)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos < n) fronts[perm[pos]] = front_sorted[pos];
}

__global__ void nds_reset_counters(int* counters)
{
    if (threadIdx.x < 4) counters[threadIdx.x] = 0;
    if (threadIdx.x == 4) counters[4] = 0;
}

template <int M>
void launch_tiles(const Workspace& ws, int n, cudaStream_t stream)
{
    const int nqb = ceil_div(n, kQB);
    const int maxw = ceil_div(n, 32);
    if (M > 1) {
        const int warps = maxw * (M - 1);
        nds_chunks<<<ceil_div(warps, 8), 256, 0, stream>>>(ws.sorted_f, ws.n_max, n, maxw, M - 1,
                                                         ws.chunk_keys, ws.chunk_bits);
    }
    dim3 grid(ceil_div(maxw, TileCfg<M>::kPW), nqb);
    nds_tiles<M><<<grid, kTileThreads, 0, stream>>>(ws.sorted_f, ws.n_max, ws.qinfo, ws.chunk_keys,
                                                     ws.chunk_bits, n, ws.words, maxw, ws.rows,
                                                     ws.blocker);
}

}  // namespace

size_t cub_temp_bytes_needed(int n_max)
{
    size_t a = 0, b = 0, c = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, a, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (int*)nullptr, (int*)nullptr, n_max);
    cub::DeviceRadixSort::SortPairs(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (int*)nullptr, (int*)nullptr, n_max);
    cub::DeviceScan::InclusiveScan(nullptr, c, (int*)nullptr, (int*)nullptr, cub::Max(), n_max);
    size_t m = a > b ? a : b;
    return m > c ? m : c;
}

int run_ndsort(Workspace& ws, const SplitPop& pop, int M, int target, int* out_fronts,
               cudaStream_t stream)
{
    const int n = pop.n;
    if (n <= 0) return MOEA_OK;
    if (n > ws.n_max || M < 1 || M > ws.m_max)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "ndsort: n=%d M=%d exceed the workspace (%d, %d)",
                         n, M, ws.n_max, ws.m_max);
    if (target > n) target = n;
    if (target < 1) target = 1;
    int* fronts = out_fronts ? out_fronts : ws.fronts;
    int* feas = ws.counters;
    const int T = 256, G = ceil_div(n, T);

    nds_reset_counters<<<1, 32, 0, stream>>>(ws.counters);
    nds_classify<<<G, T, 0, stream>>>(pop, M, ws.key0, ws.perm[0], feas);
    MOEA_CUDA_TRY(cudaGetLastError());
    const uint64_t* key0 = ws.key0;
    int cur = 0;
    size_t tmp = ws.cub_bytes;
    for (int m = M - 1; m >= 1; --m) {
        nds_gather_key<<<G, T, 0, stream>>>(pop, m, key0, ws.perm[cur], ws.key32[0]);
        MOEA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp, tmp, ws.key32[0], ws.key32[1],
                                                      ws.perm[cur], ws.perm[cur ^ 1], n, 0, 32,
                                                      stream));
        cur ^= 1;
    }
    nds_gather_key0<<<G, T, 0, stream>>>(n, key0, ws.perm[cur], ws.key64[0]);
    MOEA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp, tmp, ws.key64[0],
                                                  ws.key64[1], ws.perm[cur],
                                                  ws.perm[cur ^ 1], n, 0, 34, stream));
    cur ^= 1;
    const int* perm = ws.perm[cur];

    nds_sorted_soa<<<G, T, 0, stream>>>(pop, M, key0, perm, ws.sorted_f, ws.n_max, ws.head);
    MOEA_CUDA_TRY(cub::DeviceScan::InclusiveScan(ws.cub_tmp, tmp, ws.head, ws.run_start,
                                                 cub::Max(), n, stream));
    int* qinfo = ws.qinfo;
    nds_finalize_rows<<<G, T, 0, stream>>>(n, key0, perm, ws.run_start, feas, qinfo, ws.blocker,
                                           ws.front_sorted);
    MOEA_CUDA_TRY(cudaGetLastError());
    stage_mark("ndsort.lexsort", stream);

    switch (M) {
    case 1: launch_tiles<1>(ws, n, stream); break;
    case 2: launch_tiles<2>(ws, n, stream); break;
    case 3: launch_tiles<3>(ws, n, stream); break;
    case 4: launch_tiles<4>(ws, n, stream); break;
    case 5: launch_tiles<5>(ws, n, stream); break;
    case 6: launch_tiles<6>(ws, n, stream); break;
    case 7: launch_tiles<7>(ws, n, stream); break;
    case 8: launch_tiles<8>(ws, n, stream); break;
    case 9: launch_tiles<9>(ws, n, stream); break;
    case 10: launch_tiles<10>(ws, n, stream); break;
    case 11: launch_tiles<11>(ws, n, stream); break;
    case 12: launch_tiles<12>(ws, n, stream); break;
    case 13: launch_tiles<13>(ws, n, stream); break;
    case 14: launch_tiles<14>(ws, n, stream); break;
    case 15: launch_tiles<15>(ws, n, stream); break;
    case 16: launch_tiles<16>(ws, n, stream); break;
    default: return set_error(MOEA_ERR_UNSUPPORTED, "ndsort: M=%d", M);
    }
    MOEA_CUDA_TRY(cudaGetLastError());
    stage_mark("ndsort.dominance_tiles", stream);

    // cooperative peel
    const int W = ceil_div(n, 32);
    const int wpb = kPeelThreads / 32;
    int grid = ceil_div(ceil_div(n, 32), wpb);
    if (grid > ws.peel_grid) grid = ws.peel_grid;
    if (grid < 1 || ws.peel_single_cta) grid = 1;
    const uint32_t* rows = ws.rows;
    int Wp = ws.words;
    int nn = n, tt = target;
    const int* qi = qinfo;
    int* blk = ws.blocker;
    int* fs = ws.front_sorted;
    int* list = ws.front_list;
    int* ctr = ws.counters;
    (void)W;
    void* args[] = {(void*)&rows, (void*)&Wp, (void*)&nn, (void*)&tt, (void*)&qi,
                    (void*)&blk, (void*)&fs, (void*)&list, (void*)&ctr};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kPeelThreads);
    cfg.dynamicSmemBytes = (size_t)ws.words * sizeof(uint32_t);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (grid == 1) {
        // one CTA needs no co-residency guarantee: an ordinary launch, which
        // may run beside other work (batched instances)
        nds_peel<<<1, kPeelThreads, cfg.dynamicSmemBytes, stream>>>(rows, Wp, nn, tt, qi, blk, fs, list,
                                                                    ctr);
    } else {
        MOEA_CUDA_TRY(cudaLaunchKernelExC(&cfg, (const void*)nds_peel, args));
    }

    nds_scatter_fronts<<<G, T, 0, stream>>>(n, perm, ws.front_sorted, fronts);
    MOEA_CUDA_TRY(cudaGetLastError());
    stage_mark("ndsort.peel", stream);
    return MOEA_OK;
}

// Configure the co-resident grid of the peel kernel for this device.
int configure_peel(Workspace& ws)
{
    const size_t smem = (size_t)ws.words * sizeof(uint32_t);
    if (smem > 48 * 1024)
        MOEA_CUDA_TRY(cudaFuncSetAttribute(nds_peel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
    int per_sm = 0;
    MOEA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, nds_peel, kPeelThreads,
                                                                smem));
    int sms = 0;
    MOEA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws.device));
    if (per_sm < 1)
        return set_error(MOEA_ERR_UNSUPPORTED, "peel kernel does not fit on an SM (smem %zu)", smem);
    ws.peel_grid = sms * (per_sm > 2 ? 2 : per_sm);
    ws.peel_smem = (int)smem;
    return MOEA_OK;
}

}  // namespace moea
