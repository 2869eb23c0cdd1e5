// Constraint-dominance non-dominated sorting for sm_100a.
//
// Replaces run_ndsort / run_ndsort_init and the COO / CSR / bitmask paths of
// CUDA-MOEA (nat/src/selection/nsga3/kernels/non_dominated_sort.cu:158-1574).
// Same result (front index per point, -1 past the stop rule, index of the last
// front), different mechanism:
//
//  1. Sort of the points by (class, f0 | cv, S) with one 56-bit radix sort,
//     S the top 22 bits of the order key of the FP32 sum f1 + ... + f_{M-1}.
//     Class 0 = feasible, 1 = feasible with a NaN objective, 2 = infeasible,
//     3 = infeasible with NaN violation.  FP32 addition rounds monotonically,
//     so a feasible dominator p of q has f0(p) <= f0(q) and S(p) <= S(q); runs
//     of equal keys in class 0 are then ordered lexicographically by
//     (f1, ..., f_{M-1}, index) (nds_tie_fix, nds_tie_fix_long).  In this
//     order every dominator of a point lies strictly before it, identical
//     vectors are adjacent, and a feasible dominator already satisfies
//     f0 <= q0.
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
#include <algorithm>

#include <cub/cub.cuh>

#include "internal.cuh"

namespace moea {
namespace {

constexpr int kQB = 128;      // sorted positions (dominatees) per tile CTA
constexpr int kTileThreads = 256;
constexpr int kPeelThreads = 1024;
constexpr int kScanQueue = 1024;   // rows per CTA and front for the chunked scan
constexpr int kProbeWords = 16;    // row words probed below an assigned blocker
constexpr int kScanChunk = 512;    // words per chunk (16 per lane)
constexpr uint32_t kInfeasibleBit = 0x80000000u;
// Sort key: class (2 bits), the order key of f0 or of the violation (32
// bits), the top kSortSBits bits of the order key of S.  22 bits of S keep
// runs of equal keys as rare as 30 did while saving a radix pass; with 14
// the runs grew and the tie fix-up cost more than the pass it saved.
constexpr int kSortSBits = 22;
constexpr int kSortKeyBits = 2 + 32 + kSortSBits;
constexpr int kSortClassShift = 32 + kSortSBits;

// ---------------------------------------------------------------------------
// 1. classification and lexicographic sort
// ---------------------------------------------------------------------------

// Sort key of point i of class cls with key0 low word val: class << 54 |
// val << 22 | S (class 0), kSortKeyBits bits (seven radix passes of 8 bits),
// S the top 22 bits of the order key of the FP32 sum f1 + ... + f_{M-1}
// (monotone in every f_m; +inf + -inf (NaN) sorts with +inf sums).
__device__ __forceinline__ uint64_t sort_key(const SplitPop& pop, int M, int i, uint32_t cls, uint32_t val)
{
    uint32_t s30 = 0;
    if (cls == 0u) {
        float sum = 0.0f;
        for (int m = 1; m < M; ++m) sum = __fadd_rn(sum, pop.obj(m, i));
        s30 = float_order_key(isnan(sum) ? INFINITY : sum) >> 2;
    }
    return ((uint64_t)cls << kSortClassShift) | ((uint64_t)val << kSortSBits) | (s30 >> (30 - kSortSBits));
}

// key0[i] = class << 32 | order key of f0 (class 0) or cv (class 2);
// skey[i] = sort_key(i).
__global__ void nds_classify(SplitPop pop, int M, uint64_t* __restrict__ key0, uint64_t* __restrict__ skey,
                             int* __restrict__ perm, int* __restrict__ feasible_count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool feasible_class = false, infeasible2 = false, infeasible3 = false;
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
        skey[i] = sort_key(pop, M, i, cls, val);
        perm[i] = i;
        feasible_class = cls <= 1u;
        infeasible2 = cls == 2u;
        infeasible3 = cls == 3u;
    }
    const unsigned fm = __ballot_sync(0xFFFFFFFFu, feasible_class);
    const unsigned m2 = __ballot_sync(0xFFFFFFFFu, infeasible2);
    const unsigned m3 = __ballot_sync(0xFFFFFFFFu, infeasible3);
    if ((threadIdx.x & 31) == 0) {
        if (fm) atomicAdd(feasible_count, __popc(fm));
        if (m2) atomicAdd(feasible_count + 10, __popc(m2));
        if (m3) atomicAdd(feasible_count + 11, __popc(m3));
    }
}

// Total order inside a run of equal sort keys of class 0: lexicographic on
// the order keys of f1 .. f_{M-1}, then the point index.
__device__ __forceinline__ bool tie_less(const SplitPop& pop, int M, int a, int b)
{
    for (int m = 1; m < M; ++m) {
        const uint32_t ka = float_order_key(pop.obj(m, a)), kb = float_order_key(pop.obj(m, b));
        if (ka != kb) return ka < kb;
    }
    return a < b;
}

constexpr int kTieShort = 32;         // runs up to this length: one thread, insertion sort
constexpr int kTieLongThreads = 1024;
constexpr int kTieLongCtas = 64;        // CTAs of nds_tie_fix_long, each taking runs in turn
constexpr int kTieSmemSort = 4096;    // longer runs: bitonic in shared memory up to this size

// One thread per run head of class 0: short runs are sorted in place, longer
// ones are listed for nds_tie_fix_long.  Runs are disjoint, so the in-place
// sorts do not race.
__global__ void nds_tie_fix(SplitPop pop, int M, const uint64_t* __restrict__ skey, int* __restrict__ perm,
                            int* __restrict__ long_runs, int* __restrict__ n_long)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = pop.n;
    if (pos >= n) return;
    const uint64_t k = skey[pos];
    if ((k >> kSortClassShift) != 0u || (pos > 0 && skey[pos - 1] == k)) return;
    int L = 1;
    while (L <= kTieShort && pos + L < n && skey[pos + L] == k) ++L;
    if (L == 1) return;
    if (L > kTieShort) {
        long_runs[atomicAdd(n_long, 1)] = pos;
        return;
    }
    int* a = perm + pos;
    for (int x = 1; x < L; ++x) {
        const int v = a[x];
        int y = x - 1;
        while (y >= 0 && tie_less(pop, M, v, a[y])) {
            a[y + 1] = a[y];
            --y;
        }
        a[y + 1] = v;
    }
}

// Ascending bitonic network over a[0, L) with virtual +inf padding to the
// power of two P >= L (pairs reaching past L are skipped: +inf already sits
// last).  Every merge opens with the mirrored comparison, so all blocks sort
// ascending.  Called by every thread of the CTA.
__device__ void tie_bitonic(const SplitPop& pop, int M, int* a, int L)
{
    int P = 1;
    while (P < L) P <<= 1;
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int q = threadIdx.x; q < P / 2; q += blockDim.x) {
                int i, p;
                if (j == k >> 1) {  // mirror inside the block of k
                    const int half = k >> 1;
                    i = (q / half) * k + (q % half);
                    p = (q / half) * k + (k - 1 - (q % half));
                } else {
                    i = (q / j) * 2 * j + (q % j);
                    p = i + j;
                }
                if (p < L) {
                    const int x = a[i], y = a[p];
                    if (tie_less(pop, M, y, x)) {
                        a[i] = y;
                        a[p] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// One CTA per listed run longer than kTieShort: its length, then a bitonic
// sort unless the run is already in order (runs of identical vectors are).
__global__ void __launch_bounds__(kTieLongThreads)
nds_tie_fix_long(SplitPop pop, int M, const uint64_t* __restrict__ skey, int* __restrict__ perm,
                 const int* __restrict__ long_runs, const int* __restrict__ n_long)
{
    __shared__ int s_arr[kTieSmemSort];
    __shared__ int s_len, s_unsorted;
    const int n = pop.n;
    const int count = *n_long;
    for (int r = blockIdx.x; r < count; r += gridDim.x) {
        const int start = long_runs[r];
        const uint64_t k = skey[start];
        if (threadIdx.x == 0) {
            s_len = n - start;
            s_unsorted = 0;
        }
        __syncthreads();
        for (int base = start; base < n; base += blockDim.x) {
            const int pos = base + threadIdx.x;
            if (pos < n && skey[pos] != k) atomicMin(&s_len, pos - start);
            __syncthreads();
            const bool found = s_len < n - start;
            __syncthreads();  // every thread has read s_len before the next atomicMin
            if (found) break;
        }
        const int L = s_len;
        int* a = perm + start;
        for (int x = threadIdx.x; x + 1 < L; x += blockDim.x)
            if (tie_less(pop, M, a[x + 1], a[x])) s_unsorted = 1;
        __syncthreads();
        if (s_unsorted) {
            if (L <= kTieSmemSort) {
                for (int x = threadIdx.x; x < L; x += blockDim.x) s_arr[x] = a[x];
                __syncthreads();
                tie_bitonic(pop, M, s_arr, L);
                for (int x = threadIdx.x; x < L; x += blockDim.x) a[x] = s_arr[x];
            } else {
                tie_bitonic(pop, M, a, L);
            }
        }
        __syncthreads();
    }
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
__device__ __forceinline__ void chunk_warp(int gw, int lane, const float* __restrict__ sf, int sf_stride,
                                           int n, int W, uint32_t* __restrict__ ckeys,
                                           uint32_t* __restrict__ cbits)
{
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

__global__ void nds_chunks(const float* __restrict__ sf, int sf_stride, int n, int W, int MF,
                           uint32_t* __restrict__ ckeys, uint32_t* __restrict__ cbits)
{
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (gw >= W * MF) return;
    chunk_warp(gw, threadIdx.x & 31, sf, sf_stride, n, W, ckeys, cbits);
}

// Dominator words per tile CTA (32 positions each), sized so that the staged
// word tables and the transposed output fit in 48 KB of shared memory.
template <int M>
struct TileCfg {
    static constexpr int kPW = (M <= 4) ? 32 : ((M <= 8) ? 16 : 8);
    static constexpr int kMF = (M > 1) ? M - 1 : 1;   // objectives 1..M-1
};

// Words per tile CTA of a tile shape: shape 0 is TileCfg's, shape 1 half of
// it (twice the CTAs, each with half the staged word tables).  The batch's
// autotuner picks the shape per objective count by measured time.
template <int M, int S>
struct TileShape {
    static constexpr int kPW = S == 0 ? TileCfg<M>::kPW : TileCfg<M>::kPW / 2;
};

// Count of the 32 ascending keys at shared address a that are <= v, as the
// byte offset 4 * count: binary search with steps of 16, 8, 4, 2, 1 keys and
// a last probe that reaches 32 only from 31.  Each probe is one shared load
// with an immediate offset, one compare and one predicated add.
__device__ __forceinline__ uint32_t word_count_bytes(uint32_t a, uint32_t v)
{
    const uint32_t a0 = a;
    asm("{\n\t.reg .pred p;\n\t.reg .u32 t;\n\t"
        "ld.shared.u32 t, [%0+60];\n\tsetp.le.u32 p, t, %1;\n\t@p add.u32 %0, %0, 64;\n\t"
        "ld.shared.u32 t, [%0+28];\n\tsetp.le.u32 p, t, %1;\n\t@p add.u32 %0, %0, 32;\n\t"
        "ld.shared.u32 t, [%0+12];\n\tsetp.le.u32 p, t, %1;\n\t@p add.u32 %0, %0, 16;\n\t"
        "ld.shared.u32 t, [%0+4];\n\tsetp.le.u32 p, t, %1;\n\t@p add.u32 %0, %0, 8;\n\t"
        "ld.shared.u32 t, [%0];\n\tsetp.le.u32 p, t, %1;\n\t@p add.u32 %0, %0, 4;\n\t"
        "ld.shared.u32 t, [%0];\n\tsetp.le.u32 p, t, %1;\n\t@p add.u32 %0, %0, 4;\n\t}"
        : "+r"(a)
        : "r"(v)
        : "memory");
    return a - a0;
}

__device__ __forceinline__ uint32_t ld_shared_u32(uint32_t a)
{
    uint32_t x;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(x) : "r"(a) : "memory");
    return x;
}

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
template <int M, int PW = TileCfg<M>::kPW>
__device__ __forceinline__ void tile_block(int bx, int by, const float* __restrict__ sf, int sf_stride,
                                           const int* __restrict__ qinfo,
                                           const uint32_t* __restrict__ ckeys,
                                           const uint32_t* __restrict__ cbits, int n, int W, int Wc,
                                           uint32_t* __restrict__ rows, int* __restrict__ blocker)
{
    constexpr int MF = TileCfg<M>::kMF;
    const int q0 = by * kQB;
    if (q0 >= n) return;
    const int qend = min(q0 + kQB, n);
    // dominators of the block lie at positions < qend - 1
    const int nwords = (qend - 1 + 31) >> 5;
    const int w0 = bx * PW;
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
    const int wend = min(wb + kHalf, wcount);
    // words whose 32 positions lie below dup[q] for every lane of the warp
    // need no dup mask (most of them)
    uint32_t key_addr[MF], bits_addr[MF];
#pragma unroll
    for (int m = 0; m < MF; ++m) {
        key_addr[m] = (uint32_t)__cvta_generic_to_shared(&s_key[m][0]);
        bits_addr[m] = (uint32_t)__cvta_generic_to_shared(&s_bits[m][0]);
    }
    const int lane_full = (q < n) ? (dup >> 5) - w0 : 0x7FFFFFFF;
    const int wfull = min(wend, max(wb, __reduce_min_sync(0xFFFFFFFFu, lane_full)));
    // Every lane searches (the masks decide).  The prefix set of count c
    // sits at byte 4 c of the word's bit table.  Running shared addresses
    // step by one word table per iteration.
#pragma unroll
    for (int m = 0; m < MF; ++m) {
        key_addr[m] += (uint32_t)wb * 128u;
        bits_addr[m] += (uint32_t)wb * 132u;
    }
    uint32_t* so_row = &so[ql][0];
    const uint32_t infm = inf ? 0xFFFFFFFFu : 0u;
    auto word_bits = [&]() -> uint32_t {
        uint32_t cmp = 0xFFFFFFFFu;
        if (M > 1) {
#pragma unroll
            for (int m = 0; m < MF; ++m) {
                const uint32_t off = word_count_bytes(key_addr[m], qk[m]);
                cmp &= ld_shared_u32(bits_addr[m] + off);
                key_addr[m] += 128u;
                bits_addr[m] += 132u;
            }
        }
        return cmp | infm;
    };
    // The peel never reaches an infeasible point (each is dominated by every
    // feasible one, and the peel ends with the feasible fronts), so its row is
    // never read: a warp of infeasible q (they sort last, so whole warps are)
    // computes nothing, and a CTA of them stores nothing.  Rows of infeasible
    // q in a mixed CTA hold unspecified words.
    const bool all_inf = __all_sync(0xFFFFFFFFu, inf || q >= n);
    if (!all_inf) {
        int wl = wb;
        for (; wl < wfull; ++wl) so_row[wl] = word_bits();   // all positions below dup[q]
        for (; wl < wend; ++wl) {
            // positions p < dup[q] of this word
            const int rem = dup - (w0 + wl) * 32;
            const uint32_t mask = rem >= 32 ? 0xFFFFFFFFu : (rem <= 0 ? 0u : ((1u << rem) - 1u));
            so_row[wl] = mask & word_bits();
        }
    }
    if (__syncthreads_and(all_inf)) return;
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

template <int M>
__global__ void __launch_bounds__(kTileThreads)
nds_tiles(const float* __restrict__ sf, int sf_stride, const int* __restrict__ qinfo,
          const uint32_t* __restrict__ ckeys, const uint32_t* __restrict__ cbits, int n, int W,
          int Wc, uint32_t* __restrict__ rows, int* __restrict__ blocker)
{
    tile_block<M>(blockIdx.x, blockIdx.y, sf, sf_stride, qinfo, ckeys, cbits, n, W, Wc, rows, blocker);
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

__device__ __forceinline__ int ld_acquire_gpu(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier over co-resident CTAs.  The arrivals count up during one
// launch (counters[4] is zeroed before it): barrier number `epoch` is passed
// when the count reaches epoch * nblocks, so no CTA resets or releases
// anything and the wait ends one acquire load after the last arrival.
// Waits at most limit_ns (2 s in the peel), then records kDevBarrierTimeout
// in the status word and returns false.  Every thread of the CTA passes the
// same epoch.
__device__ bool grid_barrier(int* counters, unsigned nblocks, int epoch,
                             unsigned long long limit_ns = 2000000000ull)
{
    __shared__ int s_ok;
    __syncthreads();
    if (nblocks == 1) {  // single-CTA peel: a block barrier suffices
        __syncthreads();
        return true;
    }
    if (threadIdx.x == 0) {
        const int target = epoch * (int)nblocks;
        // release at GPU scope: with the CTA barrier above it orders every
        // thread's earlier writes before the arrival
        asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(counters + 4) : "memory");
        int ok = 1;
        const unsigned long long t0 = global_ns();
        while (ld_acquire_gpu(counters + 4) < target) {
            if (*((volatile int*)counters + 6) != 0) { ok = 0; break; }
            if (global_ns() - t0 > limit_ns) {
                atomicExch(counters + 6, kDevBarrierTimeout);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Marks the free lanes of a warp, all in the 32-position group of word gw,
// as members of front k: one atomicOr into the front's mask per warp.
__device__ __forceinline__ void peel_mark_group(bool is_free, int q, int gw, int k, int lane, uint32_t* G,
                                                int* front_sorted)
{
    const unsigned fm = __ballot_sync(0xFFFFFFFFu, is_free);
    if (!fm) return;
    if (lane == 0) atomicOr(G + gw, fm);
    if (is_free) front_sorted[q] = k;
}

// Body of the peel, run by CTA `block` of `nblocks` co-resident CTAs; U is the
// CTA's bitmask of unassigned positions (W words of shared memory), the same
// in every CTA.  Per front k:
//   1. groups: every alive point whose blocker (an unassigned dominator) was
//      assigned probes the blocker's row word and the one below; a hit is the
//      new blocker, no dominator at all makes the point free, and the other
//      rows are queued;
//   2. the CTA scans its queued rows in chunks of kScanChunk words, level by
//      level (the top chunk of every row first);
//   3. free points set their bit in the front's mask (fmask, three in
//      rotation, so no CTA appends to a shared list); after one grid barrier
//      every CTA removes the front from U and counts it.
template <int kInflight>
__device__ __forceinline__ void peel_body(int block, int nblocks, uint32_t* U,
                                          const uint32_t* __restrict__ rows, int W, int n, int target,
                                          const int* __restrict__ qinfo, int* __restrict__ blocker,
                                          int* __restrict__ front_sorted, uint32_t* __restrict__ fmask,
                                          int* counters)
{
    __shared__ int s_nscan, s_ntask;
    __shared__ int s_sq[kScanQueue], s_sw[kScanQueue], s_found[kScanQueue];
    __shared__ int s_wsum[32];
    if (threadIdx.x == 0) s_nscan = 0;
    // Feasible positions come first in the sorted order.  Infeasible ones are
    // never assigned here (each is dominated by every feasible point, and the
    // peel ends with the feasible fronts or the target), so they start out of
    // the unassigned set: they are never examined and their rows never read.
    const int nf = min(n, counters[0]);
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        const int lo = w * 32;
        U[w] = (lo + 32 <= nf) ? 0xFFFFFFFFu : (lo >= nf ? 0u : ((1u << (nf - lo)) - 1u));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    // groups of 32 positions interleaved over the CTAs: every CTA holds low
    // (short rows) and high (long rows) positions alike
    const int gwarp = warp * nblocks + block;
    const int twarps = nblocks * wpb;
    const int ngroups = (n + 31) >> 5;
    int total = 0, k = 0, epoch = 0;
    // With fewer feasible points than the target, the peel covers the
    // feasible fronts only; the infeasible fronts follow in closed form
    // (nds_infeasible_fronts).  Without feasible points there is nothing to peel.
    const int feasible = counters[0];
    const bool feasible_only = feasible < target;
    __syncthreads();
    if (feasible_only && feasible == 0) {
        if (block == 0 && threadIdx.x == 0) {
            counters[2] = -1;
            counters[12] = -1;
        }
        return;
    }

    for (;;) {
        uint32_t* G = fmask + (size_t)(k % 3) * W;  // members of front k
        // the mask front k + 1 will write: last read (as front k - 2's) before
        // the barrier of front k - 1, written again only after this front's
        const uint32_t nextw = (uint32_t)((k + 1) % 3);
        for (int w = block * blockDim.x + threadIdx.x; w < W; w += nblocks * blockDim.x)
            fmask[(size_t)nextw * W + w] = 0u;
        for (int g0 = gwarp; g0 < ngroups; g0 += twarps * kInflight) {
            int qv[kInflight], bv[kInflight];
            uint32_t pw[kInflight][kProbeWords];
            bool alive[kInflight], probe[kInflight];
#pragma unroll
            for (int u = 0; u < kInflight; ++u) {
                const int g = g0 + u * twarps;
                const int q = g * 32 + lane;
                qv[u] = q;
                alive[u] = g < ngroups && q < n && ((U[q >> 5] >> (q & 31)) & 1u);
                // blocker[q] is an unassigned dominator of q, or -1 when nothing
                // dominates q; whichever CTA resolved q's row wrote it: read through L2
                bv[u] = alive[u] ? __ldcg(blocker + q) : -1;
            }
#pragma unroll
            for (int u = 0; u < kInflight; ++u) {
                const int b = bv[u];
                // blocker assigned: probe its word and the kProbeWords - 1
                // below it; bits above it were already free of unassigned
                // dominators
                probe[u] = alive[u] && b >= 0 && !((U[b >> 5] >> (b & 31)) & 1u);
#pragma unroll
                for (int i = 0; i < kProbeWords; ++i) pw[u][i] = 0u;
                if (probe[u]) {
                    const uint32_t* row = rows + (size_t)qv[u] * W;
                    const int w = b >> 5;
#pragma unroll
                    for (int i = 0; i < kProbeWords; ++i)
                        if (w - i >= 0) pw[u][i] = __ldg(row + w - i);
                }
            }
#pragma unroll
            for (int u = 0; u < kInflight; ++u) {
                const int g = g0 + u * twarps;
                if (g >= ngroups) break;  // warp-uniform
                const int q = qv[u];
                bool is_free = false, need = false;
                int start_w = -1;
                if (alive[u]) {
                    const int b = bv[u];
                    if (b < 0) {
                        is_free = true;
                    } else if (probe[u]) {
                        const int w = b >> 5;
                        int hit = -1;
#pragma unroll
                        for (int i = 0; i < kProbeWords; ++i) {
                            const uint32_t bits = (w - i >= 0) ? (pw[u][i] & U[w - i]) : 0u;
                            if (hit < 0 && bits) hit = (w - i) * 32 + (31 - __clz(bits));
                        }
                        if (hit >= 0) {
                            blocker[q] = hit;
                        } else if (w - kProbeWords < 0) {
                            is_free = true;
                        } else {
                            need = true;
                            start_w = w - kProbeWords;
                        }
                    }
                }
                // rows not resolved by the probe go to the CTA's list; when it
                // is full the whole warp scans each of them downwards
                if (need) {
                    const int slot = atomicAdd(&s_nscan, 1);
                    if (slot < kScanQueue) {
                        s_sq[slot] = qv[u];
                        s_sw[slot] = start_w;
                        need = false;
                    }
                }
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
                peel_mark_group(is_free, q, g, k, lane, G, front_sorted);
            }
        }
        __syncthreads();
        const int nscan = min(s_nscan, kScanQueue);
        if (nscan > 0) {
            // chunks of the queued rows: row s covers words sw[s]..0 in
            // chunks of kScanChunk from the top.  Tasks go level by level (the
            // top chunk of every row first), and a chunk is skipped once an
            // unassigned dominator above it has been found: the highest one
            // found is the same, and most rows end in their top chunk.  A hit
            // found lower down (a later chunk can finish first) skips nothing.
            if (warp == 0) {
                int levels = 0;
                for (int s0 = 0; s0 < nscan; s0 += 32) {
                    const int sidx = s0 + lane;
                    if (sidx < nscan) {
                        levels = max(levels, s_sw[sidx] / kScanChunk + 1);
                        s_found[sidx] = -1;
                    }
                }
#pragma unroll
                for (int o = 16; o; o >>= 1) levels = max(levels, __shfl_xor_sync(0xFFFFFFFFu, levels, o));
                if (lane == 0) s_ntask = levels * nscan;
            }
            __syncthreads();
            const int ntask = s_ntask;
            for (int task = warp; task < ntask; task += wpb) {
                const int level = task / nscan, lo = task - level * nscan;
                if (level > s_sw[lo] / kScanChunk) continue;
                const int top = s_sw[lo] - level * kScanChunk;
                // warp-uniform: the chunk scan below is warp-collective
                const int found_hi = __shfl_sync(0xFFFFFFFFu, *((volatile int*)s_found + lo), 0);
                if (found_hi > top * 32 + 31) continue;
                const uint32_t* row = rows + (size_t)s_sq[lo] * W;
                uint32_t acc[kScanChunk / 32];
#pragma unroll
                for (int i = 0; i < kScanChunk / 32; ++i) {
                    const int w = top - lane - 32 * i;
                    acc[i] = (w >= 0 && w > top - kScanChunk) ? (__ldg(row + w) & U[w]) : 0u;
                }
#pragma unroll
                for (int i = 0; i < kScanChunk / 32; ++i) {
                    const unsigned nz = __ballot_sync(0xFFFFFFFFu, acc[i] != 0u);
                    if (nz) {
                        const int src = __ffs(nz) - 1;
                        const uint32_t bb = __shfl_sync(0xFFFFFFFFu, acc[i], src);
                        if (lane == 0) atomicMax(s_found + lo, (top - src - 32 * i) * 32 + (31 - __clz(bb)));
                        break;
                    }
                }
            }
            __syncthreads();
            // highest unassigned dominator found: new blocker; none: free
            for (int s0 = 0; s0 < nscan; s0 += blockDim.x) {
                const int sidx = s0 + threadIdx.x;
                bool is_free = false;
                int q = 0;
                if (sidx < nscan) {
                    q = s_sq[sidx];
                    const int f = s_found[sidx];
                    if (f >= 0) blocker[q] = f;
                    else is_free = true;
                }
                if (is_free) {
                    atomicOr(G + (q >> 5), 1u << (q & 31));
                    front_sorted[q] = k;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_nscan = 0;  // read again only after the barrier below
        if (!grid_barrier(counters, (unsigned)nblocks, ++epoch)) return;
        // front k is complete: remove it from U and count it
        int c = 0;
        for (int w0 = threadIdx.x; w0 < W; w0 += 4 * blockDim.x) {
            uint32_t g[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int w = w0 + i * blockDim.x;
                g[i] = (w < W) ? __ldcg(G + w) : 0u;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (g[i]) {
                    U[w0 + i * blockDim.x] &= ~g[i];
                    c += __popc(g[i]);
                }
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
        if (lane == 0) s_wsum[warp] = c;
        __syncthreads();
        int ck = 0;
        for (int w = 0; w < wpb; ++w) ck += s_wsum[w];
        __syncthreads();  // s_wsum is reused by the next front
        total += ck;
        if (total >= target || ck == 0 || (feasible_only && total >= feasible)) {
            if (block == 0 && threadIdx.x == 0) {
                counters[2] = k;
                counters[3] = total;
                counters[12] = k;
                if (ck == 0 && total < (feasible_only ? feasible : target))
                    atomicExch(counters + 6, kDevPeelInconsistent);
            }
            return;
        }
        ++k;
    }
}

__global__ void __launch_bounds__(kPeelThreads, 1)
nds_peel(const uint32_t* __restrict__ rows, int W, int n, int target, const int* __restrict__ qinfo,
         int* __restrict__ blocker, int* __restrict__ front_sorted, uint32_t* __restrict__ fmask,
         int* counters)
{
    extern __shared__ uint32_t U[];  // unassigned positions, one bit each
    peel_body<1>(blockIdx.x, gridDim.x, U, rows, W, n, target, qinfo, blocker, front_sorted, fmask, counters);
}

// ---- peel with lane-owned points ------------------------------------------
//
// When every warp of the grid owns at most one group of 32 positions
// (n <= 32 * 32 * CTAs), a lane keeps its point's state across the fronts:
// the blocker in a register and a window of at least kWin row words (the
// blocker's word and those below it) in shared memory, as three aligned
// 16-byte chunks.  The window is refilled with cp.async whenever fewer than
// kWin of its words lie at or below the blocker, so the copy lands while the
// grid waits at the barrier and the next front's probe reads only shared
// memory.  Row strides are multiples of four words (the workspace rounds
// them), which keeps every chunk 16-byte aligned.  Rows the window cannot settle go through the CTA's
// level-ordered scan as in peel_body.  The barrier carries the front sizes:
// a CTA adds (1 << 32) + (its free points) to one of two 64-bit words (front
// parity), so the front's size arrives with the barrier and no block-wide
// count is needed.  A CTA can run at most one front ahead of the slowest, so
// the word of front k holds only fronts k, k-2, ... when it is read.

constexpr int kWin = 8;        // row words cached per lane at and below its blocker
constexpr int kWinChunks = 3;  // 16-byte chunks of a window: 12 words from a multiple of 4
constexpr unsigned long long kPeelWaitNs = 2000000000ull;  // limit of one barrier wait

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(uint4* dst, const uint32_t* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Row words wlo .. wt of `row` into a lane's window (chunk stride
// kPeelThreads), wlo = wt - kWin + 1 rounded down to a multiple of 4; chunks
// below word 0 read as empty, chunks above wt are not copied.  Returns wlo.
__device__ __forceinline__ int window_fill(uint4* win, const uint32_t* row, int wt)
{
    const int wlo = (wt - (kWin - 1)) & ~3;
#pragma unroll
    for (int c = 0; c < kWinChunks; ++c) {
        const int w0 = wlo + 4 * c;
        if (w0 > wt) break;
        if (w0 >= 0) cp_async16(win + c * kPeelThreads, row + w0);
        else win[c * kPeelThreads] = make_uint4(0u, 0u, 0u, 0u);
    }
    return wlo;
}

// Arrival at a front barrier that also sums the fronts' sizes: adds
// (1 << 32) + count to *word and waits until the high half reaches `need`.
// Returns the word's value, or ~0 after `limit_ns` (status kDevBarrierTimeout)
// or when another CTA has failed.  Thread 0 only.
__device__ unsigned long long counted_arrive(unsigned long long* word, unsigned count, unsigned long long need,
                                             int* status, unsigned long long limit_ns)
{
    const unsigned long long add = (1ull << 32) | count;
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(word), "l"(add) : "memory");
    const unsigned long long t0 = global_ns();
    for (;;) {
        unsigned long long v;
        asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(word) : "memory");
        if ((v >> 32) >= need) return v;
        if (*((volatile int*)status) != 0) return ~0ull;
        if (global_ns() - t0 > limit_ns) {
            atomicExch(status, kDevBarrierTimeout);
            return ~0ull;
        }
        __nanosleep(32);
    }
}

__global__ void __launch_bounds__(kPeelThreads, 1)
nds_peel_owned(const uint32_t* __restrict__ rows, int W, int n, int target, const int* __restrict__ blocker0,
               int* __restrict__ front_sorted, uint32_t* __restrict__ fmask, int* counters)
{
    extern __shared__ uint32_t smem[];
    uint32_t* U = smem;                              // unassigned positions, one bit each
    uint4* s_win = reinterpret_cast<uint4*>(smem + ((W + 3) & ~3));  // [kWinChunks][kPeelThreads]
    __shared__ int s_nscan, s_ntask, s_cnt, s_ok, s_ck, s_total;
    __shared__ int s_sq[kScanQueue], s_sw[kScanQueue], s_found[kScanQueue];
    static_assert(kScanQueue >= kPeelThreads, "every owned point must fit the scan queue");
    const int nblocks = gridDim.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int nf = min(n, counters[0]);
    const int feasible = counters[0];
    const bool feasible_only = feasible < target;
    // feasible positions come first; infeasible ones never enter U (peel_body)
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        const int lo = w * 32;
        U[w] = (lo + 32 <= nf) ? 0xFFFFFFFFu : (lo >= nf ? 0u : ((1u << (nf - lo)) - 1u));
    }
    if (threadIdx.x == 0) {
        s_nscan = 0;
        s_cnt = 0;
    }
    // this lane's point: group g = warp * nblocks + blockIdx.x (interleaved,
    // like peel_body), at most one per warp
    const int g = warp * nblocks + blockIdx.x;
    const int q = g * 32 + lane;
    bool alive = q < nf;
    int b = -1, wlo = 0;
    uint4* win = s_win + threadIdx.x;
    const uint32_t* row = rows + (size_t)(alive ? q : 0) * W;
    if (alive) {
        b = blocker0[q];
        if (b >= 0) wlo = window_fill(win, row, b >> 5);
    }
    cp_async_commit();
    __syncthreads();
    if (feasible_only && feasible == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            counters[2] = -1;
            counters[12] = -1;
        }
        cp_async_wait_all();
        return;
    }
    unsigned long long* sizes = reinterpret_cast<unsigned long long*>(counters + 16);
    unsigned cum_even = 0u, cum_odd = 0u;  // thread 0: summed sizes of the even and odd fronts
    int k = 0;
    for (;;) {
        uint32_t* G = fmask + (size_t)(k % 3) * W;  // members of front k
        const uint32_t nextw = (uint32_t)((k + 1) % 3);
        for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += nblocks * blockDim.x)
            fmask[(size_t)nextw * W + w] = 0u;
        cp_async_wait_all();
        // 1. probe: the window of a point whose blocker was assigned
        bool is_free = false;
        int slot = -1;
        if (alive) {
            if (b < 0) {
                is_free = true;
            } else if (!((U[b >> 5] >> (b & 31)) & 1u)) {
                // the window's chunks from the top, each ANDed with the same
                // four words of U (16-byte shared loads, no data-dependent
                // branch); row words above the blocker's word are masked:
                // beyond q's own word they are not part of the row
                const int w = b >> 5;
                const int lo = max(wlo, 0);
                const uint4* U4 = reinterpret_cast<const uint4*>(U);
                int hit = -1;
#pragma unroll
                for (int c = kWinChunks - 1; c >= 0; --c) {
                    const int w0 = wlo + 4 * c;
                    if (w0 >= 0 && w0 <= w) {
                        const uint4 v = win[c * kPeelThreads];
                        const uint4 u = U4[w0 >> 2];
                        const uint32_t m[4] = {v.x & u.x, w0 + 1 <= w ? v.y & u.y : 0u,
                                               w0 + 2 <= w ? v.z & u.z : 0u, w0 + 3 <= w ? v.w & u.w : 0u};
#pragma unroll
                        for (int j = 3; j >= 0; --j)
                            if (hit < 0 && m[j]) hit = (w0 + j) * 32 + (31 - __clz(m[j]));
                    }
                }
                if (hit >= 0) {
                    b = hit;
                } else if (lo == 0) {
                    is_free = true;
                } else {
                    slot = atomicAdd(&s_nscan, 1);
                    s_sq[slot] = q;
                    s_sw[slot] = lo - 1;
                }
            }
        }
        __syncthreads();
        // 2. the CTA's level-ordered scans of the queued rows (peel_body)
        const int nscan = s_nscan;
        if (nscan > 0) {
            if (warp == 0) {
                int levels = 0;
                for (int s0 = 0; s0 < nscan; s0 += 32) {
                    const int sidx = s0 + lane;
                    if (sidx < nscan) {
                        levels = max(levels, s_sw[sidx] / kScanChunk + 1);
                        s_found[sidx] = -1;
                    }
                }
#pragma unroll
                for (int o = 16; o; o >>= 1) levels = max(levels, __shfl_xor_sync(0xFFFFFFFFu, levels, o));
                if (lane == 0) s_ntask = levels * nscan;
            }
            __syncthreads();
            const int ntask = s_ntask;
            for (int task = warp; task < ntask; task += wpb) {
                const int level = task / nscan, lo = task - level * nscan;
                if (level > s_sw[lo] / kScanChunk) continue;
                const int top = s_sw[lo] - level * kScanChunk;
                const int found_hi = __shfl_sync(0xFFFFFFFFu, *((volatile int*)s_found + lo), 0);
                if (found_hi > top * 32 + 31) continue;
                const uint32_t* srow = rows + (size_t)s_sq[lo] * W;
                uint32_t acc[kScanChunk / 32];
#pragma unroll
                for (int i = 0; i < kScanChunk / 32; ++i) {
                    const int w = top - lane - 32 * i;
                    acc[i] = (w >= 0 && w > top - kScanChunk) ? (__ldg(srow + w) & U[w]) : 0u;
                }
                // every loaded word is consumed (no load left in flight)
                int si = -1;
                unsigned snz = 0u;
                uint32_t sel = 0u;
#pragma unroll
                for (int i = 0; i < kScanChunk / 32; ++i) {
                    const unsigned nz = __ballot_sync(0xFFFFFFFFu, acc[i] != 0u);
                    if (si < 0 && nz) {
                        si = i;
                        snz = nz;
                        sel = acc[i];
                    }
                }
                if (si >= 0) {
                    const int src = __ffs(snz) - 1;
                    const uint32_t bb = __shfl_sync(0xFFFFFFFFu, sel, src);
                    if (lane == 0) atomicMax(s_found + lo, (top - src - 32 * si) * 32 + (31 - __clz(bb)));
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) s_nscan = 0;  // next written after two more CTA barriers
        }
        if (slot >= 0) {
            const int f = s_found[slot];
            if (f >= 0) b = f;
            else is_free = true;
        }
        // fewer than kWin window words at or below the blocker: refill the
        // window for the next front
        if (alive && !is_free && b >= 0 && (b >> 5) - wlo < kWin - 1) wlo = window_fill(win, row, b >> 5);
        cp_async_commit();
        // 3. members of front k: the front's mask and the CTA's count
        const unsigned fm = __ballot_sync(0xFFFFFFFFu, is_free);
        if (fm) {
            if (lane == 0) {
                atomicOr(G + g, fm);
                atomicAdd(&s_cnt, __popc(fm));
            }
            if (is_free) {
                front_sorted[q] = k;
                alive = false;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned long long v = counted_arrive(sizes + (k & 1), (unsigned)s_cnt,
                                                        (unsigned long long)(k / 2 + 1) * (unsigned)nblocks,
                                                        counters + 6, kPeelWaitNs);
            s_cnt = 0;
            s_ok = v != ~0ull;
            if (s_ok) {
                const unsigned c = (unsigned)v;
                if (k & 1) {
                    s_ck = (int)(c - cum_odd);
                    cum_odd = c;
                } else {
                    s_ck = (int)(c - cum_even);
                    cum_even = c;
                }
                s_total = (int)(cum_even + cum_odd);
            }
        }
        __syncthreads();
        if (!s_ok) {
            cp_async_wait_all();
            return;
        }
        // front k is complete: remove it from U
        for (int w = threadIdx.x; w < W; w += blockDim.x) {
            const uint32_t gv = __ldcg(G + w);
            if (gv) U[w] &= ~gv;
        }
        __syncthreads();
        const int ck = s_ck, total = s_total;
        if (total >= target || ck == 0 || (feasible_only && total >= feasible)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                counters[2] = k;
                counters[3] = total;
                counters[12] = k;
                if (ck == 0 && total < (feasible_only ? feasible : target))
                    atomicExch(counters + 6, kDevPeelInconsistent);
            }
            cp_async_wait_all();
            return;
        }
        ++k;
    }
}

// Shared memory of nds_peel_owned beyond its static arrays.
size_t peel_owned_smem(int W)
{
    return (size_t)((W + 3) & ~3) * sizeof(uint32_t) + (size_t)kWinChunks * kPeelThreads * sizeof(uint4);
}

// Run heads among the infeasible class-2 positions (sorted by violation).
__global__ void nds_infeasible_heads(int n, const int* __restrict__ qinfo, const int* __restrict__ counters,
                                     int target, int* __restrict__ flags)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    const int fc = counters[0], n2 = counters[10];
    int f = 0;
    if (fc < target && pos >= fc && pos < fc + n2)
        f = ((uint32_t)qinfo[pos] & ~kInfeasibleBit) == (uint32_t)pos ? 1 : 0;
    flags[pos] = f;
}

// Closed-form fronts of the infeasible points when the feasible ones number
// fewer than the target.  Every infeasible point is dominated by all feasible
// points, a class-2 point also by every class-2 point of smaller violation,
// a class-3 point (NaN violation) by the feasible points only.  With F the
// last feasible front (-1 without feasible points): class 3 forms front F + 1
// together with the first class-2 run, class-2 run j is front F + 1 + j.  The
// stop rule of the peel keeps the fronts up to the first whose cumulative
// count reaches the target: run j (j > 0) is kept when n3 + start_j < target.
// rank[pos] = inclusive count of run heads up to pos.
__global__ void nds_infeasible_fronts(int n, const int* __restrict__ qinfo, const int* __restrict__ rank,
                                      int* counters, int target, int* __restrict__ front_sorted)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    const int fc = counters[0], n2 = counters[10], n3 = counters[11];
    if (fc >= target) return;
    const int F1 = counters[12] + 1;
    if (pos < n && pos >= fc) {
        if (pos < fc + n2) {
            const int j = rank[pos] - 1;
            const int start = (int)((uint32_t)qinfo[pos] & ~kInfeasibleBit);
            if (j == 0 || n3 + start < target) front_sorted[pos] = F1 + j;
        } else {
            front_sorted[pos] = F1;
        }
    }
    if (pos == 0) {
        int last = F1;
        if (n2 > 0) {
            int p = target - n3 - 1;
            p = p < fc ? fc : (p > fc + n2 - 1 ? fc + n2 - 1 : p);
            last = F1 + rank[p] - 1;
        }
        counters[2] = last;
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
    if (threadIdx.x >= 10 && threadIdx.x <= 13) counters[threadIdx.x] = 0;
    if (threadIdx.x >= 16 && threadIdx.x <= 19) counters[threadIdx.x] = 0;  // front sizes (nds_peel_owned)
}

// ---------------------------------------------------------------------------
// 2b. dominance rows from block prefix sets (one workspace, any n)
// ---------------------------------------------------------------------------
//
// For every block of B sorted positions and every objective m >= 1 one table
// of BlockTable<B>::kSize words:
//   E[0]          the largest of the block's B order keys;
//   E[1 .. B-1]   the other B-1 keys as an implicit search tree (node k has
//                 children 2k and 2k+1; the in-order walk is ascending);
//   S[c], c = 0..B, from word B on: the positions of the c smallest keys
//                 (bit j of word i = position 32 i + j of the block), B/32
//                 words each.  For B = 256 the two 16-byte halves of S[c] are
//                 swapped when bit 2 of c is set, so that the 16-byte loads
//                 of eight lanes with different c spread over all eight bank
//                 groups.
// The count c of the block's keys <= v is the leaf that a log2(B)-level
// descent of the tree reaches (go right when E[k] <= v) plus (E[0] <= v); the
// block's positions whose objective is <= f_m(q) are then S[c], ties included
// whatever their order.  A lane holding q thus gets B row bits of objective m
// from log2(B) + 1 shared loads and B/128 16-byte loads, where the per-word
// tables of nds_tiles take B/32 six-probe searches.  Positions >= n carry the
// NaN key, above every key of a feasible q.
template <int B>
struct BlockTable {
    static constexpr int kWords = B / 32;                // row words per block
    static constexpr int kLevels = B == 256 ? 8 : 7;     // B = 2^kLevels
    static constexpr int kSize = B + (B + 1) * kWords;   // words per (block, objective)
};
static_assert(BlockTable<256>::kSize % 4 == 0 && BlockTable<128>::kSize % 4 == 0,
              "tables are copied in 16-byte chunks");

// Block size by objective count: up to M = 4 the double-buffered tables of
// 256 positions (9 KB per objective) leave room for several CTAs per SM;
// beyond, blocks of 128 positions (2.5 KB per objective) keep the SMs full.
template <int M>
struct BlockCfg {
    static constexpr int kB = M <= 4 ? 256 : 128;
};

// Dominatees q per row CTA, one per thread.  Every CTA stages each of its
// blocks' tables once, so more q per CTA mean fewer shared-memory writes per
// row word.
constexpr int kBlkThreads = 512;
constexpr int kBlkPerCtaMax = 8;  // blocks of dominators per row CTA, at most
constexpr int kBlkCtasPerSm = 8;  // row CTAs per SM the launch aims at (with fewer blocks per CTA)

// Count of the 32 ascending keys a[] that are <= x (six probes).
__device__ __forceinline__ int count_le32(const uint32_t* a, uint32_t x)
{
    int c = 0;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1)
        if (a[c + s - 1] <= x) c += s;
    if (a[c] <= x) ++c;
    return c;
}

// One CTA of B threads per (block, objective): each warp sorts its 32
// (key, lane) pairs with a bitonic network; the rank of a key in the block is
// its place in its warp plus, for every other warp, the count of that warp's
// keys <= it (lower warps) or < it (higher warps), which orders equal keys
// by position.  Then the tree placement of the sorted keys, and warp w builds
// word w of every prefix set with one ballot per set.
template <int B>
__global__ void __launch_bounds__(B)
nds_block_tables(const float* __restrict__ sf, int sf_stride, int n, int MF, uint32_t* __restrict__ tables)
{
    using T = BlockTable<B>;
    constexpr int NW = B / 32;
    __shared__ uint32_t s_sorted[NW][32];
    __shared__ int s_rank[B];
    const int blk = blockIdx.x / MF, m = blockIdx.x - blk * MF;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blk * B + threadIdx.x;
    const uint32_t key = p < n ? dom_key(sf[(size_t)m * sf_stride + p]) : 0xFFFFFFFFu;
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
    const uint32_t skey = (uint32_t)(kv >> 32);
    const int src = (int)(kv & 31ull);  // this lane holds the key of lane src
    s_sorted[warp][lane] = skey;
    __syncthreads();
    int r = lane;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        if (w < warp) r += count_le32(s_sorted[w], skey);
        else if (w > warp && skey > 0u) r += count_le32(s_sorted[w], skey - 1u);
    }
    s_rank[warp * 32 + src] = r;
    uint32_t* tab = tables + ((size_t)blk * MF + m) * T::kSize;
    if (r == B - 1) {
        tab[0] = skey;
    } else {
        const int i = r + 1, h = __ffs(i) - 1;  // in-order index, height above the leaves
        tab[(1 << (T::kLevels - 1 - h)) + (i >> (h + 1))] = skey;
    }
    __syncthreads();
    const int rk = s_rank[threadIdx.x];  // rank of position 32 warp + lane
    uint32_t* S = tab + B;
    for (int c0 = 0; c0 <= B; c0 += 32) {
        uint32_t mine = 0u;
#pragma unroll 8
        for (int cc = 0; cc < 32; ++cc) {
            const uint32_t bits = __ballot_sync(0xFFFFFFFFu, rk < c0 + cc);
            if (cc == lane) mine = bits;
        }
        const int c = c0 + lane;
        if (c <= B) {
            const int wj = NW == 8 ? (warp ^ (((c >> 2) & 1) << 2)) : warp;  // the half swap
            S[c * NW + wj] = mine;
        }
    }
}

__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

constexpr int kRowSegWords = 16;   // row words per lane collected before the stores
constexpr int kOutStride = 20;     // shared words per lane of the collected rows (16-byte rows, no conflicts)

// Rows are collected in shared memory for blocks of 256 positions (M <= 4).
// With blocks of 128 positions the search of the M-1 >= 4 objectives
// outweighs the stores, and the 40 KB for the collected rows would cost a
// resident CTA per SM: each lane stores its own words.
template <int B>
constexpr bool collect_rows() { return B == 256; }

// Rows of kBlkThreads dominatees (one per thread) against bpc blocks of B
// dominator positions.  The blocks' tables (all objectives) are staged in
// shared memory with cp.async, the next block's while the current one is
// searched.  Per block a lane descends the M-1 trees side by side and ANDs the
// M-1 prefix sets and the dup mask into its B/32 row words.  With
// collect_rows<B>() the lane puts them into shared memory and every
// kRowSegWords words the CTA writes the collected row segments (64 bytes per
// row), eight rows per warp instruction, where stores by the lanes themselves
// touch 32 rows per instruction; otherwise the lane stores them itself.  The lane remembers
// the highest dominator seen and raises blocker[q] to it once.  Infeasible q
// are skipped: the peel never reaches them, so their rows are never read.
template <int M, int B>
__global__ void __launch_bounds__(kBlkThreads)
nds_block_rows(const float* __restrict__ sf, int sf_stride, const int* __restrict__ qinfo,
               const uint32_t* __restrict__ tables, int n, int W, int bpc, uint32_t* __restrict__ rows,
               int* __restrict__ blocker)
{
    using T = BlockTable<B>;
    constexpr int MF = M - 1;
    constexpr int KW = T::kWords;
    constexpr int TS = T::kSize;
    constexpr int CH = MF * TS / 4;  // 16-byte chunks of one block's tables
    constexpr int G = kRowSegWords / KW;  // blocks per collected segment
    extern __shared__ uint4 s_tab[];  // [2][CH] tables, then (collect_rows) [kBlkThreads][kOutStride] row words
    __shared__ unsigned char s_live[kBlkThreads];
    uint32_t* s_out = reinterpret_cast<uint32_t*>(s_tab + 2 * CH);
    const int q0 = blockIdx.y * kBlkThreads;
    if (q0 >= n) return;
    const int qend = min(q0 + kBlkThreads, n);
    const int nb = (qend - 1 + B - 1) / B;  // blocks holding the dominators (positions < qend - 1)
    const int b_lo = blockIdx.x * bpc;
    if (b_lo >= nb) return;
    const int b_hi = min(nb, b_lo + bpc);
    const int q = q0 + threadIdx.x;
    uint32_t qk[MF];
    int dup = 0;
    bool live = false;
    if (q < n) {
        const uint32_t info = (uint32_t)qinfo[q];
        live = (info & kInfeasibleBit) == 0u;
        dup = (int)(info & ~kInfeasibleBit);
    }
#pragma unroll
    for (int m = 0; m < MF; ++m) qk[m] = live ? dom_key(sf[(size_t)m * sf_stride + q]) : 0u;
    s_live[threadIdx.x] = live ? 1 : 0;
    if (!__syncthreads_or(live)) return;

    const uint4* src = reinterpret_cast<const uint4*>(tables);
    auto stage = [&](int b, int buf) {
        const uint4* g = src + (size_t)b * CH;
        uint4* d = s_tab + buf * CH;
        for (int i = threadIdx.x; i < CH; i += kBlkThreads)
            cp_async16(d + i, reinterpret_cast<const uint32_t*>(g + i));
        cp_async_commit();
    };
    stage(b_lo, 0);
    int best = -1;
    uint32_t* my_out = s_out + threadIdx.x * kOutStride;
    int seg = b_lo;  // first block of the segment being collected
    for (int b = b_lo; b < b_hi; ++b) {
        const int buf = (b - b_lo) & 1;
        if (b + 1 < b_hi) {
            stage(b + 1, buf ^ 1);
            cp_async_wait_one();
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        if (live) {
            const int lo = b * B;
            const int rem = dup - lo;  // positions of the block below dup[q]
            uint32_t acc[KW];
#pragma unroll
            for (int j = 0; j < KW; ++j) acc[j] = rem > 0 ? 0xFFFFFFFFu : 0u;
            if (rem > 0) {
                const uint32_t* tab = reinterpret_cast<const uint32_t*>(s_tab + buf * CH);
                int k[MF];
#pragma unroll
                for (int m = 0; m < MF; ++m) k[m] = 1;
#pragma unroll
                for (int l = 0; l < T::kLevels; ++l) {
#pragma unroll
                    for (int m = 0; m < MF; ++m) k[m] = 2 * k[m] + (tab[m * TS + k[m]] <= qk[m] ? 1 : 0);
                }
#pragma unroll
                for (int m = 0; m < MF; ++m) {
                    const uint32_t* E = tab + m * TS;
                    const int c = k[m] - B + (E[0] <= qk[m] ? 1 : 0);
                    const uint4* S = reinterpret_cast<const uint4*>(E + B) + c * (KW / 4);
                    if constexpr (KW == 8) {
                        const int sw = (c >> 2) & 1;
                        const uint4 x = S[sw], y = S[sw ^ 1];
                        acc[0] &= x.x; acc[1] &= x.y; acc[2] &= x.z; acc[3] &= x.w;
                        acc[4] &= y.x; acc[5] &= y.y; acc[6] &= y.z; acc[7] &= y.w;
                    } else {
                        const uint4 x = S[0];
                        acc[0] &= x.x; acc[1] &= x.y; acc[2] &= x.z; acc[3] &= x.w;
                    }
                }
                if (rem < B) {
#pragma unroll
                    for (int j = 0; j < KW; ++j) {
                        const int r = rem - 32 * j;
                        acc[j] &= r >= 32 ? 0xFFFFFFFFu : (r <= 0 ? 0u : ((1u << r) - 1u));
                    }
                }
            }
            if constexpr (collect_rows<B>()) {
                uint4* o = reinterpret_cast<uint4*>(my_out + (b - seg) * KW);
                o[0] = make_uint4(acc[0], acc[1], acc[2], acc[3]);
                if constexpr (KW == 8) o[1] = make_uint4(acc[4], acc[5], acc[6], acc[7]);
            } else {
                uint4* dst = reinterpret_cast<uint4*>(rows + (size_t)q * W + b * KW);
                dst[0] = make_uint4(acc[0], acc[1], acc[2], acc[3]);
                if constexpr (KW == 8) {
                    if (b * KW + 8 <= W) dst[1] = make_uint4(acc[4], acc[5], acc[6], acc[7]);
                }
            }
#pragma unroll
            for (int j = 0; j < KW; ++j)
                if (acc[j]) best = lo + 32 * j + 31 - __clz(acc[j]);
        }
        if (collect_rows<B>() && (b - seg + 1 == G || b + 1 == b_hi)) {
            // the segment's words seg*KW .. seg*KW + nw - 1 of every live row:
            // a warp writes 8 rows x 4 chunks of 16 bytes, lanes 8i .. 8i+7
            // reading rows R+i and R+i+4 (distinct bank groups)
            __syncthreads();
            const int nw = (b - seg + 1) * KW;
            for (int c = threadIdx.x; c < kBlkThreads * (kRowSegWords / 4); c += kBlkThreads) {
                const int l = c & 31, rsel = l >> 2, part = l & 3;
                const int r = (c >> 5) * 8 + ((rsel & 1) << 2) + (rsel >> 1);
                const int gw = seg * KW + part * 4;
                if (part * 4 < nw && gw + 4 <= W && s_live[r])
                    *reinterpret_cast<uint4*>(rows + (size_t)(q0 + r) * W + gw) =
                        *reinterpret_cast<const uint4*>(s_out + r * kOutStride + part * 4);
            }
            seg = b + 1;
        }
        __syncthreads();  // the table buffer is staged again two blocks on, the row words rewritten
    }
    if (best >= 0) atomicMax(blocker + q, best);
}

template <int M>
constexpr int block_rows_smem()
{
    constexpr int B = BlockCfg<M>::kB;
    return 2 * (M - 1) * BlockTable<B>::kSize * 4 + (collect_rows<B>() ? kBlkThreads * kOutStride * 4 : 0);
}

template <int M>
void launch_block_rows(const Workspace& ws, int n, cudaStream_t stream)
{
    constexpr int B = BlockCfg<M>::kB;
    if (n < 2) return;  // no pairs: every blocker stays -1
    nds_block_tables<B><<<ceil_div(n, B) * (M - 1), B, 0, stream>>>(ws.sorted_f, ws.n_max, n, M - 1,
                                                                     ws.block_tables);
    // blocks per CTA: the most (up to kBlkPerCtaMax) that still give
    // kBlkCtasPerSm working CTAs per SM; fewer blocks per CTA overlap less
    // staging with searching, but small sorts need the CTAs
    const int ntiles = ceil_div(n, kBlkThreads);
    const int nb = ceil_div(n - 1, B);
    int bpc = kBlkPerCtaMax;
    for (; bpc > 1; bpc >>= 1) {
        long long ctas = 0;
        for (int t = 0; t < ntiles; ++t) ctas += ceil_div(ceil_div(std::min((t + 1) * kBlkThreads, n) - 1, B), bpc);
        if (ctas >= (long long)kBlkCtasPerSm * ws.sm_count) break;
    }
    dim3 grid(ceil_div(nb, bpc), ntiles);
    nds_block_rows<M, B><<<grid, kBlkThreads, block_rows_smem<M>(), stream>>>(
        ws.sorted_f, ws.n_max, ws.qinfo, ws.block_tables, n, ws.words, bpc, ws.rows, ws.blocker);
}

template <int M>
void launch_tiles(const Workspace& ws, int n, cudaStream_t stream)
{
    if constexpr (M > 1) {
        if (!ws.word_tiles) {
            launch_block_rows<M>(ws, n, stream);
            return;
        }
    }
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

// ---------------------------------------------------------------------------
// fused batch: one launch per stage for every instance (n = 2N <= 8192)
// ---------------------------------------------------------------------------

// Block sorts with 2, 4 or 8 items per thread: the smallest that holds the
// instance (the sort's work grows with the items).
template <int ITEMS>
using FusedSort64 = cub::BlockRadixSort<uint64_t, kFusedThreads, ITEMS, int>;
using FusedScan = cub::BlockScan<int, kFusedThreads>;
union FusedSortStorage {
    typename FusedSort64<kFusedItems>::TempStorage s64;
    typename FusedSort64<4>::TempStorage s64_4;
    typename FusedSort64<2>::TempStorage s64_2;
    typename FusedScan::TempStorage scan;
    int list[kFusedThreads + 4];  // long runs of fused_lex_onekey
};

// The order of fused_lexsort for n > kFusedThreads, as the staged path
// builds it: one block radix sort of the sort keys (sort_key) with ITEMS keys
// per thread, then each run of equal keys in class 0 put in lexicographic
// order (f1 .. f_{M-1}, index) -- runs of up to kTieShort points by one
// thread each (insertion sort), longer ones (when not already in order) by the
// whole CTA, each member counting the members that precede it.  One sort of
// kSortKeyBits bits replaces M-1 stable passes of 32 bits and one of 34.  The
// permutation goes to I.perm[0 .. n); I.key64 holds the sorted keys and
// I.vals serves the long runs as scratch.
template <int ITEMS>
__device__ __forceinline__ void fused_lex_onekey(const BatchInst& I, const SplitPop& pop, int n, int M,
                                                 FusedSortStorage& tmp)
{
    const int t = threadIdx.x;
    uint64_t keys[ITEMS];
    int vals[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int pt = t * ITEMS + j;
        vals[j] = pt;
        if (pt < n) {
            const uint64_t k0 = I.key0[pt];
            keys[j] = sort_key(pop, M, pt, (uint32_t)(k0 >> 32), (uint32_t)k0);
        } else {
            keys[j] = (1ull << kSortKeyBits) - 1ull;  // above every real key
        }
    }
    FusedSort64<ITEMS>(*reinterpret_cast<typename FusedSort64<ITEMS>::TempStorage*>(&tmp))
        .Sort(keys, vals, 0, kSortKeyBits);
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const int pos = t * ITEMS + j;
        if (pos < n) {
            I.key64[pos] = keys[j];
            I.perm[pos] = vals[j];
        }
    }
    __syncthreads();
    const uint64_t* K = I.key64;
    int* P = I.perm;
    // short runs, one thread per run head
    for (int pos = t; pos < n; pos += kFusedThreads) {
        const uint64_t k = K[pos];
        if ((k >> kSortClassShift) != 0u || (pos > 0 && K[pos - 1] == k)) continue;
        int L = 1;
        while (L <= kTieShort && pos + L < n && K[pos + L] == k) ++L;
        if (L == 1 || L > kTieShort) continue;
        for (int a = pos + 1; a < pos + L; ++a) {
            const int v = P[a];
            int b = a - 1;
            while (b >= pos && tie_less(pop, M, v, P[b])) {
                P[b + 1] = P[b];
                --b;
            }
            P[b + 1] = v;
        }
    }
    __syncthreads();
    // long runs, one after another by the whole CTA (the sort storage is free)
    int* s_heads = reinterpret_cast<int*>(&tmp);
    int* s_misc = s_heads + kFusedThreads;  // [0] heads, [1] run end, [2] out of order
    for (int base = 0; base < n; base += kFusedThreads) {
        if (t == 0) s_misc[0] = 0;
        __syncthreads();
        const int pos = base + t;
        if (pos < n) {
            const uint64_t k = K[pos];
            if ((k >> kSortClassShift) == 0u && (pos == 0 || K[pos - 1] != k) && pos + kTieShort < n &&
                K[pos + kTieShort] == k)
                s_heads[atomicAdd(s_misc, 1)] = pos;
        }
        __syncthreads();
        const int nh = s_misc[0];
        for (int h = 0; h < nh; ++h) {
            const int head = s_heads[h];
            const uint64_t k = K[head];
            if (t == 0) {
                s_misc[1] = n;
                s_misc[2] = 0;
            }
            __syncthreads();
            for (int a = head + 1 + t; a < n; a += kFusedThreads)
                if (K[a] != k) {
                    atomicMin(s_misc + 1, a);
                    break;
                }
            __syncthreads();
            const int end = s_misc[1];
            for (int a = head + 1 + t; a < end; a += kFusedThreads)
                if (tie_less(pop, M, P[a], P[a - 1])) s_misc[2] = 1;
            __syncthreads();
            if (s_misc[2]) {
                for (int a = head + t; a < end; a += kFusedThreads) {
                    const int v = P[a];
                    int r = 0;
                    for (int b = head; b < end; ++b) r += tie_less(pop, M, P[b], v) ? 1 : 0;
                    I.vals[head + r] = v;
                }
                __syncthreads();
                for (int a = head + t; a < end; a += kFusedThreads) P[a] = I.vals[a];
            }
            __syncthreads();
        }
    }
}

// Classification, sorted order, sorted objectives, dup positions and peel
// state of one instance per CTA: the stages of run_ndsort up to the
// dominance rows.  Instances of more than kFusedThreads points take the
// staged path's order (fused_lex_onekey); smaller ones count ranks under the
// lexicographic order (class and f0, f1 .. f_{M-1}, index).  Either order
// has what the rows and the peel need (dominators first, identical vectors
// adjacent, f0 non-decreasing in class 0), and the fronts depend on the
// relation only.
template <bool kLarge>
__device__ __forceinline__ void fused_lexsort_body(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    extern __shared__ __align__(16) unsigned char fused_smem[];
    FusedSortStorage& tmp = *reinterpret_cast<FusedSortStorage*>(fused_smem);
    __shared__ int s_feas;
    const BatchInst& I = insts[ids[blockIdx.x]];
    const SplitPop pop{I.objsP, I.objsO, I.cvP, I.cvO, I.N, I.N, I.N, I.n};
    const int n = I.n, M = I.M, t = threadIdx.x;
    if (t == 0) s_feas = 0;
    __syncthreads();
    int feas = 0;
    for (int i = t; i < n; i += kFusedThreads) {
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
        I.key0[i] = ((uint64_t)cls << 32) | val;
        feas += cls <= 1u;
    }
    atomicAdd(&s_feas, feas);
    __syncthreads();
    int vals[kFusedItems];
#pragma unroll
    for (int j = 0; j < kFusedItems; ++j) vals[j] = t * kFusedItems + j;
    if (n <= kFusedThreads) {
        // Small instances: the stable passes below order by (class and f0,
        // then f1 .. f_{M-1} for class 0, then the index); here each point
        // counts the points before it under that order directly, instead of
        // block sorts sized for kFusedMaxPoints.  Same permutation.
        uint64_t* s_k0 = reinterpret_cast<uint64_t*>(fused_smem);
        int* s_perm = reinterpret_cast<int*>(s_k0 + kFusedThreads);
        if (t < n) s_k0[t] = I.key0[t];
        __syncthreads();
        if (t < n) {
            const uint64_t ki = s_k0[t];
            const bool cls0 = (ki >> 32) == 0;
            int r = 0;
            for (int u = 0; u < n; ++u) {
                const uint64_t ku = s_k0[u];
                bool less = ku < ki;
                if (ku == ki) {
                    less = u < t;
                    if (cls0) {
                        for (int m = 1; m < M; ++m) {
                            const uint32_t a = float_order_key(pop.obj(m, u));
                            const uint32_t b = float_order_key(pop.obj(m, t));
                            if (a != b) {
                                less = a < b;
                                break;
                            }
                        }
                    }
                }
                r += less ? 1 : 0;
            }
            s_perm[r] = t;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kFusedItems; ++j) {
            const int pos = t * kFusedItems + j;
            vals[j] = (pos < n) ? s_perm[pos] : pos;
        }
        __syncthreads();  // the shared storage is reused below
    } else {
        if constexpr (kLarge) {
            if (n <= 2 * kFusedThreads) fused_lex_onekey<2>(I, pop, n, M, tmp);
            else if (n <= 4 * kFusedThreads) fused_lex_onekey<4>(I, pop, n, M, tmp);
            else fused_lex_onekey<kFusedItems>(I, pop, n, M, tmp);
            __syncthreads();  // the permutation in I.perm, written by every thread
#pragma unroll
            for (int j = 0; j < kFusedItems; ++j) {
                const int pos = t * kFusedItems + j;
                vals[j] = (pos < n) ? I.perm[pos] : pos;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kFusedItems; ++j) {
        const int pos = t * kFusedItems + j;
        if (pos < n) I.perm[pos] = vals[j];
    }
    __syncthreads();
    int heads[kFusedItems];
#pragma unroll
    for (int j = 0; j < kFusedItems; ++j) {
        const int pos = t * kFusedItems + j;
        heads[j] = 0;
        if (pos >= n) continue;
        const int pt = vals[j];
        const uint64_t k0 = I.key0[pt];
        const uint32_t cls = (uint32_t)(k0 >> 32);
        for (int m = 1; m < M; ++m) I.sorted_f[(size_t)(m - 1) * I.n_max + pos] = pop.obj(m, pt);
        bool is_head = true;
        if (pos > 0) {
            const int pp = I.perm[pos - 1];
            if (I.key0[pp] == k0) {
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
        heads[j] = is_head ? pos : 0;
    }
    FusedScan(tmp.scan).InclusiveScan(heads, heads, cub::Max());
    __syncthreads();
    const int feasible = s_feas;
#pragma unroll
    for (int j = 0; j < kFusedItems; ++j) {
        const int pos = t * kFusedItems + j;
        if (pos >= n) continue;
        const uint32_t cls = (uint32_t)(I.key0[vals[j]] >> 32);
        uint32_t d;
        switch (cls) {
        case 0u: d = (uint32_t)heads[j]; break;
        case 1u: d = 0u; break;
        case 2u: d = (uint32_t)heads[j] | kInfeasibleBit; break;
        default: d = (uint32_t)feasible | kInfeasibleBit; break;
        }
        I.qinfo[pos] = (int)d;
        I.blocker[pos] = -1;
        I.front_sorted[pos] = -1;
    }
    if (t == 0) {
        I.counters[0] = feasible;
        for (int c = 1; c <= 4; ++c) I.counters[c] = 0;
    }
}

__global__ void __launch_bounds__(kFusedThreads)
fused_lexsort(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    fused_lexsort_body<true>(insts, ids);
}

// Groups whose instances all have at most kFusedThreads points: the same
// body without the block sorts, a much smaller kernel (its instances are
// launch- and latency-bound, and the sort code around the counting path
// slowed them by 9%).
__global__ void __launch_bounds__(kFusedThreads)
fused_lexsort_small(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    fused_lexsort_body<false>(insts, ids);
}

// Shared memory of fused_lexsort_small: the counting path's keys and
// permutation, or the block scan's storage.
constexpr int kFusedLexSmallSmem =
    (int)(kFusedThreads * (sizeof(uint64_t) + sizeof(int)) > sizeof(FusedScan::TempStorage)
              ? kFusedThreads * (sizeof(uint64_t) + sizeof(int))
              : sizeof(FusedScan::TempStorage));

__global__ void fused_chunks(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int W = (I.n + 31) >> 5;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (gw >= W * (I.M - 1)) return;
    chunk_warp(gw, threadIdx.x & 31, I.sorted_f, I.n_max, I.n, W, I.chunk_keys, I.chunk_bits);
}

// Tile CTAs of all instances with M objectives, flattened: CTA b belongs to
// the instance whose range [prefix[k], prefix[k+1]) contains b.
template <int M, int S>
__global__ void __launch_bounds__(kTileThreads)
fused_tiles(const BatchInst* __restrict__ insts, const int* __restrict__ ids,
            const int* __restrict__ prefix, int count)
{
    const int b = blockIdx.x;
    int lo = 0, hi = count;  // largest k with prefix[k] <= b
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(prefix + mid) <= b) lo = mid; else hi = mid;
    }
    const BatchInst& I = insts[__ldg(ids + lo)];
    const int maxw = (I.n + 31) >> 5;
    constexpr int PW = TileShape<M, S>::kPW;
    const int gx = (maxw + PW - 1) / PW;
    const int lb = b - __ldg(prefix + lo);
    tile_block<M, PW>(lb % gx, lb / gx, I.sorted_f, I.n_max, I.qinfo, I.chunk_keys, I.chunk_bits, I.n, I.W, maxw,
                      I.rows, I.blocker);
}

constexpr int kFusedPeelThreads = 1024;

// Peel of one instance per CTA with the blockers, the front list and a queue
// of woken points in shared memory.  Once front k is known and removed from
// the unassigned set U, one parallel pass over the blockers queues the
// points whose blocker was in front k; each queued point (one lane each)
// probes its row from the former blocker's word downwards (bits above it stay
// free of unassigned dominators) and either records the next unassigned
// dominator found as its blocker or, having none, joins front k + 1.  A front
// costs three block barriers and one or two memory latencies.  Shared memory:
// U (W words), blocker, list and queue (n ints each).
__global__ void __launch_bounds__(kFusedPeelThreads, 1)
fused_peel(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    extern __shared__ __align__(16) uint32_t fp_smem[];
    __shared__ int s_cnt, s_qn;
    const BatchInst& I = insts[ids[blockIdx.x]];
    const int n = I.n, W = I.W, target = I.N;
    uint32_t* U = fp_smem;
    int* blk = reinterpret_cast<int*>(fp_smem + W);
    int* list = blk + n;
    int* queue = list + n;
    const uint32_t* rows = I.rows;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarps = blockDim.x >> 5;

    for (int w = t; w < W; w += blockDim.x) {
        const int lo = w * 32;
        U[w] = (lo + 32 <= n) ? 0xFFFFFFFFu : (lo >= n ? 0u : ((1u << (n - lo)) - 1u));
    }
    if (t == 0) s_cnt = 0;
    __syncthreads();
    for (int q = t; q < n; q += blockDim.x) {
        const int b = I.blocker[q];
        blk[q] = b;
        if (b < 0) {
            list[atomicAdd(&s_cnt, 1)] = q;
            I.front_sorted[q] = 0;
        }
    }
    __syncthreads();
    int len_prev = 0, len = s_cnt, total = 0, k = 0;
    for (;;) {
        const int ck = len - len_prev;
        total += ck;
        if (total >= target || ck == 0) {
            if (t == 0) {
                I.counters[1] = len;
                I.counters[2] = k;
                I.counters[3] = total;
                if (ck == 0 && total < target) atomicExch(I.counters + 6, kDevPeelInconsistent);
            }
            for (int i = t; i < len; i += blockDim.x) I.front_list[i] = list[i];
            return;
        }
        if (t == 0) s_qn = 0;
        for (int i = t; i < ck; i += blockDim.x) {
            const int p = list[len_prev + i];
            atomicAnd(U + (p >> 5), ~(1u << (p & 31)));
        }
        __syncthreads();
        // points still unassigned whose blocker has just been assigned
        for (int q = t; q < n; q += blockDim.x) {
            const int b = blk[q];
            if (b >= 0 && ((U[q >> 5] >> (q & 31)) & 1u) && !((U[b >> 5] >> (b & 31)) & 1u))
                queue[atomicAdd(&s_qn, 1)] = q;
        }
        __syncthreads();
        const int qn = s_qn;
        // entries interleaved over the warps: a short queue uses every warp
        for (int r = 0; r * 32 * nwarps < qn; ++r) {
            const int e = warp + nwarps * (r * 32 + lane);
            const bool act = e < qn;
            const int q = act ? queue[e] : 0;
            bool is_free = false, need = false;
            int start_w = -1;
            if (act) {
                const uint32_t* row = rows + (size_t)q * W;
                int w = blk[q] >> 5;
                const uint32_t hiw = __ldg(row + w);
                const uint32_t low = (w > 0) ? __ldg(row + w - 1) : 0u;
                uint32_t bits = hiw & U[w];
                if (!bits && w > 0) {
                    --w;
                    bits = low & U[w];
                }
                if (bits) {
                    blk[q] = w * 32 + (31 - __clz(bits));
                } else if (w == 0) {
                    is_free = true;
                } else {
                    need = true;
                    start_w = w - 1;
                }
            }
            // rows not resolved by the probe: the whole warp scans each of
            // them downwards over the words that still hold unassigned points
            unsigned needm = __ballot_sync(0xFFFFFFFFu, need);
            while (needm) {
                const int L = __ffs(needm) - 1;
                needm &= needm - 1;
                const int qL = __shfl_sync(0xFFFFFFFFu, q, L);
                const uint32_t* row = rows + (size_t)qL * W;
                const int sw = __shfl_sync(0xFFFFFFFFu, start_w, L);
                int found = -1;
                for (int w0 = sw; w0 >= 0 && found < 0; w0 -= 256) {
                    uint32_t acc[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int w = w0 - lane - 32 * i;
                        const uint32_t u = (w >= 0) ? U[w] : 0u;
                        acc[i] = u ? (__ldg(row + w) & u) : 0u;
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
                    if (found >= 0) blk[q] = found;
                    else is_free = true;
                }
            }
            const unsigned fm = __ballot_sync(0xFFFFFFFFu, is_free);
            if (fm) {
                int slot = 0;
                if (lane == 0) slot = atomicAdd(&s_cnt, __popc(fm));
                slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
                if (is_free) {
                    list[slot + __popc(fm & ((1u << lane) - 1u))] = q;
                    blk[q] = -1;
                    I.front_sorted[q] = k + 1;
                }
            }
        }
        __syncthreads();
        len_prev = len;
        len = s_cnt;
        ++k;
    }
}

__global__ void fused_scatter(const BatchInst* __restrict__ insts, const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos < I.n) I.fronts[I.perm[pos]] = I.front_sorted[pos];
}

template <int M>
int tile_blocks_of(int n, int shape)
{
    const int maxw = ceil_div(n, 32);
    const int pw = shape == 0 ? TileShape<M, 0>::kPW : TileShape<M, 1>::kPW;
    return ceil_div(maxw, pw) * ceil_div(n, kQB);
}

template <int M>
void launch_fused_tiles(const BatchInst* d_inst, const FusedBucket& b, cudaStream_t s)
{
    if (b.shape == 0)
        fused_tiles<M, 0><<<b.tile_blocks, kTileThreads, 0, s>>>(d_inst, b.d_ids, b.d_tile_prefix, b.count);
    else
        fused_tiles<M, 1><<<b.tile_blocks, kTileThreads, 0, s>>>(d_inst, b.d_ids, b.d_tile_prefix, b.count);
}

// Self-test of the peel's two barrier waits with a short limit: every CTA
// arrives, but the barrier asks for one arrival more than the grid has, so
// the wait runs out and records kDevBarrierTimeout.  which 0: the counted
// barrier of nds_peel_owned; 1: grid_barrier of nds_peel.
__global__ void selftest_barrier_wait(int* counters, int which, unsigned long long limit_ns)
{
    if (which == 0) {
        if (threadIdx.x == 0)
            counted_arrive(reinterpret_cast<unsigned long long*>(counters + 16), 0u,
                           (unsigned long long)gridDim.x + 1ull, counters + 6, limit_ns);
    } else {
        grid_barrier(counters, gridDim.x + 1u, 1, limit_ns);
    }
}

}  // namespace

int selftest_barrier_timeout(Workspace& ws, int which, unsigned long long limit_ns, cudaStream_t stream)
{
    nds_reset_counters<<<1, 32, 0, stream>>>(ws.counters);
    selftest_barrier_wait<<<2, 32, 0, stream>>>(ws.counters, which, limit_ns);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

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
    nds_classify<<<G, T, 0, stream>>>(pop, M, ws.key0, ws.key64[0], ws.perm[0], feas);
    MOEA_CUDA_TRY(cudaGetLastError());
    const uint64_t* key0 = ws.key0;
    size_t tmp = ws.cub_bytes;
    MOEA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws.cub_tmp, tmp, ws.key64[0], ws.key64[1], ws.perm[0],
                                                  ws.perm[1], n, 0, kSortKeyBits, stream));
    // runs of equal keys in class 0 into lexicographic order; ws.run_start
    // holds the list of long runs until the dup scan below overwrites it
    nds_tie_fix<<<G, T, 0, stream>>>(pop, M, ws.key64[1], ws.perm[1], ws.run_start, ws.counters + 13);
    nds_tie_fix_long<<<kTieLongCtas, kTieLongThreads, 0, stream>>>(pop, M, ws.key64[1], ws.perm[1], ws.run_start,
                                                               ws.counters + 13);
    MOEA_CUDA_TRY(cudaGetLastError());
    const int* perm = ws.perm[1];

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
    // every co-resident CTA with at least one group of 32 positions: each
    // CTA scans the rows of its own groups, so more CTAs mean fewer rows per
    // CTA and front (one CTA per group of 32 warps left half the SMs idle)
    int grid = ceil_div(n, 32);
    if (grid > ws.peel_grid) grid = ws.peel_grid;
    if (grid < 1 || ws.peel_single_cta) grid = 1;
    const uint32_t* rows = ws.rows;
    int Wp = ws.words;
    int nn = n, tt = target;
    const int* qi = qinfo;
    int* blk = ws.blocker;
    int* fs = ws.front_sorted;
    uint32_t* fmask = ws.peel_fmask;
    int* ctr = ws.counters;
    (void)W;
    // the three front masks start empty
    MOEA_CUDA_TRY(cudaMemsetAsync(fmask, 0, sizeof(uint32_t) * 3 * (size_t)Wp, stream));
    void* args[] = {(void*)&rows, (void*)&Wp, (void*)&nn, (void*)&tt, (void*)&qi,
                    (void*)&blk, (void*)&fs, (void*)&fmask, (void*)&ctr};
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
    // lane-owned points when every warp of the grid holds at most one group
    // of 32 positions and the rows are 16-byte aligned
    const bool owned = !ws.peel_general && ws.peel_owned_grid > 0 && ceil_div(n, 32) <= 32 * min(grid, ws.peel_owned_grid) &&
                       Wp >= kWin && (Wp & 3) == 0;
    if (owned) {
        if (grid > ws.peel_owned_grid) grid = ws.peel_owned_grid;
        const int* b0 = ws.blocker;
        void* oargs[] = {(void*)&rows, (void*)&Wp, (void*)&nn, (void*)&tt, (void*)&b0,
                         (void*)&fs, (void*)&fmask, (void*)&ctr};
        cfg.gridDim = dim3(grid);
        cfg.dynamicSmemBytes = peel_owned_smem(Wp);
        if (grid == 1) {
            nds_peel_owned<<<1, kPeelThreads, cfg.dynamicSmemBytes, stream>>>(rows, Wp, nn, tt, b0, fs, fmask,
                                                                              ctr);
        } else {
            MOEA_CUDA_TRY(cudaLaunchKernelExC(&cfg, (const void*)nds_peel_owned, oargs));
        }
    } else if (grid == 1) {
        // one CTA needs no co-residency guarantee: an ordinary launch, which
        // may run beside other work (batched instances)
        nds_peel<<<1, kPeelThreads, cfg.dynamicSmemBytes, stream>>>(rows, Wp, nn, tt, qi, blk, fs, fmask,
                                                                    ctr);
    } else {
        MOEA_CUDA_TRY(cudaLaunchKernelExC(&cfg, (const void*)nds_peel, args));
    }

    // infeasible fronts in closed form (no work when the feasible points suffice)
    nds_infeasible_heads<<<G, T, 0, stream>>>(n, qinfo, ws.counters, target, ws.head);
    MOEA_CUDA_TRY(cub::DeviceScan::InclusiveSum(ws.cub_tmp, tmp, ws.head, ws.run_start, n, stream));
    nds_infeasible_fronts<<<G, T, 0, stream>>>(n, qinfo, ws.run_start, ws.counters, target, ws.front_sorted);
    nds_scatter_fronts<<<G, T, 0, stream>>>(n, perm, ws.front_sorted, fronts);
    MOEA_CUDA_TRY(cudaGetLastError());
    stage_mark("ndsort.peel", stream);
    return MOEA_OK;
}

// Raises a kernel's dynamic shared-memory limit to at least `bytes`.  The
// limit belongs to the function, not to a workspace, so it is never lowered:
// a smaller workspace created later must not shrink the launch of a larger one.
static int raise_dynamic_smem(const void* func, size_t bytes)
{
    cudaFuncAttributes fa = {};
    MOEA_CUDA_TRY(cudaFuncGetAttributes(&fa, func));
    if ((size_t)fa.maxDynamicSharedSizeBytes < bytes)
        MOEA_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return MOEA_OK;
}

// Words of block tables a workspace of n_max points and m_max objectives
// needs for every objective count up to m_max.
size_t block_table_words(int n_max, int m_max)
{
    if (m_max < 2) return 0;
    const size_t lo = (size_t)ceil_div(n_max, 256) * (size_t)(m_max < 4 ? m_max - 1 : 3) * BlockTable<256>::kSize;
    const size_t hi = m_max >= 5 ? (size_t)ceil_div(n_max, 128) * (size_t)(m_max - 1) * BlockTable<128>::kSize : 0;
    return lo > hi ? lo : hi;
}

// Shared-memory limits of the block-row kernels beyond 48 KB.
int configure_block_rows()
{
#define MOEA_BR_CASE(K) \
    if (block_rows_smem<K>() > 48 * 1024) \
        MOEA_TRY(raise_dynamic_smem((const void*)nds_block_rows<K, BlockCfg<K>::kB>, block_rows_smem<K>()));
    MOEA_BR_CASE(2) MOEA_BR_CASE(3) MOEA_BR_CASE(4) MOEA_BR_CASE(5) MOEA_BR_CASE(6) MOEA_BR_CASE(7)
    MOEA_BR_CASE(8) MOEA_BR_CASE(9) MOEA_BR_CASE(10) MOEA_BR_CASE(11) MOEA_BR_CASE(12) MOEA_BR_CASE(13)
    MOEA_BR_CASE(14) MOEA_BR_CASE(15) MOEA_BR_CASE(16)
#undef MOEA_BR_CASE
    return MOEA_OK;
}

// Configure the co-resident grid of the peel kernel for this device.
int configure_peel(Workspace& ws)
{
    const size_t smem = (size_t)ws.words * sizeof(uint32_t);
    if (smem > 48 * 1024) MOEA_TRY(raise_dynamic_smem((const void*)nds_peel, smem));
    int per_sm = 0;
    MOEA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, nds_peel, kPeelThreads,
                                                                smem));
    int sms = 0;
    MOEA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws.device));
    ws.sm_count = sms;
    if (per_sm < 1)
        return set_error(MOEA_ERR_UNSUPPORTED, "peel kernel does not fit on an SM (smem %zu)", smem);
    ws.peel_grid = sms * (per_sm > 2 ? 2 : per_sm);
    ws.peel_smem = (int)smem;
    // the lane-owned peel: one CTA per SM
    ws.peel_owned_grid = 0;
    const size_t osmem = peel_owned_smem(ws.words);
    int optin = 0;
    MOEA_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ws.device));
    cudaFuncAttributes ofa = {};
    MOEA_CUDA_TRY(cudaFuncGetAttributes(&ofa, (const void*)nds_peel_owned));
    if (ws.words >= kWin && osmem + ofa.sharedSizeBytes <= (size_t)optin) {
        MOEA_TRY(raise_dynamic_smem((const void*)nds_peel_owned, osmem));
        int oper = 0;
        MOEA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oper, nds_peel_owned, kPeelThreads, osmem));
        if (oper >= 1) ws.peel_owned_grid = sms;
    }
    return MOEA_OK;
}

int fused_tile_blocks(int M, int n, int shape)
{
    switch (M) {
#define MOEA_TB_CASE(K) case K: return tile_blocks_of<K>(n, shape);
    MOEA_TB_CASE(1) MOEA_TB_CASE(2) MOEA_TB_CASE(3) MOEA_TB_CASE(4)
    MOEA_TB_CASE(5) MOEA_TB_CASE(6) MOEA_TB_CASE(7) MOEA_TB_CASE(8)
    MOEA_TB_CASE(9) MOEA_TB_CASE(10) MOEA_TB_CASE(11) MOEA_TB_CASE(12)
    MOEA_TB_CASE(13) MOEA_TB_CASE(14) MOEA_TB_CASE(15) MOEA_TB_CASE(16)
#undef MOEA_TB_CASE
    default: return 0;
    }
}

// U takes the workspace's row words W (4 * ceil(n / 128) for a workspace of n
// merged points), then blockers, front list and queue of n entries each.
size_t fused_peel_smem(int W, int n) { return (size_t)W * sizeof(uint32_t) + 3 * (size_t)n * sizeof(int); }

int fused_ndsort_configure()
{
    MOEA_CUDA_TRY(cudaFuncSetAttribute(fused_lexsort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(FusedSortStorage)));
    MOEA_CUDA_TRY(cudaFuncSetAttribute(fused_peel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)fused_peel_smem(4 * ceil_div(kFusedMaxPoints, 128), kFusedMaxPoints)));
    return MOEA_OK;
}

int fused_ndsort(const BatchInst* d_inst, const FusedGroup& g, cudaStream_t s)
{
    const int sort_smem = (int)sizeof(FusedSortStorage);
    if (g.max_n <= kFusedThreads)
        fused_lexsort_small<<<g.count, kFusedThreads, kFusedLexSmallSmem, s>>>(d_inst, g.d_ids);
    else
        fused_lexsort<<<g.count, kFusedThreads, sort_smem, s>>>(d_inst, g.d_ids);
    MOEA_CUDA_TRY(cudaGetLastError());
    if (g.max_M > 1) {
        const int warps = ceil_div(g.max_n, 32) * (g.max_M - 1);
        fused_chunks<<<dim3(ceil_div(warps, 8), g.count), 256, 0, s>>>(d_inst, g.d_ids);
    }
    for (const FusedBucket& b : g.buckets) {
        switch (b.M) {
#define MOEA_FT_CASE(K) case K: launch_fused_tiles<K>(d_inst, b, s); break;
        MOEA_FT_CASE(1) MOEA_FT_CASE(2) MOEA_FT_CASE(3) MOEA_FT_CASE(4)
        MOEA_FT_CASE(5) MOEA_FT_CASE(6) MOEA_FT_CASE(7) MOEA_FT_CASE(8)
        MOEA_FT_CASE(9) MOEA_FT_CASE(10) MOEA_FT_CASE(11) MOEA_FT_CASE(12)
        MOEA_FT_CASE(13) MOEA_FT_CASE(14) MOEA_FT_CASE(15) MOEA_FT_CASE(16)
#undef MOEA_FT_CASE
        default: return set_error(MOEA_ERR_UNSUPPORTED, "fused ndsort: M=%d", b.M);
        }
    }
    MOEA_CUDA_TRY(cudaGetLastError());
    fused_peel<<<g.count, kFusedPeelThreads, fused_peel_smem(g.max_W, g.max_n), s>>>(d_inst, g.d_ids);
    fused_scatter<<<dim3(ceil_div(g.max_n, 256), g.count), 256, 0, s>>>(d_inst, g.d_ids);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

}  // namespace moea
