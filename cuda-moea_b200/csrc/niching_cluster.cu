// Niche selection of the last front on one thread-block cluster.
//
// The reference selects the last front's survivors with three stable sorts
// (niching.cu:96-178): by (direction, distance); by (direction, 0 for the
// closest member of an empty niche else a random odd word); by (niche count
// + rank in the niche, random word), the survivors being the first nrem.
// The random words hash the position in the previous order, so every order
// must be reproduced exactly: each stage here is a stable LSD radix sort of
// the full 64-bit key, which gives the same order as the reference's.
//
// The sorts run over the nl members of the last front only (nl is known on
// the device alone, so a library sort has to run over the whole merged
// population).  A front of at most kNcSlice members is sorted by one CTA in
// its shared memory with CTA barriers (solo mode; the cluster's other CTAs
// leave at once).  A larger one lives in the distributed shared memory of the
// cluster's kNcCtas CTAs: CTA c holds positions [c*S, c*S + S) of the current
// order, S = ceil(nl / kNcCtas).  A pass over 8 key bits:
//   1. every CTA's count of each digit is read from the CTAs' shared memory
//      (pushed there by the previous pass), giving each digit's first
//      position for this CTA (digits before it, then lower CTAs);
//   2. each warp ranks its contiguous segment (lanes with the same digit from
//      one ballot per digit bit) into its row of a per-warp digit table
//      (stable: lanes in order, steps in order);
//   3. each member is stored into the destination CTA's other buffer, and
//      its next digit is counted there with a shared-memory atomic;
//   4. one cluster barrier.
// Digits that are the same in every key (from the cluster-wide OR and AND of
// the keys) are skipped.  Between stages the start of each direction's run is
// a segmented max-scan, carried across CTAs.
#include <cooperative_groups.h>

#include "internal.cuh"

namespace cg = cooperative_groups;

namespace moea {
namespace {

constexpr int kNcCtas = 16;
constexpr int kNcThreads = 512;
constexpr int kNcWarps = kNcThreads / 32;
constexpr int kNcSlice = 4096;                        // members per CTA
constexpr int kNcSteps = kNcSlice / kNcWarps / 32;    // 32-member steps per warp segment
constexpr int kNcPerThread = kNcSlice / kNcThreads;   // members per thread in the run scan

struct NcShared {
    uint64_t key[2][kNcSlice];
    int val[2][kNcSlice];
    int run[kNcSlice];          // global position where the member's direction run starts
    int cnt[kNcWarps][256];     // per-warp digit counts, then their prefix over warps
    int dcount[256];            // this CTA's digit totals (read by the other CTAs)
    int dtotal[256];
    int dbefore[256];
    int dbase[256];             // first global position of each digit for this CTA
    int hist[3][256];           // cluster mode: digit counts of this CTA's slice, pushed by the
                                // CTAs that scatter into it (read by all, three in rotation)
    int plan[8];                // cluster mode: shifts of the digits that differ somewhere
    uint64_t red_or, red_and;   // OR / AND of this CTA's keys (read by the other CTAs)
    uint64_t diff;              // bits that differ in some pair of keys
    uint64_t wred[kNcWarps][2];
    int wmax[kNcWarps];
    int last_head;              // highest run head in this CTA's slice, or -1 (read by the others)
    int carry;
};

__device__ __forceinline__ uint64_t shfl_xor_u64(uint64_t v, int o)
{
    const uint32_t lo = __shfl_xor_sync(0xFFFFFFFFu, (uint32_t)v, o);
    const uint32_t hi = __shfl_xor_sync(0xFFFFFFFFu, (uint32_t)(v >> 32), o);
    return ((uint64_t)hi << 32) | lo;
}

// Lanes of the warp holding the same 8-bit digit as this lane (among the
// lanes with valid set), from one ballot per digit bit.
__device__ __forceinline__ unsigned match_digit(int d, bool valid)
{
    unsigned peers = __ballot_sync(0xFFFFFFFFu, valid);
    if (!valid) peers = ~peers;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const unsigned m = __ballot_sync(0xFFFFFFFFu, (d >> b) & 1);
        peers &= ((d >> b) & 1) ? m : ~m;
    }
    return peers;
}

// Solo: one CTA holds every member (nl <= kNcSlice); its barriers are CTA
// barriers and every "remote" CTA is itself.
template <bool kSolo>
__device__ __forceinline__ void nc_sync(cg::cluster_group& cluster)
{
    if (kSolo) __syncthreads();
    else cluster.sync();
}

template <bool kSolo, class T>
__device__ __forceinline__ T* nc_map(cg::cluster_group& cluster, T* p, int r)
{
    if (kSolo) return p;
    return cluster.map_shared_rank(p, r);
}

// One stable pass over key bits [shift, shift + 8): buffer cur -> cur ^ 1.
template <bool kSolo>
__device__ void nc_pass(NcShared& sm, cg::cluster_group& cluster, int c, int cur, int len, int S, int shift)
{
    constexpr int kCtas = kSolo ? 1 : kNcCtas;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < kNcWarps * 256; i += kNcThreads) (&sm.cnt[0][0])[i] = 0;
    __syncthreads();
    // per-warp contiguous segments, a multiple of 32 members each
    const int seg = (((len + kNcWarps - 1) / kNcWarps) + 31) & ~31;
    const int b0 = warp * seg, b1 = min(len, b0 + seg);
    int rk[kNcSteps], dg[kNcSteps];
#pragma unroll
    for (int j = 0; j < kNcSteps; ++j) {
        if (b0 + 32 * j >= b1) break;  // warp-uniform: the segment has ended
        const int e = b0 + 32 * j + lane;
        const bool valid = e < b1;
        const int d = valid ? (int)((sm.key[cur][e] >> shift) & 0xFFu) : 0;
        const unsigned peers = match_digit(d, valid);
        const int leader = __ffs(peers) - 1;
        int old = 0;
        if (valid && lane == leader) {
            old = sm.cnt[warp][d];
            sm.cnt[warp][d] = old + __popc(peers);
        }
        old = __shfl_sync(0xFFFFFFFFu, old, leader);
        rk[j] = old + __popc(peers & ((1u << lane) - 1u));
        dg[j] = d;
        __syncwarp();
    }
    __syncthreads();
    if (tid < 256) {
        int run = 0;
#pragma unroll
        for (int w = 0; w < kNcWarps; ++w) {
            const int x = sm.cnt[w][tid];
            sm.cnt[w][tid] = run;
            run += x;
        }
        sm.dcount[tid] = run;
    }
    nc_sync<kSolo>(cluster);  // every CTA's digit totals are published
    if (tid < 256) {
        int total = 0, before = 0;
#pragma unroll
        for (int r = 0; r < kCtas; ++r) {
            const int x = nc_map<kSolo>(cluster, sm.dcount, r)[tid];
            total += x;
            before += (r < c) ? x : 0;
        }
        sm.dtotal[tid] = total;
        sm.dbefore[tid] = before;
    }
    __syncthreads();
    if (warp == 0) {
        // exclusive scan of the 256 digit totals, 8 consecutive digits per lane
        int part = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) part += sm.dtotal[lane * 8 + i];
        int incl = part;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        int acc = incl - part;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int d = lane * 8 + i;
            sm.dbase[d] = acc + sm.dbefore[d];
            acc += sm.dtotal[d];
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kNcSteps; ++j) {
        if (b0 + 32 * j >= b1) break;
        const int e = b0 + 32 * j + lane;
        if (e < b1) {
            const int d = dg[j];
            const int pos = sm.dbase[d] + sm.cnt[warp][d] + rk[j];
            const int dest = pos / S;
            const int slot = pos - dest * S;
            NcShared* ds = nc_map<kSolo>(cluster, &sm, dest);
            ds->key[cur ^ 1][slot] = sm.key[cur][e];
            ds->val[cur ^ 1][slot] = sm.val[cur][e];
        }
    }
    nc_sync<kSolo>(cluster);  // the other buffer is complete everywhere; this pass's totals were read
}

// Stable sort of the nl keys (with their values) held in buffer cur; returns
// the buffer that holds the result.
template <bool kSolo>
__device__ int nc_sort(NcShared& sm, cg::cluster_group& cluster, int c, int cur, int len, int S)
{
    constexpr int kCtas = kSolo ? 1 : kNcCtas;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint64_t o = 0, a = ~0ull;
    for (int e = tid; e < len; e += kNcThreads) {
        o |= sm.key[cur][e];
        a &= sm.key[cur][e];
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) {
        o |= shfl_xor_u64(o, s);
        a &= shfl_xor_u64(a, s);
    }
    if (lane == 0) {
        sm.wred[warp][0] = o;
        sm.wred[warp][1] = a;
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < kNcWarps; ++w) {
            o |= sm.wred[w][0];
            a &= sm.wred[w][1];
        }
        sm.red_or = o;
        sm.red_and = a;
    }
    nc_sync<kSolo>(cluster);
    if (tid == 0) {
        uint64_t go = 0, ga = ~0ull;
        for (int r = 0; r < kCtas; ++r) {
            const NcShared* rs = nc_map<kSolo>(cluster, &sm, r);
            go |= rs->red_or;
            ga &= rs->red_and;
        }
        sm.diff = go ^ ga;
    }
    nc_sync<kSolo>(cluster);  // the OR / AND words were read everywhere before they change again
    const uint64_t diff = sm.diff;
    for (int d = 0; d < 8; ++d) {
        if (((diff >> (8 * d)) & 0xFFu) == 0) continue;  // the same digit in every key
        nc_pass<kSolo>(sm, cluster, c, cur, len, S, 8 * d);
        cur ^= 1;
    }
    return cur;
}

// Cluster mode, one cluster barrier per pass.  Pass i reads every CTA's
// counts of its digit from hist[i % 3] (pushed by the scatter of pass i - 1,
// or counted locally before pass 0), scatters, and pushes each member's next
// digit into the destination's hist[(i + 1) % 3]; hist[(i + 2) % 3], read by
// pass i - 1 before its barrier, is cleared meanwhile.
__device__ void nc_pass_push(NcShared& sm, cg::cluster_group& cluster, int c, int cur, int len, int S, int i,
                             int shift, int next_shift)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int hb = i % 3, hn = (i + 1) % 3, hz = (i + 2) % 3;
    for (int k = tid; k < kNcWarps * 256; k += kNcThreads) (&sm.cnt[0][0])[k] = 0;
    if (tid < 256) sm.hist[hz][tid] = 0;
    // every CTA's count of each digit, and of the same digit in lower CTAs
    if (tid < 256) {
        int total = 0, before = 0;
#pragma unroll
        for (int r = 0; r < kNcCtas; ++r) {
            const int x = cluster.map_shared_rank(&sm.hist[hb][0], r)[tid];
            total += x;
            before += (r < c) ? x : 0;
        }
        sm.dtotal[tid] = total;
        sm.dbefore[tid] = before;
    }
    __syncthreads();
    const int seg = (((len + kNcWarps - 1) / kNcWarps) + 31) & ~31;
    const int b0 = warp * seg, b1 = min(len, b0 + seg);
    int rk[kNcSteps], dg[kNcSteps];
#pragma unroll
    for (int j = 0; j < kNcSteps; ++j) {
        if (b0 + 32 * j >= b1) break;  // warp-uniform: the segment has ended
        const int e = b0 + 32 * j + lane;
        const bool valid = e < b1;
        const int d = valid ? (int)((sm.key[cur][e] >> shift) & 0xFFu) : 0;
        const unsigned peers = match_digit(d, valid);
        const int leader = __ffs(peers) - 1;
        int old = 0;
        if (valid && lane == leader) {
            old = sm.cnt[warp][d];
            sm.cnt[warp][d] = old + __popc(peers);
        }
        old = __shfl_sync(0xFFFFFFFFu, old, leader);
        rk[j] = old + __popc(peers & ((1u << lane) - 1u));
        dg[j] = d;
        __syncwarp();
    }
    __syncthreads();
    if (tid < 256) {
        int run = 0;
#pragma unroll
        for (int w = 0; w < kNcWarps; ++w) {
            const int x = sm.cnt[w][tid];
            sm.cnt[w][tid] = run;
            run += x;
        }
    }
    if (warp == 0) {
        int part = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) part += sm.dtotal[lane * 8 + k];
        int incl = part;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        int acc = incl - part;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int d = lane * 8 + k;
            sm.dbase[d] = acc + sm.dbefore[d];
            acc += sm.dtotal[d];
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kNcSteps; ++j) {
        if (b0 + 32 * j >= b1) break;
        const int e = b0 + 32 * j + lane;
        if (e < b1) {
            const int d = dg[j];
            const int pos = sm.dbase[d] + sm.cnt[warp][d] + rk[j];
            const int dest = pos / S;
            const int slot = pos - dest * S;
            NcShared* ds = cluster.map_shared_rank(&sm, dest);
            const uint64_t k = sm.key[cur][e];
            ds->key[cur ^ 1][slot] = k;
            ds->val[cur ^ 1][slot] = sm.val[cur][e];
            if (next_shift >= 0) atomicAdd(&ds->hist[hn][(int)((k >> next_shift) & 0xFFu)], 1);
        }
    }
    cluster.sync();  // buffer cur ^ 1 and hist[hn] are complete everywhere; hist[hb] was read
}

// Local counts of the digit at `shift` into hist[h] (warp-aggregated).
__device__ void nc_count(NcShared& sm, int cur, int len, int shift, int h)
{
    const int tid = threadIdx.x, lane = tid & 31;
    for (int e0 = tid - lane; e0 < len; e0 += kNcThreads) {
        const int e = e0 + lane;
        const int d = (e < len) ? (int)((sm.key[cur][e] >> shift) & 0xFFu) : 0;
        const unsigned peers = match_digit(d, e < len);
        if (e < len && lane == __ffs(peers) - 1) atomicAdd(&sm.hist[h][d], __popc(peers));
    }
}

__device__ int nc_sort_cluster(NcShared& sm, cg::cluster_group& cluster, int c, int cur, int len, int S)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 256) {
        sm.hist[0][tid] = 0;
        sm.hist[1][tid] = 0;
    }
    __syncthreads();
    uint64_t o = 0, a = ~0ull;
    for (int e = tid; e < len; e += kNcThreads) {
        o |= sm.key[cur][e];
        a &= sm.key[cur][e];
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) {
        o |= shfl_xor_u64(o, s);
        a &= shfl_xor_u64(a, s);
    }
    if (lane == 0) {
        sm.wred[warp][0] = o;
        sm.wred[warp][1] = a;
    }
    // the lowest digit nearly always differs: its counts are taken now
    nc_count(sm, cur, len, 0, 0);
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < kNcWarps; ++w) {
            o |= sm.wred[w][0];
            a &= sm.wred[w][1];
        }
        sm.red_or = o;
        sm.red_and = a;
    }
    cluster.sync();  // OR / AND and the lowest digit's counts are published
    if (tid == 0) {
        uint64_t go = 0, ga = ~0ull;
        for (int r = 0; r < kNcCtas; ++r) {
            const NcShared* rs = cluster.map_shared_rank(&sm, r);
            go |= rs->red_or;
            ga &= rs->red_and;
        }
        const uint64_t diff = go ^ ga;
        int np = 0;
        for (int d = 0; d < 8; ++d)
            if ((diff >> (8 * d)) & 0xFFu) sm.plan[np++] = 8 * d;
        for (int d = np; d < 8; ++d) sm.plan[d] = -1;
    }
    __syncthreads();
    int passes = 0;
    while (passes < 8 && sm.plan[passes] >= 0) ++passes;
    if (passes > 0 && sm.plan[0] != 0) {
        // the lowest digit is the same everywhere: count the first that is not
        cluster.sync();  // hist[0] of every CTA was read by nobody; OR / AND were read
        if (tid < 256) sm.hist[0][tid] = 0;
        __syncthreads();
        nc_count(sm, cur, len, sm.plan[0], 0);
        cluster.sync();
    } else if (passes == 0) {
        cluster.sync();  // the OR / AND words were read everywhere
    }
    for (int i = 0; i < passes; ++i) {
        nc_pass_push(sm, cluster, c, cur, len, S, i, sm.plan[i], (i + 1 < passes) ? sm.plan[i + 1] : -1);
        cur ^= 1;
    }
    return cur;
}

// run[e] = global position where the direction run of member e starts
// (heads: a different direction than the member before).
template <bool kSolo>
__device__ void nc_runs(NcShared& sm, cg::cluster_group& cluster, int c, int cur, int len, int S, int lo)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t prev_dir = 0;
    if (c > 0 && len > 0) prev_dir = (uint32_t)(nc_map<kSolo>(cluster, &sm, c - 1)->key[cur][S - 1] >> 32);
    const int e0 = tid * kNcPerThread;
    int h[kNcPerThread];
    int m = -1;
#pragma unroll
    for (int i = 0; i < kNcPerThread; ++i) {
        const int e = e0 + i;
        int head = -1;
        if (e < len) {
            const uint32_t dir = (uint32_t)(sm.key[cur][e] >> 32);
            const uint32_t before = (e > 0) ? (uint32_t)(sm.key[cur][e - 1] >> 32) : prev_dir;
            if ((c == 0 && e == 0) || dir != before) head = lo + e;
        }
        m = max(m, head);
        h[i] = m;  // inclusive max within the thread's members
    }
    // exclusive max-scan of the threads' maxima
    int incl = m;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl = max(incl, y);
    }
    if (lane == 31) sm.wmax[warp] = incl;
    __syncthreads();
    if (tid == 0) {
        int best = -1;
        for (int w = 0; w < kNcWarps; ++w) best = max(best, sm.wmax[w]);
        sm.last_head = best;
    }
    int wprefix = -1;
    for (int w = 0; w < warp; ++w) wprefix = max(wprefix, sm.wmax[w]);
    int excl = __shfl_up_sync(0xFFFFFFFFu, incl, 1);
    if (lane == 0) excl = -1;
    const int base = max(wprefix, excl);
    nc_sync<kSolo>(cluster);  // last_head published
    if (tid == 0) {
        int carry = -1;
        for (int r = 0; r < c; ++r) carry = max(carry, nc_map<kSolo>(cluster, &sm, r)->last_head);
        sm.carry = carry;
    }
    __syncthreads();
    const int start = max(sm.carry, base);
#pragma unroll
    for (int i = 0; i < kNcPerThread; ++i) {
        const int e = e0 + i;
        if (e < len) sm.run[e] = max(start, h[i]);
    }
    nc_sync<kSolo>(cluster);  // last_head was read everywhere before the CTAs move on
}

template <bool kSolo>
__device__ __forceinline__ int nc_sort_any(NcShared& sm, cg::cluster_group& cluster, int c, int cur, int len,
                                           int S)
{
    if constexpr (kSolo) return nc_sort<true>(sm, cluster, c, cur, len, S);
    else return nc_sort_cluster(sm, cluster, c, cur, len, S);
}

template <bool kSolo>
__device__ void nc_niching(NcShared& sm, cg::cluster_group& cluster, int c, const int* __restrict__ idx,
                           const float* __restrict__ dist, int np, int nl, int nrem,
                           const int* __restrict__ rho, int H, uint64_t seed,
                           unsigned long long* __restrict__ offset, const int* __restrict__ nds_gidx,
                           int* __restrict__ selected)
{
    const int tid = threadIdx.x;
    const unsigned long long off = *offset;
    const int S = kSolo ? nl : (nl + kNcCtas - 1) / kNcCtas;
    const int lo = c * S;
    const int len = max(0, min(S, nl - lo));

    // stage 1: (direction, distance bits)
    for (int e = tid; e < len; e += kNcThreads) {
        const int t = lo + e;
        sm.key[0][e] = ((uint64_t)(uint32_t)idx[np + t] << 32) | __float_as_uint(dist[np + t]);
        sm.val[0][e] = t;
    }
    __syncthreads();
    int cur = nc_sort_any<kSolo>(sm, cluster, c, 0, len, S);
    nc_runs<kSolo>(sm, cluster, c, cur, len, S, lo);

    // stage 2: (direction, 0 for the closest member of an empty niche, else a random odd word)
    for (int e = tid; e < len; e += kNcThreads) {
        const int t = lo + e;
        const uint32_t ref = (uint32_t)(sm.key[cur][e] >> 32);
        const int r_i = (int)ref;
        const int rho_r = (r_i >= 0 && r_i < H) ? rho[r_i] : 0;
        const int rank = t - sm.run[e];
        const uint32_t rnd = splitmix_u32(off + (uint64_t)t, seed);
        const uint32_t low = (rho_r == 0 && rank == 0) ? 0u : (rnd | 1u);
        sm.key[cur][e] = ((uint64_t)ref << 32) | low;
    }
    __syncthreads();
    // the direction runs keep their positions: only their members move
    cur = nc_sort_any<kSolo>(sm, cluster, c, cur, len, S);

    // stage 3: (niche count + rank in the niche, random word)
    for (int e = tid; e < len; e += kNcThreads) {
        const int t = lo + e;
        const uint32_t ref = (uint32_t)(sm.key[cur][e] >> 32);
        const int r_i = (int)ref;
        const int rho_r = (r_i >= 0 && r_i < H) ? rho[r_i] : 0;
        const int rank = t - sm.run[e];
        const uint32_t rnd = splitmix_u32(off + (uint64_t)nl + (uint64_t)t, seed);
        sm.key[cur][e] = ((uint64_t)(uint32_t)(rho_r + rank) << 32) | rnd;
    }
    __syncthreads();
    cur = nc_sort_any<kSolo>(sm, cluster, c, cur, len, S);

    for (int e = tid; e < len; e += kNcThreads) {
        const int t = lo + e;
        if (t < nrem) selected[np + t] = nds_gidx[np + sm.val[cur][e]];
    }
    if (c == 0 && tid == 0) *offset = off + 2ull * (unsigned long long)nl;
}

__global__ void __launch_bounds__(kNcThreads, 1)
nich_cluster(const int* __restrict__ idx, const float* __restrict__ dist, const int* __restrict__ sizes,
             const int* __restrict__ rho, int H, uint64_t seed, unsigned long long* __restrict__ offset,
             const int* __restrict__ nds_gidx, int* __restrict__ selected, int* __restrict__ status)
{
    extern __shared__ __align__(16) unsigned char nc_raw[];
    NcShared& sm = *reinterpret_cast<NcShared*>(nc_raw);
    cg::cluster_group cluster = cg::this_cluster();
    const int c = (int)cluster.block_rank();
    const int np = sizes[0], nl = sizes[1], nrem = sizes[2];
    // every branch below is uniform over the cluster
    if (nl <= 0) return;  // no member, nothing shared
    if (nl > kNcCtas * kNcSlice) {  // excluded by the host; reported, never indexed
        if (c == 0 && threadIdx.x == 0) atomicExch(status, kDevNichingSize);
        return;
    }
    if (nl <= kNcSlice) {
        // one CTA holds the whole front: CTA barriers instead of cluster
        // barriers; the other CTAs leave at once and share nothing
        if (c == 0) nc_niching<true>(sm, cluster, 0, idx, dist, np, nl, nrem, rho, H, seed, offset, nds_gidx,
                                     selected);
        return;
    }
    nc_niching<false>(sm, cluster, c, idx, dist, np, nl, nrem, rho, H, seed, offset, nds_gidx, selected);
}

}  // namespace

int niching_cluster_capacity() { return kNcCtas * kNcSlice; }

// Whether the cluster kernel can run on the current device (attributes are
// set once per process; a device that cannot co-schedule the cluster keeps
// the library sort).
bool niching_cluster_ready()
{
    static int state = -1;  // -1 unknown, 0 no, 1 yes
    if (state >= 0) return state == 1;
    state = 0;
    if (cudaFuncSetAttribute(nich_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
        cudaFuncSetAttribute(nich_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(NcShared)) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kNcCtas);
    cfg.blockDim = dim3(kNcThreads);
    cfg.dynamicSmemBytes = sizeof(NcShared);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kNcCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, (void*)nich_cluster, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    state = clusters >= 1 ? 1 : 0;
    return state == 1;
}

int launch_niching_cluster(const int* idx, const float* dist, const int* sizes, const int* rho, int H,
                           uint64_t seed, unsigned long long* offset, const int* nds_gidx, int* selected,
                           int* status, cudaStream_t stream)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kNcCtas);
    cfg.blockDim = dim3(kNcThreads);
    cfg.dynamicSmemBytes = sizeof(NcShared);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kNcCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MOEA_CUDA_TRY(cudaLaunchKernelEx(&cfg, nich_cluster, idx, dist, sizes, rho, H, seed, offset, nds_gidx,
                                     selected, status));
    return MOEA_OK;
}

}  // namespace moea
