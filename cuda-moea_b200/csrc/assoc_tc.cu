// Association on the tensor cores: the precision form of the NSGA-III
// association (reference: nat/src/selection/nsga3/kernels/association.cu:
// 86-188, 586).
//
// The reference picks, per normalised point x, the direction r_j of least
// perpendicular distance, computed in FP32 as d2_j = |x - (x.r_j) r_j|^2
// (association.cu:139-170), ties to the smaller j.  With D_j the exact dot,
// |d2_j - (|x|^2 - D_j^2)| <= margin / 2 (assoc_margin), so every minimiser j*
// satisfies D_j*^2 >= max_k D_k^2 - margin.
//
// Here the dots of 128 points with 128 directions come from tcgen05.mma
// (kind::tf32, FP32 accumulation in tensor memory).  Each operand is split
// into TF32 parts, v = hi + lo + e with |e| <= 2^-22 |v|, placed along K as
//     A row (point)     = [x_hi, x_hi, x_lo, 0 ...]
//     B row (direction) = [r_hi, r_lo, r_hi, 0 ...]
// so one MMA forms hi.hi + hi.lo + lo.hi, within about 3 * 2^-22 sum|x_m r_m|
// of D_j before accumulation.  The kernel allows
//     E = (4M + 16) 2^-21 |x| sqrt(1 + delta)
// for the accumulated value a_j, which leaves room for an accumulator that
// truncates every partial sum.  Then
//     (|a_j*| + E)^2 >= D_j*^2 >= (max_k |a_k| - E)^2 - margin,
// and every direction passing this test is re-scored with the reference's
// FP32 formula.  The re-scored set holds every minimiser, so the packed
// (d2, j) minimum is the reference's argmin: identical to the FP32 scan.
//
// Layout: the directions are packed once (tc_pack_directions) as tiles of 128
// in the MMA's shared-memory image (K-major, no swizzle, core matrices of
// 8 rows x 16 bytes, the two 16-byte K halves of one MMA 128 bytes apart and
// 8-row groups KP * 32 bytes apart), followed by the tile's FP32 coordinates
// for the re-score.  A work item is 256 points (two 128-row point tiles that
// share every direction tile) x a range of direction tiles.  The kernel runs
// twice: launch 1 only takes each point's largest |a_j| over all directions
// (one |max| per element, no branches, merged across items by atomicMax);
// launch 2 tests every 32-column chunk against the threshold of that maximum
// and re-scores the candidate groups of 4 columns.  With a running maximum
// instead, the threshold tightens only once the sweep reaches the point's
// best direction, and until then most chunks trigger for some lane of a warp.
// Re-scoring a direction that is not a candidate is harmless (the exact
// formula decides), and the packed (d2, j) minimum makes the order of the
// re-scores irrelevant.
//
// Kernel: one persistent CTA per SM holding all 512 TMEM columns (two
// buffers x two point tiles x 128 FP32 columns).  Warp 0 streams direction
// tiles into a ring of shared-memory stages with cp.async.bulk; warp 1 issues
// the MMAs; warps 2..17 read the accumulators.  Consumer warp w reads TMEM
// lanes 32 (w & 3) .. +31 (its sub-partition) of point tile ((w - 2) >> 3)
// and columns 64 (((w - 2) >> 2) & 1) .. +63; the warps of column half 0 also
// write their point tile of each item (double buffered).  Stages,
// accumulators and point tiles are handed over through mbarriers.  Every wait
// gives up after about 1 s, records kDevTensorTimeout and lets the CTA drain
// its copies and free its tensor memory.
#include <cmath>

#include "internal.cuh"

namespace moea {
namespace {

constexpr int kTcRows = 128;            // points per point tile (MMA M)
constexpr int kTcSub = 2;               // point tiles per work item
constexpr int kTcItemRows = kTcRows * kTcSub;
constexpr int kTcCols = 128;            // directions per tile (MMA N)
constexpr int kTcConsumerWarps = 16;
constexpr int kTcThreads = 32 * (2 + kTcConsumerWarps);
constexpr int kTcTmemCols = 2 * kTcSub * kTcCols;   // all of the SM's tensor memory
constexpr int kTcTilesPerItem = 32;
constexpr int kTcSmemBudget = 200 * 1024;
// Dynamic shared memory of at least this size keeps one CTA per SM, so the
// 512 TMEM columns of a CTA are always free.
constexpr int kTcMinSmem = 116 * 1024;

__host__ __device__ constexpr int tc_k(int M) { return ((3 * M + 7) / 8) * 8; }
// floats of one packed direction tile: MMA image, then FP32 coordinates (M, 128)
__host__ __device__ constexpr int tc_tile_floats(int M) { return kTcCols * (tc_k(M) + M); }
// floats of one 128-row point tile; the CTA holds two buffers of kTcSub of them
__host__ __device__ constexpr int tc_a_floats(int M) { return kTcRows * tc_k(M); }
__host__ __device__ constexpr int tc_a_bytes(int M) { return 2 * kTcSub * 4 * tc_a_floats(M); }
__host__ __device__ constexpr int tc_stages(int M)
{
    return (kTcSmemBudget - tc_a_bytes(M)) / (4 * tc_tile_floats(M)) > 6
               ? 6
               : (kTcSmemBudget - tc_a_bytes(M)) / (4 * tc_tile_floats(M));
}
__host__ __device__ constexpr int tc_smem(int M)
{
    return tc_a_bytes(M) + 4 * tc_stages(M) * tc_tile_floats(M) > kTcMinSmem
               ? tc_a_bytes(M) + 4 * tc_stages(M) * tc_tile_floats(M)
               : kTcMinSmem;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long tc_now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Round a finite FP32 value to TF32 (10 explicit mantissa bits), to nearest
// with ties away from zero; |v - result| <= 2^-11 |v|.  The tensor core reads
// exactly these bits.  Non-finite values become 0 (their rows are re-scored
// against every direction).
__device__ __forceinline__ float tf32_round(float v)
{
    if (!isfinite(v)) return 0.0f;
    return __uint_as_float((__float_as_uint(v) + 0x1000u) & 0xFFFFE000u);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase of this parity to complete; false after limit_ns
// (about 1 s in the association kernel).
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long limit_ns = 1000000000ull)
{
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = tc_now_ns();
    while (!mbar_try(bar, parity))
        if (tc_now_ns() - t0 > limit_ns) return false;
    return true;
}

// The same wait by every lane of a warp; true only if it completed for all.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity)
{
    return __all_sync(0xFFFFFFFFu, mbar_wait(bar, parity));
}

__device__ __forceinline__ bool mbar_wait_warp_limit(uint64_t* bar, uint32_t parity, unsigned long long limit_ns)
{
    return __all_sync(0xFFFFFFFFu, mbar_wait(bar, parity, limit_ns));
}

// One contiguous global -> shared copy by the bulk-copy engine, completing
// `bytes` of transaction count on bar (addresses 16-byte aligned, size a
// multiple of 16).
__device__ __forceinline__ void bulk_copy_g2s(float* dst, const float* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory matrix descriptor (sm_100): start address, LBO and SBO in
// 16-byte units at bits 0, 16 and 32, descriptor version 1 at bit 46, base
// offset 0, layout type 0 (no swizzle) at bits 61-63.
__device__ __forceinline__ uint64_t smem_desc(const float* p, uint32_t lbo, uint32_t sbo)
{
    const uint32_t addr = smem_u32(p);
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator (bits 4-5 = 1), A and
// B TF32 (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcCols >> 3) << 17) |
                              ((uint32_t)(kTcRows >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate)
{
    const uint32_t z = 0;  // no output lane disabled
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(kTcIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// Arrive on bar once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void tc_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: lane
// = TMEM lane base of the warp + lane id), waited for in the same statement so
// that no use of the registers can be scheduled before the wait.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float (&v)[32])
{
    uint32_t u[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7]),
          "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15]),
          "=r"(u[16]), "=r"(u[17]), "=r"(u[18]), "=r"(u[19]), "=r"(u[20]), "=r"(u[21]), "=r"(u[22]), "=r"(u[23]),
          "=r"(u[24]), "=r"(u[25]), "=r"(u[26]), "=r"(u[27]), "=r"(u[28]), "=r"(u[29]), "=r"(u[30]), "=r"(u[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(u[k]);
}

// Packs the directions (M,H) into tiles of kTcCols directions, one float4 per
// thread.  Tile t: first the MMA image -- row r, K columns 4 kc .. 4 kc + 3 of
// [r_hi (M), r_lo (M), r_hi (M), 0 ...] at float offset
// (r >> 3) * 8 KP + kc * 32 + (r & 7) * 4 -- then the FP32 coordinates
// (M, kTcCols).  Directions past H are zero.
__global__ void tc_pack_directions(const float* __restrict__ refs, int M, int H, int KP, int T,
                                   float* __restrict__ out)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int image = kTcCols * KP / 4;                 // float4 of the MMA image
    const int per_tile = image + kTcCols * M / 4;
    if (c >= (long long)T * per_tile) return;
    const int t = (int)(c / per_tile), rem = (int)(c % per_tile);
    float e[4];
    if (rem < image) {
        const int g = rem / (2 * KP), w = rem % (2 * KP);
        const int kc = w >> 3, r = (g << 3) | (w & 7);
        const int j = t * kTcCols + r;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = 4 * kc + q;
            float val = 0.0f;
            if (j < H && k < 3 * M) {
                const int m = k % M;
                const float v = refs[(size_t)m * H + j];
                const float hi = tf32_round(v);
                val = (k >= M && k < 2 * M) ? tf32_round((isfinite(v) ? v : 0.0f) - hi) : hi;
            }
            e[q] = val;
        }
    } else {
        const int f = rem - image;
        const int m = f / (kTcCols / 4), c4 = f % (kTcCols / 4);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = t * kTcCols + 4 * c4 + q;
            e[q] = j < H ? refs[(size_t)m * H + j] : 0.0f;
        }
    }
    reinterpret_cast<float4*>(out)[c] = make_float4(e[0], e[1], e[2], e[3]);
}

// pass 1: row_max[i] <- max_j |a_ij| (FP32 bits; the caller zeroes it first).
// pass 2: re-score the candidates of the threshold of row_max[i]; packed
// (d2, j) minima into best_out.
template <int M>
__global__ void __launch_bounds__(kTcThreads, 1)
assoc_tensor(const float* __restrict__ x, int x_stride, const float* __restrict__ scale, int H,
             const float* __restrict__ packed, int T, int tiles_per_item, int splits, const int* __restrict__ d_n,
             int pass, unsigned* __restrict__ row_max, unsigned long long* __restrict__ best_out,
             int* __restrict__ status)
{
    constexpr int KP = tc_k(M);
    constexpr int TF = tc_tile_floats(M);
    constexpr int AF = tc_a_floats(M);
    constexpr int S = tc_stages(M);
    static_assert(S >= 2, "at least two direction stages");
    extern __shared__ float4 s_dyn[];
    float* sA = reinterpret_cast<float*>(s_dyn);   // [2 buffers][kTcSub point tiles]
    float* sB = sA + 2 * kTcSub * AF;              // S direction tiles
    __shared__ uint64_t bar_bfull[S], bar_bempty[S], bar_afull[2], bar_aempty[2], bar_accfull[2], bar_accempty[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;

    const int n = *d_n;
    const int P = (n + kTcItemRows - 1) / kTcItemRows;
    const int items = P * splits;
    if ((int)blockIdx.x >= items) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // pass 1 needs only the MMA image of a tile, pass 2 also its FP32 coordinates
    const uint32_t tile_bytes = pass == 1 ? (uint32_t)(KP * kTcCols * 4) : (uint32_t)(TF * 4);

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&bar_bfull[s], 1);
            mbar_init(&bar_bempty[s], 1 + kTcConsumerWarps);   // the MMA's commit + every consumer warp
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&bar_afull[a], kTcConsumerWarps / 2);    // the point-tile writer warps
            mbar_init(&bar_aempty[a], 1);
            mbar_init(&bar_accfull[a], 1);
            mbar_init(&bar_accempty[a], kTcConsumerWarps);
        }
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const float delta = packed[(size_t)T * TF];
    volatile int* abort_flag = &s_abort;
    auto fail = [&]() {
        *abort_flag = 1;
        atomicExch(status, kDevTensorTimeout);
    };

    // Every role walks the same sequence: items k = blockIdx.x + i * gridDim.x,
    // each with its direction tiles [t0, t1).
    if (warp == 0) {
        // ---- direction tiles into the stage ring
        if (lane == 0) {
            uint32_t gl = 0;
            int last_use[S];
            for (int s = 0; s < S; ++s) last_use[s] = -1;
            bool stop = false;
            for (int k = blockIdx.x; k < items && !stop; k += gridDim.x) {
                const int t0 = (k % splits) * tiles_per_item, t1 = min(T, t0 + tiles_per_item);
                for (int t = t0; t < t1; ++t, ++gl) {
                    const int s = (int)(gl % S);
                    const uint32_t use = gl / S;
                    if (*abort_flag || !mbar_wait(&bar_bempty[s], (use & 1u) ^ 1u)) {
                        if (!*abort_flag) fail();
                        stop = true;
                        break;
                    }
                    mbar_expect_tx(&bar_bfull[s], tile_bytes);
                    bulk_copy_g2s(sB + (size_t)s * TF, packed + (size_t)t * TF, tile_bytes, &bar_bfull[s]);
                    last_use[s] = (int)use;
                }
            }
            if (*abort_flag)  // let the copies in flight land before the CTA exits
                for (int s = 0; s < S; ++s)
                    if (last_use[s] >= 0) mbar_wait(&bar_bfull[s], (uint32_t)last_use[s] & 1u);
        }
    } else if (warp == 1) {
        // ---- MMAs: point tiles x direction tile -> accumulators
        if (lane == 0) {
            uint32_t g = 0, il = 0;
            int last_use[S], last_a[2] = {-1, -1};
            for (int s = 0; s < S; ++s) last_use[s] = -1;
            bool stop = false;
            for (int k = blockIdx.x; k < items && !stop; k += gridDim.x, ++il) {
                const int ab = il & 1;
                if (*abort_flag || !mbar_wait(&bar_afull[ab], (il >> 1) & 1u)) {
                    if (!*abort_flag) fail();
                    break;
                }
                tc_fence_after();
                const int t0 = (k % splits) * tiles_per_item, t1 = min(T, t0 + tiles_per_item);
                for (int t = t0; t < t1; ++t, ++g) {
                    const int s = (int)(g % S), b = (int)(g & 1u);
                    if (*abort_flag || !mbar_wait(&bar_bfull[s], (g / S) & 1u) ||
                        !mbar_wait(&bar_accempty[b], ((g >> 1) & 1u) ^ 1u)) {
                        if (!*abort_flag) fail();
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t b_desc = smem_desc(sB + (size_t)s * TF, 128, KP * 32);
#pragma unroll
                    for (int a = 0; a < kTcSub; ++a) {
                        const uint64_t a_desc = smem_desc(sA + (ab * kTcSub + a) * AF, 128, KP * 32);
                        const uint32_t d = tmem + (uint32_t)((b * kTcSub + a) * kTcCols);
#pragma unroll
                        for (int kk = 0; kk < KP / 8; ++kk)
                            tc_mma(d, a_desc + 16u * kk, b_desc + 16u * kk, kk > 0 ? 1u : 0u);
                    }
                    tc_commit(&bar_accfull[b]);
                    tc_commit(&bar_bempty[s]);
                    last_use[s] = (int)(g / S);
                }
                if (!stop) {
                    tc_commit(&bar_aempty[ab]);
                    last_a[ab] = (int)(il >> 1);
                }
            }
            // every MMA issued has completed before the accumulators are freed,
            // and every commit has arrived before the CTA's shared memory goes
            if (g > 0) mbar_wait(&bar_accfull[(g - 1) & 1u], ((g - 1) >> 1) & 1u);
            if (!*abort_flag) {
                for (int s = 0; s < S; ++s)
                    if (last_use[s] >= 0) mbar_wait(&bar_bempty[s], (uint32_t)last_use[s] & 1u);
                for (int a = 0; a < 2; ++a)
                    if (last_a[a] >= 0) mbar_wait(&bar_aempty[a], (uint32_t)last_a[a] & 1u);
            }
        }
    } else {
        // ---- consumers: point tile writers, then the pass's epilogue
        const int q = warp & 3;                  // TMEM sub-partition of this warp
        const int sub = (warp - 2) >> 3;         // point tile
        const int half = ((warp - 2) >> 2) & 1;  // 64-column half of each direction tile
        const int row = q * 32 + lane;
        const uint32_t lane_base = (uint32_t)(q * 32) << 16;
        uint32_t g = 0, il = 0;
        bool stop = false;
        for (int k = blockIdx.x; k < items && !stop; k += gridDim.x, ++il) {
            const int ab = il & 1;
            const int i = (k / splits) * kTcItemRows + sub * kTcRows + row;
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
            if (half == 0) {
                if (*abort_flag || !mbar_wait_warp(&bar_aempty[ab], ((il >> 1) & 1u) ^ 1u)) {
                    if (!*abort_flag && lane == 0) fail();
                    break;
                }
                float hi[M], lo[M];
#pragma unroll
                for (int m = 0; m < M; ++m) {
                    hi[m] = tf32_round(xr[m]);
                    lo[m] = tf32_round((isfinite(xr[m]) ? xr[m] : 0.0f) - hi[m]);
                }
                float* a = sA + (ab * kTcSub + sub) * AF + (row >> 3) * (8 * KP) + (row & 7) * 4;
#pragma unroll
                for (int kc = 0; kc < KP / 4; ++kc) {
                    float e[4];
#pragma unroll
                    for (int qq = 0; qq < 4; ++qq) {
                        const int kq = 4 * kc + qq;
                        e[qq] = kq < M       ? hi[kq % M]
                                : kq < 2 * M ? hi[(kq - M) % M]
                                : kq < 3 * M ? lo[(kq - 2 * M) % M]
                                             : 0.0f;
                    }
                    *reinterpret_cast<float4*>(a + kc * 32) = make_float4(e[0], e[1], e[2], e[3]);
                }
                async_proxy_fence();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar_afull[ab]);
            }
            // pass 2: threshold of the point's largest |a_j| over all directions
            float thr = INFINITY;
            if (pass == 2 && valid) {
                const float margin = assoc_margin(M, xx, delta);
                const float err =
                    (4.0f * M + 16.0f) * 4.76837158e-07f * sqrtf(xx) * sqrtf(1.0f + delta) * (1.0f + 1e-6f) + 1e-30f;
                const float lo = fmaxf(__uint_as_float(row_max[i]) - err, 0.0f);
                const float sq = lo * lo * (1.0f - 1e-6f) - margin;
                // margin = inf (non-finite point, far-from-unit directions): every direction
                thr = (margin < INFINITY && sq > 0.0f) ? sqrtf(sq) * (1.0f - 1e-6f) - err : -INFINITY;
            }
            float maxa = 0.0f;
            unsigned long long best = ~0ull;
            const int t0 = (k % splits) * tiles_per_item, t1 = min(T, t0 + tiles_per_item);
            for (int t = t0; t < t1; ++t, ++g) {
                const int s = (int)(g % S), b = (int)(g & 1u);
                // bfull: the stage's FP32 coordinates are visible to this warp too
                if (*abort_flag || !mbar_wait_warp(&bar_accfull[b], (g >> 1) & 1u) ||
                    !mbar_wait_warp(&bar_bfull[s], (g / S) & 1u)) {
                    if (!*abort_flag && lane == 0) fail();
                    stop = true;
                    break;
                }
                tc_fence_after();
                const float* dirs = sB + (size_t)s * TF + KP * kTcCols;   // (M, kTcCols) FP32
                const uint32_t col_base = tmem + lane_base + (uint32_t)((b * kTcSub + sub) * kTcCols + half * 64);
#pragma unroll 1
                for (int h = 0; h < 2; ++h) {
                    const int col0 = half * 64 + h * 32;
                    float w[32];
                    tmem_load32(col_base + (uint32_t)(h * 32), w);
                    if (h == 1) {  // the accumulator is in registers: release it
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&bar_accempty[b]);
                    }
                    // w8[k]: |max| of columns k, k + 8, k + 16, k + 24
                    float w8[8];
#pragma unroll
                    for (int kk = 0; kk < 8; ++kk)
                        w8[kk] = fmaxf(fmaxf(fabsf(w[kk]), fabsf(w[kk + 8])), fmaxf(fabsf(w[kk + 16]), fabsf(w[kk + 24])));
                    const float tmax = fmaxf(fmaxf(fmaxf(w8[0], w8[1]), fmaxf(w8[2], w8[3])),
                                             fmaxf(fmaxf(w8[4], w8[5]), fmaxf(w8[6], w8[7])));
                    if (pass == 1) {
                        maxa = fmaxf(maxa, tmax);
                        continue;
                    }
                    if (!(tmax >= thr)) continue;
                    uint32_t mask = 0u;
#pragma unroll
                    for (int kk = 0; kk < 8; ++kk)
                        if (w8[kk] >= thr) mask |= 0x01010101u << kk;
                    const int j0 = t * kTcCols + col0;
                    const int lim = H - j0;
                    if (lim < 32) mask &= lim > 0 ? ((1u << lim) - 1u) : 0u;
                    while (mask) {
                        const int kk = __ffs((int)mask) - 1;
                        mask &= mask - 1u;
                        float r[M];
#pragma unroll
                        for (int m = 0; m < M; ++m) r[m] = dirs[m * kTcCols + col0 + kk];
                        float dot = 0.0f;
#pragma unroll
                        for (int m = 0; m < M; ++m) dot = fmaf(xr[m], r[m], dot);
                        float d2 = 0.0f;
#pragma unroll
                        for (int m = 0; m < M; ++m) {
                            const float res = fmaf(-dot, r[m], xr[m]);
                            d2 = fmaf(res, res, d2);
                        }
                        if (d2 < INFINITY) {  // the reference keeps only d2 < best, best starting at inf
                            const unsigned long long c =
                                ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)(j0 + kk);
                            best = c < best ? c : best;
                        }
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar_bempty[s]);
            }
            if (valid) {
                if (pass == 1) atomicMax(row_max + i, __float_as_uint(maxa));
                else if (best != ~0ull) atomicMin(best_out + i, best);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols)
                     : "memory");
}

template <int M>
int configure_tensor_kernel()
{
    MOEA_CUDA_TRY(cudaFuncSetAttribute(assoc_tensor<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem(M)));
    return MOEA_OK;
}

int tc_sm_count()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
            sms = 148;
    }
    return sms;
}

template <int M>
void launch_tensor(const float* x, int x_stride, const float* scale, int H, const float* packed, const int* d_n,
                   int n_cap, unsigned* row_max, unsigned long long* best, int* status, cudaStream_t stream)
{
    const int T = ceil_div(H, kTcCols);
    const int p_cap = ceil_div(n_cap, kTcItemRows);
    const int sms = tc_sm_count();
    // items of at most kTcTilesPerItem tiles, and enough of them to fill the SMs
    int splits = ceil_div(T, kTcTilesPerItem);
    const int fill = ceil_div(2 * sms, p_cap);
    if (splits < fill) splits = fill < T ? fill : T;
    const int per_item = ceil_div(T, splits);
    splits = ceil_div(T, per_item);
    const int items_cap = p_cap * splits;
    const int grid = items_cap < sms ? items_cap : sms;
    for (int pass = 1; pass <= 2; ++pass)
        assoc_tensor<M><<<grid, kTcThreads, tc_smem(M), stream>>>(x, x_stride, scale, H, packed, T, per_item,
                                                                 splits, d_n, pass, row_max, best, status);
}

// Self-test of the association's mbarrier wait with a short limit: the
// barrier expects one arrival that never comes, so every warp's wait runs
// out and the kernel records kDevTensorTimeout, as the association kernel
// does before it drains.
__global__ void selftest_mbar_wait(int* status, unsigned long long limit_ns)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const bool ok = mbar_wait_warp_limit(&bar, 0u, limit_ns);
    if (!ok && threadIdx.x == 0) atomicExch(status, kDevTensorTimeout);
}

}  // namespace

bool tensor_directions_ready(const Workspace& ws, const float* d_refs, int M, int H)
{
    return d_refs && ws.tc_src == d_refs && ws.tc_M == M && ws.tc_H == H && ws.tc_dirs;
}

int prepare_tensor_directions(Workspace& ws, const float* d_refs, int M, int H, cudaStream_t stream)
{
    if (!d_refs || M < 1 || M > kMaxObjectives || H < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "tensor association: bad arguments");
    const int KP = tc_k(M), T = ceil_div(H, kTcCols);
    const size_t body = (size_t)T * kTcCols * (KP + M);
    const size_t need = body + 4;  // + delta, padded to 16 bytes
    ws.tc_src = nullptr;
    if (!ws.tc_rowmax) MOEA_CUDA_TRY(cudaMalloc((void**)&ws.tc_rowmax, sizeof(unsigned) * ws.n_max));
    if (need > ws.tc_cap) {
        cudaFree(ws.tc_dirs);
        ws.tc_dirs = nullptr;
        ws.tc_cap = 0;
        MOEA_CUDA_TRY(cudaMalloc((void**)&ws.tc_dirs, sizeof(float) * need));
        ws.tc_cap = need;
    }
    const long long chunks = (long long)body / 4;
    tc_pack_directions<<<ceil_div(chunks, 256), 256, 0, stream>>>(d_refs, M, H, KP, T, ws.tc_dirs);
    MOEA_CUDA_TRY(cudaGetLastError());
    MOEA_TRY(run_dir_delta(d_refs, M, H, ws.tc_dirs + body, stream));
    switch (M) {
#define MOEA_TC_CFG(K) case K: MOEA_TRY(configure_tensor_kernel<K>()); break;
    MOEA_TC_CFG(1) MOEA_TC_CFG(2) MOEA_TC_CFG(3) MOEA_TC_CFG(4)
    MOEA_TC_CFG(5) MOEA_TC_CFG(6) MOEA_TC_CFG(7) MOEA_TC_CFG(8)
    MOEA_TC_CFG(9) MOEA_TC_CFG(10) MOEA_TC_CFG(11) MOEA_TC_CFG(12)
    MOEA_TC_CFG(13) MOEA_TC_CFG(14) MOEA_TC_CFG(15) MOEA_TC_CFG(16)
#undef MOEA_TC_CFG
    default: return set_error(MOEA_ERR_UNSUPPORTED, "tensor association: M=%d", M);
    }
    tc_sm_count();
    ws.tc_src = d_refs;
    ws.tc_M = M;
    ws.tc_H = H;
    return MOEA_OK;
}

int run_associate_tensor(Workspace& ws, const float* x, int x_stride, const float* scale, const float* refs,
                         int M, const int* d_n, int n_cap, int H, int* idx, float* dist, cudaStream_t stream)
{
    if (n_cap <= 0) return MOEA_OK;
    if (!tensor_directions_ready(ws, refs, M, H))
        return set_error(MOEA_ERR_STATE, "tensor association: directions not prepared");
    MOEA_TRY(run_assoc_reset(ws.assoc_best, n_cap, stream));
    MOEA_CUDA_TRY(cudaMemsetAsync(ws.tc_rowmax, 0, sizeof(unsigned) * n_cap, stream));
    int* status = ws.counters + 6;
    switch (M) {
#define MOEA_TC_CASE(K) case K: launch_tensor<K>(x, x_stride, scale, H, ws.tc_dirs, d_n, n_cap, ws.tc_rowmax, ws.assoc_best, status, stream); break;
    MOEA_TC_CASE(1) MOEA_TC_CASE(2) MOEA_TC_CASE(3) MOEA_TC_CASE(4)
    MOEA_TC_CASE(5) MOEA_TC_CASE(6) MOEA_TC_CASE(7) MOEA_TC_CASE(8)
    MOEA_TC_CASE(9) MOEA_TC_CASE(10) MOEA_TC_CASE(11) MOEA_TC_CASE(12)
    MOEA_TC_CASE(13) MOEA_TC_CASE(14) MOEA_TC_CASE(15) MOEA_TC_CASE(16)
#undef MOEA_TC_CASE
    default: return set_error(MOEA_ERR_UNSUPPORTED, "tensor association: M=%d", M);
    }
    MOEA_CUDA_TRY(cudaGetLastError());
    return run_assoc_finish(ws.assoc_best, d_n, n_cap, idx, dist, stream);
}

int selftest_mbar_timeout(Workspace& ws, unsigned long long limit_ns, cudaStream_t stream)
{
    selftest_mbar_wait<<<1, 64, 0, stream>>>(ws.counters + 6, limit_ns);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

}  // namespace moea
