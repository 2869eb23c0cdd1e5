// Built-in test problems (DTLZ family, constrained variants, CSDP) for sm_100a.
//
// Reference: python/csrc/native/src/problem/dtlz/dtlz_kernels.cu:28-1176.
// Objectives are written straight into the objective-major (M,N) layout (the
// reference writes (N,M) and transposes, :748-819).  The g-term reduction
// keeps the reference's summation order -- virtual thread t of a 256-thread
// row accumulates terms t, t+256, ..., each group of 32 folds with a
// shuffle-down tree, and the eight partials are added in order (DTLZ5 folds
// them with a second tree) -- and every formula keeps the reference's
// expression shape (double-precision pi products, the same fused
// multiply-adds), so the FP32 objectives are the reference's bit for bit on
// the GPU.  Rows with at most 256 g-terms use one warp per row; longer rows
// (large D) use one 256-thread block per row reading the row coalesced.
#include <math_constants.h>

#include "internal.cuh"

namespace moea {
namespace {

enum Base { kDTLZ1 = 1, kDTLZ2, kDTLZ3, kDTLZ4, kDTLZ5, kDTLZ6, kDTLZ7, kConvexDTLZ2 };

__host__ __device__ inline int base_kind(int kind)
{
    switch (kind) {
    case 9: return kDTLZ1;    // C1-DTLZ1
    case 10: return kDTLZ3;   // C1-DTLZ3
    case 11: return kDTLZ2;   // C2-DTLZ2
    case 12: return kConvexDTLZ2;
    case 13: return kDTLZ1;   // C3-DTLZ1
    case 14: return kDTLZ4;   // C3-DTLZ4
    default: return kind;
    }
}

// One g-term added to a running partial.
template <int B>
__device__ __forceinline__ float g_accumulate(float thread_sum, float xv)
{
    if (B == kDTLZ1 || B == kDTLZ3) {
        const float val = xv - 0.5f;
        thread_sum += val * val - cosf(20.0f * M_PI * val);
    } else if (B == kDTLZ6) {
        thread_sum += powf(xv, 0.1f);
    } else if (B == kDTLZ7) {
        thread_sum += xv;
    } else {
        const float val = xv - 0.5f;
        thread_sum += val * val;
    }
    return thread_sum;
}

__device__ __forceinline__ float warp_tree(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Final fold of the eight warp partials (lane 0 holds them in ws).
template <int B>
__device__ __forceinline__ float fold_partials(const float* ws)
{
    if (B == kDTLZ5) {
        // warp-0 shuffle tree over the partials, lanes 8..31 zero
        const float a = ws[0] + ws[4], b = ws[1] + ws[5], c = ws[2] + ws[6], d = ws[3] + ws[7];
        return (a + c) + (b + d);
    }
    float total = 0.0f;
#pragma unroll
    for (int w = 0; w < 8; ++w) total += ws[w];
    return total;
}

__device__ __forceinline__ float safe_cos_hp(float v) { return fmaxf(0.0f, cosf(v * M_PI / 2.0f)); }

// Objective m of one row from its g sum; x points at the row.  Each
// objective is the reference's expression for it (dtlz_kernels.cu:28-716),
// evaluated independently, so different threads may compute different m.
template <int B>
__device__ float row_objective(int m, float total_sum, const float* __restrict__ x, int D, int M)
{
    const int k = D - (M - 1);
    if (B == kDTLZ1) {
        const float g = 100.0f * (static_cast<float>(k) + total_sum);
        const float scalar = 0.5f * (1.0f + g);
        float f = scalar;
        for (int j = 0; j < M - 1 - m; ++j) f *= fmaxf(0.0f, fminf(1.0f, x[j]));
        if (m > 0) f *= fmaxf(0.0f, 1.0f - x[M - 1 - m]);
        return f;
    } else if (B == kDTLZ2 || B == kDTLZ3 || B == kConvexDTLZ2 || B == kDTLZ4) {
        const float g = (B == kDTLZ3) ? 100.0f * (static_cast<float>(k) + total_sum) : total_sum;
        float f = 1.0f + g;
        for (int j = 0; j < M - 1 - m; ++j)
            f *= (B == kDTLZ4) ? fmaxf(0.0f, cosf(powf(x[j], 100.0f) * M_PI / 2.0f))
                               : safe_cos_hp(x[j]);
        if (m > 0)
            f *= (B == kDTLZ4) ? sinf(powf(x[M - 1 - m], 100.0f) * M_PI / 2.0f)
                               : sinf(x[M - 1 - m] * M_PI / 2.0f);
        if (B == kConvexDTLZ2) {
            if (m < M - 1) { f = f * f; f = f * f; } else { f = f * f; }
        }
        return f;
    } else if (B == kDTLZ5 || B == kDTLZ6) {
        const float g = total_sum;
        const float denom = 2.0f * (1.0f + g);
        auto theta = [&](int i) -> float {
            if (i == 0) return x[0];
            float t = (1.0f + 2.0f * g * x[i]) / denom;
            if (B == kDTLZ5) t = fmaxf(0.0f, fminf(1.0f, t));
            return t;
        };
        float f = 1.0f + g;
        for (int j = 0; j < M - 1 - m; ++j)
            f *= (B == kDTLZ5) ? fmaxf(0.0f, __cosf(theta(j) * M_PI * 0.5f))
                               : fmaxf(0.0f, cosf(theta(j) * M_PI * 0.5f));
        if (m > 0)
            f *= (B == kDTLZ5) ? __sinf(theta(M - 1 - m) * M_PI * 0.5f)
                               : sinf(theta(M - 1 - m) * M_PI * 0.5f);
        return f;
    } else {  // kDTLZ7
        if (m < M - 1) return x[m];
        const float g = 1.0f + (9.0f / static_cast<float>(k)) * total_sum;
        float h_sum = 0.0f;
        for (int i = 0; i < M - 1; ++i) {
            const float fi = x[i];
            h_sum += (fi / (1.0f + g)) * (1.0f + sinf(3.0f * M_PI * fi));
        }
        const float h = static_cast<float>(M) - h_sum;
        return (1.0f + g) * h;
    }
}

// One warp per row; valid when the row has at most 256 g-terms.
template <int B>
__device__ __forceinline__ void dtlz_warp_row(int row, int lane, const float* __restrict__ vars, int N,
                                              int D, int M, float* __restrict__ objs)
{
    const float* x = vars + (size_t)row * D;
    const int start = (B == kDTLZ7) ? D - (D - M + 1) : M - 1;
    const int k = D - start;
    float ws[8];
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const int t = lane + 32 * w;
        float a = 0.0f;
        if (t < k) a = g_accumulate<B>(a, x[start + t]);
        ws[w] = warp_tree(a);
    }
    float total = (lane == 0) ? fold_partials<B>(ws) : 0.0f;
    total = __shfl_sync(0xFFFFFFFFu, total, 0);
    if (lane < M) objs[(size_t)lane * N + row] = row_objective<B>(lane, total, x, D, M);
}

template <int B>
__global__ void __launch_bounds__(256)
dtlz_warp_rows(const float* __restrict__ vars, int N, int D, int M, float* __restrict__ objs)
{
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (row >= N) return;
    dtlz_warp_row<B>(row, threadIdx.x & 31, vars, N, D, M, objs);
}

// Fused batch: offspring objectives of every instance (blockIdx.y), problem
// kinds 1..8 with at most 256 g-terms; their constraint violation is zero.
__global__ void __launch_bounds__(256) fused_dtlz(const BatchInst* __restrict__ insts,
                                                  const int* __restrict__ ids)
{
    const BatchInst& I = insts[ids[blockIdx.y]];
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (row >= I.N) return;
    const int lane = threadIdx.x & 31;
    switch (I.kind) {
    case kDTLZ1: dtlz_warp_row<kDTLZ1>(row, lane, I.varsO, I.N, I.D, I.M, I.objsO); break;
    case kDTLZ2: dtlz_warp_row<kDTLZ2>(row, lane, I.varsO, I.N, I.D, I.M, I.objsO); break;
    case kDTLZ3: dtlz_warp_row<kDTLZ3>(row, lane, I.varsO, I.N, I.D, I.M, I.objsO); break;
    case kDTLZ4: dtlz_warp_row<kDTLZ4>(row, lane, I.varsO, I.N, I.D, I.M, I.objsO); break;
    case kDTLZ5: dtlz_warp_row<kDTLZ5>(row, lane, I.varsO, I.N, I.D, I.M, I.objsO); break;
    case kDTLZ6: dtlz_warp_row<kDTLZ6>(row, lane, I.varsO, I.N, I.D, I.M, I.objsO); break;
    case kDTLZ7: dtlz_warp_row<kDTLZ7>(row, lane, I.varsO, I.N, I.D, I.M, I.objsO); break;
    case kConvexDTLZ2: dtlz_warp_row<kConvexDTLZ2>(row, lane, I.varsO, I.N, I.D, I.M, I.objsO); break;
    default: break;
    }
    if (lane == 0) I.cvO[row] = 0.0f;
}

// One 256-thread block per row, the reference's strided accumulation.
template <int B>
__global__ void __launch_bounds__(256)
dtlz_block_rows(const float* __restrict__ vars, int N, int D, int M, float* __restrict__ objs)
{
    const int row = blockIdx.x;
    if (row >= N) return;
    const float* x = vars + (size_t)row * D;
    const int start = (B == kDTLZ7) ? D - (D - M + 1) : M - 1;
    const int k = D - start;
    float a = 0.0f;
    for (int i = threadIdx.x; i < k; i += 256) a = g_accumulate<B>(a, __ldg(x + start + i));
    a = warp_tree(a);
    __shared__ float ws[8];
    __shared__ float s_total;
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        float w8[8];
        for (int w = 0; w < 8; ++w) w8[w] = ws[w];
        s_total = fold_partials<B>(w8);
    }
    __syncthreads();
    if ((int)threadIdx.x < M) objs[(size_t)threadIdx.x * N + row] = row_objective<B>(threadIdx.x, s_total, x, D, M);
}

// Constraint violation from the objectives (dtlz_kernels.cu:824-1090).
__global__ void cv_kernel(int kind, const float* __restrict__ objs, int N, int M, float R,
                          float* __restrict__ cvout)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float* f = objs + i;  // f[m * N]
    float cv = 0.0f;
    switch (kind) {
    case 9: {
        float constraint = f[(size_t)(M - 1) * N] / 0.6f;
        for (int m = 0; m < M - 1; m++) {
            const float f_m = f[(size_t)m * N];
            constraint += f_m / 0.5f;
        }
        cv = fmaxf(constraint - 1.0f, 0.0f);
        break;
    }
    case 10: {
        const float R_sqr = R * R;
        float fv_sqr = 0.0f;
        for (int m = 0; m < M; m++) {
            const float f_m = f[(size_t)m * N];
            fv_sqr += f_m * f_m;
        }
        cv = fmaxf((fv_sqr - 16.0f) * (R_sqr - fv_sqr), 0.0f);
        break;
    }
    case 11: {
        const float inv_sqrt_M = 1.0f / sqrtf((float)M);
        const float r2 = R * R;
        const float inv_r2 = 1.0f / r2;
        float sum_f2 = 0.0f;
        for (int m = 0; m < M; ++m) {
            const float fm = f[(size_t)m * N];
            sum_f2 = fmaf(fm, fm, sum_f2);
        }
        float min_cv = CUDART_INF_F;
        for (int m = 0; m < M; ++m) {
            const float fm = f[(size_t)m * N];
            const float diff = fm - 1.0f;
            const float dist2 = fmaf(diff, diff, sum_f2 - fm * fm);
            min_cv = fminf(min_cv, dist2 * inv_r2 - 1.0f);
        }
        float center_sum2 = 0.0f;
        for (int m = 0; m < M; ++m) {
            const float df = f[(size_t)m * N] - inv_sqrt_M;
            center_sum2 = fmaf(df, df, center_sum2);
        }
        cv = fmaxf(fminf(min_cv, center_sum2 * inv_r2 - 1.0f), 0.0f);
        break;
    }
    case 12: {
        const float inv_M = 1.0f / static_cast<float>(M);
        const float inv_R_sqr = 1.0f / (R * R);
        float sum = 0.0f, sum_sq = 0.0f;
        for (int m = 0; m < M; m++) {
            const float f_m = f[(size_t)m * N];
            sum += f_m;
            sum_sq += f_m * f_m;
        }
        const float mean = sum * inv_M;
        const float variance = sum_sq - static_cast<float>(M) * mean * mean;
        cv = fmaxf(1.0f - variance * inv_R_sqr, 0.0f);
        break;
    }
    case 13: {
        float fv_sum = 0.0f;
        for (int m = 0; m < M; m++) fv_sum += f[(size_t)m * N];
        fv_sum *= 2.0f;
        for (int m = 0; m < M; m++) {
            float c = f[(size_t)m * N] + 1.0f - fv_sum;
            cv += fmaxf(c, 0.0f);
        }
        break;
    }
    case 14: {
        float fv_sqr = 0.0f;
        for (int m = 0; m < M; m++) {
            const float f_m = f[(size_t)m * N];
            fv_sqr += f_m * f_m;
        }
        for (int m = 0; m < M; m++) {
            const float f_m = f[(size_t)m * N];
            float c = 0.75f * (f_m * f_m) - fv_sqr;
            c += 1.0f;
            cv += fmaxf(c, 0.0f);
        }
        break;
    }
    default: break;
    }
    cvout[i] = cv;
}

// CSDP car-side-impact problem (dtlz_kernels.cu:719-747, 1046-1092).
__global__ void csdp_kernel(const float* __restrict__ vars, int N, float* __restrict__ objs,
                            float* __restrict__ cvout)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float* x = vars + (size_t)i * 7;
    const float x1 = x[0], x2 = x[1], x3 = x[2], x4 = x[3], x5 = x[4], x6 = x[5], x7 = x[6];
    {
        const float F = 4.72 - 0.5 * x4 - 0.19 * x2 * x3;
        const float V_MBP = 10.58 - 0.674 * x1 * x2 - 0.67275 * x2;
        const float V_FD = 16.45 - 0.489 * x3 * x7 - 0.843 * x5 * x6;
        objs[i] = 1.98 + 4.9 * x1 + 6.67 * x2 + 6.98 * x3 + 4.01 * x4 + 1.78 * x5 + 0.00001 * x6 + 2.73 * x7;
        objs[(size_t)N + i] = F;
        objs[(size_t)2 * N + i] = 0.5f * (V_MBP + V_FD);
    }
    const float F = 4.72f - 0.5f * x4 - 0.19f * x2 * x3;
    const float V_MBP = 10.58f - 0.674f * x1 * x2 - 0.67275f * x2;
    const float V_FD = 16.45f - 0.489f * x3 * x7 - 0.843f * x5 * x6;
    float g[10];
    g[0] = 1.16f - 0.3717f * x2 * x4 - 0.0092928f * x3 - 1.0f;
    g[1] = 0.261f - 0.0159f * x1 * x2 - 0.06486f * x1 - 0.019f * x2 * x7 + 0.0144f * x3 * x5 + 0.0154464f * x6 - 0.32f;
    g[2] = 0.214f + 0.00817f * x5 - 0.045195f * x1 - 0.0135168f * x1 + 0.03099f * x2 * x6 - 0.018f * x2 * x7
         + 0.007176f * x3 + 0.023232f * x3 - 0.00364f * x5 * x6 - 0.018f * x2 * x2 - 0.32f;
    g[3] = 0.74f - 0.61f * x2 - 0.031296f * x3 - 0.031872f * x7 + 0.227f * x2 * x2 - 0.32f;
    g[4] = 28.98f + 3.818f * x3 - 4.2f * x1 * x2 + 1.27296f * x6 - 2.68065f * x7 - 32.0f;
    g[5] = 33.86f + 2.95f * x3 - 5.057f * x1 * x2 - 3.795f * x2 - 3.4431f * x7 + 1.45728f - 32.0f;
    g[6] = 46.36f - 9.9f * x2 - 4.4505f * x1 - 32.0f;
    g[7] = F - 4.0f;
    g[8] = V_MBP - 9.9f;
    g[9] = V_FD - 15.7f;
    float s = 0.0f;
    for (int j = 0; j < 10; ++j) s += fmaxf(g[j], 0.0f);
    cvout[i] = s;
}

__global__ void zero_kernel(float* p, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = 0.0f;
}

template <int B>
void launch_rows(const float* x, int N, int D, int M, float* objs, cudaStream_t s)
{
    const int k = (B == kDTLZ7) ? D - M + 1 : D - (M - 1);
    if (k <= 256)
        dtlz_warp_rows<B><<<ceil_div(N, 8), 256, 0, s>>>(x, N, D, M, objs);
    else
        dtlz_block_rows<B><<<N, 256, 0, s>>>(x, N, D, M, objs);
}

}  // namespace

int fused_evaluate(const BatchInst* d_inst, const FusedGroup& g, cudaStream_t s)
{
    fused_dtlz<<<dim3(ceil_div(g.max_N, 8), g.count), 256, 0, s>>>(d_inst, g.d_ids);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

namespace {

float cv_radius(int kind, int M)
{
    switch (kind) {
    case 10: return M == 2 ? 6.0f : M == 3 ? 5.0f : M == 5 ? 12.5f : 15.0f;
    case 11: return M == 2 ? 0.15f : M == 3 ? 0.40f : 1.0f;
    case 12: return M == 3 ? 0.20f : M == 5 ? 0.225f : (M == 8 || M == 10) ? 0.26f : M == 15 ? 0.27f : 0.225f;
    default: return 0.0f;
    }
}

}  // namespace

// Validates a built-in problem configuration (problem_factory / dtlz_problem.cu).
int validate_problem(int kind, int D, int M)
{
    if (kind < 1 || kind > 15) return set_error(MOEA_ERR_INVALID_ARGUMENT, "unknown problem kind %d", kind);
    if (M < 1 || M > kMaxObjectives)
        return set_error(MOEA_ERR_UNSUPPORTED, "problem: objectives=%d (1..%d)", M, kMaxObjectives);
    if (kind == 15) {
        if (D != 7 || M != 3) return set_error(MOEA_ERR_INVALID_ARGUMENT, "CSDP requires D=7, M=3");
        return MOEA_OK;
    }
    if (D < M) return set_error(MOEA_ERR_INVALID_ARGUMENT, "problem: dimension %d < objectives %d", D, M);
    if (kind == 10 && !(M == 2 || M == 3 || M == 5 || M == 8 || M == 10 || M == 15))
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "C1-DTLZ3 supports M in {2,3,5,8,10,15}");
    if (kind == 11 && !(M == 2 || M == 3 || M == 5 || M == 8 || M == 10 || M == 15))
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "C2-DTLZ2 supports M in {2,3,5,8,10,15}");
    if (kind == 12 && !(M == 3 || M == 5 || M == 8 || M == 10 || M == 15))
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "C2-ConvexDTLZ2 supports M in {3,5,8,10,15}");
    return MOEA_OK;
}

int run_problem(int kind, const float* x, int N, int D, int M, float* objs, float* cv,
                cudaStream_t s)
{
    MOEA_TRY(validate_problem(kind, D, M));
    if (N <= 0) return MOEA_OK;
    if (kind == 15) {
        csdp_kernel<<<ceil_div(N, 256), 256, 0, s>>>(x, N, objs, cv);
        MOEA_CUDA_TRY(cudaGetLastError());
        return MOEA_OK;
    }
    switch (base_kind(kind)) {
    case kDTLZ1: launch_rows<kDTLZ1>(x, N, D, M, objs, s); break;
    case kDTLZ2: launch_rows<kDTLZ2>(x, N, D, M, objs, s); break;
    case kDTLZ3: launch_rows<kDTLZ3>(x, N, D, M, objs, s); break;
    case kDTLZ4: launch_rows<kDTLZ4>(x, N, D, M, objs, s); break;
    case kDTLZ5: launch_rows<kDTLZ5>(x, N, D, M, objs, s); break;
    case kDTLZ6: launch_rows<kDTLZ6>(x, N, D, M, objs, s); break;
    case kDTLZ7: launch_rows<kDTLZ7>(x, N, D, M, objs, s); break;
    case kConvexDTLZ2: launch_rows<kConvexDTLZ2>(x, N, D, M, objs, s); break;
    default: return set_error(MOEA_ERR_INVALID_ARGUMENT, "unknown problem kind %d", kind);
    }
    if (kind >= 9)
        cv_kernel<<<ceil_div(N, 256), 256, 0, s>>>(kind, objs, N, M, cv_radius(kind, M), cv);
    else
        zero_kernel<<<ceil_div(N, 256), 256, 0, s>>>(cv, N);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

}  // namespace moea

extern "C" moea_status moea_problem_evaluate(int kind, const float* d_x, int N, int D, int M,
                                             float* d_objs, float* d_cv, void* stream)
{
    if (!d_x || !d_objs || !d_cv || N < 0)
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "problem_evaluate: bad arguments");
    return moea::run_problem(kind, d_x, N, D, M, d_objs, d_cv, (cudaStream_t)stream);
}
