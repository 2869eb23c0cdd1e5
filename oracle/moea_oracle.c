/*
 * CPU oracle for the CUDA-MOEA generation hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates the reference algorithm so that the CUDA kernels of the
 * product can be checked against it.  Nothing in the product links or calls it;
 * tests/, the smoke check and the CPU-baseline leg of bench.py load it through
 * oracle/oracle.py.
 *
 * Floating-point policy.  Built with -ffp-contract=off: every fused
 * multiply-add that the reference's nvcc build forms (explicit fmaf, or a
 * single-use product feeding an add/sub, which nvcc contracts by default) is
 * written as fmaf() here, everything else rounds per operation.  Transcendental
 * functions come from the host libm, so stages that use cosf/sinf/powf/acosf/
 * rsqrtf agree with the GPU to a few ulp, not bit for bit; the integer stages
 * (dominance, fronts, sorting keys, niching, elitism) are exact.
 *
 * Paths cited as `nat/...` are relative to python/csrc/native/ of CUDA-MOEA.
 */
#include "moea_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_INF (INFINITY)

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* ======================================================================== */
/* random numbers                                                           */
/* ======================================================================== */

/* nat/src/core/cuda/cuda_random.cu:1606-1613 */
uint32_t orc_splitmix_u32(uint64_t counter, uint64_t seed)
{
    uint64_t z = counter ^ seed;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (uint32_t)z;
}

/* nat/src/core/cuda/cuda_manager.cu:27-40 (island 0) */
uint64_t orc_derive_seed(uint64_t seed)
{
    uint64_t x = seed;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

/* Philox4x32-10, Salmon et al., "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11: ten rounds of two 32x32->64 multiplies with the Weyl key schedule. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void orc_philox_stream(uint64_t seed, uint32_t generation, uint32_t tag,
                       int64_t count, uint32_t* out)
{
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < count; ++e) {
        const uint32_t ctr[4] = {(uint32_t)e, (uint32_t)((uint64_t)e >> 32), generation, tag};
        orc_philox4x32_10(ctr, key, out + 4 * e);
    }
}

/* ======================================================================== */
/* stable sort of (uint64 key, int value) pairs                             */
/* ======================================================================== */

typedef struct { uint64_t key; int pos; int val; } kv_t;

static int kv_cmp(const void* a, const void* b)
{
    const kv_t* x = (const kv_t*)a;
    const kv_t* y = (const kv_t*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

/* Stable ascending sort of keys with their values (CUB radix sort semantics). */
static void stable_sort_kv(uint64_t* keys, int* vals, int n)
{
    if (n <= 1) return;
    kv_t* t = (kv_t*)malloc(sizeof(kv_t) * (size_t)n);
    for (int i = 0; i < n; ++i) { t[i].key = keys[i]; t[i].pos = i; t[i].val = vals[i]; }
    qsort(t, (size_t)n, sizeof(kv_t), kv_cmp);
    for (int i = 0; i < n; ++i) { keys[i] = t[i].key; vals[i] = t[i].val; }
    free(t);
}

static int int_cmp(const void* a, const void* b)
{
    const int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* ======================================================================== */
/* non-dominated sorting                                                    */
/* ======================================================================== */

/* Constraint dominance of p over q; feasibility is cv == 0 exactly
 * (non_dominated_sort.cu:190-239, cuda_globals.cuh FEASIBLE_CV). */
int orc_dominates(const float* cv, const float* objs, int M, int n, int p, int q)
{
    if (p == q) return 0;
    const float cp = cv[p], cq = cv[q];
    const int pf = (cp == 0.0f), qf = (cq == 0.0f);
    if (pf && !qf) return 1;
    if (!pf && !qf) return cp < cq;
    if (!pf) return 0;
    int le = 1, lt = 0;
    for (int m = 0; m < M; ++m) {
        const float a = objs[(size_t)m * n + p], b = objs[(size_t)m * n + q];
        le &= (a <= b);
        lt |= (a < b);
    }
    return le && lt;
}

int orc_ndsort(const float* cv, const float* objs, int M, int n, int target, int* fronts)
{
    for (int i = 0; i < n; ++i) fronts[i] = -1;
    if (n <= 0) return 0;
    int* cnt = (int*)malloc(sizeof(int) * (size_t)n);
    int* cur = (int*)malloc(sizeof(int) * (size_t)n);
    int* nxt = (int*)malloc(sizeof(int) * (size_t)n);
    #pragma omp parallel for schedule(dynamic, 64)
    for (int q = 0; q < n; ++q) {
        int c = 0;
        for (int p = 0; p < n; ++p) c += orc_dominates(cv, objs, M, n, p, q);
        cnt[q] = c;
    }
    int ncur = 0;
    for (int q = 0; q < n; ++q) if (cnt[q] == 0) { fronts[q] = 0; cur[ncur++] = q; }
    int assigned = ncur, k = 0;
    while (assigned < target && ncur > 0) {
        /* peel front k: dominatees whose count drops to zero form front k+1 */
        #pragma omp parallel for schedule(dynamic, 64)
        for (int q = 0; q < n; ++q) {
            if (fronts[q] != -1) continue;
            int dec = 0;
            for (int i = 0; i < ncur; ++i) dec += orc_dominates(cv, objs, M, n, cur[i], q);
            cnt[q] -= dec;
        }
        int nn = 0;
        for (int q = 0; q < n; ++q)
            if (fronts[q] == -1 && cnt[q] == 0) { fronts[q] = k + 1; nxt[nn++] = q; }
        ++k;
        assigned += nn;
        int* t = cur; cur = nxt; nxt = t; ncur = nn;
    }
    free(cnt); free(cur); free(nxt);
    return k;
}

/* ======================================================================== */
/* NSGA-III selection stages                                                */
/* ======================================================================== */

void orc_nds_extract(const int* fronts, int n_mix, int max_front, int N,
                     int* nds_gidx, int sizes[4])
{
    int np = 0, nl = 0;
    for (int i = 0; i < n_mix; ++i) {
        if (fronts[i] >= 0 && fronts[i] < max_front) ++np;
        else if (fronts[i] == max_front) ++nl;
    }
    int a = 0, b = np;
    for (int i = 0; i < n_mix; ++i) {
        if (fronts[i] >= 0 && fronts[i] < max_front) nds_gidx[a++] = i;
        else if (fronts[i] == max_front) nds_gidx[b++] = i;
    }
    sizes[0] = np; sizes[1] = nl; sizes[2] = N - np; sizes[3] = np + nl;
}

void orc_ideal_point(const float* objs, int M, int n, float* ideal)
{
    for (int m = 0; m < M; ++m) {
        float z = ORC_INF;
        for (int i = 0; i < n; ++i) z = fminf(z, objs[(size_t)m * n + i]);
        ideal[m] = z;
    }
}

/* One-sided Jacobi SVD of the square matrix a (n x n, row-major, FP64).
 * On return the columns of a hold U*Sigma, v holds V, sigma the column norms.
 * Returns 1 (ill-conditioned, nothing else set) when the column norms fail
 * the conditioning test before convergence. */
static int jacobi_svd(double* a, double* v, double* sigma, int n)
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) v[i * n + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 60; ++sweep) {
        /* column norms only spread under rotations (each pair ends at the
         * eigenvalues of its 2x2 Gram matrix): once they fail the
         * conditioning test the result is the fallback, so stop */
        double cmax = 0.0, cmin = INFINITY;
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += a[k * n + i] * a[k * n + i];
            cmax = fmax(cmax, sqrt(s));
            cmin = fmin(cmin, sqrt(s));
        }
        if (cmin < 1e-10 || cmax / cmin > 1e6) return 1;
        /* round-robin order (circle method over P = n rounded up to even
         * columns, column P - 1 a bye when n is odd): in round r column
         * P - 1 meets column r and, for k >= 1, (r + k) mod (P - 1) meets
         * (r - k) mod (P - 1); the pairs of a round share no column, so the
         * GPU rotates them at once and the order inside a round is free */
        int rotated = 0;
        const int P = (n + 1) & ~1;
        for (int r = 0; r < P - 1; ++r) {
            for (int k = 0; k < P / 2; ++k) {
                int i = (k == 0) ? r : (r + k) % (P - 1);
                int j = (k == 0) ? P - 1 : (r - k + (P - 1)) % (P - 1);
                if (i > j) { const int tmp = i; i = j; j = tmp; }
                if (j >= n) continue;  /* the bye */
                double al = 0.0, be = 0.0, ga = 0.0;
                for (int q = 0; q < n; ++q) {
                    const double x = a[q * n + i], y = a[q * n + j];
                    al += x * x; be += y * y; ga += x * y;
                }
                if (ga == 0.0 || fabs(ga) <= 1e-15 * sqrt(al * be)) continue;
                rotated = 1;
                const double zeta = (be - al) / (2.0 * ga);
                const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / sqrt(1.0 + t * t);
                const double s = c * t;
                for (int q = 0; q < n; ++q) {
                    const double x = a[q * n + i], y = a[q * n + j];
                    a[q * n + i] = c * x - s * y;
                    a[q * n + j] = s * x + c * y;
                    const double vx = v[q * n + i], vy = v[q * n + j];
                    v[q * n + i] = c * vx - s * vy;
                    v[q * n + j] = s * vx + c * vy;
                }
            }
        }
        if (!rotated) break;
    }
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += a[k * n + i] * a[k * n + i];
        sigma[i] = sqrt(s);
    }
    return 0;
}

/* Reciprocal intercepts from the extreme points (normalization.cu:739-856,
 * 1302-1394).  A has one row per extreme point: A[j][m] = f'_m(extreme_j).
 * Returns 1 for the ill-conditioned fallback. */
static int intercepts_fp64(const float* E /* row-major [m][j] */, int M, double* rcp)
{
    double a[16 * 16], v[16 * 16], sg[16];
    for (int j = 0; j < M; ++j)
        for (int m = 0; m < M; ++m) {
            const float e = E[m * M + j];
            if (!isfinite(e)) return 1;
            a[j * M + m] = (double)e;
        }
    if (jacobi_svd(a, v, sg, M)) return 1;
    double smax = 0.0, smin = INFINITY;
    for (int i = 0; i < M; ++i) {
        if (!isfinite(sg[i])) return 1;
        smax = fmax(smax, sg[i]);
        smin = fmin(smin, sg[i]);
    }
    if (smin < 1e-10) return 1;
    if (smax / smin > 1e6) return 1;
    /* pinv(A) * 1 = V diag(1/sigma masked) U^T 1, U_i = column_i(a) / sigma_i */
    double coef[16];
    for (int i = 0; i < M; ++i) {
        double ut1 = 0.0;
        for (int k = 0; k < M; ++k) ut1 += a[k * M + i];
        coef[i] = (sg[i] > 1e-5) ? ut1 / (sg[i] * sg[i]) : 0.0;
    }
    for (int m = 0; m < M; ++m) {
        double s = 0.0;
        for (int i = 0; i < M; ++i) s += v[m * M + i] * coef[i];
        rcp[m] = s;
    }
    return 0;
}

int orc_normalize(float* f, const float* ideal, int M, int n, float* rcp_b, int* extreme)
{
    /* translate + clamp (normalization.cu:370-444) */
    for (int m = 0; m < M; ++m)
        for (int i = 0; i < n; ++i) {
            float v = f[(size_t)m * n + i] - ideal[m];
            if (isfinite(v)) v = fmaxf(v, 0.0f);
            f[(size_t)m * n + i] = v;
        }
    /* ASF extreme points, ties to the smaller index (normalization.cu:454-540, 648-729) */
    for (int j = 0; j < M; ++j) {
        float best = ORC_INF; int bi = -1;
        for (int i = 0; i < n; ++i) {
            float mx = -ORC_INF;
            for (int m = 0; m < M; ++m) {
                float v = f[(size_t)m * n + i];
                v = isnan(v) ? ORC_INF : v;
                mx = fmaxf(mx, v * ((m == j) ? 1.0f : 1e6f));
            }
            if (mx < best) { best = mx; bi = i; }
        }
        extreme[j] = bi;
    }
    float E[16 * 16];
    for (int m = 0; m < M; ++m)
        for (int j = 0; j < M; ++j)
            E[m * M + j] = (extreme[j] >= 0) ? f[(size_t)m * n + extreme[j]] : ORC_INF;
    double rcp[16];
    const int ill = intercepts_fp64(E, M, rcp);
    for (int m = 0; m < M; ++m) {
        float r;
        if (!ill) {
            r = (float)rcp[m];
        } else {
            /* row-maximum fallback (normalization.cu:803-856) */
            float mx = -ORC_INF;
            for (int i = 0; i < n; ++i) {
                float v = f[(size_t)m * n + i];
                mx = fmaxf(mx, isnan(v) ? -ORC_INF : v);
            }
            r = (mx > 1e-10f) ? 1.0f / fmaxf(mx, 1e-6f) : 1.0f;
        }
        if (!isfinite(r) || r <= 0.0f) r = 1.0f;  /* sanitize (normalization.cu:572-586) */
        rcp_b[m] = r;
    }
    for (int m = 0; m < M; ++m)
        for (int i = 0; i < n; ++i) f[(size_t)m * n + i] = f[(size_t)m * n + i] * rcp_b[m];
    return ill;
}

void orc_associate(const float* x, const float* refs, int M, int n, int H, int* idx, float* dist)
{
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        float xr[16];
        for (int m = 0; m < M; ++m) xr[m] = x[(size_t)m * n + i];
        float best = ORC_INF; int bj = -1;
        for (int j = 0; j < H; ++j) {
            float dot = 0.0f;
            for (int m = 0; m < M; ++m) dot = fmaf(xr[m], refs[(size_t)m * H + j], dot);
            float d2 = 0.0f;
            for (int m = 0; m < M; ++m) {
                const float r = fmaf(-dot, refs[(size_t)m * H + j], xr[m]);
                d2 = fmaf(r, r, d2);
            }
            if (d2 < best) { best = d2; bj = j; }
        }
        idx[i] = bj;
        dist[i] = (best != ORC_INF) ? sqrtf(best) : ORC_INF;
    }
}

/* segment rank within runs of equal (key >> 32) (cuda_ref_segment_ops.cu:17-45) */
static void segment_rank(const uint64_t* keys, int n, int* rank)
{
    int head = 0;
    for (int t = 0; t < n; ++t) {
        if (t == 0 || (uint32_t)(keys[t] >> 32) != (uint32_t)(keys[t - 1] >> 32)) head = t;
        rank[t] = t - head;
    }
}

void orc_niching(uint64_t seed, uint64_t* offset, const int* nds_gidx,
                 const float* dist, const int* idx, const int sizes[4], int H,
                 int N, int* selected)
{
    const int np = sizes[0], nl = sizes[1], nrem = sizes[2];
    (void)N;
    int* rho = (int*)calloc((size_t)(H > 0 ? H : 1), sizeof(int));
    for (int i = 0; i < np; ++i) {
        selected[i] = nds_gidx[i];
        if (idx[i] >= 0 && idx[i] < H) rho[idx[i]]++;
    }
    if (nrem <= 0 || nl <= 0) { free(rho); return; }
    uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nl);
    int* val = (int*)malloc(sizeof(int) * (size_t)nl);
    int* rk = (int*)malloc(sizeof(int) * (size_t)nl);
    for (int t = 0; t < nl; ++t) {
        key[t] = ((uint64_t)(uint32_t)idx[np + t] << 32) | f2u(dist[np + t]);
        val[t] = t;
    }
    stable_sort_kv(key, val, nl);
    segment_rank(key, nl, rk);
    for (int t = 0; t < nl; ++t) {
        const int ref = (int)(uint32_t)(key[t] >> 32);
        const int rho_r = (ref >= 0 && ref < H) ? rho[ref] : 0;
        const uint32_t r = orc_splitmix_u32(*offset + (uint64_t)t, seed);
        const uint32_t low = (rho_r == 0 && rk[t] == 0) ? 0u : (r | 1u);
        key[t] = ((uint64_t)(uint32_t)ref << 32) | low;
    }
    *offset += (uint64_t)nl;
    stable_sort_kv(key, val, nl);
    segment_rank(key, nl, rk);
    for (int t = 0; t < nl; ++t) {
        const int ref = (int)(uint32_t)(key[t] >> 32);
        const int rho_r = (ref >= 0 && ref < H) ? rho[ref] : 0;
        const uint32_t r = orc_splitmix_u32(*offset + (uint64_t)t, seed);
        key[t] = ((uint64_t)(uint32_t)(rho_r + rk[t]) << 32) | r;
    }
    *offset += (uint64_t)nl;
    stable_sort_kv(key, val, nl);
    for (int i = 0; i < nrem; ++i) selected[np + i] = nds_gidx[np + val[i]];
    free(key); free(val); free(rk); free(rho);
}

void orc_quantize_cv(const float* cv, float* out, int n, float eps_feas,
                     float clip_upper, float log_alpha, int bins)
{
    const float inv_clip_upper = 1.0f / clip_upper;
    const float inv_clip_log = (log_alpha > 0.0f) ? 1.0f / log1pf(log_alpha * clip_upper) : 0.0f;
    for (int i = 0; i < n; ++i) {
        const float raw = cv[i];
        const float u = fminf(fmaxf(raw, 0.0f), clip_upper);
        const float x = (log_alpha > 0.0f) ? log1pf(log_alpha * u) * inv_clip_log : u * inv_clip_upper;
        int bin = 1 + (int)floorf(x * (float)bins);
        if (bin < 1) bin = 1;
        if (bin > bins) bin = bins;
        const int infeas = (eps_feas == 0.0f) ? (raw != 0.0f) : (raw > eps_feas);
        out[i] = infeas ? (float)bin : 0.0f;
    }
}

int orc_nsga3_select(const float* mix_cv, const float* mix_objs, int M, int N,
                     const float* refs, int H, uint64_t seed, uint64_t* offset,
                     float* ideal_last, const float* off_objs_unused,
                     int* survivors, int* survivor_fronts, int sizes_out[4])
{
    (void)off_objs_unused;
    const int n_mix = 2 * N;
    int* fronts = (int*)malloc(sizeof(int) * (size_t)n_mix);
    const int max_front = orc_ndsort(mix_cv, mix_objs, M, n_mix, N, fronts);
    int* gidx = (int*)malloc(sizeof(int) * (size_t)n_mix);
    int sizes[4];
    orc_nds_extract(fronts, n_mix, max_front, N, gidx, sizes);
    const int nds = sizes[3];
    float* f = (float*)malloc(sizeof(float) * (size_t)M * (size_t)(nds > 0 ? nds : 1));
    for (int m = 0; m < M; ++m)
        for (int i = 0; i < nds; ++i) f[(size_t)m * nds + i] = mix_objs[(size_t)m * n_mix + gidx[i]];
    /* ideal point: running minimum over all offspring (ideal_point.cu:97-165) */
    float ideal[16];
    for (int m = 0; m < M; ++m) {
        float z = ORC_INF;
        for (int i = 0; i < N; ++i) z = fminf(z, mix_objs[(size_t)m * n_mix + N + i]);
        ideal[m] = fminf(ideal_last[m], z);
        ideal_last[m] = ideal[m];
    }
    if (sizes[2] > 0) {
        float rcp[16]; int ext[16];
        orc_normalize(f, ideal, M, nds, rcp, ext);
        int* aidx = (int*)malloc(sizeof(int) * (size_t)(nds > 0 ? nds : 1));
        float* adist = (float*)malloc(sizeof(float) * (size_t)(nds > 0 ? nds : 1));
        orc_associate(f, refs, M, nds, H, aidx, adist);
        orc_niching(seed, offset, gidx, adist, aidx, sizes, H, N, survivors);
        free(aidx); free(adist);
    } else {
        for (int i = 0; i < N; ++i) survivors[i] = gidx[i];
    }
    qsort(survivors, (size_t)N, sizeof(int), int_cmp);
    for (int i = 0; i < N; ++i) survivor_fronts[i] = fronts[survivors[i]];
    if (sizes_out) memcpy(sizes_out, sizes, sizeof(sizes));
    free(fronts); free(gidx); free(f);
    return max_front;
}

/* ======================================================================== */
/* RVEA stages                                                              */
/* ======================================================================== */

void orc_rvea_translate(const float* objs, int M, int n, float* out, float* zmin)
{
    for (int m = 0; m < M; ++m) {
        float z = ORC_INF;
        for (int i = 0; i < n; ++i) z = fminf(z, objs[(size_t)m * n + i]);
        zmin[m] = z;
        for (int i = 0; i < n; ++i) out[(size_t)m * n + i] = fmaxf(objs[(size_t)m * n + i] - z, 1e-32f);
    }
}

void orc_rvea_partition(const float* t, const float* refs, int M, int n, int K,
                        int n_active, int n_parent, float* theta, int* idx)
{
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        float x[16], sq = 0.0f;
        for (int m = 0; m < M; ++m) { x[m] = t[(size_t)m * n + i]; sq = fmaf(x[m], x[m], sq); }
        const float inv = 1.0f / sqrtf(sq + 1e-12f);
        float best = -ORC_INF; int bj = -1;
        for (int j = 0; j < K; ++j) {
            float dot = 0.0f;
            for (int m = 0; m < M; ++m) dot = fmaf(x[m], refs[(size_t)m * K + j], dot);
            const float c = dot * inv;
            if (c > best) { best = c; bj = j; }
        }
        theta[i] = (best > -ORC_INF) ? acosf(fminf(fmaxf(best, 0.0f), 1.0f)) : ORC_INF;
        idx[i] = bj;
    }
    for (int i = n_active; i < n_parent; ++i) idx[i] = K;
}

void orc_rvea_gamma(const float* refs, int M, int K, float* gamma)
{
    if (K == 1) { gamma[0] = 3.14159265358979323846f; return; }
    for (int j = 0; j < K; ++j) {
        float mx = -ORC_INF;
        for (int k = 0; k < K; ++k) {
            if (k == j) continue;
            float dot = 0.0f;
            for (int m = 0; m < M; ++m) dot = fmaf(refs[(size_t)m * K + j], refs[(size_t)m * K + k], dot);
            mx = fmaxf(mx, dot);
        }
        gamma[j] = (mx > -ORC_INF) ? acosf(fminf(fmaxf(mx, 0.0f), 1.0f)) : 3.14159265358979323846f;
    }
}

void orc_rvea_apd(const float* t, const float* theta, const float* gamma,
                  const int* idx, int M, int n, int K, int gen, int max_gen,
                  float alpha, float* apd)
{
    const float total = fmaxf((float)max_gen, 1.0f);
    const float progress = fminf(fmaxf((float)gen / total, 0.0f), 1.0f);
    const float ps = (float)M * powf(progress, alpha);
    for (int i = 0; i < n; ++i) {
        float sq = 0.0f;
        for (int m = 0; m < M; ++m) { const float v = t[(size_t)m * n + i]; sq = fmaf(v, v, sq); }
        const float norm = sqrtf(sq);
        if (norm > 1e-12f) {
            const int r = idx[i];
            if (r < 0 || r >= K) { apd[i] = 1e30f; continue; }
            const float th = fminf(fmaxf(theta[i], 0.0f), 3.14159265358979323846f);
            const float ga = fmaxf(gamma[r], 1e-6f);
            const float a = (1.0f + ps * th / ga) * norm;
            apd[i] = (!isfinite(a) || a < 0.0f) ? 1e30f : a;
        } else {
            apd[i] = 0.0f;
        }
    }
}

static inline uint32_t rvea_metric_bits(float cv, float apd, uint32_t* flag)
{
    const int feas = (cv <= 1e-8f);
    float m = feas ? apd : cv;
    if (!(isfinite(m) && m >= 0.0f)) m = 1e30f;
    *flag = feas ? 0u : 1u;
    return f2u(m) & 0x7FFFFFFFu;
}

int orc_rvea_elitism(const int* idx, const float* cv, const float* apd, int N,
                     int n_mix, int K, int* selected)
{
    if (N <= 0 || n_mix <= 0) return 0;
    uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n_mix);
    int* val = (int*)malloc(sizeof(int) * (size_t)n_mix);
    int* rk = (int*)malloc(sizeof(int) * (size_t)n_mix);
    for (int i = 0; i < n_mix; ++i) {
        uint32_t flag;
        const uint32_t mb = rvea_metric_bits(cv[i], apd[i], &flag);
        key[i] = ((uint64_t)(uint32_t)idx[i] << 32) | ((uint64_t)flag << 31) | mb;
        val[i] = i;
    }
    stable_sort_kv(key, val, n_mix);
    segment_rank(key, n_mix, rk);
    int* win = (int*)malloc(sizeof(int) * (size_t)n_mix);
    int nw = 0;
    for (int t = 0; t < n_mix; ++t) {
        const int ref = (int)(uint32_t)(key[t] >> 32);
        if (rk[t] == 0 && ref >= 0 && ref < K) win[nw++] = val[t];
    }
    int active;
    if (nw == 0) {
        for (int i = 0; i < N; ++i) selected[i] = val[i];
        active = N;
    } else if (nw <= N) {
        for (int i = 0; i < nw; ++i) selected[i] = win[i];
        active = nw;
    } else {
        uint64_t* tk = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nw);
        int* tv = (int*)malloc(sizeof(int) * (size_t)nw);
        for (int i = 0; i < nw; ++i) {
            uint32_t flag;
            const uint32_t mb = rvea_metric_bits(cv[win[i]], apd[win[i]], &flag);
            tk[i] = ((uint64_t)flag << 63) | ((uint64_t)mb << 32) | (uint32_t)win[i];
            tv[i] = i;
        }
        stable_sort_kv(tk, tv, nw);
        for (int i = 0; i < N; ++i) selected[i] = win[tv[i]];
        active = N;
        free(tk); free(tv);
    }
    qsort(selected, (size_t)active, sizeof(int), int_cmp);
    free(key); free(val); free(rk); free(win);
    return active;
}

void orc_rvea_adapt(const float* v0, const float* objs, int M, int K,
                    int n_active, int n_stride, float* v)
{
    float range[16];
    for (int m = 0; m < M; ++m) {
        float lo = ORC_INF, hi = -ORC_INF;
        for (int i = 0; i < n_active; ++i) {
            lo = fminf(lo, objs[(size_t)m * n_stride + i]);
            hi = fmaxf(hi, objs[(size_t)m * n_stride + i]);
        }
        float r = hi - lo;
        if (!isfinite(r) || r < 1e-12f) r = 1e-12f;
        range[m] = r;
    }
    for (int j = 0; j < K; ++j) {
        float base[16], sc[16], bs = 0.0f, ss = 0.0f;
        for (int m = 0; m < M; ++m) {
            float b = v0[(size_t)m * K + j];
            if (!isfinite(b)) b = 0.0f;
            base[m] = b; bs = fmaf(b, b, bs);
            float s = b * range[m];
            if (!isfinite(s)) s = 0.0f;
            sc[m] = s; ss = fmaf(s, s, ss);
        }
        const int us = isfinite(ss) && ss > 1e-12f;
        const int ub = isfinite(bs) && bs > 1e-12f;
        const float is = us ? 1.0f / sqrtf(ss) : 0.0f;
        const float ib = ub ? 1.0f / sqrtf(bs) : 0.0f;
        for (int m = 0; m < M; ++m)
            v[(size_t)m * K + j] = us ? sc[m] * is : (ub ? base[m] * ib : (m == 0 ? 1.0f : 0.0f));
    }
}

/* ======================================================================== */
/* reproduction                                                             */
/* ======================================================================== */

void orc_tournament(const int* cand, const int* rank, const float* cv, int n, int* winners)
{
    for (int i = 0; i < n; ++i) {
        const int a = cand[2 * i], b = cand[2 * i + 1];
        const float ca = cv[a], cb = cv[b];
        if (ca == 0.0f && cb != 0.0f) winners[i] = a;
        else if (ca != 0.0f && cb == 0.0f) winners[i] = b;
        else if (ca != 0.0f && cb != 0.0f) winners[i] = (ca <= cb) ? a : b;
        else winners[i] = (rank[a] <= rank[b]) ? a : b;
    }
}

float orc_annealed(float begin, float end, int gen, int total)
{
    float p = 1.0f;
    if (total > 0) {
        p = (float)gen / (float)total;
        p = p < 0.0f ? 0.0f : (p > 1.0f ? 1.0f : p);
    }
    return begin + (end - begin) * p;
}

void orc_sbx(const float* parents, const int* pidx, const float* bounds,
             const float* u, const int* sign, const float* copy, float* off,
             float eta, float prob, float copy_prob, int n_off, int D)
{
    const int pairs = n_off / 2;
    for (int p = 0; p < pairs; ++p) {
        const int ca = 2 * p, cb = ca + 1;
        const int pa = pidx[ca], pb = pidx[cb];
        for (int d = 0; d < D; ++d) {
            const size_t e = (size_t)p * D + d;
            const float x1 = parents[(size_t)pa * D + d], x2 = parents[(size_t)pb * D + d];
            const float u1 = u[2 * e], u2 = u[2 * e + 1];
            if (u2 >= prob || copy[e] < copy_prob) {
                off[(size_t)ca * D + d] = x1;
                off[(size_t)cb * D + d] = x2;
                continue;
            }
            const float power = 1.0f / (1.0f + eta);
            float beta = (u1 < 0.5f) ? powf(2.0f * u1, power)
                                     : powf(1.0f / fmaf(-2.0f, u1, 2.0f), power);
            beta *= (float)(2 * sign[e] - 1);
            const float mid = 0.5f * (x1 + x2);
            const float delta = 0.5f * beta * (x1 - x2);
            const float lo = bounds[2 * d], hi = bounds[2 * d + 1];
            off[(size_t)ca * D + d] = fminf(fmaxf(mid + delta, lo), hi);
            off[(size_t)cb * D + d] = fminf(fmaxf(mid - delta, lo), hi);
        }
    }
    if (n_off % 2) {
        const int c = n_off - 1;
        for (int d = 0; d < D; ++d) off[(size_t)c * D + d] = parents[(size_t)pidx[c] * D + d];
    }
}

void orc_pm(float* off, const float* bounds, const float* u, float eta, float prob, int n, int D)
{
    const size_t count = (size_t)n * D;
    for (size_t i = 0; i < count; ++i) {
        const int d = (int)(i % (size_t)D);
        const float u1 = u[2 * i], u2 = u[2 * i + 1];
        if (u1 >= prob / (float)D) continue;
        const float lo = bounds[2 * d], hi = bounds[2 * d + 1];
        const float range = hi - lo;
        const float value = off[i];
        const float nv = (value - lo) / range;
        const float ex = eta + 1.0f;
        float delta;
        if (u2 <= 0.5f) {
            const float xy = 1.0f - nv;
            const float vm = fmaf(fmaf(-2.0f, u2, 1.0f), powf(xy, ex), 2.0f * u2);
            delta = powf(vm, 1.0f / ex) - 1.0f;
        } else {
            const float xy = nv;
            const float vm = fmaf(2.0f * (u2 - 0.5f), powf(xy, ex), 2.0f * (1.0f - u2));
            delta = 1.0f - powf(vm, 1.0f / ex);
        }
        off[i] = fminf(fmaxf(fmaf(delta, range, value), lo), hi);
    }
}

/* ======================================================================== */
/* problems                                                                 */
/* ======================================================================== */

/* g-term reduction in the order of the reference's 256-thread block reduction
 * (dtlz_kernels.cu:28-160): thread t accumulates terms t, t+256, ... in turn,
 * each warp folds its 32 partials with a shuffle-down tree, and the 8 warp
 * sums are added in warp order (warp_tree_final=0) or folded by a second
 * shuffle tree (warp_tree_final=1, DTLZ5 :435-541).  accumulate(acc, i)
 * returns the new per-thread partial for term i. */
typedef float (*acc_fn)(float acc, const float* x, int i, const void* ctx);

static float warp_tree(float* v)
{
    for (int off = 16; off > 0; off >>= 1)
        for (int l = 0; l < off; ++l) v[l] = v[l] + v[l + off];
    return v[0];
}

static float block_reduce(const float* row, int k, acc_fn fn, const void* ctx, int warp_tree_final)
{
    float part[256];
    for (int t = 0; t < 256; ++t) {
        float a = 0.0f;
        for (int i = t; i < k; i += 256) a = fn(a, row, i, ctx);
        part[t] = a;
    }
    float ws[32];
    for (int w = 0; w < 8; ++w) ws[w] = warp_tree(part + 32 * w);
    if (warp_tree_final) {
        for (int w = 8; w < 32; ++w) ws[w] = 0.0f;
        return warp_tree(ws);
    }
    float total = 0.0f;
    for (int w = 0; w < 8; ++w) total += ws[w];
    return total;
}

static float acc_rastrigin(float a, const float* x, int i, const void* ctx)
{
    const int start = *(const int*)ctx;
    const float val = x[start + i] - 0.5f;
    return a + fmaf(val, val, -cosf(20.0f * M_PI * val));
}
static float acc_square(float a, const float* x, int i, const void* ctx)
{
    const int start = *(const int*)ctx;
    const float val = x[start + i] - 0.5f;
    return fmaf(val, val, a);
}
static float acc_pow01(float a, const float* x, int i, const void* ctx)
{
    const int start = *(const int*)ctx;
    return a + powf(x[start + i], 0.1f);
}
static float acc_plain(float a, const float* x, int i, const void* ctx)
{
    const int start = *(const int*)ctx;
    return a + x[start + i];
}

static inline float clamp01(float v) { return fmaxf(0.0f, fminf(1.0f, v)); }
static inline float cos_half_pi(float v) { return fmaxf(0.0f, cosf(v * M_PI / 2.0f)); }
static inline float sin_half_pi(float v) { return sinf(v * M_PI / 2.0f); }

/* FP32 restatement of one row (dtlz_kernels.cu:28-747).  out has M entries. */
static void dtlz_row_f32(int base, const float* x, int D, int M, float* out)
{
    const int start = M - 1, k = D - start;
    switch (base) {
    case 1: {
        const float s = block_reduce(x, k, acc_rastrigin, &start, 0);
        const float g = 100.0f * ((float)k + s);
        const float scal = 0.5f * (1.0f + g);
        for (int m = 0; m < M; ++m) {
            float f = scal;
            for (int j = 0; j < M - 1 - m; ++j) f *= clamp01(x[j]);
            if (m > 0) f *= fmaxf(0.0f, 1.0f - x[M - 1 - m]);
            out[m] = f;
        }
        break;
    }
    case 2: case 8: case 3: case 4: {
        float g;
        if (base == 3) {
            const float s = block_reduce(x, k, acc_rastrigin, &start, 0);
            g = 100.0f * ((float)k + s);
        } else {
            g = block_reduce(x, k, acc_square, &start, 0);
        }
        for (int m = 0; m < M; ++m) {
            float f = 1.0f + g;
            for (int j = 0; j < M - 1 - m; ++j)
                f *= (base == 4) ? fmaxf(0.0f, cosf(powf(x[j], 100.0f) * M_PI / 2.0f)) : cos_half_pi(x[j]);
            if (m > 0)
                f *= (base == 4) ? sinf(powf(x[M - 1 - m], 100.0f) * M_PI / 2.0f) : sin_half_pi(x[M - 1 - m]);
            if (base == 8) {
                if (m < M - 1) { f = f * f; f = f * f; } else { f = f * f; }
            }
            out[m] = f;
        }
        break;
    }
    case 5: case 6: {
        const float g = (base == 5) ? block_reduce(x, k, acc_square, &start, 1)
                                    : block_reduce(x, k, acc_pow01, &start, 0);
        float th[32];
        th[0] = x[0];
        const float denom = 2.0f * (1.0f + g);
        for (int i = 1; i < M - 1; ++i) {
            th[i] = fmaf(2.0f * g, x[i], 1.0f) / denom;
            if (base == 5) th[i] = fmaxf(0.0f, fminf(1.0f, th[i]));
        }
        for (int m = 0; m < M; ++m) {
            float f = 1.0f + g;
            for (int j = 0; j < M - 1 - m; ++j) f *= fmaxf(0.0f, cosf(th[j] * M_PI * 0.5f));
            if (m > 0) f *= sinf(th[M - 1 - m] * M_PI * 0.5f);
            out[m] = f;
        }
        break;
    }
    case 7: {
        const float s = block_reduce(x, k, acc_plain, &start, 0);
        const float g = fmaf(9.0f / (float)k, s, 1.0f);
        float hs = 0.0f;
        for (int i = 0; i < M - 1; ++i) {
            out[i] = x[i];
            hs = fmaf(x[i] / (1.0f + g), 1.0f + sinf(3.0f * M_PI * x[i]), hs);
        }
        out[M - 1] = (1.0f + g) * ((float)M - hs);
        break;
    }
    default: break;
    }
}

/* FP64 evaluation of one row (the error reference). */
static void dtlz_row_f64(int base, const float* xf, int D, int M, double* out)
{
    const int start = M - 1, k = D - start;
    double x[64];
    for (int i = 0; i < M && i < 64; ++i) x[i] = xf[i];
    double g = 0.0;
    if (base == 1 || base == 3) {
        for (int i = 0; i < k; ++i) { const double v = (double)xf[start + i] - 0.5; g += v * v - cos(20.0 * M_PI * v); }
        g = 100.0 * ((double)k + g);
    } else if (base == 6) {
        for (int i = 0; i < k; ++i) g += pow((double)xf[start + i], 0.1);
    } else if (base == 7) {
        for (int i = 0; i < k; ++i) g += (double)xf[start + i];
        g = 1.0 + 9.0 / (double)k * g;
    } else {
        for (int i = 0; i < k; ++i) { const double v = (double)xf[start + i] - 0.5; g += v * v; }
    }
    switch (base) {
    case 1:
        for (int m = 0; m < M; ++m) {
            double f = 0.5 * (1.0 + g);
            for (int j = 0; j < M - 1 - m; ++j) f *= fmax(0.0, fmin(1.0, x[j]));
            if (m > 0) f *= fmax(0.0, 1.0 - x[M - 1 - m]);
            out[m] = f;
        }
        break;
    case 2: case 3: case 4: case 8:
        for (int m = 0; m < M; ++m) {
            double f = 1.0 + g;
            for (int j = 0; j < M - 1 - m; ++j)
                f *= fmax(0.0, cos(((base == 4) ? pow(x[j], 100.0) : x[j]) * M_PI / 2.0));
            if (m > 0) f *= sin(((base == 4) ? pow(x[M - 1 - m], 100.0) : x[M - 1 - m]) * M_PI / 2.0);
            if (base == 8) f = (m < M - 1) ? f * f * f * f : f * f;
            out[m] = f;
        }
        break;
    case 5: case 6: {
        double th[64];
        th[0] = x[0];
        for (int i = 1; i < M - 1; ++i) {
            th[i] = (1.0 + 2.0 * g * x[i]) / (2.0 * (1.0 + g));
            if (base == 5) th[i] = fmax(0.0, fmin(1.0, th[i]));
        }
        for (int m = 0; m < M; ++m) {
            double f = 1.0 + g;
            for (int j = 0; j < M - 1 - m; ++j) f *= fmax(0.0, cos(th[j] * M_PI * 0.5));
            if (m > 0) f *= sin(th[M - 1 - m] * M_PI * 0.5);
            out[m] = f;
        }
        break;
    }
    case 7: {
        double hs = 0.0;
        for (int i = 0; i < M - 1; ++i) { out[i] = x[i]; hs += x[i] / (1.0 + g) * (1.0 + sin(3.0 * M_PI * x[i])); }
        out[M - 1] = (1.0 + g) * ((double)M - hs);
        break;
    }
    default: break;
    }
}

/* constraint violation of one column from its objectives (dtlz_kernels.cu:824-1090) */
static float cv_f32(int kind, const float* f, int M)
{
    switch (kind) {
    case 9: {  /* C1-DTLZ1 */
        float c = f[M - 1] / 0.6f;
        for (int m = 0; m < M - 1; ++m) c += f[m] / 0.5f;
        return fmaxf(c - 1.0f, 0.0f);
    }
    case 10: {  /* C1-DTLZ3 */
        float R = 15.0f;
        if (M == 2) R = 6.0f; else if (M == 3) R = 5.0f; else if (M == 5) R = 12.5f;
        float s = 0.0f;
        for (int m = 0; m < M; ++m) s = fmaf(f[m], f[m], s);
        return fmaxf((s - 16.0f) * (R * R - s), 0.0f);
    }
    case 11: {  /* C2-DTLZ2 */
        float R = 1.0f;
        if (M == 2) R = 0.15f; else if (M == 3) R = 0.40f;
        const float inv_sqrt_m = 1.0f / sqrtf((float)M);
        const float inv_r2 = 1.0f / (R * R);
        float s = 0.0f;
        for (int m = 0; m < M; ++m) s = fmaf(f[m], f[m], s);
        float mn = ORC_INF;
        for (int m = 0; m < M; ++m) {
            const float diff = f[m] - 1.0f;
            const float d2 = fmaf(diff, diff, fmaf(-f[m], f[m], s));
            mn = fminf(mn, fmaf(d2, inv_r2, -1.0f));
        }
        float cs = 0.0f;
        for (int m = 0; m < M; ++m) { const float df = f[m] - inv_sqrt_m; cs = fmaf(df, df, cs); }
        return fmaxf(fminf(mn, fmaf(cs, inv_r2, -1.0f)), 0.0f);
    }
    case 12: {  /* C2-ConvexDTLZ2 */
        float R = 0.225f;
        if (M == 3) R = 0.20f; else if (M == 8 || M == 10) R = 0.26f; else if (M == 15) R = 0.27f;
        const float inv_m = 1.0f / (float)M;
        const float inv_r2 = 1.0f / (R * R);
        float s = 0.0f, sq = 0.0f;
        for (int m = 0; m < M; ++m) { s += f[m]; sq = fmaf(f[m], f[m], sq); }
        const float mean = s * inv_m;
        const float var = fmaf(-((float)M * mean), mean, sq);
        return fmaxf(fmaf(-var, inv_r2, 1.0f), 0.0f);
    }
    case 13: {  /* C3-DTLZ1 */
        float s = 0.0f;
        for (int m = 0; m < M; ++m) s += f[m];
        s *= 2.0f;
        float cv = 0.0f;
        for (int m = 0; m < M; ++m) cv += fmaxf((f[m] + 1.0f) - s, 0.0f);
        return cv;
    }
    case 14: {  /* C3-DTLZ4 */
        float s = 0.0f;
        for (int m = 0; m < M; ++m) s = fmaf(f[m], f[m], s);
        float cv = 0.0f;
        for (int m = 0; m < M; ++m) {
            float c = fmaf(0.75f, f[m] * f[m], -s);
            c += 1.0f;
            cv += fmaxf(c, 0.0f);
        }
        return cv;
    }
    default: return 0.0f;
    }
}

static double cv_f64(int kind, const double* f, int M)
{
    switch (kind) {
    case 9: { double c = f[M - 1] / 0.6; for (int m = 0; m < M - 1; ++m) c += f[m] / 0.5; return fmax(c - 1.0, 0.0); }
    case 10: {
        double R = 15.0; if (M == 2) R = 6.0; else if (M == 3) R = 5.0; else if (M == 5) R = 12.5;
        double s = 0.0; for (int m = 0; m < M; ++m) s += f[m] * f[m];
        return fmax((s - 16.0) * (R * R - s), 0.0);
    }
    case 11: {
        double R = 1.0; if (M == 2) R = 0.15; else if (M == 3) R = 0.40;
        double s = 0.0; for (int m = 0; m < M; ++m) s += f[m] * f[m];
        double mn = INFINITY;
        for (int m = 0; m < M; ++m) mn = fmin(mn, ((f[m] - 1.0) * (f[m] - 1.0) + s - f[m] * f[m]) / (R * R) - 1.0);
        double cs = 0.0; for (int m = 0; m < M; ++m) cs += (f[m] - 1.0 / sqrt((double)M)) * (f[m] - 1.0 / sqrt((double)M));
        return fmax(fmin(mn, cs / (R * R) - 1.0), 0.0);
    }
    case 12: {
        double R = 0.225; if (M == 3) R = 0.20; else if (M == 8 || M == 10) R = 0.26; else if (M == 15) R = 0.27;
        double s = 0.0, sq = 0.0; for (int m = 0; m < M; ++m) { s += f[m]; sq += f[m] * f[m]; }
        const double mean = s / M;
        return fmax(1.0 - (sq - M * mean * mean) / (R * R), 0.0);
    }
    case 13: {
        double s = 0.0; for (int m = 0; m < M; ++m) s += f[m];
        double cv = 0.0; for (int m = 0; m < M; ++m) cv += fmax(f[m] + 1.0 - 2.0 * s, 0.0);
        return cv;
    }
    case 14: {
        double s = 0.0; for (int m = 0; m < M; ++m) s += f[m] * f[m];
        double cv = 0.0; for (int m = 0; m < M; ++m) cv += fmax(0.75 * f[m] * f[m] - s + 1.0, 0.0);
        return cv;
    }
    default: return 0.0;
    }
}

/* CSDP (dtlz_kernels.cu:719-747, 1046-1092): double-literal arithmetic as written */
static void csdp_row(const float* x, float* f, float* cv)
{
    const float x1 = x[0], x2 = x[1], x3 = x[2], x4 = x[3], x5 = x[4], x6 = x[5], x7 = x[6];
    const float F = 4.72 - 0.5 * x4 - 0.19 * x2 * x3;
    const float V_MBP = 10.58 - 0.674 * x1 * x2 - 0.67275 * x2;
    const float V_FD = 16.45 - 0.489 * x3 * x7 - 0.843 * x5 * x6;
    f[0] = 1.98 + 4.9 * x1 + 6.67 * x2 + 6.98 * x3 + 4.01 * x4 + 1.78 * x5 + 0.00001 * x6 + 2.73 * x7;
    f[1] = F;
    f[2] = 0.5f * (V_MBP + V_FD);
    const float Ff = 4.72f - 0.5f * x4 - 0.19f * x2 * x3;
    const float Vm = 10.58f - 0.674f * x1 * x2 - 0.67275f * x2;
    const float Vf = 16.45f - 0.489f * x3 * x7 - 0.843f * x5 * x6;
    float g[10];
    g[0] = 1.16f - 0.3717f * x2 * x4 - 0.0092928f * x3 - 1.0f;
    g[1] = 0.261f - 0.0159f * x1 * x2 - 0.06486f * x1 - 0.019f * x2 * x7 + 0.0144f * x3 * x5 + 0.0154464f * x6 - 0.32f;
    g[2] = 0.214f + 0.00817f * x5 - 0.045195f * x1 - 0.0135168f * x1 + 0.03099f * x2 * x6 - 0.018f * x2 * x7
         + 0.007176f * x3 + 0.023232f * x3 - 0.00364f * x5 * x6 - 0.018f * x2 * x2 - 0.32f;
    g[3] = 0.74f - 0.61f * x2 - 0.031296f * x3 - 0.031872f * x7 + 0.227f * x2 * x2 - 0.32f;
    g[4] = 28.98f + 3.818f * x3 - 4.2f * x1 * x2 + 1.27296f * x6 - 2.68065f * x7 - 32.0f;
    g[5] = 33.86f + 2.95f * x3 - 5.057f * x1 * x2 - 3.795f * x2 - 3.4431f * x7 + 1.45728f - 32.0f;
    g[6] = 46.36f - 9.9f * x2 - 4.4505f * x1 - 32.0f;
    g[7] = Ff - 4.0f;
    g[8] = Vm - 9.9f;
    g[9] = Vf - 15.7f;
    float s = 0.0f;
    for (int i = 0; i < 10; ++i) s += fmaxf(g[i], 0.0f);
    *cv = s;
}

int orc_problem_evaluate(int kind, const float* x, int N, int D, int M,
                         float* objs, float* cv, int precision)
{
    if (kind < 1 || kind > 15 || M < 1 || M > 32 || D < 1) return -1;
    if (kind == 15 && (D != 7 || M != 3)) return -1;
    if (kind != 15 && kind != 7 && D < M) return -1;
    static const int base_of[16] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 1, 3, 2, 8, 1, 4, 0};
    #pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        const float* row = x + (size_t)i * D;
        float f32[32]; double f64[64];
        if (kind == 15) {
            float c;
            csdp_row(row, f32, &c);
            for (int m = 0; m < 3; ++m) objs[(size_t)m * N + i] = f32[m];
            cv[i] = c;
            continue;
        }
        const int base = base_of[kind];
        if (precision == 0) {
            dtlz_row_f32(base, row, D, M, f32);
            for (int m = 0; m < M; ++m) objs[(size_t)m * N + i] = f32[m];
            cv[i] = (kind >= 9) ? cv_f32(kind, f32, M) : 0.0f;
        } else {
            dtlz_row_f64(base, row, D, M, f64);
            for (int m = 0; m < M; ++m) objs[(size_t)m * N + i] = (float)f64[m];
            cv[i] = (kind >= 9) ? (float)cv_f64(kind, f64, M) : 0.0f;
        }
    }
    return 0;
}

/* ======================================================================== */
/* reference directions                                                     */
/* ======================================================================== */

static long long comb_ll(int n, int k)
{
    if (k > n) return 0;
    if (k == 0 || k == n) return 1;
    if (k > n - k) k = n - k;
    long long r = 1;
    for (int i = 1; i <= k; ++i) { r *= (n - k + i); r /= i; }
    return r;
}

/* std::prev_permutation on a 0/1 sequence; returns 0 after the smallest one. */
static int prev_perm01(unsigned char* a, int n)
{
    int i = n - 1;
    while (i > 0 && !(a[i - 1] > a[i])) --i;
    if (i == 0) {
        for (int l = 0, r = n - 1; l < r; ++l, --r) { unsigned char t = a[l]; a[l] = a[r]; a[r] = t; }
        return 0;
    }
    int j = n - 1;
    while (!(a[j] < a[i - 1])) --j;
    unsigned char t = a[i - 1]; a[i - 1] = a[j]; a[j] = t;
    for (int l = i, r = n - 1; l < r; ++l, --r) { t = a[l]; a[l] = a[r]; a[r] = t; }
    return 1;
}

/* One Das-Dennis layer in prev_permutation order (nsga3_reference_generator.cu:28-60). */
static int single_layer(int h, int M, float* out /* (M, count) or NULL */, int stride, int col0)
{
    const int len = h + M - 1;
    const int count = (int)comb_ll(len, M - 1);
    if (!out || len <= 0 || h <= 0) return count;
    unsigned char* mask = (unsigned char*)calloc((size_t)(len > 0 ? len : 1), 1);
    int* combo = (int*)malloc(sizeof(int) * (size_t)(M + 1));
    for (int i = 0; i < M - 1; ++i) mask[i] = 1;
    int pt = 0;
    do {
        int c = 0;
        combo[c++] = -1;
        for (int i = 0; i < len; ++i) if (mask[i]) combo[c++] = i;
        combo[c++] = len;
        for (int d = 0; d < M; ++d)
            out[(size_t)d * stride + col0 + pt] = (float)(combo[d + 1] - combo[d] - 1) / (float)h;
        ++pt;
    } while (prev_perm01(mask, len));
    free(mask); free(combo);
    return count;
}

int orc_reference_directions(int mode, int np, int M, float* out)
{
    if (M <= 0) return -1;
    if (mode == 1) {
        if (np <= 0) return -1;
        const int count = single_layer(np, M, NULL, 0, 0);
        if (!out) return count;
        single_layer(np, M, out, count, 0);
        for (int p = 0; p < count; ++p) {
            float n2 = 0.0f;
            for (int m = 0; m < M; ++m) { const float v = out[(size_t)m * count + p]; n2 += v * v; }
            const float inv = 1.0f / sqrtf(n2);
            for (int m = 0; m < M; ++m) out[(size_t)m * count + p] = out[(size_t)m * count + p] * inv;
        }
        return count;
    }
    /* auto layers from the population size (nsga3_reference_generator.cu:62-130) */
    int h1 = 0;
    while (comb_ll(h1 + M - 1, M - 1) <= np) ++h1;
    --h1;
    const int n1 = (int)comb_ll(h1 + M - 1, M - 1);
    int h2 = 0, n2 = 0;
    if (h1 < M) {
        h2 = 1;
        while (comb_ll(h1 + M - 1, M - 1) + comb_ll(h2 + M - 1, M - 1) <= np) ++h2;
        --h2;
        if (h2 > 0) n2 = (int)comb_ll(h2 + M - 1, M - 1);
    }
    const int count = n1 + n2;
    if (!out) return count;
    single_layer(h1, M, out, count, 0);
    if (n2 > 0) {
        single_layer(h2, M, out, count, n1);
        const float centroid = 1.0f / (float)M;
        for (int p = 0; p < n2; ++p)
            for (int m = 0; m < M; ++m)
                out[(size_t)m * count + n1 + p] = 0.5f * (out[(size_t)m * count + n1 + p] + centroid);
    }
    if (mode == 2)
        for (size_t i = 0; i < (size_t)M * count; ++i) out[i] = fmaxf(out[i], 1e-6f);
    for (int p = 0; p < count; ++p) {
        float s = 0.0f;
        for (int m = 0; m < M; ++m) { const float v = out[(size_t)m * count + p]; s += v * v; }
        const float nrm = sqrtf(s);
        for (int m = 0; m < M; ++m) out[(size_t)m * count + p] = out[(size_t)m * count + p] / nrm;
    }
    return count;
}
