/*
 * CPU oracle for the CUDA-MOEA generation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This restatement of the reference algorithm is the
 * checker that the CUDA kernels are compared against; only tests/, the smoke
 * check and the CPU-baseline leg of bench.py may load it.  The product path never
 * calls it and has no CPU fallback.
 *
 * Every function cites the reference file:line it restates (paths are relative
 * to the CUDA-MOEA project root; `nat/` = python/csrc/native/).
 *
 * Layouts follow the reference: variables (N,D) row-major, objectives (M,N)
 * objective-major, constraint violation (N,), bounds interleaved [lb0,ub0,...],
 * reference directions (M,H) objective-major.
 */
#ifndef MOEA_ORACLE_H
#define MOEA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- random numbers ---------------- */
/* SplitMix64 counter hash used by the niching draws
 * (nat/src/core/cuda/cuda_random.cu:1606-1613). */
uint32_t orc_splitmix_u32(uint64_t counter, uint64_t seed);
/* Seed derivation of RNDManager (nat/src/core/cuda/cuda_manager.cu:27-40). */
uint64_t orc_derive_seed(uint64_t seed);
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) -- the product RNG. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Product draw streams (see cuda-moea_b200/csrc/rng.cuh): fills out[4*count]
 * with the Philox outputs for element indices [0,count) of (generation, tag). */
void orc_philox_stream(uint64_t seed, uint32_t generation, uint32_t tag,
                       int64_t count, uint32_t* out);

/* ---------------- non-dominated sorting ---------------- */
/* Constraint-dominance p over q (nat/src/selection/nsga3/kernels/non_dominated_sort.cu:158-281). */
int orc_dominates(const float* cv, const float* objs, int M, int n, int p, int q);
/* Fronts with the reference stop rule: fronts are peeled until at least
 * `target` individuals are assigned; later individuals stay -1.  Returns the
 * index of the last (partially selected) front.  Restates run_ndsort /
 * run_ndsort_init (non_dominated_sort.cu:1337-1574) and the front propagation
 * loops (:735-843, :1070-1279). */
int orc_ndsort(const float* cv, const float* objs, int M, int n, int target, int* fronts);

/* ---------------- NSGA-III selection stages ---------------- */
/* Sizes and [prior; last] ascending-index compaction
 * (non_dominated_sort.cu:1580-1781).  sizes = {N_prior, N_last, N_rem, N_nds}. */
void orc_nds_extract(const int* fronts, int n_mix, int max_front, int N,
                     int* nds_gidx, int sizes[4]);
/* Ideal point: per-objective minimum with fminf semantics (ideal_point.cu:36-129). */
void orc_ideal_point(const float* objs, int M, int n, float* ideal);
/* Normalisation (normalization.cu:370-856, 1217-1394, 1593-1636) with the SVD
 * restated in FP64 (one-sided Jacobi).  objs_nds (M,N_nds) is overwritten with
 * the normalised values; rcp_b receives the sanitised reciprocal intercepts;
 * extreme receives the extreme-point indices; returns 1 when the fallback
 * (row maxima) was taken. */
int orc_normalize(float* objs_nds, const float* ideal, int M, int n_nds,
                  float* rcp_b, int* extreme);
/* Association (association.cu:86-188, 397-447): exact FP32 formula, ties to
 * the smaller direction index. */
void orc_associate(const float* x, const float* refs, int M, int n, int H,
                   int* idx, float* dist);
/* Niching (niching.cu:250-400, cuda_ref_segment_ops.cu:17-138).  *offset is
 * advanced by 2*N_last like the reference.  selected receives N global indices
 * ([prior; chosen last] before the final ascending sort). */
void orc_niching(uint64_t seed, uint64_t* offset, const int* nds_gidx,
                 const float* dist, const int* idx, const int sizes[4], int H,
                 int N, int* selected);
/* One complete NSGA-III environmental selection (nsga3_environment_selector.cu:289-538).
 * parent/offspring populations are merged implicitly (index < N: parent).
 * ideal_last is updated in place.  Outputs the sorted survivor indices (N),
 * the survivor fronts (N) and returns max_front.  cv_sort may be NULL (no
 * quantisation) or the CV used for sorting. */
int orc_nsga3_select(const float* mix_cv, const float* mix_objs, int M, int N,
                     const float* refs, int H, uint64_t seed, uint64_t* offset,
                     float* ideal_last, const float* off_objs,
                     int* survivors, int* survivor_fronts, int sizes_out[4]);
/* Optional CV quantisation (cv_quantization.cu:11-95). */
void orc_quantize_cv(const float* cv, float* out, int n, float eps_feas,
                     float clip_upper, float log_alpha, int bins);

/* ---------------- RVEA stages ---------------- */
/* z_min and translation (objective_translation.cu:15-167). */
void orc_rvea_translate(const float* objs, int M, int n, float* out, float* zmin);
/* Partition (reference_partition.cu:48-356).  rsqrtf is restated as 1/sqrtf. */
void orc_rvea_partition(const float* t, const float* refs, int M, int n, int K,
                        int n_active, int n_parent, float* theta, int* idx);
/* gamma (angle_penalized_distance.cu:197-417). */
void orc_rvea_gamma(const float* refs, int M, int K, float* gamma);
/* APD (angle_penalized_distance.cu:45-184). */
void orc_rvea_apd(const float* t, const float* theta, const float* gamma,
                  const int* idx, int M, int n, int K, int gen, int max_gen,
                  float alpha, float* apd);
/* Elitism (elitism_selection.cu:68-419).  Returns the active count; writes
 * the survivor set sorted ascending into selected (active entries). */
int orc_rvea_elitism(const int* idx, const float* cv, const float* apd, int N,
                     int n_mix, int K, int* selected);
/* Direction adaptation (rvea_reference_adaptation.cu:126-317). */
void orc_rvea_adapt(const float* v0, const float* objs, int M, int K,
                    int n_active, int n_stride, float* v);

/* ---------------- reproduction ---------------- */
/* Tournament winner (mating_selection.cu:11-35) from explicit candidates. */
void orc_tournament(const int* cand /* (n,2) */, const int* rank, const float* cv,
                    int n, int* winners);
/* SBX (sbx_crossover.cu:20-70) from explicit draws: u (pairs*D,2), sign
 * (pairs*D), copy (pairs*D). */
void orc_sbx(const float* parents, const int* pidx, const float* bounds,
             const float* u, const int* sign, const float* copy, float* off,
             float eta, float prob, float copy_prob, int n_off, int D);
/* Polynomial mutation (polynomial_mutation.cu:20-60) from explicit draws u (n*D,2). */
void orc_pm(float* off, const float* bounds, const float* u, float eta,
            float prob, int n, int D);
/* Annealed distribution index (sbx_crossover.cu:12-18). */
float orc_annealed(float begin, float end, int gen, int total);

/* ---------------- problems ---------------- */
/* kinds follow the reference problem names (dtlz_kernels.cu:28-1176):
 * 1..7 DTLZ1-7, 8 ConvexDTLZ2, 9 C1-DTLZ1, 10 C1-DTLZ3, 11 C2-DTLZ2,
 * 12 C2-ConvexDTLZ2, 13 C3-DTLZ1, 14 C3-DTLZ4, 15 CSDP.
 * objs is (M,N); cv (N) is written for constrained kinds, zero otherwise.
 * precision 0 = FP32 restatement, 1 = FP64 evaluation (error reference). */
int orc_problem_evaluate(int kind, const float* x, int N, int D, int M,
                         float* objs, float* cv, int precision);

/* ---------------- reference directions ---------------- */
/* Das-Dennis directions (nsga3_reference_generator.cu:28-221,
 * rvea_reference_generator.cu:182-205).  mode 0 = NSGA-III auto from the
 * population size, 1 = NSGA-III by partitions, 2 = RVEA auto (clamped).
 * Returns the count; when out is non-NULL writes (M,count) normalised values. */
int orc_reference_directions(int mode, int n_or_partitions, int M, float* out);

#ifdef __cplusplus
}
#endif
#endif
