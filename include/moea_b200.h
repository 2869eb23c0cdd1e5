/*
 * moea_b200 -- C ABI of the B200 implementation of the CUDA-MOEA generation
 * hot path (NSGA-III / RVEA environmental selection, SBX, polynomial mutation,
 * tournament/random mating and DTLZ evaluation).
 *
 * Conventions
 *   - Plain pointers and sizes only.  Pointers named d_* are CUDA device
 *     pointers, h_* are host pointers.  `stream` is a cudaStream_t passed as
 *     void* (NULL = legacy default stream).  All device work is stream-ordered.
 *   - Layouts follow the reference: variables (N,D) row-major, objectives (M,N)
 *     objective-major, constraint violation (N,), bounds interleaved
 *     [lb0,ub0,lb1,ub1,...], reference directions (M,H) objective-major.
 *   - Every function returns a moea_status; the message of the last failure on
 *     the calling thread is available from moea_last_error().  Nothing in this
 *     library calls exit() (the reference's CUDA_CHECK does,
 *     nat/include/cuda_moea/core/cuda/cuda_utils.cuh:16-22).
 *
 * Reference paths below are inside CUDA-MOEA; nat/ stands for python/csrc/native/.
 */
#ifndef MOEA_B200_H
#define MOEA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MOEA_ABI_VERSION 1

typedef int moea_status;
enum {
    MOEA_OK = 0,
    MOEA_ERR_INVALID_ARGUMENT = 1, /* reference: std::invalid_argument */
    MOEA_ERR_CUDA = 2,             /* CUDA runtime error */
    MOEA_ERR_UNSUPPORTED = 3,      /* configuration outside what the kernels support */
    MOEA_ERR_STATE = 4,            /* reference: std::logic_error */
    MOEA_ERR_DEVICE_TIMEOUT = 5,   /* a bounded device-side wait gave up */
    MOEA_ERR_OUT_OF_MEMORY = 6,
    MOEA_ERR_CALLBACK = 7,         /* a user callback reported failure */
    MOEA_ERR_LOAD = 8              /* a plugin library did not load (reference: std::runtime_error) */
};

/* Version of this ABI (MOEA_ABI_VERSION). No reference counterpart: a binding
 * checks it once before its first call. */
int moea_abi_version(void);
/* Message of the last failure on the calling thread ("" if none). */
const char* moea_last_error(void);

/* ========================================================================
 * Workspace for the stage-level entry points.  Owns the device scratch a
 * stage needs (dominance rows, sort buffers, partial reductions).  Replaces
 * the per-generation pool allocations of the reference
 * (nat/src/selection/nsga3/kernels/dynamic_workspace.cu:3-125).
 * ====================================================================== */
typedef struct moea_workspace moea_workspace;

/* max_points: largest merged population (2N); max_objectives <= 16;
 * max_directions: largest reference-direction count. */
moea_status moea_workspace_create(int device, int max_points, int max_objectives,
                                  int max_directions, moea_workspace** out);
void moea_workspace_destroy(moea_workspace* ws);
/* Bytes of device memory held by the workspace (the reference's selector scratch
 * pool, nat/src/selection/nsga3/kernels/dynamic_workspace.cu, reports none). */
size_t moea_workspace_bytes(const moea_workspace* ws);
/* Front-peeling kernel of the workspace's sorts: MOEA_PEEL_AUTO (default) takes
 * the lane-owned peel whenever every warp of the grid holds at most one group
 * of 32 points (up to 151,552 merged points on a B200) and the general peel
 * beyond; MOEA_PEEL_GENERAL always takes the general one.  Both give the same
 * fronts.  No counterpart in the reference (one peel path there). */
#define MOEA_PEEL_AUTO 0
#define MOEA_PEEL_GENERAL 1
moea_status moea_workspace_set_peel(moea_workspace* ws, int mode);
/* Dominance-row kernel of the workspace's sorts: MOEA_TILES_AUTO (default)
 * builds the rows from prefix sets of blocks of 256 sorted positions (128
 * beyond four objectives) with search trees of their keys; MOEA_TILES_WORD
 * from the per-word tables (32 positions) with six-probe searches.  Both give
 * the same fronts.  No counterpart in the reference. */
#define MOEA_TILES_AUTO 0
#define MOEA_TILES_WORD 1
moea_status moea_workspace_set_tiles(moea_workspace* ws, int mode);

/* ========================================================================
 * Stage-level entry points (one hot-path stage each).
 * ====================================================================== */

/* Constraint-dominance non-dominated sort of n points with the reference stop
 * rule: fronts are peeled until >= target points are assigned; later points
 * get -1.  d_fronts (n) receives front indices; *h_max_front the index of the
 * last (partially selected) front.  Synchronises the stream before returning.
 * Replaces run_ndsort / run_ndsort_init
 * (nat/src/selection/nsga3/kernels/non_dominated_sort.cu:1337, :1407). */
moea_status moea_ndsort(moea_workspace* ws, const float* d_cv, const float* d_objs,
                        int M, int n, int target, int* d_fronts, int* h_max_front,
                        void* stream);

/* Prior/last-front sizes and the [prior; last] ascending-index compaction.
 * d_sizes receives {N_prior, N_last, N_rem, N_nds}; d_nds_gidx (n_mix).
 * max_front is read from d_max_front.  Replaces get_nds_mask_size +
 * extract_ndsfit_mskidx (non_dominated_sort.cu:1636, :1720). */
moea_status moea_nds_extract(moea_workspace* ws, const int* d_fronts, int n_mix,
                             const int* d_max_front, int N, int* d_nds_gidx,
                             int* d_sizes, void* stream);

/* Per-objective minimum (fminf semantics) of d_objs (M,n) into d_ideal (M).
 * Replaces get_idpts (nat/src/selection/nsga3/kernels/ideal_point.cu:97). */
moea_status moea_ideal_point(moea_workspace* ws, const float* d_objs, int M, int n,
                             float* d_ideal, void* stream);

/* Hyperplane normalisation of d_objs (M,n) in place: translate by d_ideal,
 * ASF extreme points, FP64 intercept solve with the reference's degeneracy
 * fallback, sanitise, scale.  d_rcp_b (M) receives the reciprocal intercepts,
 * d_extreme (M) the extreme-point indices (may be NULL).  Replaces
 * execute_normalization (nat/src/selection/nsga3/kernels/normalization.cu:1593). */
moea_status moea_normalize(moea_workspace* ws, float* d_objs, const float* d_ideal, int M,
                           int n, float* d_rcp_b, int* d_extreme, void* stream);

/* Association modes; all give the reference's exact argmin. */
#define MOEA_ASSOC_TREE 0    /* cone tree over the directions, one warp per point, subtrees
                                pruned by a conservative bound on dot^2 (default); above 5
                                objectives the tensor-core search of MOEA_ASSOC_TENSOR when
                                points x directions >= 2^24, else the scan */
#define MOEA_ASSOC_SCAN 1    /* every direction visited, FP32 re-score of the dot^2 candidates */
#define MOEA_ASSOC_TENSOR 2  /* precision form: the point x direction dots on the tensor cores
                                (split TF32 operands, FP32 accumulation), FP32 re-score of every
                                direction within the proven error bound of the best */

/* Association of normalised points d_x (M,n) to directions d_refs (M,H):
 * perpendicular distance with the reference's FP32 formula, ties to the
 * smaller direction index.  mode MOEA_ASSOC_TREE builds the cone tree of
 * d_refs on the host on every call (a read-back that synchronises the
 * stream); the algorithm object builds it once.  mode MOEA_ASSOC_TENSOR packs
 * the split TF32 operand of d_refs on the device on every call (the algorithm
 * object packs it once) and reports a timed-out tensor-core wait as
 * MOEA_ERR_DEVICE_TIMEOUT.  Replaces
 * execute_association (nat/src/selection/nsga3/kernels/association.cu:586). */
moea_status moea_associate(moea_workspace* ws, const float* d_x, const float* d_refs, int M,
                           int n, int H, int* d_idx, float* d_dist, int mode, void* stream);

/* Allocation-free variant of moea_associate in MOEA_ASSOC_SCAN mode: no
 * workspace, no device allocation.  Scratch lives in static device arrays
 * sized for at most 65536 points (larger n -> MOEA_ERR_INVALID_ARGUMENT).
 * For callers that hold no workspace and may not allocate during a
 * generation (strategies that receive only borrowed views).  Calls whose work
 * overlaps on the device share the scratch and race; the first call on a
 * device resolves the scratch addresses (not stream-ordered), so make it
 * before any stream capture that includes this function.  No counterpart in
 * the reference. */
moea_status moea_associate_static(const float* d_x, const float* d_refs, int M, int n, int H,
                                  int* d_idx, float* d_dist, void* stream);

/* NSGA-III niche selection.  d_sizes as produced by moea_nds_extract; the
 * tie-break draws use SplitMix64(offset + i, seed) like the reference and
 * *h_offset is advanced by 2*N_last.  d_selected (N) receives mixed indices
 * [prior; chosen]. Replaces execute_niching
 * (nat/src/selection/nsga3/kernels/niching.cu:250). */
moea_status moea_niching(moea_workspace* ws, uint64_t seed, uint64_t* h_offset,
                         const int* d_nds_gidx, const float* d_dist, const int* d_idx,
                         const int* d_sizes, int H, int N, int* d_selected, void* stream);

/* One complete NSGA-III environmental selection over the merged population
 * (parents are mixed indices [0,N), offspring [N,2N)).  d_ideal_last (M) is
 * the running ideal point (updated).  Outputs: d_survivors (N, ascending mixed
 * indices), d_survivor_fronts (N), d_sizes (4).  *h_offset as for
 * moea_niching.  Replaces NSGA3EnvironmentSelector::select
 * (nat/src/selection/nsga3/nsga3_environment_selector.cu:289-538). */
moea_status moea_nsga3_select(moea_workspace* ws, const float* d_mix_cv,
                              const float* d_mix_objs, int M, int N, const float* d_refs,
                              int H, uint64_t seed, uint64_t* h_offset, float* d_ideal_last,
                              int* d_survivors, int* d_survivor_fronts, int* d_sizes,
                              int assoc_mode, void* stream);

/* Inverted generational distance in FP64: d_objs (M,n) objective-major
 * approximation, d_ref (r,M) row-major FP64 reference front.  Rows with a
 * non-finite objective are dropped; with filter_nondominated only the
 * non-dominated rows count.  d_min_dist (r) receives each reference point's
 * distance to its nearest kept row, *h_igd their mean (synchronises the
 * stream).  Replaces igd / nondominated_mask of the reference's evaluation
 * tooling (tests/evaluation/metrics/igd.py:8-47). */
moea_status moea_igd(moea_workspace* ws, const float* d_objs, int n, int M, const double* d_ref, int r,
                     int filter_nondominated, double* d_min_dist, double* h_igd, void* stream);

/* Optional CV quantisation (nat/src/selection/nsga3/kernels/cv_quantization.cu:65). */
moea_status moea_quantize_cv(const float* d_cv, float* d_out, int n, float eps_feas,
                             float clip_upper, float log_alpha, int bins, void* stream);

/* ---- RVEA ---- */
/* z_min translation (nat/src/selection/rvea/kernels/objective_translation.cu:125). */
moea_status moea_rvea_translate(moea_workspace* ws, const float* d_objs, int M, int n,
                                float* d_out, float* d_zmin, void* stream);
/* Max-cosine partition with dead parent slots [n_active, n_parent) marked K
 * (nat/src/selection/rvea/kernels/reference_partition.cu:407). */
moea_status moea_rvea_partition(moea_workspace* ws, const float* d_t, const float* d_refs,
                                int M, int n, int K, int n_active, int n_parent,
                                float* d_theta, int* d_idx, void* stream);
/* gamma per direction (angle_penalized_distance.cu:387). */
moea_status moea_rvea_gamma(moea_workspace* ws, const float* d_refs, int M, int K,
                            float* d_gamma, void* stream);
/* APD with penalty M*progress^alpha, progress = gen/max_gen clamped
 * (angle_penalized_distance.cu:159). */
moea_status moea_rvea_apd(moea_workspace* ws, const float* d_t, const float* d_theta,
                          const float* d_gamma, const int* d_idx, int M, int n, int K,
                          int gen, int max_gen, float alpha, float* d_apd, void* stream);
/* Elitism: per-direction winner, truncation to N; d_selected (N) receives the
 * survivor set sorted ascending, *h_active the active count
 * (nat/src/selection/rvea/kernels/elitism_selection.cu:194). */
moea_status moea_rvea_elitism(moea_workspace* ws, const int* d_idx, const float* d_cv,
                              const float* d_apd, int N, int n_mix, int K, int* d_selected,
                              int* h_active, void* stream);
/* Direction adaptation V = normalize(V0 * (zmax - zmin)) over the first
 * n_active columns (nat/src/reference/rvea_reference_adaptation.cu:279). */
moea_status moea_rvea_adapt(moea_workspace* ws, const float* d_v0, const float* d_objs,
                            int M, int K, int n_active, int n_stride, float* d_v,
                            void* stream);

/* ---- reproduction ---- */
/* Tournament winners from explicit candidate pairs d_cand (n,2)
 * (nat/src/reproduction/mating_selection.cu:11-35, :74). */
moea_status moea_tournament(const int* d_cand, const int* d_rank, const float* d_cv, int n,
                            int* d_winners, void* stream);
/* SBX from explicit draws: d_u (pairs*D,2), d_sign (pairs*D), d_copy (pairs*D)
 * (nat/src/reproduction/sbx_crossover.cu:20-70, :123). */
moea_status moea_sbx(const float* d_parents, const int* d_pidx, const float* d_bounds,
                     const float* d_u, const int* d_sign, const float* d_copy, float* d_off,
                     float eta, float prob, float copy_prob, int n_off, int D, void* stream);
/* Polynomial mutation in place from explicit draws d_u (n*D,2)
 * (nat/src/reproduction/polynomial_mutation.cu:20-60, :95). */
moea_status moea_pm(float* d_off, const float* d_bounds, const float* d_u, float eta,
                    float prob, int n, int D, void* stream);
/* Fused tournament (or random, mating=0) + SBX + PM with in-register Philox
 * draws for (seed, generation).  d_rank may be NULL for random mating.
 * d_parent_idx (n_off) receives the chosen parents (may be NULL). */
moea_status moea_reproduce(const float* d_parents, const float* d_parent_cv,
                           const int* d_rank, int active, const float* d_bounds,
                           float* d_off, int* d_parent_idx, int n_parents, int n_off, int D,
                           int mating, float sbx_eta, float sbx_prob, float sbx_copy_prob,
                           int mutate, float pm_eta, float pm_prob, uint64_t seed,
                           uint32_t generation, void* stream);
/* Random initial population x = lb + u (ub - lb), u uniform in [0, 1) from
 * the product's Philox stream of the run seed (CudaConfig.seed, derived as
 * the algorithm object derives it) and reset epoch (0 for the first run):
 * the algorithm object's own initial population.  Replaces
 * Population::initialize_random (nat/src/core/population.cu:97-115). */
moea_status moea_initialize_population(uint64_t seed, uint32_t epoch, const float* d_bounds, int N, int D,
                                      float* d_vars, void* stream);
/* The raw product draws of moea_reproduce, for checking: d_out (count,4). */
moea_status moea_rng_blocks(uint64_t seed, uint32_t generation, uint32_t tag, int64_t count,
                            uint32_t* d_out, void* stream);

/* ---- problems ---- */
/* Built-in problems (nat/src/problem/dtlz/dtlz_kernels.cu:28-1176): kind
 * 1..7 DTLZ1-7, 8 ConvexDTLZ2, 9 C1-DTLZ1, 10 C1-DTLZ3, 11 C2-DTLZ2,
 * 12 C2-ConvexDTLZ2, 13 C3-DTLZ1, 14 C3-DTLZ4, 15 CSDP.  d_objs (M,N),
 * d_cv (N) (zeros for unconstrained kinds). */
moea_status moea_problem_evaluate(int kind, const float* d_x, int N, int D, int M,
                                  float* d_objs, float* d_cv, void* stream);

/* ---- reference directions ---- */
/* Das-Dennis directions (nat/src/reference/nsga3_reference_generator.cu:153,
 * :184; rvea_reference_generator.cu:182).  mode 0 = NSGA-III auto layers for
 * n points, 1 = NSGA-III single layer with n partitions, 2 = RVEA auto
 * (clamped to >= 1e-6).  *h_count receives the count; h_out (M,count) is
 * written when non-NULL and capacity (floats) suffices. */
moea_status moea_reference_directions(int mode, int n, int M, float* h_out, size_t capacity,
                                      int* h_count);

/* ========================================================================
 * Strategy handles: the reference's strategy interfaces as opaque objects, so
 * a host program can assemble a generation from them the way
 * EvolutionaryAlgorithm::step does (nat/src/algorithm/algorithm.cu:104-286):
 * mating -> crossover -> mutation -> evaluation -> environmental selection ->
 * direction update.  Every call is ordered on `stream` and returns without
 * waiting for the device; sizes that the reference keeps on the host (the
 * RVEA active count, the front sizes) stay on the device.  Populations are
 * borrowed views for the duration of a call, as in the reference.
 * ====================================================================== */

/* A borrowed population (the reference's PopulationView,
 * nat/include/cuda_moea/core/types.cuh:21-51): variables (size, dimension)
 * row-major, objectives (objectives, size) objective-major, constraint
 * violation (size), bounds interleaved (2 * dimension). */
typedef struct moea_population_desc {
    float* d_variables;
    float* d_objectives;
    float* d_constraints;
    const float* d_bounds;
    int size, dimension, objectives;
} moea_population_desc;

/* The reference's GenerationContext (nat/include/cuda_moea/core/contexts.cuh):
 * the generation index, the horizon and the run's seed (CudaConfig.seed; every
 * handle derives its draws from it the way the algorithm object does, so a
 * generation assembled from handles equals the algorithm's). */
typedef struct moea_generation_desc {
    int generation;
    int max_generations;
    uint64_t seed;
} moea_generation_desc;

/* ---- reference directions (IReferenceDirectionProvider,
 * nat/include/cuda_moea/reference/reference_direction_provider.cuh:11-26) ---- */
typedef struct moea_directions moea_directions;
/* DasDennisDirections{partitions} (0: from the requested count). */
moea_status moea_create_dasdennis(int partitions, moea_directions** out);
/* AdaptiveRVEADirections{frequency} (reference_directions.cu:61-162). */
moea_status moea_create_adaptive_directions(float frequency, moea_directions** out);
/* UserDefinedDirections: h_values (M, count) objective-major, copied
 * (reference_directions.cu:180-237). */
moea_status moea_create_user_directions(const float* h_values, int M, int count, int normalize,
                                        moea_directions** out);
moea_status moea_directions_initialize(moea_directions* d, int requested_count, int M, int device,
                                       void* stream);
/* view(): directions, initial directions, gamma (NULL unless adaptive), M, count. */
moea_status moea_directions_view(moea_directions* d, const float** d_values, const float** d_initial,
                                 const float** d_gamma, int* M, int* count);
/* update(): adaptive directions adapt on the reference's schedule (every
 * max(1, lround(frequency * max_generations)) completed generations) to the
 * first *d_active columns of pop's objectives (d_active NULL: all). */
moea_status moea_directions_update(moea_directions* d, const moea_population_desc* pop, const int* d_active,
                                   const moea_generation_desc* ctx, void* stream);
moea_status moea_directions_reset(moea_directions* d, void* stream);
void moea_directions_destroy(moea_directions* d);

/* ---- mating (IMatingSelector, nat/include/cuda_moea/reproduction/mating_selector.cuh:9-19) ---- */
typedef struct moea_mating moea_mating;
moea_status moea_create_tournament(moea_mating** out);   /* TournamentMating (mating_selection.cu:74) */
moea_status moea_create_random_mating(moea_mating** out); /* RandomMating (mating_selection.cu:39) */
/* select(): d_parent_idx (count) from parents; d_rank (tournament: required,
 * mating_selection.cu:80-86) and d_active (NULL: parents->size) come from the
 * selector's mating state. */
moea_status moea_mating_select(moea_mating* m, const moea_population_desc* parents, const int* d_rank,
                               const int* d_active, int* d_parent_idx, int count,
                               const moea_generation_desc* ctx, void* stream);
void moea_mating_destroy(moea_mating* m);

/* ---- crossover (ICrossoverOperator, crossover_operator.cuh:9-19) ---- */
typedef struct moea_crossover moea_crossover;
/* SimulatedBinaryCrossover{eta_initial, eta_final, probability,
 * variable_copy_probability} (sbx_crossover.cu:73-190). */
moea_status moea_create_sbx(float eta_initial, float eta_final, float probability, float copy_probability,
                            moea_crossover** out);
/* apply(): offspring->size children from parents and d_parent_idx (size). */
moea_status moea_crossover_apply(moea_crossover* c, const moea_population_desc* parents, const int* d_parent_idx,
                                 moea_population_desc* offspring, const moea_generation_desc* ctx, void* stream);
void moea_crossover_destroy(moea_crossover* c);

/* ---- mutation (IMutationOperator, mutation_operator.cuh:9-17) ---- */
typedef struct moea_mutation moea_mutation;
/* PolynomialMutation{eta_initial, eta_final, probability} (polynomial_mutation.cu:63-124). */
moea_status moea_create_pm(float eta_initial, float eta_final, float probability, moea_mutation** out);
/* mutate(): offspring variables in place. */
moea_status moea_mutation_apply(moea_mutation* m, moea_population_desc* offspring, const moea_generation_desc* ctx,
                                void* stream);
void moea_mutation_destroy(moea_mutation* m);

/* ---- environmental selection (IEnvironmentSelector,
 * nat/include/cuda_moea/selection/environment_selector.cuh:9-33) ---- */
typedef struct moea_selector moea_selector;
typedef struct moea_nsga3_selector_config {
    float sparse_ratio;       /* validated; the bitmask relation needs no pair buffer */
    int cv_bins;              /* CVQuantizationConfig (0: off) */
    float cv_clip_upper, cv_log_alpha, feasibility_epsilon;
    int association_mode;     /* MOEA_ASSOC_* */
} moea_nsga3_selector_config;
/* NSGA3EnvironmentSelector (nsga3_environment_selector.cu:50-566); cfg NULL:
 * the reference defaults. */
moea_status moea_create_nsga3_selector(const moea_nsga3_selector_config* cfg, moea_selector** out);
/* RVEAEnvironmentSelector{alpha} (rvea_environment_selector.cu:52-324). */
moea_status moea_create_rvea_selector(float alpha, moea_selector** out);
/* initialize(AlgorithmInfo, provider, CudaContext): allocates the selector's
 * scratch for population_size N (merged 2N) once.  The provider must be
 * initialized and outlive the selector (the reference keeps a raw pointer). */
moea_status moea_selector_initialize(moea_selector* s, int population_size, int dimension, int objectives,
                                     int max_generations, moea_directions* directions, int device, void* stream);
/* prepare(): NSGA-III sorts the parents (mating ranks, running ideal point on
 * the first call); RVEA keeps its active count. */
moea_status moea_selector_prepare(moea_selector* s, const moea_population_desc* parents,
                                  const moea_generation_desc* ctx, void* stream);
/* select(): the next population from parents + offspring, written to next. */
moea_status moea_selector_select(moea_selector* s, const moea_population_desc* parents,
                                 const moea_population_desc* offspring, moea_population_desc* next,
                                 const moea_generation_desc* ctx, void* stream);
/* mating_state(): device pointers of the parents' ranks (NSGA-III; NULL for
 * RVEA) and of the active count (one int). */
moea_status moea_selector_mating_state(moea_selector* s, const int** d_rank, const int** d_active);
/* active_count(): reads the device count back (synchronises the stream). */
moea_status moea_selector_active_count(moea_selector* s, int* h_active, void* stream);
/* finalize(): RVEA computes the front-0 indices of the active parents
 * (front_zero.cu:244-293; synchronises); NSGA-III does nothing. */
moea_status moea_selector_finalize(moea_selector* s, const moea_population_desc* population, void* stream);
/* result_indices(): NSGA-III the parents' fronts (count = size), RVEA the
 * front-0 indices of the last finalize. */
moea_status moea_selector_result_indices(moea_selector* s, const int** d_indices, int* count);
moea_status moea_selector_reset(moea_selector* s, void* stream);
void moea_selector_destroy(moea_selector* s);

/* ========================================================================
 * Algorithm (the NSGA3 / RVEA entry points, Algorithm / AlgorithmBuilder).
 * Replaces EvolutionaryAlgorithm (nat/src/algorithm/algorithm.cu:104-432)
 * built by AlgorithmFactory::create (nat/src/factory/algorithm_factory.cu:66).
 * ====================================================================== */
typedef struct moea_algorithm moea_algorithm;

enum { MOEA_NSGA3 = 0, MOEA_RVEA = 1 };
enum { MOEA_MATING_RANDOM = 0, MOEA_MATING_TOURNAMENT = 1, MOEA_MATING_CALLBACK = 2 };
enum { MOEA_DIRS_DAS_DENNIS = 0, MOEA_DIRS_ADAPTIVE = 1, MOEA_DIRS_USER = 2 };

/* Problem evaluated by the caller (a PythonProblem or a native plugin): writes
 * objectives (M,N) and constraint violation (N) for d_vars (N,D) on stream.
 * Returns 0 on success.  generation is -1 for the initial population. */
typedef int (*moea_evaluate_fn)(void* user, const float* d_vars, float* d_objs, float* d_cv,
                                int N, int D, int M, int generation, int max_generations,
                                void* stream);
/* Mating selection by the caller: writes N parent indices (int32) for the
 * current parents.  d_rank may be NULL. */
typedef int (*moea_mating_fn)(void* user, const float* d_vars, const float* d_objs,
                              const float* d_cv, const int* d_rank, int active, int* d_out,
                              int N, int D, int M, int generation, void* stream);
/* Runs before each generation on the parents of a callback problem
 * (IProblemEvaluator::prepare_parent, nat/src/algorithm/algorithm.cu:230-237);
 * a nonzero *h_changed makes the algorithm sort the parents again.  Returns 0
 * on success. */
typedef int (*moea_prepare_fn)(void* user, float* d_vars, float* d_objs, float* d_cv, int N, int D, int M,
                               int generation, int max_generations, void* stream, int* h_changed);
/* Called when the algorithm is reset (IProblemEvaluator::reset, algorithm.cu:413). */
typedef void (*moea_problem_reset_fn)(void* user);

typedef struct moea_algorithm_config {
    int algorithm;            /* MOEA_NSGA3 / MOEA_RVEA */
    int population_size;
    int max_generations;
    int device;
    uint64_t seed;            /* CudaConfig.seed, default 2887 */
    void* stream;             /* stream to run on; NULL = an internal stream */
    /* problem */
    int problem_kind;         /* 1..15 built-in, 0 = callback */
    int dimension;
    int objectives;
    float constraint_activation_ratio;
    const float* h_lower;     /* (D) bounds, used for callback problems; NULL = [0,1] */
    const float* h_upper;
    moea_evaluate_fn evaluate;
    void* evaluate_user;
    /* mating */
    int mating;               /* MOEA_MATING_* */
    moea_mating_fn mate;
    void* mate_user;
    /* SBX */
    float sbx_eta_initial, sbx_eta_final, sbx_probability, sbx_copy_probability;
    /* polynomial mutation (mutation = 0 -> NoMutation) */
    int mutation;
    float pm_eta_initial, pm_eta_final, pm_probability;
    /* reference directions */
    int directions;           /* MOEA_DIRS_* */
    int partitions;           /* Das-Dennis partitions (0 = from population size) */
    float adapt_frequency;    /* AdaptiveRVEADirections.frequency */
    const float* h_user_directions; /* (M,count) objective-major */
    int user_direction_count;
    int normalize_user_directions;
    /* NSGA-III selector */
    float sparse_ratio;       /* validated for compatibility; the bitmask path needs no pair buffer */
    int cv_bins;
    float cv_clip_upper, cv_log_alpha, feasibility_epsilon;
    int association_mode;     /* MOEA_ASSOC_TREE, MOEA_ASSOC_SCAN or MOEA_ASSOC_TENSOR */
    /* RVEA selector */
    float rvea_alpha;
    /* initial population (N,D) row-major on the host, or NULL */
    const float* h_initial_population;
    int use_graphs;           /* capture one generation into a CUDA graph when possible */
    int fused_small;          /* run an eligible population with 2N <= 8192 (NSGA-III, built-in
                                 unconstrained DTLZ, fixed directions) as the fused generation:
                                 same results, about 20 launches instead of about 80 */
    /* Snapshots in the reference's data-recorder format
     * (nat/src/algorithm/data_recorder.cu:128-292): generation 0, every
     * save_interval-th generation and the last one, under save_directory
     * (NULL: no snapshots; save_interval must then be positive).  Written from
     * pinned host copies by a side stream: the compute stream waits for the
     * device-to-host copies only.  Each generation directory also holds
     * resume.bin for moea_algorithm_load_snapshot. */
    const char* save_directory;
    int save_interval;
    const char* problem_name; /* metadata name of a callback problem (NULL: null) */
    int constraint_count;     /* metadata constraint count of a callback problem */
    /* optional hooks of a callback problem, called with evaluate_user */
    moea_prepare_fn prepare;
    moea_problem_reset_fn problem_reset;
} moea_algorithm_config;

/* Fills cfg with the reference defaults (nat/src/factory/algorithm_factory.cu:25-118). */
void moea_algorithm_config_defaults(moea_algorithm_config* cfg, int algorithm);

moea_status moea_algorithm_create(const moea_algorithm_config* cfg, moea_algorithm** out);
void moea_algorithm_destroy(moea_algorithm* alg);
moea_status moea_algorithm_initialize(moea_algorithm* alg);
moea_status moea_algorithm_step(moea_algorithm* alg);
/* Runs the remaining generations; *h_total_ms receives the device time of
 * the loop (CUDA events, like run_device, algorithm.cu:313-329). */
moea_status moea_algorithm_run(moea_algorithm* alg, double* h_total_ms);
moea_status moea_algorithm_reset(moea_algorithm* alg);
moea_status moea_algorithm_synchronize(moea_algorithm* alg);
/* Runs finalize (front-0 indices for RVEA) before results are read, saves
 * the current generation's snapshot when one is due and waits for the
 * snapshot files (the reference saves at result(), algorithm.cu:357-366). */
moea_status moea_algorithm_finalize(moea_algorithm* alg);
/* Waits until every snapshot queued so far is on disk and returns the first
 * file error since the last call.  No counterpart in the reference, whose
 * recorder writes synchronously (data_recorder.cu:219-292). */
moea_status moea_algorithm_flush_snapshots(moea_algorithm* alg);
/* Resume.  Replaces the state of an algorithm (initialized first if needed)
 * by a generation directory of its snapshots: population, ranks or active
 * count, adapted directions, running ideal point, niching counter and
 * generation.  The following steps equal those of the run that wrote it,
 * bit for bit, when the configuration is the same.  Sizes are checked
 * against the configuration.  No counterpart in the reference, which only
 * saves. */
moea_status moea_algorithm_load_snapshot(moea_algorithm* alg, const char* generation_directory);

typedef struct moea_population_view {
    float* d_variables;       /* (N,D) */
    float* d_objectives;      /* (M,N) */
    float* d_constraints;     /* (N) */
    const int* d_auxiliary;   /* result indices (fronts for NSGA-III, front-0 for RVEA) */
    int auxiliary_count;
    int size, dimension, objectives;
    int active_count;
    int generation;
    int initialized, finished;
    int device;
    double total_ms;
    int kernels_per_generation; /* kernel nodes of the captured generation graph (0 if not captured) */
    int graph_active;           /* 1 when generations replay a CUDA graph */
    int last_max_front;         /* reserved (-1); see moea_algorithm_selection_stats */
    int last_sizes[4];
} moea_population_view;

/* NSGA-III: index of the last front and {N_prior, N_last, N_rem, N_nds} of the
 * latest selection (synchronises the algorithm's stream).  Replaces run_ndsort's
 * max_front and NumNDSData (nat/src/selection/nsga3/kernels/non_dominated_sort.cu:1407,
 * :1636). */
moea_status moea_algorithm_selection_stats(moea_algorithm* alg, int* h_max_front, int* h_sizes);

moea_status moea_algorithm_view(moea_algorithm* alg, moea_population_view* out);
/* Reference directions in use: d_values (M,count).  Replaces
 * IReferenceDirectionProvider::view()
 * (nat/include/cuda_moea/reference/reference_direction_provider.cuh:18). */
moea_status moea_algorithm_directions(moea_algorithm* alg, const float** d_values, int* count);
/* Runs one generation with direct launches and CUDA events between its
 * stages: h_ms[i] is the device time of stage i, h_names the '\n'-separated
 * stage names (both up to cap / names_cap). */
moea_status moea_algorithm_profile_step(moea_algorithm* alg, char* h_names, size_t names_cap,
                                        float* h_ms, int cap, int* h_count);
/* Device status of the last generation (0 ok); also returned as a status by step.
 * Replaces the reference's CUDA error path, which exits the process
 * (nat/include/cuda_moea/core/cuda/cuda_utils.cuh:16-22). */
moea_status moea_algorithm_device_status(moea_algorithm* alg, int* h_status);

/* ========================================================================
 * Batched instances (the batching form; no counterpart in the reference,
 * whose algorithms run one at a time).  count independent algorithms with
 * built-in problems and mating, one device and one max_generations, advance
 * together with one CUDA graph launch per generation.  Each instance's
 * results equal those of running it alone with moea_algorithm_*.
 *   Fused mode (when every instance is NSGA-III on a built-in unconstrained
 *   problem with at most 256 g-terms, 2N <= 8192, fixed directions, no CV
 *   quantisation): every stage is one launch for all instances.
 *   The fused instances are split into groups of similar pair-test load
 *   (MOEA_BATCH_GROUPS(g) in flags, default 16); each group's chain of
 *   kernels is a parallel branch of the graph.
 *   Otherwise (or with MOEA_BATCH_NO_FUSION): each instance's generation is
 *   a parallel branch of the graph.
 * cfgs[i].stream and use_graphs are ignored; stream (NULL = internal) orders
 * all of the batch's work.
 * ====================================================================== */
typedef struct moea_batch moea_batch;
#define MOEA_BATCH_NO_FUSION 1
/* Autotuned schedule (fused mode, unless MOEA_BATCH_GROUPS is given): a
 * scratch copy of the batch runs min(10, max_generations/4) generations, times
 * every instance's fused generation alone, then times the default schedule and
 * longest-processing-time schedules on those measured costs for 1, 2, 4, ...
 * groups (graph branches); the fastest is used.  On that schedule each
 * objective count present then tries the half-width dominance tiles (below)
 * and keeps them where the generation got faster.  The choice is cached per
 * device and instance mix for the life of the process.  Results do not depend
 * on the schedule or the tile shape. */
#define MOEA_BATCH_AUTOTUNE 2
/* Fused mode: half-width dominance tiles for every objective count (twice the
 * tile CTAs, each staging half the word tables).  Without it, and without
 * MOEA_BATCH_AUTOTUNE, every objective count uses the full-width tiles. */
#define MOEA_BATCH_HALF_TILES 4
#define MOEA_BATCH_GROUPS(g) (((g) & 0xFF) << 8)
moea_status moea_batch_create(const moea_algorithm_config* cfgs, int count, void* stream, int flags,
                              moea_batch** out);
void moea_batch_destroy(moea_batch* b);
moea_status moea_batch_step(moea_batch* b);
/* generations < 0: run to max_generations.  *h_total_ms: device time. */
moea_status moea_batch_run(moea_batch* b, int generations, double* h_total_ms);
moea_status moea_batch_synchronize(moea_batch* b);
moea_status moea_batch_info(moea_batch* b, int* h_count, int* h_generation, int* h_graph_kernels,
                            int* h_fused);
/* The batch's schedule: number of groups (graph branches of the fused
 * generation; 0 when not fused), how it was chosen (0 the default pair-test
 * assignment, 1 autotuned by this batch, 2 autotuned earlier for the same
 * mix), the autotuner's measured generation time of the chosen and of the
 * default schedule, of the slowest instance run alone and of all instances
 * run alone one after another (ms; 0 when not tuned), and the group of each
 * instance (h_group_of, count entries, may be NULL).  No counterpart in the
 * reference. */
moea_status moea_batch_schedule(moea_batch* b, int* h_groups, int* h_source, float* h_tuned_ms,
                                float* h_default_ms, float* h_slowest_ms, float* h_serial_ms, int* h_group_of);
/* Dominance tile shape of the fused generation per objective count:
 * h_shapes[m] for m = 0 .. cap-1 (0 full-width tiles, 1 half-width; entries
 * of objective counts absent from the batch are 0).  No counterpart in the
 * reference. */
moea_status moea_batch_tile_shapes(moea_batch* b, int* h_shapes, int cap);
/* Population view of instance `index` (same contract as moea_algorithm_view). */
moea_status moea_batch_view(moea_batch* b, int index, moea_population_view* out);

/* ---- problem plugins: C++ IProblemEvaluator libraries ------------------
 * A plugin is a shared library built against the plugin SDK
 * (cuda-moea_b200/sdk/include: IProblemEvaluator, PopulationView,
 * ProblemConfig, CUDA_MOEA_REGISTER_PROBLEM), which repeats the names of the
 * reference's SDK (nat/include/cuda_moea/native/plugin.cuh:35-58,
 * problem/problem_evaluator.cuh:10-31), so reference problem sources build
 * against it unchanged.  Replaces the reference's loader
 * (python/csrc/native_problem.cpp). */
typedef struct moea_native_problem moea_native_problem;

/* Loads a problem library and checks its registration (entry point
 * cuda_moea_problem_v1: ABI 1, this SDK's build id, a name, unique parameter
 * names). */
moea_status moea_native_open(const char* library_path, moea_native_problem** out);
/* Waits for the problem's stream, destroys the problem, unloads the library. */
void moea_native_close(moea_native_problem* p);
/* The registration as JSON: {"name", "build_id", "parameters": {name:
 * {"type", "default", "description"}}}, types int, float, bool, str,
 * float_list.  *needed receives the size with the terminating zero. */
moea_status moea_native_schema(const moea_native_problem* p, char* buf, size_t cap, size_t* needed);
/* A parameter value for moea_native_create.  Its type must be the type of
 * the registered default (a float parameter also takes an integer); unknown
 * names are rejected. */
moea_status moea_native_set_int(moea_native_problem* p, const char* name, long long value);
moea_status moea_native_set_float(moea_native_problem* p, const char* name, double value);
moea_status moea_native_set_bool(moea_native_problem* p, const char* name, int value);
moea_status moea_native_set_string(moea_native_problem* p, const char* name, const char* value);
moea_status moea_native_set_floats(moea_native_problem* p, const char* name, const double* values, int count);
/* Constructs the problem (the plugin's constructor) with the values set and
 * the defaults of the rest.  name must be the registered name; the problem's
 * ProblemInfo must repeat dimension, objectives and the bounds. */
moea_status moea_native_create(moea_native_problem* p, const char* name, int dimension, int objectives,
                               const float* h_lower, const float* h_upper);
moea_status moea_native_constraint_count(const moea_native_problem* p, int* out);
/* The problem as callback hooks of moea_algorithm_config (evaluate, prepare,
 * problem_reset with evaluate_user = the handle).  moea_native_evaluate can
 * also be called directly: it evaluates d_vars (N,D) into d_objs (M,N) and
 * d_cv (N) on stream.  The first call runs the plugin's initialize. */
int moea_native_evaluate(void* p, const float* d_vars, float* d_objs, float* d_cv, int N, int D, int M,
                         int generation, int max_generations, void* stream);
int moea_native_prepare(void* p, float* d_vars, float* d_objs, float* d_cv, int N, int D, int M, int generation,
                        int max_generations, void* stream, int* h_changed);
void moea_native_reset(void* p);

/* Diagnostic for the bounded device waits.  Runs one of them against a
 * condition that never completes, with a limit of limit_ns (1 ns .. 2 s),
 * and reports what a caller of the real kernel would see: which 0 is the
 * counted front barrier of the lane-owned peel, 1 the grid barrier of the
 * general peel (both report MOEA_ERR_DEVICE_TIMEOUT "front peeling"), 2 the
 * mbarrier wait of the tensor-core association (MOEA_ERR_DEVICE_TIMEOUT
 * "association").  The wait gives up, the kernel returns and the workspace
 * stays usable; nothing faults.  No counterpart in the reference, whose
 * device waits are unbounded. */
moea_status moea_selftest_wait_timeout(moea_workspace* ws, int which, unsigned long long limit_ns, void* stream);

#ifdef __cplusplus
}
#endif
#endif
