// Strategy handles of the C ABI: the reference's strategy interfaces
// (IReferenceDirectionProvider, IMatingSelector, ICrossoverOperator,
// IMutationOperator, IEnvironmentSelector; nat/include/cuda_moea/...) as
// opaque objects over the same stage functions the algorithm object runs.
//
// Semantics follow the reference's strategy classes:
//   DasDennisDirections / AdaptiveRVEADirections / UserDefinedDirections
//       nat/src/reference/reference_directions.cu:16-237
//   RandomMating / TournamentMating        nat/src/reproduction/mating_selection.cu:37-108
//   SimulatedBinaryCrossover               nat/src/reproduction/sbx_crossover.cu:73-190
//   PolynomialMutation                     nat/src/reproduction/polynomial_mutation.cu:63-124
//   NSGA3EnvironmentSelector               nat/src/selection/nsga3/nsga3_environment_selector.cu:50-566
//   RVEAEnvironmentSelector                nat/src/selection/rvea/rvea_environment_selector.cu:52-324
//
// The mechanism differs where the algorithm object's does: every quantity the
// reference reads back to the host (front sizes, the RVEA active count) stays
// on the device, so no call below waits for the GPU except those documented
// as synchronising (active_count, RVEA finalize).  Draws come from the same
// Philox streams as the algorithm object's, keyed by the derived run seed and
// the generation, so a generation assembled from handles equals the
// algorithm's generation bit for bit.
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "internal.cuh"

namespace moea {

int workspace_init(Workspace& ws, int device, int n_max, int m_max, int h_max);
void workspace_free(Workspace& ws);
int workspace_check_status(Workspace& ws, cudaStream_t stream);
int run_nsga3_select(Workspace& ws, const SplitPop& pop, int M, int N, const float* refs, int H,
                     uint64_t seed, float* ideal_last, int* survivors, int* survivor_fronts,
                     int assoc_mode, cudaStream_t stream, const SplitPop* sort_pop);
int run_quantize_cv(const float* cv, float* out, int n, float eps, float clip, float log_alpha,
                    int bins, cudaStream_t stream);
int run_mating(const float* cv, const int* rank, const int* d_active, int active, int n_off,
               uint64_t seed, const int* d_gen, uint32_t gen, int* pidx, cudaStream_t stream);
int run_rvea_translate(const SplitPop& pop, int M, float* t, int t_stride, float* zmin,
                       cudaStream_t s);
int run_rvea_partition(const float* t, int t_stride, int n, const float* refs, int M, int K,
                       const int* d_active, int n_active, int n_parent, float* theta, int* idx,
                       cudaStream_t s);
int run_rvea_gamma(const float* refs, int M, int K, float* gamma, cudaStream_t s);
int run_rvea_apd(const float* t, int t_stride, int n, const float* theta, const float* gamma,
                 const int* idx, int M, int K, const float* ps_table, const int* d_gen,
                 float ps_host, float* apd, cudaStream_t s);
float rvea_penalty_scale(int M, int gen, int max_gen, float alpha);
int run_rvea_elitism(Workspace& ws, const int* idx, const SplitPop& pop, const float* apd, int N,
                     int K, int* survivors, int* d_active, cudaStream_t s);
int run_rvea_update(const SplitPop& pop, const float* vars_a, const float* vars_b,
                    const int* survivors, const int* d_active, int N, int D, int M, float* vars,
                    float* objs, float* cv, cudaStream_t s, int* nan_rows = nullptr);
int run_rvea_adapt(const float* v0, const float* objs, int stride, const int* d_active,
                   int n_active, int M, int K, float* range_tmp, float* v, cudaStream_t s);
int run_gather_next(const float* vars_a, const float* vars_b, const SplitPop& pop, const int* survivors,
                    const int* fronts, int N, int D, int M, float* vars, float* objs, float* cv, int* rank,
                    cudaStream_t stream);
int run_front_zero(Workspace& ws, const float* objs, const float* cv, int n_stride, int active, int M,
                   int* out, int* h_count, cudaStream_t stream);
int das_dennis(int mode, int n, int M, std::vector<float>& out);
int normalize_user_directions(std::vector<float>& v, int M, int count);

namespace {

template <class T>
int dmalloc(T** p, size_t count)
{
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (count > 0 ? count : 1));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(e == cudaErrorMemoryAllocation ? MOEA_ERR_OUT_OF_MEMORY : MOEA_ERR_CUDA,
                         "cudaMalloc: %s", cudaGetErrorString(e));
    }
    return MOEA_OK;
}

template <class T>
void dfree(T*& p)
{
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// AnnealedValue of the SBX / PM distribution indices: the kernels anneal on
// the device from (begin, end, generation, total), as the fused pass does.
bool valid_pop(const moea_population_desc* p, bool need_objs)
{
    return p && p->d_variables && p->d_bounds && p->size > 0 && p->dimension > 0 &&
           (!need_objs || (p->d_objectives && p->d_constraints && p->objectives > 0));
}

__global__ void set_int(int* p, int v) { *p = v; }

}  // namespace
}  // namespace moea

using namespace moea;

enum { kDirsDasDennis = 0, kDirsAdaptive = 1, kDirsUser = 2 };

struct moea_directions {
    int kind = kDirsDasDennis;
    int partitions = 0;
    float frequency = 0.1f;
    std::vector<float> user;
    int user_M = 0, user_count = 0;
    bool normalize = true;
    int M = 0, count = 0, device = 0;
    float* values = nullptr;
    float* initial = nullptr;
    float* gamma = nullptr;
    float* range_tmp = nullptr;
    bool ready = false;

    void release()
    {
        dfree(values);
        dfree(initial);
        dfree(gamma);
        dfree(range_tmp);
        ready = false;
    }
    ~moea_directions() { release(); }
};

enum { kMatingRandom = 0, kMatingTournament = 1 };

struct moea_mating {
    int kind = kMatingTournament;
};

struct moea_crossover {
    float eta0 = 30.0f, eta1 = 30.0f, prob = 1.0f, copy = 0.0f;
};

struct moea_mutation {
    float eta0 = 20.0f, eta1 = 20.0f, prob = 1.0f;
};

struct moea_selector {
    bool nsga3 = true;
    moea_nsga3_selector_config ncfg{};
    float alpha = 2.0f;
    int N = 0, D = 0, M = 0, T = 0, device = 0;
    moea_directions* dirs = nullptr;
    Workspace ws;
    bool ws_ready = false;
    int assoc_mode = MOEA_ASSOC_TREE;
    // NSGA-III state
    int* rank = nullptr;             // (N) fronts of the current parents
    float* ideal_last = nullptr;     // (M) running ideal point
    bool ideal_ready = false;
    float* cv_sort[2] = {};          // quantised violations (parents, offspring)
    // RVEA state
    int* d_active = nullptr;         // (1)
    float* t_buf = nullptr;          // (M, 2N)
    float* theta = nullptr;          // (2N)
    float* apd = nullptr;            // (2N)
    int* part_idx = nullptr;         // (2N)
    float* zmin = nullptr;           // (M)
    float* own_gamma = nullptr;      // (H) for providers without gamma
    int* frontzero = nullptr;        // (N)
    int frontzero_count = 0;
    int* survivors = nullptr;        // (2N)

    void release()
    {
        void* ptrs[] = {rank, ideal_last, cv_sort[0], cv_sort[1], d_active, t_buf, theta, apd, part_idx, zmin,
                        own_gamma, frontzero, survivors};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        rank = part_idx = d_active = frontzero = survivors = nullptr;
        ideal_last = t_buf = theta = apd = zmin = own_gamma = nullptr;
        cv_sort[0] = cv_sort[1] = nullptr;
        if (ws_ready) {
            workspace_free(ws);
            ws_ready = false;
        }
    }
    ~moea_selector() { release(); }

    const float* gamma() const { return (dirs && dirs->gamma) ? dirs->gamma : own_gamma; }
};

namespace {

template <class T>
moea_status make_handle(T** out)
{
    if (!out) return set_error(MOEA_ERR_INVALID_ARGUMENT, "null output handle");
    *out = new (std::nothrow) T();
    if (!*out) return set_error(MOEA_ERR_OUT_OF_MEMORY, "out of host memory");
    return MOEA_OK;
}

uint64_t run_seed(const moea_generation_desc* ctx) { return derive_seed(ctx->seed); }

}  // namespace

extern "C" {

// ---------------------------------------------------------------- directions
moea_status moea_create_dasdennis(int partitions, moea_directions** out)
{
    if (partitions < 0) return set_error(MOEA_ERR_INVALID_ARGUMENT, "Das-Dennis partitions cannot be negative");
    MOEA_TRY(make_handle(out));
    (*out)->kind = kDirsDasDennis;
    (*out)->partitions = partitions;
    return MOEA_OK;
}

moea_status moea_create_adaptive_directions(float frequency, moea_directions** out)
{
    MOEA_TRY(make_handle(out));
    (*out)->kind = kDirsAdaptive;
    (*out)->frequency = frequency;  // checked at initialize, as in the reference
    return MOEA_OK;
}

moea_status moea_create_user_directions(const float* h_values, int M, int count, int normalize,
                                        moea_directions** out)
{
    if (!h_values || M <= 0 || count <= 0)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "User directions must have shape (objective_count, count)");
    MOEA_TRY(make_handle(out));
    moea_directions* d = *out;
    d->kind = kDirsUser;
    d->user.assign(h_values, h_values + (size_t)M * count);
    d->user_M = M;
    d->user_count = count;
    d->normalize = normalize != 0;
    return MOEA_OK;
}

moea_status moea_directions_initialize(moea_directions* d, int requested_count, int M, int device, void* stream)
{
    if (!d || M <= 0 || M > kMaxObjectives)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "directions_initialize: bad arguments");
    const cudaStream_t s = (cudaStream_t)stream;
    std::vector<float> host;
    int count = 0;
    if (d->kind == kDirsUser) {
        if (M != d->user_M)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "User direction objective count does not match the problem");
        host = d->user;
        count = d->user_count;
        if (d->normalize) MOEA_TRY(normalize_user_directions(host, M, count));
    } else if (d->kind == kDirsAdaptive) {
        if (!(d->frequency > 0.0f && d->frequency <= 1.0f))
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "RVEA reference adaptation frequency must be in (0, 1]");
        count = das_dennis(2, requested_count, M, host);
    } else {
        count = das_dennis(d->partitions > 0 ? 1 : 0, d->partitions > 0 ? d->partitions : requested_count, M, host);
    }
    if (count < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "no reference directions for %d points and %d objectives",
                         requested_count, M);
    MOEA_CUDA_TRY(cudaSetDevice(device));
    d->release();
    d->M = M;
    d->count = count;
    d->device = device;
    MOEA_TRY(dmalloc(&d->values, (size_t)M * count));
    MOEA_TRY(dmalloc(&d->initial, (size_t)M * count));
    MOEA_CUDA_TRY(cudaMemcpyAsync(d->values, host.data(), sizeof(float) * host.size(), cudaMemcpyHostToDevice, s));
    MOEA_CUDA_TRY(cudaMemcpyAsync(d->initial, host.data(), sizeof(float) * host.size(), cudaMemcpyHostToDevice, s));
    if (d->kind == kDirsAdaptive) {
        MOEA_TRY(dmalloc(&d->gamma, (size_t)count));
        MOEA_TRY(dmalloc(&d->range_tmp, (size_t)M));
        MOEA_TRY(run_rvea_gamma(d->values, M, count, d->gamma, s));
    }
    // the host vector goes out of scope: the copies must have read it
    MOEA_CUDA_TRY(cudaStreamSynchronize(s));
    d->ready = true;
    return MOEA_OK;
}

moea_status moea_directions_view(moea_directions* d, const float** d_values, const float** d_initial,
                                 const float** d_gamma, int* M, int* count)
{
    if (!d || !d->ready) return set_error(MOEA_ERR_STATE, "reference directions are not initialized");
    if (d_values) *d_values = d->values;
    if (d_initial) *d_initial = d->initial;
    if (d_gamma) *d_gamma = d->gamma;
    if (M) *M = d->M;
    if (count) *count = d->count;
    return MOEA_OK;
}

moea_status moea_directions_update(moea_directions* d, const moea_population_desc* pop, const int* d_active,
                                   const moea_generation_desc* ctx, void* stream)
{
    if (!d || !d->ready || !ctx) return set_error(MOEA_ERR_STATE, "reference directions are not initialized");
    if (d->kind != kDirsAdaptive) return MOEA_OK;  // fixed providers do not update
    if (!pop || !pop->d_objectives || pop->objectives != d->M || pop->size <= 0)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "directions_update: population does not match the directions");
    const int interval = std::max(1, (int)std::lround(d->frequency * ctx->max_generations));
    if ((ctx->generation + 1) % interval != 0) return MOEA_OK;
    const cudaStream_t s = (cudaStream_t)stream;
    MOEA_TRY(run_rvea_adapt(d->initial, pop->d_objectives, pop->size, d_active, pop->size, d->M, d->count,
                            d->range_tmp, d->values, s));
    return run_rvea_gamma(d->values, d->M, d->count, d->gamma, s);
}

moea_status moea_directions_reset(moea_directions* d, void* stream)
{
    if (!d || !d->ready) return MOEA_OK;
    const cudaStream_t s = (cudaStream_t)stream;
    MOEA_CUDA_TRY(cudaMemcpyAsync(d->values, d->initial, sizeof(float) * (size_t)d->M * d->count,
                                  cudaMemcpyDeviceToDevice, s));
    if (d->gamma) MOEA_TRY(run_rvea_gamma(d->values, d->M, d->count, d->gamma, s));
    return MOEA_OK;
}

void moea_directions_destroy(moea_directions* d) { delete d; }

// ---------------------------------------------------------------- mating
moea_status moea_create_tournament(moea_mating** out)
{
    MOEA_TRY(make_handle(out));
    (*out)->kind = kMatingTournament;
    return MOEA_OK;
}

moea_status moea_create_random_mating(moea_mating** out)
{
    MOEA_TRY(make_handle(out));
    (*out)->kind = kMatingRandom;
    return MOEA_OK;
}

moea_status moea_mating_select(moea_mating* m, const moea_population_desc* parents, const int* d_rank,
                               const int* d_active, int* d_parent_idx, int count,
                               const moea_generation_desc* ctx, void* stream)
{
    if (!m || !parents || !parents->d_constraints || parents->size <= 0 || !d_parent_idx || count < 0 || !ctx)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "mating_select: bad arguments");
    if (m->kind == kMatingTournament && !d_rank)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "TournamentMating requires a rank array for every parent");
    if (count == 0) return MOEA_OK;
    return run_mating(parents->d_constraints, m->kind == kMatingTournament ? d_rank : nullptr, d_active,
                      parents->size, count, run_seed(ctx), nullptr, (uint32_t)ctx->generation, d_parent_idx,
                      (cudaStream_t)stream);
}

void moea_mating_destroy(moea_mating* m) { delete m; }

// ---------------------------------------------------------------- crossover / mutation
moea_status moea_create_sbx(float eta_initial, float eta_final, float probability, float copy_probability,
                            moea_crossover** out)
{
    if (eta_initial <= 0.0f || eta_final <= 0.0f || probability < 0.0f || probability > 1.0f ||
        copy_probability < 0.0f || copy_probability > 1.0f)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "Invalid SBX configuration");
    MOEA_TRY(make_handle(out));
    **out = moea_crossover{eta_initial, eta_final, probability, copy_probability};
    return MOEA_OK;
}

moea_status moea_crossover_apply(moea_crossover* c, const moea_population_desc* parents, const int* d_parent_idx,
                                 moea_population_desc* offspring, const moea_generation_desc* ctx, void* stream)
{
    if (!c || !valid_pop(parents, false) || !valid_pop(offspring, false) || !d_parent_idx || !ctx ||
        parents->dimension != offspring->dimension)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "crossover_apply: bad arguments");
    return run_variation_pass(kPassCrossover, parents->d_variables, d_parent_idx, parents->d_bounds,
                              offspring->d_variables, offspring->size, offspring->dimension, c->eta0, c->eta1,
                              c->prob, c->copy, 0, 20.0f, 20.0f, 1.0f, ctx->max_generations, run_seed(ctx), nullptr,
                              (uint32_t)ctx->generation, (cudaStream_t)stream);
}

void moea_crossover_destroy(moea_crossover* c) { delete c; }

moea_status moea_create_pm(float eta_initial, float eta_final, float probability, moea_mutation** out)
{
    if (eta_initial <= 0.0f || eta_final <= 0.0f || probability < 0.0f || probability > 1.0f)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "Invalid polynomial-mutation configuration");
    MOEA_TRY(make_handle(out));
    **out = moea_mutation{eta_initial, eta_final, probability};
    return MOEA_OK;
}

moea_status moea_mutation_apply(moea_mutation* m, moea_population_desc* offspring, const moea_generation_desc* ctx,
                                void* stream)
{
    if (!m || !valid_pop(offspring, false) || !ctx)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "mutation_apply: bad arguments");
    return run_variation_pass(kPassMutation, nullptr, nullptr, offspring->d_bounds, offspring->d_variables,
                              offspring->size, offspring->dimension, 30.0f, 30.0f, 1.0f, 0.0f, 1, m->eta0, m->eta1,
                              m->prob, ctx->max_generations, run_seed(ctx), nullptr, (uint32_t)ctx->generation,
                              (cudaStream_t)stream);
}

void moea_mutation_destroy(moea_mutation* m) { delete m; }

// ---------------------------------------------------------------- environmental selection
moea_status moea_create_nsga3_selector(const moea_nsga3_selector_config* cfg, moea_selector** out)
{
    moea_nsga3_selector_config c{0.5f, 0, 0.0f, 0.0f, 0.0f, MOEA_ASSOC_TREE};  // NSGA3SelectionConfig defaults
    if (cfg) c = *cfg;
    if (!(c.sparse_ratio > 0.0f)) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NSGA-III sparse_ratio must be positive");
    if (c.cv_bins > 0) {
        const bool ok = std::isfinite(c.cv_clip_upper) && c.cv_clip_upper > 0.0f && std::isfinite(c.cv_log_alpha) &&
                        c.cv_log_alpha >= 0.0f && std::isfinite(c.feasibility_epsilon) &&
                        c.feasibility_epsilon >= 0.0f &&
                        (c.cv_log_alpha == 0.0f || std::log1p(c.cv_log_alpha * c.cv_clip_upper) > 0.0f);
        if (!ok) return set_error(MOEA_ERR_INVALID_ARGUMENT, "Invalid NSGA-III CV quantization configuration");
    }
    if (c.association_mode != MOEA_ASSOC_TREE && c.association_mode != MOEA_ASSOC_SCAN &&
        c.association_mode != MOEA_ASSOC_TENSOR)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "association_mode must be %d, %d or %d", MOEA_ASSOC_TREE,
                         MOEA_ASSOC_SCAN, MOEA_ASSOC_TENSOR);
    MOEA_TRY(make_handle(out));
    (*out)->nsga3 = true;
    (*out)->ncfg = c;
    return MOEA_OK;
}

moea_status moea_create_rvea_selector(float alpha, moea_selector** out)
{
    MOEA_TRY(make_handle(out));
    (*out)->nsga3 = false;
    (*out)->alpha = alpha;  // checked at initialize, as in the reference
    return MOEA_OK;
}

moea_status moea_selector_initialize(moea_selector* s, int population_size, int dimension, int objectives,
                                     int max_generations, moea_directions* directions, int device, void* stream)
{
    if (!s || population_size <= 0 || dimension <= 0 || objectives <= 0 || max_generations <= 0)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "selector_initialize: bad arguments");
    if (objectives > kMaxObjectives)
        return set_error(MOEA_ERR_UNSUPPORTED, "at most %d objectives are supported", kMaxObjectives);
    if (!directions || !directions->ready)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, s->nsga3 ? "NSGA3EnvironmentSelector requires reference directions"
                                                           : "RVEAEnvironmentSelector requires reference directions");
    if (directions->M != objectives)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "reference directions have %d objectives, the problem %d",
                         directions->M, objectives);
    if (s->nsga3 && population_size % 2 != 0)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "The current NSGA-III CUDA backend requires an even population size");
    if (!s->nsga3 && !(s->alpha > 0.0f)) return set_error(MOEA_ERR_INVALID_ARGUMENT, "RVEA alpha must be positive");
    const cudaStream_t st = (cudaStream_t)stream;
    MOEA_CUDA_TRY(cudaSetDevice(device));
    s->release();
    s->N = population_size;
    s->D = dimension;
    s->M = objectives;
    s->T = max_generations;
    s->device = device;
    s->dirs = directions;
    const int N = s->N, M = s->M, H = directions->count;
    MOEA_TRY(workspace_init(s->ws, device, 2 * N, M, H));
    s->ws_ready = true;
    MOEA_TRY(dmalloc(&s->d_active, 1));
    MOEA_TRY(dmalloc(&s->survivors, (size_t)2 * N));
    set_int<<<1, 1, 0, st>>>(s->d_active, N);
    MOEA_CUDA_TRY(cudaGetLastError());
    if (s->nsga3) {
        MOEA_TRY(dmalloc(&s->rank, (size_t)N));
        MOEA_TRY(dmalloc(&s->ideal_last, (size_t)M));
        MOEA_TRY(dmalloc(&s->cv_sort[0], (size_t)N));
        MOEA_TRY(dmalloc(&s->cv_sort[1], (size_t)N));
        MOEA_CUDA_TRY(cudaMemsetAsync(s->rank, 0, sizeof(int) * N, st));
        // adaptive directions change on the device, so they are always scanned
        s->assoc_mode = directions->kind == kDirsAdaptive ? MOEA_ASSOC_SCAN : s->ncfg.association_mode;
        if (s->assoc_mode == MOEA_ASSOC_TREE)
            MOEA_TRY(prepare_direction_tree(s->ws, directions->values, nullptr, M, H, st));
        if (s->assoc_mode == MOEA_ASSOC_TENSOR || (s->assoc_mode == MOEA_ASSOC_TREE && tensor_preferred(M, 2 * N, H)))
            MOEA_TRY(prepare_tensor_directions(s->ws, directions->values, M, H, st));
        s->ideal_ready = false;
    } else {
        MOEA_TRY(dmalloc(&s->t_buf, (size_t)M * 2 * N));
        MOEA_TRY(dmalloc(&s->theta, (size_t)2 * N));
        MOEA_TRY(dmalloc(&s->apd, (size_t)2 * N));
        MOEA_TRY(dmalloc(&s->part_idx, (size_t)2 * N));
        MOEA_TRY(dmalloc(&s->zmin, (size_t)M));
        MOEA_TRY(dmalloc(&s->frontzero, (size_t)N));
        if (!directions->gamma) {  // fixed directions: gamma once (the algorithm object does the same)
            MOEA_TRY(dmalloc(&s->own_gamma, (size_t)H));
            MOEA_TRY(run_rvea_gamma(directions->values, M, H, s->own_gamma, st));
        }
    }
    s->frontzero_count = 0;
    return MOEA_OK;
}

moea_status moea_selector_prepare(moea_selector* s, const moea_population_desc* parents,
                                  const moea_generation_desc* ctx, void* stream)
{
    if (!s || !s->ws_ready) return set_error(MOEA_ERR_STATE, "environment selector is not initialized");
    if (!valid_pop(parents, true) || parents->size != s->N || parents->objectives != s->M || !ctx)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "selector_prepare: population does not match the selector");
    if (!s->nsga3) return MOEA_OK;  // RVEA keeps its active count (rvea_environment_selector.cu:153-159)
    const cudaStream_t st = (cudaStream_t)stream;
    const float* cvp = parents->d_constraints;
    if (s->ncfg.cv_bins > 0) {
        MOEA_TRY(run_quantize_cv(parents->d_constraints, s->cv_sort[0], s->N, s->ncfg.feasibility_epsilon,
                                 s->ncfg.cv_clip_upper, s->ncfg.cv_log_alpha, s->ncfg.cv_bins, st));
        cvp = s->cv_sort[0];
    }
    MOEA_TRY(run_ndsort(s->ws, merged_view(parents->d_objectives, cvp, s->N), s->M, s->N, s->rank, st));
    if (!s->ideal_ready) {
        MOEA_TRY(run_ideal(parents->d_objectives, s->N, s->M, s->N, nullptr, s->ideal_last, st));
        s->ideal_ready = true;
    }
    return MOEA_OK;
}

moea_status moea_selector_select(moea_selector* s, const moea_population_desc* parents,
                                 const moea_population_desc* offspring, moea_population_desc* next,
                                 const moea_generation_desc* ctx, void* stream)
{
    if (!s || !s->ws_ready) return set_error(MOEA_ERR_STATE, "environment selector is not initialized");
    const int N = s->N, D = s->D, M = s->M;
    for (const moea_population_desc* p : {parents, offspring, (const moea_population_desc*)next})
        if (!valid_pop(p, true) || p->size != N || p->dimension != D || p->objectives != M)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "selector_select: a population does not match the selector");
    if (!ctx) return set_error(MOEA_ERR_INVALID_ARGUMENT, "selector_select: no generation context");
    if (s->nsga3 && !s->ideal_ready) return set_error(MOEA_ERR_STATE, "NSGA-III select before prepare");
    const cudaStream_t st = (cudaStream_t)stream;
    SplitPop pop{parents->d_objectives, offspring->d_objectives, parents->d_constraints, offspring->d_constraints,
                 N, N, N, 2 * N};
    const int H = s->dirs->count;
    const float* refs = s->dirs->values;
    if (s->nsga3) {
        SplitPop sort_pop = pop;
        if (s->ncfg.cv_bins > 0) {
            MOEA_TRY(run_quantize_cv(parents->d_constraints, s->cv_sort[0], N, s->ncfg.feasibility_epsilon,
                                     s->ncfg.cv_clip_upper, s->ncfg.cv_log_alpha, s->ncfg.cv_bins, st));
            MOEA_TRY(run_quantize_cv(offspring->d_constraints, s->cv_sort[1], N, s->ncfg.feasibility_epsilon,
                                     s->ncfg.cv_clip_upper, s->ncfg.cv_log_alpha, s->ncfg.cv_bins, st));
            sort_pop.cv_a = s->cv_sort[0];
            sort_pop.cv_b = s->cv_sort[1];
        }
        MOEA_TRY(run_nsga3_select(s->ws, pop, M, N, refs, H, run_seed(ctx), s->ideal_last, s->survivors, nullptr,
                                  s->assoc_mode, st, &sort_pop));
        return run_gather_next(parents->d_variables, offspring->d_variables, pop, s->survivors, s->ws.fronts, N, D,
                               M, next->d_variables, next->d_objectives, next->d_constraints, s->rank, st);
    }
    MOEA_TRY(run_rvea_translate(pop, M, s->t_buf, 2 * N, s->zmin, st));
    MOEA_TRY(run_rvea_partition(s->t_buf, 2 * N, 2 * N, refs, M, H, s->d_active, N, N, s->theta, s->part_idx, st));
    // EvoX's generation count: the first selection uses 1 / max_gen (rvea_environment_selector.cu:236-238)
    MOEA_TRY(run_rvea_apd(s->t_buf, 2 * N, 2 * N, s->theta, s->gamma(), s->part_idx, M, H, nullptr, nullptr,
                          rvea_penalty_scale(M, ctx->generation + 1, ctx->max_generations, s->alpha), s->apd, st));
    MOEA_TRY(run_rvea_elitism(s->ws, s->part_idx, pop, s->apd, N, H, s->survivors, s->d_active, st));
    return run_rvea_update(pop, parents->d_variables, offspring->d_variables, s->survivors, s->d_active, N, D, M,
                           next->d_variables, next->d_objectives, next->d_constraints, st);
}

moea_status moea_selector_mating_state(moea_selector* s, const int** d_rank, const int** d_active)
{
    if (!s || !s->ws_ready) return set_error(MOEA_ERR_STATE, "environment selector is not initialized");
    if (d_rank) *d_rank = s->nsga3 ? s->rank : nullptr;
    if (d_active) *d_active = s->d_active;
    return MOEA_OK;
}

moea_status moea_selector_active_count(moea_selector* s, int* h_active, void* stream)
{
    if (!s || !s->ws_ready || !h_active) return set_error(MOEA_ERR_STATE, "environment selector is not initialized");
    const cudaStream_t st = (cudaStream_t)stream;
    MOEA_CUDA_TRY(cudaMemcpyAsync(h_active, s->d_active, sizeof(int), cudaMemcpyDeviceToHost, st));
    MOEA_CUDA_TRY(cudaStreamSynchronize(st));
    return MOEA_OK;
}

moea_status moea_selector_finalize(moea_selector* s, const moea_population_desc* population, void* stream)
{
    if (!s || !s->ws_ready) return set_error(MOEA_ERR_STATE, "environment selector is not initialized");
    if (s->nsga3) return MOEA_OK;
    if (!valid_pop(population, true) || population->size != s->N || population->objectives != s->M)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "selector_finalize: population does not match the selector");
    int active = 0;
    MOEA_TRY(moea_selector_active_count(s, &active, stream));
    return run_front_zero(s->ws, population->d_objectives, population->d_constraints, s->N, active, s->M,
                          s->frontzero, &s->frontzero_count, (cudaStream_t)stream);
}

moea_status moea_selector_result_indices(moea_selector* s, const int** d_indices, int* count)
{
    if (!s || !s->ws_ready) return set_error(MOEA_ERR_STATE, "environment selector is not initialized");
    if (d_indices) *d_indices = s->nsga3 ? s->rank : s->frontzero;
    if (count) *count = s->nsga3 ? s->N : s->frontzero_count;
    return MOEA_OK;
}

moea_status moea_selector_reset(moea_selector* s, void* stream)
{
    if (!s || !s->ws_ready) return MOEA_OK;
    const cudaStream_t st = (cudaStream_t)stream;
    set_int<<<1, 1, 0, st>>>(s->d_active, s->N);
    MOEA_CUDA_TRY(cudaGetLastError());
    MOEA_CUDA_TRY(cudaMemsetAsync(s->ws.offset_dev, 0, sizeof(unsigned long long), st));
    s->ideal_ready = false;
    s->frontzero_count = 0;
    return MOEA_OK;
}

void moea_selector_destroy(moea_selector* s) { delete s; }

}  // extern "C"
