// The generational algorithm loop behind the NSGA3 / RVEA entry points.
//
// Reference: EvolutionaryAlgorithm (python/csrc/native/src/algorithm/algorithm.cu:104-432),
// the strategy defaults of AlgorithmFactory (src/factory/algorithm_factory.cu:25-118),
// NSGA3EnvironmentSelector (src/selection/nsga3/nsga3_environment_selector.cu) and
// RVEAEnvironmentSelector (src/selection/rvea/rvea_environment_selector.cu).
//
// Differences in mechanism (not in results):
//  - one stream; every per-generation quantity the reference keeps on the host
//    (generation index, RVEA active count, niching RNG offset, APD penalty,
//    constraint activation) lives in device memory, so a generation is a fixed
//    sequence of launches with no host synchronisation and can be captured
//    once into a CUDA graph per population-slot parity and replayed;
//  - the merged parent+offspring population is never materialised (SplitPop);
//  - buffers are allocated once at initialisation (no per-generation pool
//    allocation, dynamic_workspace.cu:3-125).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "internal.cuh"
#include "snapshot.h"

namespace moea {

int workspace_init(Workspace& ws, int device, int n_max, int m_max, int h_max);
void workspace_free(Workspace& ws);
int workspace_check_status(Workspace& ws, cudaStream_t stream);
int run_nsga3_select(Workspace& ws, const SplitPop& pop, int M, int N, const float* refs, int H,
                     uint64_t seed, float* ideal_last, int* survivors, int* survivor_fronts,
                     int assoc_mode, cudaStream_t stream, const SplitPop* sort_pop);
int run_quantize_cv(const float* cv, float* out, int n, float eps, float clip, float log_alpha,
                    int bins, cudaStream_t stream);
int run_problem(int kind, const float* x, int N, int D, int M, float* objs, float* cv,
                cudaStream_t s);
int validate_problem(int kind, int D, int M);
int run_mating(const float* cv, const int* rank, const int* d_active, int active, int n_off,
               uint64_t seed, const int* d_gen, uint32_t gen, int* pidx, cudaStream_t stream);
int run_variation(const float* parents, const int* pidx, const float* bounds, float* off,
                  int n_off, int D, float sbx_eta0, float sbx_eta1, float sbx_prob, float copy_prob,
                  int mutate, float pm_eta0, float pm_eta1, float pm_prob, int total,
                  uint64_t seed, const int* d_gen, uint32_t gen, cudaStream_t stream);
int run_init_uniform(float* vars, const float* bounds, int N, int D, uint64_t seed,
                     cudaStream_t stream);
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
bool rvea_block_eligible(int n, int M, int K);
int run_rvea_select_block(const SplitPop& pop, const float* refs, int M, int K, const float* gamma, int* d_active,
                          int N, const float* ps_table, const int* d_gen, float ps_host, float* t, int t_stride,
                          float* zmin, float* theta, int* idx, float* apd, int* survivors, cudaStream_t s);
int run_rvea_update(const SplitPop& pop, const float* vars_a, const float* vars_b,
                    const int* survivors, const int* d_active, int N, int D, int M, float* vars,
                    float* objs, float* cv, cudaStream_t s, int* nan_rows = nullptr);
int run_fill_int(int* p, int count, int value, cudaStream_t s);
int run_rvea_adapt(const float* v0, const float* objs, int stride, const int* d_active,
                   int n_active, int M, int K, float* range_tmp, float* v, cudaStream_t s);
int das_dennis(int mode, int n, int M, std::vector<float>& out);
int normalize_user_directions(std::vector<float>& v, int M, int count);

namespace {

// Next parents from the survivors: variables row by row (float4 when D is a
// multiple of 4, several rows per block when rows are short), then
// objectives, violations and fronts.
__global__ void gather_next(const float* __restrict__ vars_a, const float* __restrict__ vars_b,
                            SplitPop pop, const int* __restrict__ surv, const int* __restrict__ fronts,
                            int N, int D, int M, float* __restrict__ vars, float* __restrict__ objs,
                            float* __restrict__ cv, int* __restrict__ rank)
{
    const int vec = (D & 3) == 0 ? 4 : 1;
    const int units = D / vec;                                    // per row
    const int lanes = units >= (int)blockDim.x ? (int)blockDim.x : (units < 1 ? 1 : units);
    const int rows_per_block = (int)blockDim.x / lanes;
    const int sub = (int)threadIdx.x / lanes, lane = (int)threadIdx.x % lanes;
    for (int r = blockIdx.x * rows_per_block + sub; r < N && sub < rows_per_block;
         r += gridDim.x * rows_per_block) {
        const int s = surv[r];
        const float* src = (s < pop.n_a) ? vars_a + (size_t)s * D : vars_b + (size_t)(s - pop.n_a) * D;
        float* dst = vars + (size_t)r * D;
        if (vec == 4) {
            copy_units4(reinterpret_cast<float4*>(dst), reinterpret_cast<const float4*>(src), units, lane, lanes);
        } else {
            for (int u = lane; u < units; u += lanes) dst[u] = __ldg(src + u);
        }
    }
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
        const int s = surv[r];
        for (int m = 0; m < M; ++m) objs[(size_t)m * N + r] = pop.obj(m, s);
        cv[r] = pop.cvv(s);
        if (rank) rank[r] = fronts[s];
    }
}

// Blocks of gather_next: its rows per block (as the kernel derives them), at
// most 16 blocks per SM of a 148-SM part, at least enough for the objectives.
int gather_blocks(int N, int D)
{
    const int units = (D % 4 == 0) ? D / 4 : D;
    const int lanes = std::max(1, std::min(256, units));
    const int rows_per_block = 256 / lanes;
    const int blocks = std::max(ceil_div(N, rows_per_block), ceil_div(N, 256));
    return std::max(1, std::min(148 * 16, blocks));
}

__global__ void bump_generation(int* gen) { *gen += 1; }

__global__ void zero_cv_if_inactive(float* cv, int n, const int* __restrict__ active_table,
                                    const int* __restrict__ d_gen)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !active_table[*d_gen]) cv[i] = 0.0f;
}

__global__ void zero_front_pick(const int* __restrict__ fronts, int n, int* __restrict__ flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = fronts[i] == 0 ? 1 : 0;
}

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

}  // namespace

// The next parents from NSGA-III survivors (ascending mixed indices): rows of
// variables, objectives, violations and, when rank is given, the survivors'
// fronts (nsga3_population_update.cu:248-300).
int run_gather_next(const float* vars_a, const float* vars_b, const SplitPop& pop, const int* survivors,
                    const int* fronts, int N, int D, int M, float* vars, float* objs, float* cv, int* rank,
                    cudaStream_t stream)
{
    gather_next<<<gather_blocks(N, D), 256, 0, stream>>>(vars_a, vars_b, pop, survivors, fronts, N, D, M, vars,
                                                          objs, cv, rank);
    MOEA_CUDA_TRY(cudaGetLastError());
    return MOEA_OK;
}

// Front-0 indices of the first `active` points (RVEAEnvironmentSelector::
// finalize, front_zero.cu:200-293): *h_count receives their number (the
// stream is synchronised).
int run_front_zero(Workspace& ws, const float* objs, const float* cv, int n_stride, int active, int M,
                   int* out, int* h_count, cudaStream_t stream)
{
    *h_count = 0;
    if (active <= 0) return MOEA_OK;
    SplitPop pop{objs, objs, cv, cv, n_stride, n_stride, active, active};
    MOEA_TRY(run_ndsort(ws, pop, M, 1, ws.selected, stream));
    zero_front_pick<<<ceil_div(active, 256), 256, 0, stream>>>(ws.selected, active, ws.flags);
    MOEA_TRY(run_flag_compaction(ws, active, out, stream));
    std::vector<int> flags(active);
    MOEA_CUDA_TRY(cudaMemcpyAsync(flags.data(), ws.flags, sizeof(int) * active, cudaMemcpyDeviceToHost, stream));
    MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
    int c = 0;
    for (int v : flags) c += v != 0;
    *h_count = c;
    return workspace_check_status(ws, stream);
}

}  // namespace moea

using namespace moea;

struct moea_algorithm;

namespace {
// Fused generation (one launch per stage for a group of instances): whether
// an algorithm qualifies, its descriptor for one parity of the slot
// rotation, and the launch plan of a group of instances.
bool fused_eligible(const moea_algorithm* a);
BatchInst fused_describe(moea_algorithm* a, int P, int X);
int fused_build_group(const std::vector<moea_algorithm*>& inst, const std::vector<int>& ids, FusedGroup& g,
                      const int* tile_shape = nullptr);
void fused_free_group(FusedGroup& g);
}  // namespace

struct moea_algorithm {
    moea_algorithm_config cfg{};
    std::vector<float> lower, upper, user_dirs, init_pop;
    int N = 0, D = 0, M = 0, T = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Workspace ws;
    bool ws_ready = false;

    float* vars[3] = {};
    float* objs[3] = {};
    float* cv[3] = {};
    int* rank[3] = {};
    float* cv_sort[2] = {};  // quantised violations of parents / offspring
    int P = 0, O = 1, X = 2;
    float* bounds = nullptr;
    int* parent_idx = nullptr;
    float* refs = nullptr;
    float* refs0 = nullptr;
    float* gamma = nullptr;
    int H = 0;
    float* ideal_last = nullptr;
    bool ideal_ready = false;
    int* d_gen = nullptr;
    int* d_active = nullptr;
    float* ps_table = nullptr;
    int* cv_table = nullptr;
    float* t_buf = nullptr;
    float* theta = nullptr;
    float* apd = nullptr;
    int* part_idx = nullptr;
    float* zmin = nullptr;
    int* survivors = nullptr;
    int* frontzero = nullptr;
    int frontzero_count = 0;
    // RVEA: per population slot, the first row from which every row is known
    // to hold the dead-slot NaN sentinels (N: nothing known).  The update
    // fills only the dead rows below it.  Reset whenever the rows may have
    // been written outside the update (start, snapshot load, a population
    // view handed out).
    int* nan_rows = nullptr;
    uint64_t seed = 0;
    uint32_t epoch = 0;
    int generation = 0;
    bool initialized = false;
    double total_ms = 0.0;
    int last_prepared_target = -2;
    cudaGraphExec_t graph[2] = {};
    bool graph_failed = false;
    int graph_kernels = 0;
    // small populations: the generation as the fused kernels of a one-instance group
    bool fused_single = false;
    BatchInst* f_inst[2] = {};
    FusedGroup f_group;
    // snapshots (data-recorder format) and their metadata
    std::string save_dir, problem_label;
    std::unique_ptr<SnapshotWriter> recorder;

    int setup_single_fused();
    int describe_single_fused();

    void drop_graphs()
    {
        for (auto& g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    ~moea_algorithm() { release(); }

    void release()
    {
        recorder.reset();  // waits for queued snapshots
        for (auto& g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        for (auto& d : f_inst)
            if (d) { cudaFree(d); d = nullptr; }
        fused_free_group(f_group);
        fused_single = false;
        void* ptrs[] = {vars[0], vars[1], vars[2], objs[0], objs[1], objs[2], cv[0], cv[1], cv[2],
                        rank[0], rank[1], rank[2], cv_sort[0], cv_sort[1], bounds, parent_idx, refs,
                        refs0, gamma, ideal_last, d_gen, d_active, ps_table, cv_table, t_buf, theta,
                        apd, part_idx, zmin, survivors, frontzero, nan_rows};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        std::memset(vars, 0, sizeof(vars));
        std::memset(objs, 0, sizeof(objs));
        std::memset(cv, 0, sizeof(cv));
        std::memset(rank, 0, sizeof(rank));
        cv_sort[0] = cv_sort[1] = nullptr;
        bounds = refs = refs0 = gamma = ideal_last = ps_table = t_buf = theta = apd = zmin = nullptr;
        parent_idx = d_gen = d_active = cv_table = part_idx = survivors = frontzero = nan_rows = nullptr;
        if (ws_ready) { workspace_free(ws); ws_ready = false; }
        if (own_stream && stream) { cudaStreamDestroy(stream); stream = nullptr; }
    }

    bool nsga3() const { return cfg.algorithm == MOEA_NSGA3; }

    // A callback returned rc: keep the reason it gave, if any.
    static int callback_failed(const char* what, int rc)
    {
        const std::string reason = last_error();
        if (reason.empty()) return set_error(MOEA_ERR_CALLBACK, "%s callback failed (%d)", what, rc);
        return set_error(MOEA_ERR_CALLBACK, "%s callback failed (%d): %s", what, rc, reason.c_str());
    }
    bool constrained() const { return cfg.problem_kind >= 9 && cfg.problem_kind <= 15; }

    // MOEAStdTestEvaluator::is_cv_active (dtlz_kernels.cu:1302-1312)
    bool cv_active(int eval_iter) const
    {
        if (cfg.constraint_activation_ratio <= 0.0f) return true;
        if (eval_iter < 0 || T <= 0) return false;
        const float progress = static_cast<float>(eval_iter + 1) / static_cast<float>(T);
        return progress >= cfg.constraint_activation_ratio;
    }
    bool cv_switch_node(int target) const
    {
        if (target < 0 || last_prepared_target == target) return false;
        if (target == 0) return cv_active(0);
        return !cv_active(target - 1) && cv_active(target);
    }

    int evaluate(int slot, int gen_index)
    {
        if (cfg.problem_kind == 0) {
            set_error(MOEA_OK, "");  // a failing callback may leave its reason
            const int rc = cfg.evaluate(cfg.evaluate_user, vars[slot], objs[slot], cv[slot], N, D, M,
                                        gen_index, T, (void*)stream);
            if (rc != 0) return callback_failed("problem evaluate", rc);
            return MOEA_OK;
        }
        MOEA_TRY(run_problem(cfg.problem_kind, vars[slot], N, D, M, objs[slot], cv[slot], stream));
        if (constrained() && cfg.problem_kind != 15 && !cv_active(gen_index))
            MOEA_CUDA_TRY(cudaMemsetAsync(cv[slot], 0, sizeof(float) * N, stream));
        return MOEA_OK;
    }

    // NSGA3EnvironmentSelector::prepare (nsga3_environment_selector.cu:236-287)
    int prepare()
    {
        if (!nsga3()) return MOEA_OK;
        const float* cvp = cv[P];
        if (cfg.cv_bins > 0) {
            MOEA_TRY(run_quantize_cv(cv[P], cv_sort[0], N, cfg.feasibility_epsilon, cfg.cv_clip_upper,
                                     cfg.cv_log_alpha, cfg.cv_bins, stream));
            cvp = cv_sort[0];
        }
        MOEA_TRY(run_ndsort(ws, merged_view(objs[P], cvp, N), M, N, rank[P], stream));
        if (!ideal_ready) {
            MOEA_TRY(run_ideal(objs[P], N, M, N, nullptr, ideal_last, stream));
            ideal_ready = true;
        }
        return MOEA_OK;
    }

    int directions_init()
    {
        std::vector<float> host;
        int count = 0;
        if (cfg.directions == MOEA_DIRS_USER) {
            if (user_dirs.empty() || cfg.user_direction_count < 1)
                return set_error(MOEA_ERR_INVALID_ARGUMENT, "User directions must have shape (objective_count, count)");
            count = cfg.user_direction_count;
            host = user_dirs;
            if (cfg.normalize_user_directions) MOEA_TRY(normalize_user_directions(host, M, count));
        } else if (cfg.directions == MOEA_DIRS_ADAPTIVE) {
            if (!(cfg.adapt_frequency > 0.0f && cfg.adapt_frequency <= 1.0f))
                return set_error(MOEA_ERR_INVALID_ARGUMENT, "RVEA reference adaptation frequency must be in (0, 1]");
            count = das_dennis(2, N, M, host);
        } else {
            count = das_dennis(cfg.partitions > 0 ? 1 : 0, cfg.partitions > 0 ? cfg.partitions : N, M, host);
        }
        if (count < 1) return set_error(MOEA_ERR_INVALID_ARGUMENT, "no reference directions for N=%d M=%d", N, M);
        H = count;
        MOEA_TRY(dmalloc(&refs, (size_t)M * H));
        MOEA_TRY(dmalloc(&refs0, (size_t)M * H));
        MOEA_TRY(dmalloc(&gamma, (size_t)H));
        MOEA_CUDA_TRY(cudaMemcpyAsync(refs, host.data(), sizeof(float) * host.size(), cudaMemcpyHostToDevice, stream));
        MOEA_CUDA_TRY(cudaMemcpyAsync(refs0, host.data(), sizeof(float) * host.size(), cudaMemcpyHostToDevice, stream));
        MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
        if (!nsga3()) MOEA_TRY(run_rvea_gamma(refs, M, H, gamma, stream));
        return MOEA_OK;
    }

    // Adapted directions change on the device, so they are always scanned.
    int assoc_mode() const
    {
        return cfg.directions == MOEA_DIRS_ADAPTIVE ? MOEA_ASSOC_SCAN : cfg.association_mode;
    }

    int validate()
    {
        if (cfg.population_size <= 0 || cfg.max_generations <= 0)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "Algorithm requires positive population_size and max_generations");
        if (cfg.algorithm != MOEA_NSGA3 && cfg.algorithm != MOEA_RVEA)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "algorithm must be NSGA3 or RVEA");
        if (cfg.dimension <= 0 || cfg.objectives <= 0)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "Problem must provide positive dimensions");
        if (cfg.objectives > kMaxObjectives)
            return set_error(MOEA_ERR_UNSUPPORTED, "at most %d objectives are supported", kMaxObjectives);
        if (cfg.problem_kind == 0 && !cfg.evaluate)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "callback problem without an evaluate function");
        if (cfg.problem_kind != 0) MOEA_TRY(validate_problem(cfg.problem_kind, cfg.dimension, cfg.objectives));
        if (nsga3()) {
            if (cfg.population_size % 2 != 0)
                return set_error(MOEA_ERR_INVALID_ARGUMENT, "The current NSGA-III CUDA backend requires an even population size");
            if (!(cfg.sparse_ratio > 0.0f))
                return set_error(MOEA_ERR_INVALID_ARGUMENT, "NSGA-III sparse_ratio must be positive");
            if (cfg.cv_bins > 0) {
                const bool ok = std::isfinite(cfg.cv_clip_upper) && cfg.cv_clip_upper > 0.0f &&
                                std::isfinite(cfg.cv_log_alpha) && cfg.cv_log_alpha >= 0.0f &&
                                std::isfinite(cfg.feasibility_epsilon) && cfg.feasibility_epsilon >= 0.0f &&
                                (cfg.cv_log_alpha == 0.0f ||
                                 (std::log1p(cfg.cv_log_alpha * cfg.cv_clip_upper) > 0.0f));
                if (!ok) return set_error(MOEA_ERR_INVALID_ARGUMENT, "Invalid NSGA-III CV quantization configuration");
            }
        } else if (!(cfg.rvea_alpha > 0.0f)) {
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "RVEA alpha must be positive");
        }
        if (cfg.sbx_eta_initial <= 0.0f || cfg.sbx_eta_final <= 0.0f || cfg.sbx_probability < 0.0f ||
            cfg.sbx_probability > 1.0f || cfg.sbx_copy_probability < 0.0f || cfg.sbx_copy_probability > 1.0f)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "Invalid SBX configuration");
        if (cfg.mutation && (cfg.pm_eta_initial <= 0.0f || cfg.pm_eta_final <= 0.0f ||
                             cfg.pm_probability < 0.0f || cfg.pm_probability > 1.0f))
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "Invalid polynomial-mutation configuration");
        if (cfg.association_mode != MOEA_ASSOC_TREE && cfg.association_mode != MOEA_ASSOC_SCAN &&
            cfg.association_mode != MOEA_ASSOC_TENSOR)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "association_mode must be %d, %d or %d", MOEA_ASSOC_TREE,
                             MOEA_ASSOC_SCAN, MOEA_ASSOC_TENSOR);
        if (!save_dir.empty() && cfg.save_interval <= 0)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "saveData generation interval must be positive");
        if (cfg.mating == MOEA_MATING_CALLBACK && !cfg.mate)
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "callback mating without a function");
        // only the NSGA-III selector provides ranks (mating_selection.cu:80-86)
        if (cfg.mating == MOEA_MATING_TOURNAMENT && !nsga3())
            return set_error(MOEA_ERR_INVALID_ARGUMENT, "TournamentMating requires a rank array for every parent");
        return MOEA_OK;
    }

    int initialize()
    {
        if (initialized) return MOEA_OK;
        MOEA_TRY(validate());
        N = cfg.population_size;
        D = cfg.dimension;
        M = cfg.objectives;
        T = cfg.max_generations;
        MOEA_CUDA_TRY(cudaSetDevice(cfg.device));
        if (cfg.stream) {
            stream = (cudaStream_t)cfg.stream;
            own_stream = false;
        } else {
            MOEA_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
            own_stream = true;
        }
        seed = derive_seed(cfg.seed);
        for (int s = 0; s < 3; ++s) {
            MOEA_TRY(dmalloc(&vars[s], (size_t)N * D));
            MOEA_TRY(dmalloc(&objs[s], (size_t)M * N));
            MOEA_TRY(dmalloc(&cv[s], (size_t)N));
            MOEA_TRY(dmalloc(&rank[s], (size_t)N));
            MOEA_CUDA_TRY(cudaMemsetAsync(objs[s], 0, sizeof(float) * M * N, stream));
            MOEA_CUDA_TRY(cudaMemsetAsync(cv[s], 0, sizeof(float) * N, stream));
            MOEA_CUDA_TRY(cudaMemsetAsync(rank[s], 0, sizeof(int) * N, stream));
        }
        MOEA_TRY(dmalloc(&cv_sort[0], (size_t)N));
        MOEA_TRY(dmalloc(&cv_sort[1], (size_t)N));
        MOEA_TRY(dmalloc(&bounds, (size_t)2 * D));
        MOEA_TRY(dmalloc(&parent_idx, (size_t)N));
        MOEA_TRY(dmalloc(&ideal_last, (size_t)M));
        MOEA_TRY(dmalloc(&d_gen, 1));
        MOEA_TRY(dmalloc(&d_active, 1));
        MOEA_TRY(dmalloc(&ps_table, (size_t)T + 2));
        MOEA_TRY(dmalloc(&cv_table, (size_t)T + 2));
        MOEA_TRY(dmalloc(&t_buf, (size_t)M * 2 * N));
        MOEA_TRY(dmalloc(&theta, (size_t)2 * N));
        MOEA_TRY(dmalloc(&apd, (size_t)2 * N));
        MOEA_TRY(dmalloc(&part_idx, (size_t)2 * N));
        MOEA_TRY(dmalloc(&zmin, (size_t)M));
        MOEA_TRY(dmalloc(&survivors, (size_t)2 * N));
        MOEA_TRY(dmalloc(&frontzero, (size_t)N));
        MOEA_TRY(dmalloc(&nan_rows, 3));
        std::vector<float> hb(2 * (size_t)D);
        for (int d = 0; d < D; ++d) {
            hb[2 * d] = lower.empty() ? 0.0f : lower[d];
            hb[2 * d + 1] = upper.empty() ? 1.0f : upper[d];
            if (cfg.problem_kind == 15) {  // CSDP box (dtlz_problem.cu)
                static const float lo[7] = {0.5f, 0.45f, 0.5f, 0.5f, 0.875f, 0.4f, 0.4f};
                static const float hi[7] = {1.5f, 1.35f, 1.5f, 1.5f, 2.625f, 1.2f, 1.2f};
                hb[2 * d] = lo[d];
                hb[2 * d + 1] = hi[d];
            }
        }
        MOEA_CUDA_TRY(cudaMemcpyAsync(bounds, hb.data(), sizeof(float) * hb.size(), cudaMemcpyHostToDevice, stream));
        std::vector<float> ps(T + 2);
        std::vector<int> ct(T + 2);
        for (int g = 0; g < T + 2; ++g) {
            ps[g] = rvea_penalty_scale(M, g + 1, T, cfg.rvea_alpha);
            ct[g] = cv_active(g) ? 1 : 0;
        }
        MOEA_CUDA_TRY(cudaMemcpyAsync(ps_table, ps.data(), sizeof(float) * ps.size(), cudaMemcpyHostToDevice, stream));
        MOEA_CUDA_TRY(cudaMemcpyAsync(cv_table, ct.data(), sizeof(int) * ct.size(), cudaMemcpyHostToDevice, stream));
        MOEA_TRY(directions_init());
        MOEA_TRY(workspace_init(ws, cfg.device, 2 * N, M, H));
        ws_ready = true;
        if (nsga3() && assoc_mode() == MOEA_ASSOC_TREE)
            MOEA_TRY(prepare_direction_tree(ws, refs, nullptr, M, H, stream));
        if (nsga3() && (assoc_mode() == MOEA_ASSOC_TENSOR ||
                        (assoc_mode() == MOEA_ASSOC_TREE && tensor_preferred(M, 2 * N, H))))
            MOEA_TRY(prepare_tensor_directions(ws, refs, M, H, stream));
        if (!init_pop.empty()) {
            for (int r = 0; r < N; ++r)
                for (int d = 0; d < D; ++d) {
                    const float v = init_pop[(size_t)r * D + d];
                    if (!std::isfinite(v) || v < hb[2 * d] || v > hb[2 * d + 1])
                        return set_error(MOEA_ERR_INVALID_ARGUMENT,
                                         "initial_population contains a non-finite or out-of-bounds value");
                }
        }
        MOEA_TRY(start_population());
        initialized = true;
        if (cfg.fused_small && fused_eligible(this)) MOEA_TRY(setup_single_fused());
        if (!save_dir.empty()) {
            std::vector<float> lo(D), hi(D);
            for (int d = 0; d < D; ++d) {
                lo[d] = hb[2 * d];
                hi[d] = hb[2 * d + 1];
            }
            recorder.reset(new SnapshotWriter());
            MOEA_TRY(recorder->open(save_dir, cfg.save_interval, snapshot_meta(), lo, hi, refs0, stream));
            MOEA_TRY(snapshot_now());
        }
        return MOEA_OK;
    }

    SnapshotMeta snapshot_meta() const
    {
        static const char* kNames[16] = {nullptr, "DTLZ1", "DTLZ2", "DTLZ3", "DTLZ4", "DTLZ5", "DTLZ6", "DTLZ7",
                                         "ConvexDTLZ2", "C1DTLZ1", "C1DTLZ3", "C2DTLZ2", "C2ConvexDTLZ2",
                                         "C3DTLZ1", "C3DTLZ4", "CSDP"};
        SnapshotMeta m;
        m.algorithm_name = nsga3() ? "NSGA-III" : "RVEA";  // algorithm_factory.cu:16-17
        const int k = cfg.problem_kind;
        m.problem_name = (k >= 1 && k <= 15) ? kNames[k] : problem_label;
        m.N = N;
        m.D = D;
        m.M = M;
        m.H = H;
        m.T = T;
        m.constraint_count = k == 0 ? cfg.constraint_count : (constrained() ? 1 : 0);
        m.seed = cfg.seed;
        return m;
    }

    // Queues the snapshot of the current parents when one is due.
    int snapshot_now()
    {
        if (!recorder) return MOEA_OK;
        SnapshotSave s;
        s.generation = generation;
        s.vars = vars[P];
        s.objs = objs[P];
        s.cv = cv[P];
        s.refs = refs;
        if (nsga3()) {
            s.aux = rank[P];
            s.aux_count = N;
            s.active = N;
        } else {
            s.aux = frontzero;
            s.aux_count = frontzero_count;
            s.d_active = d_active;
        }
        s.ideal = ideal_last;
        s.offset = ws.offset_dev;
        s.epoch = epoch;
        s.last_prepared_target = last_prepared_target;
        s.ideal_ready = ideal_ready ? 1 : 0;
        return recorder->save(s, stream);
    }

    int load_snapshot(const char* dir)
    {
        if (!dir || !*dir) return set_error(MOEA_ERR_INVALID_ARGUMENT, "snapshot: empty directory");
        if (!initialized) MOEA_TRY(initialize());
        MOEA_CUDA_TRY(cudaSetDevice(cfg.device));
        MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
        SnapshotLoad L;
        MOEA_TRY(load_snapshot_files(dir, snapshot_meta(), nsga3(), L));
        auto up = [&](void* dst, const void* src, size_t bytes) {
            return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
        };
        MOEA_CUDA_TRY(up(vars[P], L.vars.data(), sizeof(float) * L.vars.size()));
        MOEA_CUDA_TRY(up(objs[P], L.objs.data(), sizeof(float) * L.objs.size()));
        MOEA_CUDA_TRY(up(cv[P], L.cv.data(), sizeof(float) * L.cv.size()));
        if (nsga3()) MOEA_CUDA_TRY(up(rank[P], L.aux.data(), sizeof(int) * L.aux.size()));
        // adapted directions change during a run; fixed ones were built at initialize
        if (cfg.directions == MOEA_DIRS_ADAPTIVE && H > 0) {
            MOEA_CUDA_TRY(up(refs, L.refs.data(), sizeof(float) * L.refs.size()));
            if (!nsga3()) MOEA_TRY(run_rvea_gamma(refs, M, H, gamma, stream));
        }
        const int active = nsga3() ? N : L.active;
        MOEA_CUDA_TRY(up(d_active, &active, sizeof(int)));
        MOEA_CUDA_TRY(up(d_gen, &L.generation, sizeof(int)));
        MOEA_CUDA_TRY(up(ws.offset_dev, &L.niching_offset, sizeof(unsigned long long)));
        MOEA_CUDA_TRY(up(ideal_last, L.ideal.data(), sizeof(float) * L.ideal.size()));
        MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
        generation = L.generation;
        epoch = L.epoch;
        last_prepared_target = L.last_prepared_target;
        ideal_ready = L.ideal_ready != 0;
        frontzero_count = 0;
        MOEA_TRY(forget_nan_rows());
        drop_graphs();  // captured generations hold the seed of their epoch
        if (fused_single) MOEA_TRY(describe_single_fused());
        return MOEA_OK;
    }

    // Random (or given) parents, their evaluation and the first sort.
    int start_population()
    {
        P = 0; O = 1; X = 2;
        if (!init_pop.empty() && epoch == 0) {
            MOEA_CUDA_TRY(cudaMemcpyAsync(vars[P], init_pop.data(), sizeof(float) * init_pop.size(),
                                          cudaMemcpyHostToDevice, stream));
        } else {
            MOEA_TRY(run_init_uniform(vars[P], bounds, N, D, seed ^ ((uint64_t)epoch << 48), stream));
        }
        MOEA_TRY(evaluate(P, -1));
        generation = 0;
        const int zero = 0;
        MOEA_CUDA_TRY(cudaMemcpyAsync(d_gen, &zero, sizeof(int), cudaMemcpyHostToDevice, stream));
        MOEA_CUDA_TRY(cudaMemcpyAsync(d_active, &N, sizeof(int), cudaMemcpyHostToDevice, stream));
        MOEA_CUDA_TRY(cudaMemsetAsync(ws.offset_dev, 0, sizeof(unsigned long long), stream));
        MOEA_TRY(forget_nan_rows());
        ideal_ready = false;
        last_prepared_target = -2;
        MOEA_TRY(prepare());
        MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
        return workspace_check_status(ws, stream);
    }

    uint64_t gen_seed() const { return seed ^ ((uint64_t)epoch << 48); }

    // No slot's rows are known to hold the sentinels any more.
    int forget_nan_rows()
    {
        return nan_rows ? run_fill_int(nan_rows, 3, N, stream) : MOEA_OK;
    }

    // Reproduction, evaluation and selection of one generation: the part that
    // is replayed from a CUDA graph.
    int generation_body()
    {
        if (fused_single) {
            const BatchInst* d = f_inst[P == 0 ? 0 : 1];
            MOEA_TRY(fused_reproduce(d, f_group, stream));
            MOEA_TRY(fused_evaluate(d, f_group, stream));
            MOEA_TRY(fused_ndsort(d, f_group, stream));
            return fused_select(d, f_group, stream);
        }
        const uint64_t s = gen_seed();
        if (cfg.mating == MOEA_MATING_CALLBACK) {
            const int rc = cfg.mate(cfg.mate_user, vars[P], objs[P], cv[P], nsga3() ? rank[P] : nullptr,
                                    nsga3() ? N : active_count_sync(), parent_idx, N, D, M, generation,
                                    (void*)stream);
            if (rc != 0) return set_error(MOEA_ERR_CALLBACK, "mating callback failed (%d)", rc);
        } else {
            const bool tournament = cfg.mating == MOEA_MATING_TOURNAMENT;
            MOEA_TRY(run_mating(cv[P], tournament ? rank[P] : nullptr, nsga3() ? nullptr : d_active, N, N,
                                s, d_gen, 0, parent_idx, stream));
        }
        stage_mark("mating", stream);
        MOEA_TRY(run_variation(vars[P], parent_idx, bounds, vars[O], N, D, cfg.sbx_eta_initial,
                               cfg.sbx_eta_final, cfg.sbx_probability, cfg.sbx_copy_probability,
                               cfg.mutation, cfg.pm_eta_initial, cfg.pm_eta_final, cfg.pm_probability, T,
                               s, d_gen, 0, stream));
        stage_mark("variation", stream);
        if (cfg.problem_kind == 0) {
            MOEA_TRY(evaluate(O, generation));
        } else {
            MOEA_TRY(run_problem(cfg.problem_kind, vars[O], N, D, M, objs[O], cv[O], stream));
            if (constrained() && cfg.problem_kind != 15)
                zero_cv_if_inactive<<<ceil_div(N, 256), 256, 0, stream>>>(cv[O], N, cv_table, d_gen);
        }
        stage_mark("evaluate", stream);
        SplitPop pop{objs[P], objs[O], cv[P], cv[O], N, N, N, 2 * N};
        if (nsga3()) {
            SplitPop sort_pop = pop;
            if (cfg.cv_bins > 0) {
                MOEA_TRY(run_quantize_cv(cv[P], cv_sort[0], N, cfg.feasibility_epsilon, cfg.cv_clip_upper,
                                         cfg.cv_log_alpha, cfg.cv_bins, stream));
                MOEA_TRY(run_quantize_cv(cv[O], cv_sort[1], N, cfg.feasibility_epsilon, cfg.cv_clip_upper,
                                         cfg.cv_log_alpha, cfg.cv_bins, stream));
                sort_pop.cv_a = cv_sort[0];
                sort_pop.cv_b = cv_sort[1];
            }
            MOEA_TRY(run_nsga3_select(ws, pop, M, N, refs, H, seed, ideal_last, survivors, nullptr,
                                      assoc_mode(), stream, &sort_pop));
            gather_next<<<gather_blocks(N, D), 256, 0, stream>>>(
                vars[P], vars[O], pop, survivors, ws.fronts, N, D, M, vars[X], objs[X], cv[X], rank[X]);
            MOEA_CUDA_TRY(cudaGetLastError());
        } else {
            if (rvea_block_eligible(2 * N, M, H)) {
                // small merged populations: the whole selection in one CTA
                MOEA_TRY(run_rvea_select_block(pop, refs, M, H, gamma, d_active, N, ps_table, d_gen, 0.0f, t_buf,
                                               2 * N, zmin, theta, part_idx, apd, survivors, stream));
            } else {
                MOEA_TRY(run_rvea_translate(pop, M, t_buf, 2 * N, zmin, stream));
                MOEA_TRY(run_rvea_partition(t_buf, 2 * N, 2 * N, refs, M, H, d_active, N, N, theta, part_idx,
                                            stream));
                MOEA_TRY(run_rvea_apd(t_buf, 2 * N, 2 * N, theta, gamma, part_idx, M, H, ps_table, d_gen, 0.0f,
                                      apd, stream));
                MOEA_TRY(run_rvea_elitism(ws, part_idx, pop, apd, N, H, survivors, d_active, stream));
            }
            MOEA_TRY(run_rvea_update(pop, vars[P], vars[O], survivors, d_active, N, D, M, vars[X], objs[X],
                                     cv[X], stream, nan_rows + X));
        }
        bump_generation<<<1, 1, 0, stream>>>(d_gen);
        MOEA_CUDA_TRY(cudaGetLastError());
        stage_mark("survivors", stream);
        return MOEA_OK;
    }

    bool graphable() const
    {
        return cfg.use_graphs && cfg.problem_kind != 0 && cfg.mating != MOEA_MATING_CALLBACK;
    }

    // Work before a generation's body: the constraint activation switch
    // refreshes parent violations and re-sorts them (problem_evaluator
    // prepare_parent, dtlz_kernels.cu:1361-1394).
    int pre_step()
    {
        if (cfg.problem_kind == 0 && cfg.prepare) {
            int changed = 0;
            set_error(MOEA_OK, "");
            const int rc = cfg.prepare(cfg.evaluate_user, vars[P], objs[P], cv[P], N, D, M, generation, T,
                                       (void*)stream, &changed);
            if (rc != 0) return callback_failed("problem prepare", rc);
            if (changed) MOEA_TRY(prepare());
        }
        if (constrained() && cfg.problem_kind != 0 && cv_switch_node(generation)) {
            MOEA_TRY(run_problem(cfg.problem_kind, vars[P], N, D, M, objs[P], cv[P], stream));
            last_prepared_target = generation;
            MOEA_TRY(prepare());
        }
        return MOEA_OK;
    }

    // Work after a generation's body: RVEA direction adaptation
    // (reference_directions.cu:132-162) and the slot rotation.
    int post_step()
    {
        if (cfg.directions == MOEA_DIRS_ADAPTIVE) {
            const int interval = std::max(1, (int)std::lround(cfg.adapt_frequency * T));
            if ((generation + 1) % interval == 0) {
                MOEA_TRY(run_rvea_adapt(refs0, objs[X], N, nsga3() ? nullptr : d_active, N, M, H, zmin,
                                        refs, stream));
                if (!nsga3()) MOEA_TRY(run_rvea_gamma(refs, M, H, gamma, stream));
            }
        }
        std::swap(P, X);
        ++generation;
        return MOEA_OK;
    }

    int step()
    {
        if (!initialized) MOEA_TRY(initialize());
        if (generation >= T) return MOEA_OK;
        MOEA_CUDA_TRY(cudaSetDevice(cfg.device));
        MOEA_TRY(pre_step());
        bool done = false;
        if (graphable() && !graph_failed) {
            const int parity = (P == 0) ? 0 : 1;
            if (!graph[parity]) {
                cudaGraph_t g = nullptr;
                MOEA_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                const int st = generation_body();
                cudaError_t ce = cudaStreamEndCapture(stream, &g);
                if (st == MOEA_OK && ce == cudaSuccess) {
                    size_t count = 0;
                    if (cudaGraphGetNodes(g, nullptr, &count) == cudaSuccess && count > 0) {
                        std::vector<cudaGraphNode_t> nodes(count);
                        cudaGraphGetNodes(g, nodes.data(), &count);
                        int k = 0;
                        for (auto nd : nodes) {
                            cudaGraphNodeType ty;
                            if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++k;
                        }
                        graph_kernels = k;
                    }
                    ce = cudaGraphInstantiate(&graph[parity], g, 0);
                }
                if (g) cudaGraphDestroy(g);
                if (st != MOEA_OK || ce != cudaSuccess) {
                    // capture is an optimisation: fall back to direct launches
                    cudaGetLastError();
                    graph[parity] = nullptr;
                    graph_failed = true;
                }
            }
            if (graph[parity]) {
                MOEA_CUDA_TRY(cudaGraphLaunch(graph[parity], stream));
                done = true;
            }
        }
        if (!done) MOEA_TRY(generation_body());
        MOEA_TRY(post_step());
        return snapshot_now();
    }

    int active_count_sync()
    {
        if (nsga3() || !initialized) return N;
        int a = N;
        cudaMemcpyAsync(&a, d_active, sizeof(int), cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);
        return a;
    }

    // RVEAEnvironmentSelector::finalize: front-0 of the active parents
    // (front_zero.cu:200-293).
    int finalize()
    {
        if (!initialized) return set_error(MOEA_ERR_STATE, "Algorithm has not been initialized");
        if (nsga3()) return MOEA_OK;
        const int active = active_count_sync();
        frontzero_count = 0;
        return run_front_zero(ws, objs[P], cv[P], N, active, M, frontzero, &frontzero_count, stream);
    }

    // finalize plus the snapshot of the current generation (reference result())
    int finalize_and_save()
    {
        MOEA_TRY(finalize());
        if (!recorder) return MOEA_OK;
        MOEA_TRY(snapshot_now());
        return recorder->flush();
    }

    int reset()
    {
        if (!initialized) return MOEA_OK;
        MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
        drop_graphs();  // the draws of the new epoch use a different seed
        ++epoch;
        if (H > 0) {
            MOEA_CUDA_TRY(cudaMemcpyAsync(refs, refs0, sizeof(float) * (size_t)M * H, cudaMemcpyDeviceToDevice,
                                          stream));
            if (!nsga3()) MOEA_TRY(run_rvea_gamma(refs, M, H, gamma, stream));
        }
        total_ms = 0.0;
        frontzero_count = 0;
        if (cfg.problem_kind == 0 && cfg.problem_reset) cfg.problem_reset(cfg.evaluate_user);
        MOEA_TRY(start_population());
        // the draws of the new epoch use another seed
        if (fused_single) MOEA_TRY(describe_single_fused());
        return snapshot_now();
    }
};

extern "C" {

void moea_algorithm_config_defaults(moea_algorithm_config* c, int algorithm)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->algorithm = algorithm;
    c->population_size = 1024;
    c->max_generations = 100;
    c->device = 0;
    c->seed = 2887;
    c->problem_kind = 2;  // DTLZ2
    c->dimension = 12;
    c->objectives = 3;
    c->mating = algorithm == MOEA_NSGA3 ? MOEA_MATING_TOURNAMENT : MOEA_MATING_RANDOM;
    c->sbx_eta_initial = c->sbx_eta_final = 30.0f;
    c->sbx_probability = 1.0f;
    c->sbx_copy_probability = 0.0f;
    c->mutation = 1;
    c->pm_eta_initial = c->pm_eta_final = 20.0f;
    c->pm_probability = 1.0f;
    c->directions = algorithm == MOEA_NSGA3 ? MOEA_DIRS_DAS_DENNIS : MOEA_DIRS_ADAPTIVE;
    c->partitions = 0;
    c->adapt_frequency = 0.1f;
    c->normalize_user_directions = 1;
    c->sparse_ratio = 0.5f;
    c->rvea_alpha = 2.0f;
    c->use_graphs = 1;
    c->fused_small = 1;
}

moea_status moea_algorithm_create(const moea_algorithm_config* cfg, moea_algorithm** out)
{
    if (!cfg || !out) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    moea_algorithm* a = new (std::nothrow) moea_algorithm();
    if (!a) return set_error(MOEA_ERR_OUT_OF_MEMORY, "host allocation failed");
    a->cfg = *cfg;
    const int D = cfg->dimension, M = cfg->objectives, N = cfg->population_size;
    if (cfg->h_lower && D > 0) a->lower.assign(cfg->h_lower, cfg->h_lower + D);
    if (cfg->h_upper && D > 0) a->upper.assign(cfg->h_upper, cfg->h_upper + D);
    if (cfg->h_user_directions && cfg->user_direction_count > 0 && M > 0)
        a->user_dirs.assign(cfg->h_user_directions, cfg->h_user_directions + (size_t)M * cfg->user_direction_count);
    if (cfg->h_initial_population && N > 0 && D > 0)
        a->init_pop.assign(cfg->h_initial_population, cfg->h_initial_population + (size_t)N * D);
    a->cfg.h_lower = a->cfg.h_upper = a->cfg.h_user_directions = a->cfg.h_initial_population = nullptr;
    if (cfg->save_directory) a->save_dir = cfg->save_directory;
    if (cfg->problem_name) a->problem_label = cfg->problem_name;
    a->cfg.save_directory = a->cfg.problem_name = nullptr;
    *out = a;
    return MOEA_OK;
}

void moea_algorithm_destroy(moea_algorithm* a)
{
    if (!a) return;
    if (a->stream) cudaStreamSynchronize(a->stream);
    delete a;
}

moea_status moea_algorithm_initialize(moea_algorithm* a)
{
    if (!a) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL algorithm");
    const int st = a->initialize();
    if (st != MOEA_OK && !a->initialized) a->release();
    return st;
}

moea_status moea_algorithm_step(moea_algorithm* a)
{
    if (!a) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL algorithm");
    return a->step();
}

moea_status moea_algorithm_run(moea_algorithm* a, double* h_total_ms)
{
    if (!a) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL algorithm");
    if (!a->initialized) MOEA_TRY(a->initialize());
    cudaEvent_t e0, e1;
    MOEA_CUDA_TRY(cudaEventCreate(&e0));
    MOEA_CUDA_TRY(cudaEventCreate(&e1));
    MOEA_CUDA_TRY(cudaEventRecord(e0, a->stream));
    int st = MOEA_OK;
    while (st == MOEA_OK && a->generation < a->T) st = a->step();
    cudaEventRecord(e1, a->stream);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != MOEA_OK) return st;
    a->total_ms = ms;
    if (h_total_ms) *h_total_ms = ms;
    return workspace_check_status(a->ws, a->stream);
}

moea_status moea_algorithm_reset(moea_algorithm* a)
{
    if (!a) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL algorithm");
    return a->reset();
}

moea_status moea_algorithm_synchronize(moea_algorithm* a)
{
    if (!a) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL algorithm");
    if (!a->initialized) return MOEA_OK;
    MOEA_CUDA_TRY(cudaStreamSynchronize(a->stream));
    return workspace_check_status(a->ws, a->stream);
}

moea_status moea_algorithm_finalize(moea_algorithm* a)
{
    if (!a) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL algorithm");
    return a->finalize_and_save();
}

moea_status moea_algorithm_flush_snapshots(moea_algorithm* a)
{
    if (!a) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL algorithm");
    return a->recorder ? a->recorder->flush() : MOEA_OK;
}

moea_status moea_algorithm_load_snapshot(moea_algorithm* a, const char* generation_directory)
{
    if (!a) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL algorithm");
    return a->load_snapshot(generation_directory);
}

moea_status moea_algorithm_view(moea_algorithm* a, moea_population_view* v)
{
    if (!a || !v) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(v, 0, sizeof(*v));
    v->size = a->cfg.population_size;
    v->dimension = a->cfg.dimension;
    v->objectives = a->cfg.objectives;
    v->generation = a->generation;
    v->initialized = a->initialized;
    v->finished = a->initialized && a->generation >= a->T;
    v->device = a->cfg.device;
    v->total_ms = a->total_ms;
    v->kernels_per_generation = a->graph_kernels;
    v->graph_active = (a->graph[0] || a->graph[1]) ? 1 : 0;
    v->last_max_front = -1;
    if (!a->initialized) return MOEA_OK;
    // the caller may write the rows it is given
    MOEA_TRY(a->forget_nan_rows());
    v->d_variables = a->vars[a->P];
    v->d_objectives = a->objs[a->P];
    v->d_constraints = a->cv[a->P];
    if (a->nsga3()) {
        v->d_auxiliary = a->rank[a->P];
        v->auxiliary_count = a->N;
    } else {
        v->d_auxiliary = a->frontzero;
        v->auxiliary_count = a->frontzero_count;
    }
    v->active_count = a->active_count_sync();
    return MOEA_OK;
}

moea_status moea_algorithm_selection_stats(moea_algorithm* a, int* h_max_front, int* h_sizes)
{
    if (!a || !h_max_front || !h_sizes) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL argument");
    *h_max_front = -1;
    if (!a->initialized || !a->nsga3()) return MOEA_OK;
    MOEA_CUDA_TRY(cudaMemcpyAsync(h_max_front, a->ws.counters + 2, sizeof(int), cudaMemcpyDeviceToHost, a->stream));
    MOEA_CUDA_TRY(cudaMemcpyAsync(h_sizes, a->ws.sizes, 4 * sizeof(int), cudaMemcpyDeviceToHost, a->stream));
    MOEA_CUDA_TRY(cudaStreamSynchronize(a->stream));
    return MOEA_OK;
}

moea_status moea_algorithm_directions(moea_algorithm* a, const float** d_values, int* count)
{
    if (!a || !d_values || !count) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL argument");
    *d_values = a->refs;
    *count = a->H;
    return MOEA_OK;
}

moea_status moea_algorithm_profile_step(moea_algorithm* a, char* h_names, size_t names_cap,
                                        float* h_ms, int cap, int* h_count)
{
    if (!a || !h_ms || !h_count || cap < 1) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!a->initialized) MOEA_TRY(a->initialize());
    *h_count = 0;
    if (a->generation >= a->T) return set_error(MOEA_ERR_STATE, "algorithm finished");
    StageProfile prof;
    stage_profile() = &prof;
    stage_mark("start", a->stream);
    const bool saved = a->graph_failed;
    a->graph_failed = true;  // direct launches: events between stages
    const int st = a->step();
    a->graph_failed = saved;
    stage_profile() = nullptr;
    cudaStreamSynchronize(a->stream);
    int n = 0;
    size_t used = 0;
    for (size_t i = 1; i < prof.events.size() && n < cap; ++i) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, prof.events[i - 1], prof.events[i]);
        h_ms[n++] = ms;
        if (h_names) {
            const size_t len = std::strlen(prof.names[i]);
            if (used + len + 2 <= names_cap) {
                std::memcpy(h_names + used, prof.names[i], len);
                used += len;
                h_names[used++] = '\n';
                h_names[used] = '\0';
            }
        }
    }
    for (cudaEvent_t e : prof.events) cudaEventDestroy(e);
    *h_count = n;
    if (st != MOEA_OK) return st;
    return workspace_check_status(a->ws, a->stream);
}

moea_status moea_algorithm_device_status(moea_algorithm* a, int* h_status)
{
    if (!a || !h_status) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL argument");
    *h_status = 0;
    if (!a->initialized) return MOEA_OK;
    MOEA_CUDA_TRY(cudaMemcpy(h_status, a->ws.counters + 6, sizeof(int), cudaMemcpyDeviceToHost));
    return MOEA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched instances: many independent algorithms advance one generation per
// CUDA graph launch.  Each instance keeps its own buffers, workspace and
// generation body (so its results are those of running it alone); the batch
// captures all bodies into one graph as parallel branches forked from and
// joined into the batch stream.  Work outside the bodies (initialisation, the
// constraint-activation switch, direction adaptation, views) runs on the
// batch stream, so it is ordered with the graph launches.  Instances peel
// their fronts with one ordinary CTA instead of a cooperative grid, so that
// branches may run side by side.
// ---------------------------------------------------------------------------

namespace {

// Every instance of a fused generation: NSGA-III, built-in unconstrained
// problems with at most 256 g-terms, built-in mating, fixed directions
// searched by the cone tree, no CV quantisation, 2N <= 8192, slots at the
// start of their rotation.
bool fused_eligible(const moea_algorithm* a)
{
    const moea_algorithm_config& c = a->cfg;
    const int k = c.problem_kind == 7 ? a->D - a->M + 1 : a->D - (a->M - 1);
    return a->nsga3() && c.problem_kind >= 1 && c.problem_kind <= 8 && k >= 1 && k <= 256 &&
           2 * a->N <= kFusedMaxPoints && c.mating != MOEA_MATING_CALLBACK &&
           c.directions != MOEA_DIRS_ADAPTIVE && c.cv_bins <= 0 && a->assoc_mode() == MOEA_ASSOC_TREE &&
           direction_tree_ready(a->ws, a->refs, a->M, a->H) && a->ws.tree_depth <= kDirTreeMaxDepth &&
           a->P == 0 && a->X == 2;
}

BatchInst fused_describe(moea_algorithm* a, int P, int X)
{
    const moea_algorithm_config& c = a->cfg;
    Workspace& w = a->ws;
    BatchInst b{};
    b.N = a->N; b.D = a->D; b.M = a->M; b.H = a->H; b.n = 2 * a->N; b.n_max = w.n_max; b.W = w.words;
    b.kind = c.problem_kind; b.tournament = c.mating == MOEA_MATING_TOURNAMENT; b.mutate = c.mutation;
    b.T = a->T;
    b.sbx_eta0 = c.sbx_eta_initial; b.sbx_eta1 = c.sbx_eta_final; b.sbx_prob = c.sbx_probability;
    b.sbx_copy = c.sbx_copy_probability; b.pm_eta0 = c.pm_eta_initial; b.pm_eta1 = c.pm_eta_final;
    b.pm_prob = c.pm_probability;
    b.seed = a->gen_seed(); b.nich_seed = a->seed;
    b.varsP = a->vars[P]; b.objsP = a->objs[P]; b.cvP = a->cv[P]; b.rankP = a->rank[P];
    b.varsO = a->vars[1]; b.objsO = a->objs[1]; b.cvO = a->cv[1];
    b.varsX = a->vars[X]; b.objsX = a->objs[X]; b.cvX = a->cv[X]; b.rankX = a->rank[X];
    b.bounds = a->bounds; b.pidx = a->parent_idx; b.d_gen = a->d_gen; b.ideal = a->ideal_last;
    b.key0 = w.key0; b.key64 = w.key64[0]; b.perm = w.perm[0]; b.vals = w.sel_vals[0];
    b.sorted_f = w.sorted_f; b.qinfo = w.qinfo; b.blocker = w.blocker; b.front_sorted = w.front_sorted;
    b.front_list = w.front_list; b.counters = w.counters; b.rows = w.rows; b.chunk_keys = w.chunk_keys;
    b.chunk_bits = w.chunk_bits; b.fronts = w.fronts; b.nds_gidx = w.nds_gidx; b.sizes = w.sizes;
    b.nds_objs = w.nds_objs; b.rcp_b = w.rcp_b; b.extreme = w.extreme; b.assoc_idx = w.assoc_idx;
    b.assoc_best = w.assoc_best;
    b.assoc_dist = w.assoc_dist; b.rho = w.rho; b.selected = w.selected; b.flags = w.flags;
    b.survivors = a->survivors; b.offset = w.offset_dev;
    b.t_dirs_orig = a->refs;
    b.t_dirs = w.tree_dirs; b.t_order = w.tree_order; b.t_center = w.tree_center; b.t_cos = w.tree_cos;
    b.t_sin = w.tree_sin; b.t_link = w.tree_link; b.t_nodes = w.tree_nodes; b.t_delta = w.tree_delta;
    return b;
}

// tile_shape[m]: the dominance tile shape of the instances with m objectives
// (nullptr: shape 0 for all).
int fused_build_group(const std::vector<moea_algorithm*>& inst, const std::vector<int>& ids, FusedGroup& g,
                      const int* tile_shape)
{
    g = FusedGroup{};
    g.count = (int)ids.size();
    for (int i : ids) {
        g.max_n = std::max(g.max_n, 2 * inst[i]->N);
        g.max_W = std::max(g.max_W, inst[i]->ws.words);
        g.max_N = std::max(g.max_N, inst[i]->N);
        g.max_D = std::max(g.max_D, inst[i]->D);
        g.max_M = std::max(g.max_M, inst[i]->M);
    }
    MOEA_CUDA_TRY(cudaMalloc((void**)&g.d_ids, sizeof(int) * ids.size()));
    MOEA_CUDA_TRY(cudaMemcpy(g.d_ids, ids.data(), sizeof(int) * ids.size(), cudaMemcpyHostToDevice));
    for (int m = 1; m <= kMaxObjectives; ++m) {
        std::vector<int> bids, prefix{0};
        int mn = 0, mh = 0;
        const int shape = tile_shape ? tile_shape[m] : 0;
        for (int i : ids) {
            if (inst[i]->M != m) continue;
            bids.push_back(i);
            mh = std::max(mh, inst[i]->H);
            const int n = 2 * inst[i]->N;
            prefix.push_back(prefix.back() + fused_tile_blocks(m, n, shape));
            mn = std::max(mn, n);
        }
        if (bids.empty()) continue;
        FusedBucket b;
        b.M = m;
        b.count = (int)bids.size();
        b.max_n = mn;
        b.tile_blocks = prefix.back();
        b.shape = shape;
        b.max_H = mh;
        MOEA_CUDA_TRY(cudaMalloc((void**)&b.d_ids, sizeof(int) * bids.size()));
        MOEA_CUDA_TRY(cudaMalloc((void**)&b.d_tile_prefix, sizeof(int) * prefix.size()));
        MOEA_CUDA_TRY(cudaMemcpy(b.d_ids, bids.data(), sizeof(int) * bids.size(), cudaMemcpyHostToDevice));
        MOEA_CUDA_TRY(cudaMemcpy(b.d_tile_prefix, prefix.data(), sizeof(int) * prefix.size(),
                                 cudaMemcpyHostToDevice));
        g.buckets.push_back(b);
    }
    return MOEA_OK;
}

void fused_free_group(FusedGroup& g)
{
    if (g.d_ids) cudaFree(g.d_ids);
    for (auto& b : g.buckets) {
        if (b.d_ids) cudaFree(b.d_ids);
        if (b.d_tile_prefix) cudaFree(b.d_tile_prefix);
    }
    g = FusedGroup{};
}

}  // namespace

// One-instance fused plan: descriptors of both parities (instance index 0).
int moea_algorithm::describe_single_fused()
{
    for (int parity = 0; parity < 2; ++parity) {
        const BatchInst h = fused_describe(this, parity == 0 ? 0 : 2, parity == 0 ? 2 : 0);
        if (!f_inst[parity]) MOEA_CUDA_TRY(cudaMalloc((void**)&f_inst[parity], sizeof(BatchInst)));
        MOEA_CUDA_TRY(cudaMemcpy(f_inst[parity], &h, sizeof(BatchInst), cudaMemcpyHostToDevice));
    }
    return MOEA_OK;
}

int moea_algorithm::setup_single_fused()
{
    MOEA_TRY(fused_ndsort_configure());
    MOEA_TRY(fused_select_configure());
    MOEA_TRY(describe_single_fused());
    std::vector<moea_algorithm*> self{this};
    MOEA_TRY(fused_build_group(self, {0}, f_group));
    fused_single = true;
    return MOEA_OK;
}

struct moea_batch {
    std::vector<moea_algorithm*> inst;
    // fused mode: one launch per stage for each group of instances; the
    // groups run side by side on their own streams (graph branches)
    bool fused = false;
    int fused_groups = 16;
    BatchInst* d_inst[2] = {};
    std::vector<FusedGroup> groups;
    std::vector<cudaStream_t> gstream;
    std::vector<cudaEvent_t> gjoin;
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0;
    int T = 0;
    int generation = 0;
    bool use_fused = true;
    cudaGraphExec_t graph[2] = {};
    int graph_kernels = 0;
    // the schedule: group of each instance (fused mode), and how it was chosen
    std::vector<int> group_of;
    std::array<int, kMaxObjectives + 1> tile_shape{};  // dominance tile shape per objective count
    int schedule_source = 0;    // 0 pair-test LPT, 1 autotuned now, 2 autotuned earlier (cache)
    std::vector<double> inst_cost;  // measured generation of each instance alone (autotuner), or empty
    float tuned_ms = 0.0f;      // measured generation of the chosen schedule (autotuner)
    float default_ms = 0.0f;    // measured generation of the default schedule (autotuner)
    float slowest_ms = 0.0f;    // the slowest instance's generation run alone (autotuner probe)
    float serial_ms = 0.0f;     // all instances' generations run alone one after another

    ~moea_batch()
    {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto& d : d_inst)
            if (d) cudaFree(d);
        for (auto& g : groups) fused_free_group(g);
        for (cudaStream_t gs : gstream) cudaStreamDestroy(gs);
        for (cudaEvent_t e : gjoin) cudaEventDestroy(e);
        for (moea_algorithm* a : inst) delete a;
        for (cudaStream_t s : branch) cudaStreamDestroy(s);
        for (cudaEvent_t e : join) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    bool fused_possible() const
    {
        for (moea_algorithm* a : inst)
            if (!fused_eligible(a) || a->P != 0 || a->X != 2) return false;
        return true;
    }

    int setup_fused(const std::vector<int>* schedule = nullptr)
    {
        if (!fused_possible()) return MOEA_OK;
        MOEA_TRY(fused_ndsort_configure());
        MOEA_TRY(fused_select_configure());
        const int count = (int)inst.size();
        for (int parity = 0; parity < 2; ++parity) {
            std::vector<BatchInst> h(count);
            for (int i = 0; i < count; ++i) h[i] = fused_describe(inst[i], parity == 0 ? 0 : 2, parity == 0 ? 2 : 0);
            MOEA_CUDA_TRY(cudaMalloc((void**)&d_inst[parity], sizeof(BatchInst) * count));
            MOEA_CUDA_TRY(cudaMemcpy(d_inst[parity], h.data(), sizeof(BatchInst) * count, cudaMemcpyHostToDevice));
        }
        fused = true;
        if (schedule) return build_groups(*schedule);
        // default: longest-processing-time assignment by the pair tests of
        // one generation, (2N)^2, so that every group carries a similar share
        std::vector<double> cost(count);
        for (int i = 0; i < count; ++i) cost[i] = (double)inst[i]->N * inst[i]->N;
        return build_groups(lpt(cost, std::max(1, std::min(fused_groups, count))));
    }

    // Longest-processing-time assignment of the instances to G groups.
    static std::vector<int> lpt(const std::vector<double>& cost, int G)
    {
        const int count = (int)cost.size();
        std::vector<int> order(count), group(count, 0);
        for (int i = 0; i < count; ++i) order[i] = i;
        std::sort(order.begin(), order.end(), [&](int x, int y) {
            return cost[x] > cost[y] || (cost[x] == cost[y] && x < y);
        });
        std::vector<double> load(G, 0.0);
        for (int i : order) {
            const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            group[i] = g;
            load[g] += cost[i];
        }
        return group;
    }

    void free_groups()
    {
        drop_graphs();
        for (auto& g : groups) fused_free_group(g);
        for (cudaStream_t gs : gstream) cudaStreamDestroy(gs);
        for (cudaEvent_t e : gjoin) cudaEventDestroy(e);
        groups.clear();
        gstream.clear();
        gjoin.clear();
    }

    void drop_graphs()
    {
        for (auto& g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    // One fused group per value of group_of (instance -> group); each group's
    // chain of kernels is one branch of the generation's graph.
    int build_groups(const std::vector<int>& schedule)
    {
        free_groups();
        group_of = schedule;
        const int G = schedule.empty() ? 0 : *std::max_element(schedule.begin(), schedule.end()) + 1;
        for (int gi = 0; gi < G; ++gi) {
            std::vector<int> ids;
            for (int i = 0; i < (int)schedule.size(); ++i)
                if (schedule[i] == gi) ids.push_back(i);
            // the costliest instances first: a group's CTAs start in this
            // order, so the long ones do not start last (list scheduling)
            if (inst_cost.size() == schedule.size())
                std::stable_sort(ids.begin(), ids.end(), [&](int x, int y) { return inst_cost[x] > inst_cost[y]; });
            if (ids.empty()) continue;
            FusedGroup g;
            MOEA_TRY(fused_build_group(inst, ids, g, tile_shape.data()));
            groups.push_back(std::move(g));
            cudaStream_t gs = nullptr;
            cudaEvent_t ge = nullptr;
            MOEA_CUDA_TRY(cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking));
            gstream.push_back(gs);
            MOEA_CUDA_TRY(cudaEventCreateWithFlags(&ge, cudaEventDisableTiming));
            gjoin.push_back(ge);
        }
        return MOEA_OK;
    }

    // ---- autotuner (runs on a scratch copy of a batch: it advances and
    // re-runs that copy's generations freely) ----

    // Device time of each instance's fused generation run alone (one group of
    // one instance, direct launches), at the current parity.  The outputs go
    // to the next-population slots and are discarded.
    int probe_costs(std::vector<double>& cost)
    {
        const int count = (int)inst.size();
        const int parity = (inst[0]->P == 0) ? 0 : 1;
        cost.assign(count, 0.0);
        cudaEvent_t e0, e1;
        MOEA_CUDA_TRY(cudaEventCreate(&e0));
        MOEA_CUDA_TRY(cudaEventCreate(&e1));
        int st = MOEA_OK;
        for (int i = 0; i < count && st == MOEA_OK; ++i) {
            FusedGroup g;
            st = fused_build_group(inst, std::vector<int>{i}, g, tile_shape.data());
            if (st != MOEA_OK) break;
            cudaEventRecord(e0, stream);
            st = fused_reproduce(d_inst[parity], g, stream);
            if (st == MOEA_OK) st = fused_evaluate(d_inst[parity], g, stream);
            if (st == MOEA_OK) st = fused_ndsort(d_inst[parity], g, stream);
            if (st == MOEA_OK) st = fused_select(d_inst[parity], g, stream);
            cudaEventRecord(e1, stream);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            cost[i] = ms;
            fused_free_group(g);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st == MOEA_OK) MOEA_CUDA_TRY(cudaGetLastError());
        return st;
    }

    // Best of `reps` replays of the captured generation of a schedule (the
    // same parents each time, so each replay is the same generation's work).
    int time_schedule(const std::vector<int>& schedule, int reps, float* best_ms)
    {
        MOEA_TRY(build_groups(schedule));
        const int parity = (inst[0]->P == 0) ? 0 : 1;
        cudaGraphExec_t g = nullptr;
        MOEA_TRY(capture(&g, parity));
        cudaEvent_t e0, e1;
        MOEA_CUDA_TRY(cudaEventCreate(&e0));
        MOEA_CUDA_TRY(cudaEventCreate(&e1));
        float best = 1e30f;
        cudaGraphLaunch(g, stream);  // warm
        for (int r = 0; r < reps; ++r) {
            cudaEventRecord(e0, stream);
            cudaGraphLaunch(g, stream);
            cudaEventRecord(e1, stream);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            best = std::min(best, ms);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaGraphExecDestroy(g);
        MOEA_CUDA_TRY(cudaGetLastError());
        *best_ms = best;
        return MOEA_OK;
    }

    // Runs `warm` generations, measures every instance alone, then times the
    // pair-test LPT schedule of the default group count and measured-cost LPT
    // schedules of 1, 2, 4, ... count groups (instances in a group ordered by
    // cost, costliest first); *chosen receives the fastest.  Then, on the
    // chosen schedule, each objective count present tries the second
    // dominance tile shape and keeps it where the generation got faster;
    // *shapes receives the result.
    int autotune(int warm, std::vector<int>* chosen, float* chosen_ms, float* dflt_ms, float* slowest,
                 float* serial, std::vector<double>* cost_out, std::array<int, kMaxObjectives + 1>* shapes)
    {
        const int count = (int)inst.size();
        for (int g = 0; g < warm && generation < T - 1; ++g) MOEA_TRY(step());
        std::vector<double> measured;
        MOEA_TRY(probe_costs(measured));
        *cost_out = measured;
        inst_cost = measured;
        *slowest = (float)*std::max_element(measured.begin(), measured.end());
        double total = 0.0;
        for (double c : measured) total += c;
        *serial = (float)total;
        std::vector<double> pairs(count);
        for (int i = 0; i < count; ++i) pairs[i] = (double)inst[i]->N * inst[i]->N;
        std::vector<std::vector<int>> cands;
        cands.push_back(lpt(pairs, std::max(1, std::min(fused_groups, count))));
        for (int G = 1; G <= count; G *= 2) cands.push_back(lpt(measured, G));
        if ((count & (count - 1)) != 0) cands.push_back(lpt(measured, count));
        float best = 1e30f;
        for (size_t c = 0; c < cands.size(); ++c) {
            float ms = 0.0f;
            MOEA_TRY(time_schedule(cands[c], 3, &ms));
            if (c == 0) *dflt_ms = ms;
            if (ms < best) {
                best = ms;
                *chosen = cands[c];
            }
        }
        for (int m = 1; m <= kMaxObjectives; ++m) {
            bool present = false;
            for (moea_algorithm* a : inst) present |= a->M == m;
            if (!present) continue;
            tile_shape[m] = 1;
            float ms = 0.0f;
            MOEA_TRY(time_schedule(*chosen, 3, &ms));
            if (ms < best) best = ms;
            else tile_shape[m] = 0;
        }
        *shapes = tile_shape;
        *chosen_ms = best;
        return MOEA_OK;
    }

    int fused_body(int parity)
    {
        const BatchInst* d = d_inst[parity];
        MOEA_CUDA_TRY(cudaEventRecord(fork, stream));
        for (size_t gi = 0; gi < groups.size(); ++gi) {
            const FusedGroup& g = groups[gi];
            cudaStream_t gs = gstream[gi];
            MOEA_CUDA_TRY(cudaStreamWaitEvent(gs, fork, 0));
            MOEA_TRY(fused_reproduce(d, g, gs));
            MOEA_TRY(fused_evaluate(d, g, gs));
            MOEA_TRY(fused_ndsort(d, g, gs));
            MOEA_TRY(fused_select(d, g, gs));
            MOEA_CUDA_TRY(cudaEventRecord(gjoin[gi], gs));
            MOEA_CUDA_TRY(cudaStreamWaitEvent(stream, gjoin[gi], 0));
        }
        return MOEA_OK;
    }

    int capture(cudaGraphExec_t* out, int parity)
    {
        MOEA_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int st = MOEA_OK;
        cudaError_t ce = cudaSuccess;
        if (fused) {
            st = fused_body(parity);
        } else {
            ce = cudaEventRecord(fork, stream);
        }
        for (size_t i = 0; !fused && i < inst.size() && st == MOEA_OK && ce == cudaSuccess; ++i) {
            moea_algorithm* a = inst[i];
            ce = cudaStreamWaitEvent(branch[i], fork, 0);
            if (ce != cudaSuccess) break;
            a->stream = branch[i];
            st = a->generation_body();
            a->stream = stream;
            if (st == MOEA_OK) ce = cudaEventRecord(join[i], branch[i]);
            if (st == MOEA_OK && ce == cudaSuccess) ce = cudaStreamWaitEvent(stream, join[i], 0);
        }
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(stream, &g);
        if (st == MOEA_OK && ce == cudaSuccess && ee == cudaSuccess) {
            size_t count = 0;
            if (cudaGraphGetNodes(g, nullptr, &count) == cudaSuccess && count > 0) {
                std::vector<cudaGraphNode_t> nodes(count);
                cudaGraphGetNodes(g, nodes.data(), &count);
                int k = 0;
                for (auto nd : nodes) {
                    cudaGraphNodeType ty;
                    if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++k;
                }
                graph_kernels = k;
            }
            ce = cudaGraphInstantiate(out, g, 0);
        }
        if (g) cudaGraphDestroy(g);
        if (st != MOEA_OK) return st;
        if (ce != cudaSuccess || ee != cudaSuccess) {
            const cudaError_t e = ce != cudaSuccess ? ce : ee;
            cudaGetLastError();
            return set_error(MOEA_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
        }
        return MOEA_OK;
    }

    int step()
    {
        if (generation >= T) return MOEA_OK;
        MOEA_CUDA_TRY(cudaSetDevice(device));
        for (moea_algorithm* a : inst) MOEA_TRY(a->pre_step());
        const int parity = (inst[0]->P == 0) ? 0 : 1;
        if (!graph[parity]) MOEA_TRY(capture(&graph[parity], parity));
        MOEA_CUDA_TRY(cudaGraphLaunch(graph[parity], stream));
        for (moea_algorithm* a : inst) MOEA_TRY(a->post_step());
        ++generation;
        return MOEA_OK;
    }
};

namespace {

struct TunedSchedule {
    std::vector<int> schedule;
    std::array<int, kMaxObjectives + 1> tile_shape{};
    std::vector<double> cost;  // each instance's generation alone
    float tuned_ms = 0.0f, default_ms = 0.0f, slowest_ms = 0.0f, serial_ms = 0.0f;
};

std::map<std::string, TunedSchedule>& tuning_cache()
{
    static std::map<std::string, TunedSchedule> cache;
    return cache;
}

std::mutex& tuning_mutex()
{
    static std::mutex m;
    return m;
}

// The instance mix a schedule is tuned for: the device and, per instance in
// order, everything that sets its work (problem, sizes, directions, operators).
std::string batch_signature(const moea_algorithm_config* cfgs, int count)
{
    std::string key;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, cfgs[0].device) == cudaSuccess) key += prop.name;
    key += "|" + std::to_string(count) + "|" + std::to_string(cfgs[0].max_generations);
    for (int i = 0; i < count; ++i) {
        const moea_algorithm_config& c = cfgs[i];
        char buf[256];
        std::snprintf(buf, sizeof(buf), "|%d,%d,%d,%d,%d,%d,%d,%d,%g,%g,%d,%d", c.algorithm, c.problem_kind,
                      c.population_size, c.dimension, c.objectives, c.directions, c.partitions, c.mating,
                      (double)c.sbx_probability, (double)c.sbx_copy_probability, c.mutation, c.association_mode);
        key += buf;
    }
    return key;
}

}  // namespace

extern "C" {

moea_status moea_batch_create(const moea_algorithm_config* cfgs, int count, void* stream, int flags,
                              moea_batch** out)
{
    if (!cfgs || count < 1 || !out) return set_error(MOEA_ERR_INVALID_ARGUMENT, "batch: bad arguments");
    *out = nullptr;
    const int device = cfgs[0].device, T = cfgs[0].max_generations;
    for (int i = 0; i < count; ++i) {
        const moea_algorithm_config& c = cfgs[i];
        if (c.device != device || c.max_generations != T)
            return set_error(MOEA_ERR_INVALID_ARGUMENT,
                             "batch: instance %d differs in device or max_generations from instance 0", i);
        if (c.problem_kind == 0 || c.mating == MOEA_MATING_CALLBACK)
            return set_error(MOEA_ERR_INVALID_ARGUMENT,
                             "batch: instance %d uses a callback; batched instances need built-in problems "
                             "and mating", i);
        if (c.save_directory)
            return set_error(MOEA_ERR_INVALID_ARGUMENT,
                             "batch: instance %d saves snapshots; run it alone to save them", i);
    }
    MOEA_CUDA_TRY(cudaSetDevice(device));
    moea_batch* b = new (std::nothrow) moea_batch();
    if (!b) return set_error(MOEA_ERR_OUT_OF_MEMORY, "host allocation failed");
    b->device = device;
    b->T = T;
    b->use_fused = (flags & MOEA_BATCH_NO_FUSION) == 0;
    if (flags & MOEA_BATCH_HALF_TILES) b->tile_shape.fill(1);
    if (((flags >> 8) & 0xFF) > 0) b->fused_groups = (flags >> 8) & 0xFF;
    int st = MOEA_OK;
    cudaError_t ce = cudaSuccess;
    if (stream) {
        b->stream = (cudaStream_t)stream;
    } else {
        ce = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        b->own_stream = ce == cudaSuccess;
    }
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int i = 0; i < count && st == MOEA_OK && ce == cudaSuccess; ++i) {
        moea_algorithm_config c = cfgs[i];
        c.stream = b->stream;
        c.use_graphs = 0;
        c.fused_small = 0;  // the batch fuses its instances itself
        moea_algorithm* a = nullptr;
        st = moea_algorithm_create(&c, &a);
        if (st != MOEA_OK) break;
        b->inst.push_back(a);
        st = a->initialize();
        if (st != MOEA_OK) {
            const std::string msg = last_error();  // set_error rewrites the buffer it returns
            st = set_error(st, "batch instance %d: %s", i, msg.c_str());
            break;
        }
        a->ws.peel_single_cta = true;
        cudaStream_t s = nullptr;
        cudaEvent_t e = nullptr;
        ce = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (ce == cudaSuccess) b->branch.push_back(s);
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        if (ce == cudaSuccess) b->join.push_back(e);
    }
    if (st == MOEA_OK && ce != cudaSuccess) {
        cudaGetLastError();
        st = set_error(MOEA_ERR_CUDA, "batch: %s", cudaGetErrorString(ce));
    }
    const bool groups_given = ((flags >> 8) & 0xFF) > 0;
    if (st == MOEA_OK && b->use_fused && (flags & MOEA_BATCH_AUTOTUNE) && !groups_given && b->fused_possible()) {
        // the schedule of this instance mix: from the cache, or tuned now on a
        // scratch copy of the batch (same configurations, so the same work)
        const std::string key = batch_signature(cfgs, count);
        std::lock_guard<std::mutex> lock(tuning_mutex());
        auto it = tuning_cache().find(key);
        if (it != tuning_cache().end()) {
            b->inst_cost = it->second.cost;
            b->tile_shape = it->second.tile_shape;
            st = b->setup_fused(&it->second.schedule);
            b->schedule_source = 2;
            b->tuned_ms = it->second.tuned_ms;
            b->default_ms = it->second.default_ms;
            b->slowest_ms = it->second.slowest_ms;
            b->serial_ms = it->second.serial_ms;
        } else {
            moea_batch* scratch = nullptr;
            st = moea_batch_create(cfgs, count, nullptr, flags & ~MOEA_BATCH_AUTOTUNE, &scratch);
            TunedSchedule ts;
            if (st == MOEA_OK) {
                st = scratch->autotune(std::min(10, T / 4), &ts.schedule, &ts.tuned_ms, &ts.default_ms,
                                       &ts.slowest_ms, &ts.serial_ms, &ts.cost, &ts.tile_shape);
                delete scratch;
            }
            if (st == MOEA_OK) {
                tuning_cache()[key] = ts;
                b->inst_cost = ts.cost;
                b->tile_shape = ts.tile_shape;
                st = b->setup_fused(&ts.schedule);
                b->schedule_source = 1;
                b->tuned_ms = ts.tuned_ms;
                b->default_ms = ts.default_ms;
                b->slowest_ms = ts.slowest_ms;
                b->serial_ms = ts.serial_ms;
            }
        }
    } else if (st == MOEA_OK && b->use_fused) {
        st = b->setup_fused();
    }
    if (st != MOEA_OK) {
        delete b;
        return st;
    }
    *out = b;
    return MOEA_OK;
}

moea_status moea_batch_schedule(moea_batch* b, int* h_groups, int* h_source, float* h_tuned_ms,
                                float* h_default_ms, float* h_slowest_ms, float* h_serial_ms, int* h_group_of)
{
    if (!b) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL batch");
    if (h_slowest_ms) *h_slowest_ms = b->slowest_ms;
    if (h_serial_ms) *h_serial_ms = b->serial_ms;
    if (h_groups) *h_groups = (int)b->groups.size();
    if (h_source) *h_source = b->schedule_source;
    if (h_tuned_ms) *h_tuned_ms = b->tuned_ms;
    if (h_default_ms) *h_default_ms = b->default_ms;
    if (h_group_of)
        for (size_t i = 0; i < b->inst.size(); ++i) h_group_of[i] = i < b->group_of.size() ? b->group_of[i] : -1;
    return MOEA_OK;
}

moea_status moea_batch_tile_shapes(moea_batch* b, int* h_shapes, int cap)
{
    if (!b || (!h_shapes && cap > 0) || cap < 0) return set_error(MOEA_ERR_INVALID_ARGUMENT, "tile shapes: bad arguments");
    for (int m = 0; m < cap; ++m) {
        bool present = false;
        for (moea_algorithm* a : b->inst) present |= a->M == m;
        h_shapes[m] = (present && m <= kMaxObjectives && b->fused) ? b->tile_shape[m] : 0;
    }
    return MOEA_OK;
}

void moea_batch_destroy(moea_batch* b) { delete b; }

moea_status moea_batch_step(moea_batch* b)
{
    if (!b) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL batch");
    return b->step();
}

moea_status moea_batch_run(moea_batch* b, int generations, double* h_total_ms)
{
    if (!b) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL batch");
    MOEA_CUDA_TRY(cudaSetDevice(b->device));
    cudaEvent_t e0, e1;
    MOEA_CUDA_TRY(cudaEventCreate(&e0));
    MOEA_CUDA_TRY(cudaEventCreate(&e1));
    MOEA_CUDA_TRY(cudaEventRecord(e0, b->stream));
    int st = MOEA_OK;
    for (int g = 0; (generations < 0 || g < generations) && b->generation < b->T && st == MOEA_OK; ++g)
        st = b->step();
    cudaEventRecord(e1, b->stream);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != MOEA_OK) return st;
    if (h_total_ms) *h_total_ms = ms;
    for (moea_algorithm* a : b->inst) MOEA_TRY(workspace_check_status(a->ws, b->stream));
    return MOEA_OK;
}

moea_status moea_batch_synchronize(moea_batch* b)
{
    if (!b) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL batch");
    MOEA_CUDA_TRY(cudaStreamSynchronize(b->stream));
    for (moea_algorithm* a : b->inst) MOEA_TRY(workspace_check_status(a->ws, b->stream));
    return MOEA_OK;
}

moea_status moea_batch_info(moea_batch* b, int* h_count, int* h_generation, int* h_graph_kernels,
                            int* h_fused)
{
    if (!b) return set_error(MOEA_ERR_INVALID_ARGUMENT, "NULL batch");
    if (h_fused) *h_fused = b->fused ? 1 : 0;
    if (h_count) *h_count = (int)b->inst.size();
    if (h_generation) *h_generation = b->generation;
    if (h_graph_kernels) *h_graph_kernels = b->graph_kernels;
    return MOEA_OK;
}

moea_status moea_batch_view(moea_batch* b, int index, moea_population_view* out)
{
    if (!b || !out || index < 0 || index >= (int)b->inst.size())
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "batch_view: bad arguments");
    return moea_algorithm_view(b->inst[index], out);
}

}  // extern "C"
