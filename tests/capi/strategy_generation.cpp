// Drives NSGA-III and RVEA generations through the strategy handles of
// include/moea_b200.h (directions, mating, crossover, mutation, selector:
// the reference's strategy interfaces) the way the reference's
// EvolutionaryAlgorithm::step does (algorithm.cu:221-286), and checks every
// generation bit for bit against the algorithm object run with the same
// configuration.  Built and run by tests/test_gpu_strategies.py.
//
//   strategy_generation <algorithm 0|1> <problem kind> <D> <M> <N> <generations>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

#include "moea_b200.h"

#define CHECK(x)                                                                          \
    do {                                                                                  \
        const int rc_ = (x);                                                              \
        if (rc_ != 0) {                                                                   \
            std::fprintf(stderr, "%s failed (%d): %s\n", #x, rc_, moea_last_error());   \
            std::exit(2);                                                                 \
        }                                                                                 \
    } while (0)
#define CUDA(x)                                                                           \
    do {                                                                                  \
        const cudaError_t e_ = (x);                                                       \
        if (e_ != cudaSuccess) {                                                          \
            std::fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));                \
            std::exit(2);                                                                 \
        }                                                                                 \
    } while (0)

struct Slot {
    float *x = nullptr, *f = nullptr, *cv = nullptr;
    moea_population_desc desc{};
};

static void make_slot(Slot& s, const float* bounds, int N, int D, int M)
{
    CUDA(cudaMalloc(&s.x, sizeof(float) * N * D));
    CUDA(cudaMalloc(&s.f, sizeof(float) * N * M));
    CUDA(cudaMalloc(&s.cv, sizeof(float) * N));
    s.desc = moea_population_desc{s.x, s.f, s.cv, bounds, N, D, M};
}

static bool same_bytes(const void* d_a, const void* d_b, size_t bytes, const char* what, int g)
{
    std::vector<unsigned char> a(bytes), b(bytes);
    CUDA(cudaMemcpy(a.data(), d_a, bytes, cudaMemcpyDeviceToHost));
    CUDA(cudaMemcpy(b.data(), d_b, bytes, cudaMemcpyDeviceToHost));
    if (std::memcmp(a.data(), b.data(), bytes) != 0) {
        std::printf("MISMATCH %s at generation %d\n", what, g);
        return false;
    }
    return true;
}

int main(int argc, char** argv)
{
    if (argc < 7) {
        std::fprintf(stderr, "usage: %s algorithm kind D M N generations\n", argv[0]);
        return 2;
    }
    const int algo = std::atoi(argv[1]), kind = std::atoi(argv[2]), D = std::atoi(argv[3]),
              M = std::atoi(argv[4]), N = std::atoi(argv[5]), G = std::atoi(argv[6]);
    const int T = 3 * G;  // horizon: annealing and the RVEA penalty see the same T on both sides
    const uint64_t seed = 2887;
    cudaStream_t stream;
    CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));

    // the algorithm object
    moea_algorithm_config cfg;
    moea_algorithm_config_defaults(&cfg, algo);
    cfg.population_size = N;
    cfg.max_generations = T;
    cfg.seed = seed;
    cfg.problem_kind = kind;
    cfg.dimension = D;
    cfg.objectives = M;
    cfg.stream = stream;
    cfg.sbx_copy_probability = 0.25f;
    cfg.sbx_eta_final = 10.0f;  // annealed index
    if (algo == MOEA_RVEA) {
        cfg.directions = MOEA_DIRS_ADAPTIVE;
        cfg.adapt_frequency = 0.5f;  // adapts every lround(0.5 T) generations
    }
    moea_algorithm* alg = nullptr;
    CHECK(moea_algorithm_create(&cfg, &alg));
    CHECK(moea_algorithm_initialize(alg));
    moea_population_view v{};
    CHECK(moea_algorithm_view(alg, &v));

    // the same generation from the strategy handles
    std::vector<float> hb(2 * D);
    for (int d = 0; d < D; ++d) { hb[2 * d] = 0.0f; hb[2 * d + 1] = 1.0f; }
    float* bounds = nullptr;
    CUDA(cudaMalloc(&bounds, sizeof(float) * 2 * D));
    CUDA(cudaMemcpy(bounds, hb.data(), sizeof(float) * 2 * D, cudaMemcpyHostToDevice));
    Slot P, O, X;
    make_slot(P, bounds, N, D, M);
    make_slot(O, bounds, N, D, M);
    make_slot(X, bounds, N, D, M);
    CUDA(cudaMemcpyAsync(P.x, v.d_variables, sizeof(float) * N * D, cudaMemcpyDeviceToDevice, stream));
    CUDA(cudaMemcpyAsync(P.f, v.d_objectives, sizeof(float) * N * M, cudaMemcpyDeviceToDevice, stream));
    CUDA(cudaMemcpyAsync(P.cv, v.d_constraints, sizeof(float) * N, cudaMemcpyDeviceToDevice, stream));

    moea_directions* dirs = nullptr;
    moea_mating* mate = nullptr;
    moea_crossover* cx = nullptr;
    moea_mutation* mu = nullptr;
    moea_selector* sel = nullptr;
    if (algo == MOEA_NSGA3) {
        CHECK(moea_create_dasdennis(0, &dirs));
        CHECK(moea_create_tournament(&mate));
        CHECK(moea_create_nsga3_selector(nullptr, &sel));
    } else {
        CHECK(moea_create_adaptive_directions(0.5f, &dirs));
        CHECK(moea_create_random_mating(&mate));
        CHECK(moea_create_rvea_selector(2.0f, &sel));
    }
    CHECK(moea_create_sbx(cfg.sbx_eta_initial, cfg.sbx_eta_final, 1.0f, 0.25f, &cx));
    CHECK(moea_create_pm(20.0f, 20.0f, 1.0f, &mu));
    CHECK(moea_directions_initialize(dirs, N, M, 0, stream));
    CHECK(moea_selector_initialize(sel, N, D, M, T, dirs, 0, stream));
    moea_generation_desc ctx{0, T, seed};
    CHECK(moea_selector_prepare(sel, &P.desc, &ctx, stream));
    int* pidx = nullptr;
    CUDA(cudaMalloc(&pidx, sizeof(int) * N));

    bool ok = true;
    for (int g = 0; g < G && ok; ++g) {
        ctx.generation = g;
        const int *rank = nullptr, *active = nullptr;
        CHECK(moea_selector_mating_state(sel, &rank, &active));
        CHECK(moea_mating_select(mate, &P.desc, rank, active, pidx, N, &ctx, stream));
        CHECK(moea_crossover_apply(cx, &P.desc, pidx, &O.desc, &ctx, stream));
        CHECK(moea_mutation_apply(mu, &O.desc, &ctx, stream));
        CHECK(moea_problem_evaluate(kind, O.x, N, D, M, O.f, O.cv, stream));
        CHECK(moea_selector_select(sel, &P.desc, &O.desc, &X.desc, &ctx, stream));
        CHECK(moea_directions_update(dirs, &X.desc, active, &ctx, stream));
        std::swap(P, X);

        CHECK(moea_algorithm_step(alg));
        CHECK(moea_algorithm_view(alg, &v));
        CUDA(cudaStreamSynchronize(stream));
        ok = same_bytes(P.x, v.d_variables, sizeof(float) * N * D, "variables", g) &&
             same_bytes(P.f, v.d_objectives, sizeof(float) * N * M, "objectives", g) &&
             same_bytes(P.cv, v.d_constraints, sizeof(float) * N, "violations", g);
        const float* d_alg_dirs = nullptr;
        const float* d_dirs = nullptr;
        int count = 0, dm = 0;
        CHECK(moea_algorithm_directions(alg, &d_alg_dirs, &count));
        CHECK(moea_directions_view(dirs, &d_dirs, nullptr, nullptr, &dm, nullptr));
        ok = ok && same_bytes(d_dirs, d_alg_dirs, sizeof(float) * (size_t)M * count, "directions", g);
        if (algo == MOEA_NSGA3) {
            const int* d_idx = nullptr;
            int n_idx = 0;
            CHECK(moea_selector_result_indices(sel, &d_idx, &n_idx));
            ok = ok && n_idx == N && same_bytes(d_idx, v.d_auxiliary, sizeof(int) * N, "ranks", g);
        } else {
            int h_active = 0;
            CHECK(moea_selector_active_count(sel, &h_active, stream));
            if (h_active != v.active_count) {
                std::printf("MISMATCH active count at generation %d: %d vs %d\n", g, h_active, v.active_count);
                ok = false;
            }
        }
    }
    if (ok && algo == MOEA_RVEA) {  // front-0 indices of the final parents
        CHECK(moea_selector_finalize(sel, &P.desc, stream));
        CHECK(moea_algorithm_finalize(alg));
        CHECK(moea_algorithm_view(alg, &v));
        const int* d_idx = nullptr;
        int n_idx = 0;
        CHECK(moea_selector_result_indices(sel, &d_idx, &n_idx));
        ok = n_idx == v.auxiliary_count && n_idx > 0 &&
             same_bytes(d_idx, v.d_auxiliary, sizeof(int) * n_idx, "front-0 indices", G);
    }
    moea_selector_destroy(sel);
    moea_mutation_destroy(mu);
    moea_crossover_destroy(cx);
    moea_mating_destroy(mate);
    moea_directions_destroy(dirs);
    moea_algorithm_destroy(alg);
    std::printf(ok ? "OK %d generations\n" : "FAILED\n", G);
    return ok ? 0 : 1;
}
