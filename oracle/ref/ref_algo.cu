// TEST AND BASELINE INFRASTRUCTURE ONLY -- C entry point over CUDA-MOEA's own
// complete algorithm (python/csrc/native/src/**, every source of its native
// library compiled in place by oracle/ref/Makefile into
// oracle/_ref/libmoea_ref_algo.so).  The reference arm of bench.py calls it to
// time the reference's own NSGA-III / RVEA generation on the same GPU, as a
// second baseline beside the CPU restatement.
//
// The algorithm is built through the reference's C++ builders
// (src/builder/nsga3_builder.cu, rvea_builder.cu) and stepped through
// EvolutionaryAlgorithm::step (src/algorithm/algorithm.cu:104-286).  Each
// timed step is bracketed by a device synchronise on both sides: the
// reference's step itself waits on the host for its front peeling and its
// selection sizes, so host time around a synchronised step is its generation
// time.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "cuda_moea/algorithms/nsga3.cuh"
#include "cuda_moea/algorithms/rvea.cuh"
#include "cuda_moea/factory/algorithm_factory.cuh"
#include "cuda_moea/factory/operator_factory.cuh"
#include "cuda_moea/factory/problem_factory.cuh"

using namespace cuda_moea;

extern "C" int ref_algo_time(int algorithm, int problem_kind, int D, int M, int N, int partitions, int max_gen,
                             float sparse_ratio, unsigned long long seed, int warmup, int steps, double* h_step_ms,
                             char* err, size_t err_cap)
{
    try {
        const ProblemKind kind = static_cast<ProblemKind>(problem_kind - 1);
        SBXConfig sbx{30.0f, 30.0f, 1.0f, 0.0f};
        PolynomialMutationConfig pm{20.0f, 20.0f, 1.0f};
        auto configure = [&](auto& b) {
            b.populationSize(N).maxGenerations(max_gen).problem(kind, D, M).randomSeed(seed).printProgress(false)
                .cudaWarmup(false).crossover(CrossoverKind::SBX, sbx).mutation(MutationKind::Polynomial, pm);
        };
        auto run = [&](Algorithm& a) {
            a.initialize();
            for (int i = 0; i < warmup; ++i) a.step();
            for (int i = 0; i < steps; ++i) {
                cudaDeviceSynchronize();
                const auto t0 = std::chrono::steady_clock::now();
                a.step();
                cudaDeviceSynchronize();
                const auto t1 = std::chrono::steady_clock::now();
                h_step_ms[i] = std::chrono::duration<double, std::milli>(t1 - t0).count();
            }
        };
        if (algorithm == 0) {
            NSGA3::Builder b;
            configure(b);
            b.mating(MatingKind::Tournament).sparseRatio(sparse_ratio);
            if (partitions > 0) b.referencePointPartition(partitions);
            Algorithm a = b.build();
            run(a);
        } else {
            RVEA::Builder b;
            configure(b);
            Algorithm a = b.build();
            run(a);
        }
        const cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            std::snprintf(err, err_cap, "CUDA: %s", cudaGetErrorString(e));
            return 2;
        }
        return 0;
    } catch (const std::exception& ex) {
        std::snprintf(err, err_cap, "%s", ex.what());
        return 1;
    }
}

// A whole run of the reference's algorithm the way its published quality
// benchmark configures it (tests/benchmark/adapters/dtlz.py _run_cuda): a given
// initial population (N, D) row-major, SBX {eta, eta, 1, copy_prob}, PM
// {20, 20, 1}, NSGA-III with sparse ratio 1 and the given user directions
// (M, H) objective-major (normalised by the provider), RVEA with alpha 2 and
// adaptive directions of the given frequency.  After max_gen generations the
// final objectives (M, N) objective-major, the active count and the run's own
// device time (RunResult.total_ms) are returned.
extern "C" int ref_algo_run(int algorithm, int problem_kind, int D, int M, int N, int max_gen,
                            unsigned long long seed, float sbx_eta, float copy_prob, const float* h_init,
                            const float* h_dirs, int H, float frequency, float* h_objs, int* h_active,
                            double* h_total_ms, char* err, size_t err_cap)
{
    try {
        auto st = AlgorithmFactory::defaults(algorithm == 0 ? AlgorithmKind::NSGA3 : AlgorithmKind::RVEA);
        st.config.population_size = N;
        st.config.max_generations = max_gen;
        st.config.print_progress = false;
        st.config.cuda.seed = seed;
        st.config.cuda.enable_warmup = false;
        if (h_init) st.config.initial_population.assign(h_init, h_init + (size_t)N * D);
        st.strategies.problem = ProblemFactory::create(static_cast<ProblemKind>(problem_kind - 1), D, M, 0.0f);
        st.strategies.crossover = OperatorFactory::crossover(CrossoverKind::SBX, SBXConfig{sbx_eta, sbx_eta, 1.0f, copy_prob});
        st.strategies.mutation = OperatorFactory::mutation(MutationKind::Polynomial, PolynomialMutationConfig{20.0f, 20.0f, 1.0f});
        if (algorithm == 0) {
            st.strategies.environment_selector = std::make_unique<NSGA3EnvironmentSelector>(NSGA3SelectionConfig{1.0f, {}});
            if (h_dirs)
                st.strategies.reference_directions = std::make_unique<UserDefinedDirections>(
                    std::vector<float>(h_dirs, h_dirs + (size_t)M * H), M, true);
        } else {
            st.strategies.environment_selector = std::make_unique<RVEAEnvironmentSelector>(RVEASelectionConfig{2.0f});
            st.strategies.reference_directions = std::make_unique<AdaptiveRVEADirections>(AdaptiveDirectionConfig{frequency});
        }
        Algorithm a = AlgorithmFactory::create(std::move(st));
        RunResult r = a.run();
        std::memcpy(h_objs, r.objectives.data(), sizeof(float) * (size_t)M * N);
        *h_active = r.active_count;
        *h_total_ms = r.total_ms;
        return 0;
    } catch (const std::exception& ex) {
        std::snprintf(err, err_cap, "%s", ex.what());
        return 1;
    }
}
