// Plugin SDK of libmoea_b200: the problem interface a plugin implements
// (CUDA-MOEA's IProblemEvaluator,
// nat/include/cuda_moea/problem/problem_evaluator.cuh:10-31).
//
//   evaluate        writes objectives (M, N) and violations (N) of the
//                   population on the stream;
//   prepare_parent  runs before each generation on the current parents;
//                   returning true makes the algorithm re-sort them (a
//                   problem whose constraints switch on mid-run);
//   initialize      once, before the first evaluation;
//   reset           when the algorithm restarts.
#pragma once

#include "cuda_moea/core/contexts.cuh"
#include "cuda_moea/core/types.cuh"

namespace cuda_moea {

class IProblemEvaluator {
public:
    virtual ~IProblemEvaluator() = default;

    virtual const ProblemInfo& info() const noexcept = 0;
    virtual void initialize(CudaContext&) {}
    virtual void evaluate(PopulationView population, const EvaluationContext& context, cudaStream_t stream) = 0;
    virtual bool prepare_parent(PopulationView, const EvaluationContext&, cudaStream_t) { return false; }
    virtual void reset() {}
};

}  // namespace cuda_moea
