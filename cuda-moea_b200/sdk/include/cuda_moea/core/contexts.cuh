// Plugin SDK of libmoea_b200: per-call contexts (the generation being made;
// -1 for the initial population), as in CUDA-MOEA's
// nat/include/cuda_moea/core/contexts.cuh.
#pragma once

#include "cuda_moea/core/cuda_context.cuh"

namespace cuda_moea {

struct GenerationContext {
    int generation = 0;
    int max_generations = 0;
    CudaContext& cuda;
};

struct EvaluationContext {
    int generation = 0;
    int max_generations = 0;
    CudaContext& cuda;
};

}  // namespace cuda_moea
