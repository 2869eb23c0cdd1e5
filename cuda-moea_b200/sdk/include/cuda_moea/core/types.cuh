// Plugin SDK of libmoea_b200: the view types a problem plugin receives.
// Names and field order are those of CUDA-MOEA's core types
// (nat/include/cuda_moea/core/types.cuh), so plugin sources written for it
// compile unchanged against this SDK.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace cuda_moea {

// Non-owning device array.
template <typename T>
struct DeviceSpan {
    T* data = nullptr;
    std::size_t size = 0;

    bool empty() const noexcept { return data == nullptr || size == 0; }
    explicit operator bool() const noexcept { return !empty(); }
};

// Read-only population: variables (N, D) row-major, objectives (M, N)
// objective-major, violations (N), bounds interleaved [lb0, ub0, lb1, ...].
struct ConstPopulationView {
    const float* variables = nullptr;
    const float* objectives = nullptr;
    const float* constraints = nullptr;
    const float* bounds = nullptr;
    int size = 0;
    int dimension = 0;
    int objective_count = 0;
};

// Population the problem writes objectives and violations into.
struct PopulationView {
    float* variables = nullptr;
    float* objectives = nullptr;
    float* constraints = nullptr;
    const float* bounds = nullptr;
    int size = 0;
    int dimension = 0;
    int objective_count = 0;

    operator ConstPopulationView() const noexcept
    {
        return {variables, objectives, constraints, bounds, size, dimension, objective_count};
    }
};

// What a problem reports about itself; the host checks it against the
// requested dimension, objective count and bounds.
struct ProblemInfo {
    std::string name;
    int dimension = 0;
    int objective_count = 0;
    int constraint_count = 0;
    std::vector<float> lower_bounds;
    std::vector<float> upper_bounds;
};

}  // namespace cuda_moea
