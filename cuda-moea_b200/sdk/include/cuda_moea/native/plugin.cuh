// Plugin SDK of libmoea_b200: registration of a problem library.
//
// A problem library defines a class derived from IProblemEvaluator whose
// constructor takes a ProblemConfig, lists its parameters with defaults, and
// registers both in exactly one translation unit:
//
//     const std::vector<cuda_moea::native::ParameterSpec> params{
//         {"scale", 1.0, "multiplier of the first objective"}};
//     CUDA_MOEA_REGISTER_PROBLEM(MyProblem, "MyProblem", params)
//
// The registration (entry point cuda_moea_problem_v1, version 1) is the one
// of CUDA-MOEA's nat/include/cuda_moea/native/plugin.cuh:35-58, so problem
// sources written for it build against this SDK unchanged.  The type of a
// parameter is the type of its default: int64, double, bool, string or a
// list of doubles.
#pragma once

#include <cstdint>
#include <string>
#include <unordered_map>
#include <variant>
#include <vector>

#include "cuda_moea/native/build_id.h"
#include "cuda_moea/problem/problem_evaluator.cuh"

namespace cuda_moea::native {

using Parameter = std::variant<std::int64_t, double, bool, std::string, std::vector<double>>;

struct ParameterSpec {
    const char* name;
    Parameter default_value;
    const char* description;
};

// What the problem is constructed with: the requested sizes and bounds and
// a value for every registered parameter.
struct ProblemConfig {
    int dimension;
    int objectives;
    std::vector<float> lower_bounds;
    std::vector<float> upper_bounds;
    std::unordered_map<std::string, Parameter> parameters;

    template <class T>
    const T& get(const std::string& name) const
    {
        return std::get<T>(parameters.at(name));
    }
};

// The library checks abi and build_id before it touches anything else.
struct Plugin {
    std::uint32_t abi;
    const char* build_id;
    const char* name;
    const std::vector<ParameterSpec>* parameters;
    IProblemEvaluator* (*create)(const ProblemConfig&);
    void (*destroy)(IProblemEvaluator*) noexcept;
};
using Entry = const Plugin* (*)();

}  // namespace cuda_moea::native

#define CUDA_MOEA_REGISTER_PROBLEM(Type, Name, Schema)                                                  \
    extern "C" __attribute__((visibility("default"))) const ::cuda_moea::native::Plugin*              \
    cuda_moea_problem_v1()                                                                            \
    {                                                                                                 \
        static const ::cuda_moea::native::Plugin plugin{                                              \
            1, CUDA_MOEA_NATIVE_BUILD_ID, Name, &(Schema),                                            \
            [](const ::cuda_moea::native::ProblemConfig& config) -> ::cuda_moea::IProblemEvaluator* { \
                return new Type(config);                                                              \
            },                                                                                        \
            [](::cuda_moea::IProblemEvaluator* value) noexcept { delete value; }};                    \
        return &plugin;                                                                               \
    }
