#include "problem.cuh"

namespace {
const std::vector<cuda_moea::native::ParameterSpec> parameters{
    {"shift", 0.5, "center of the second sphere"},
    {"radius", 1.0, "feasible radius around the origin"},
    {"weights", std::vector<double>{1.0, 1.0}, "weights of the two objectives"},
    {"constrained", false, "enable sum(x*x) <= radius*radius"},
    {"switch_at", std::int64_t{-1}, "generation at which the constraint starts (-1: always)"},
    {"label", std::string("WeightedSpheres"), "name the problem reports"},
    {"bad_info", false, "report a wrong dimension (tests the host's check)"},
    {"throw_at_create", false, "throw from the constructor (tests the host's check)"},
};
}  // namespace

CUDA_MOEA_REGISTER_PROBLEM(WeightedSpheres, "WeightedSpheres", parameters)
