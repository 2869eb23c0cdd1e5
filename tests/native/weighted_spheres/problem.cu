#include "problem.cuh"

#include <stdexcept>

namespace {

// One thread per individual; objectives (M, N) objective-major.
__global__ void weighted_spheres(const float* x, float* f, float* cv, int n, int d, float shift, float w0, float w1,
                                 float radius, int with_cv, int objectives)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a = 0.0f, b = 0.0f;
    for (int j = 0; j < d; ++j) {
        const float v = x[(size_t)i * d + j];
        a += v * v;
        const float t = v - shift;
        b += t * t;
    }
    if (objectives) {
        f[i] = w0 * a;
        f[n + i] = w1 * b;
    }
    cv[i] = with_cv ? fmaxf(a - radius * radius, 0.0f) : 0.0f;
}

}  // namespace

WeightedSpheres::WeightedSpheres(const cuda_moea::native::ProblemConfig& config)
    : shift_(static_cast<float>(config.get<double>("shift"))),
      radius_(static_cast<float>(config.get<double>("radius"))),
      constrained_(config.get<bool>("constrained")),
      switch_at_(config.get<std::int64_t>("switch_at"))
{
    if (config.get<bool>("throw_at_create")) throw std::invalid_argument("asked to fail");
    if (config.objectives != 2) throw std::invalid_argument("WeightedSpheres needs objectives=2");
    const auto& w = config.get<std::vector<double>>("weights");
    if (w.size() != 2) throw std::invalid_argument("weights needs two values");
    w0_ = static_cast<float>(w[0]);
    w1_ = static_cast<float>(w[1]);
    info_.name = config.get<std::string>("label");
    info_.dimension = config.get<bool>("bad_info") ? config.dimension + 1 : config.dimension;
    info_.objective_count = 2;
    info_.constraint_count = constrained_ ? 1 : 0;
    info_.lower_bounds = config.lower_bounds;
    info_.upper_bounds = config.upper_bounds;
}

void WeightedSpheres::launch(cuda_moea::PopulationView p, bool with_cv, bool objectives, cudaStream_t stream) const
{
    if (p.size == 0) return;
    weighted_spheres<<<(p.size + 127) / 128, 128, 0, stream>>>(p.variables, p.objectives, p.constraints, p.size,
                                                               p.dimension, shift_, w0_, w1_, radius_,
                                                               with_cv ? 1 : 0, objectives ? 1 : 0);
}

void WeightedSpheres::evaluate(cuda_moea::PopulationView p, const cuda_moea::EvaluationContext& context,
                               cudaStream_t stream)
{
    launch(p, active(context.generation), true, stream);
}

bool WeightedSpheres::prepare_parent(cuda_moea::PopulationView p, const cuda_moea::EvaluationContext& context,
                                     cudaStream_t stream)
{
    if (!constrained_ || switch_at_ < 0 || context.generation != switch_at_) return false;
    launch(p, true, false, stream);
    return true;
}
