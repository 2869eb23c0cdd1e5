// Test plugin: two weighted spheres, f0 = w0 sum x^2, f1 = w1 sum (x - shift)^2,
// with an optional radius constraint sum x^2 <= radius^2 that switches on at
// generation `switch_at` (-1: from the start).  Its prepare_parent turns the
// constraint on for the parents at the switch and asks for a re-sort.
#pragma once
#include <string>
#include <vector>

#include "cuda_moea/native/plugin.cuh"

class WeightedSpheres final : public cuda_moea::IProblemEvaluator {
public:
    explicit WeightedSpheres(const cuda_moea::native::ProblemConfig& config);
    const cuda_moea::ProblemInfo& info() const noexcept override { return info_; }
    void evaluate(cuda_moea::PopulationView population, const cuda_moea::EvaluationContext& context,
                  cudaStream_t stream) override;
    bool prepare_parent(cuda_moea::PopulationView population, const cuda_moea::EvaluationContext& context,
                        cudaStream_t stream) override;
    void reset() override { resets_ += 1; }

private:
    bool active(int generation) const { return constrained_ && (switch_at_ < 0 || generation >= switch_at_); }
    void launch(cuda_moea::PopulationView p, bool with_cv, bool objectives, cudaStream_t stream) const;

    cuda_moea::ProblemInfo info_;
    float shift_, radius_, w0_, w1_;
    bool constrained_;
    long long switch_at_;
    int resets_ = 0;
};
