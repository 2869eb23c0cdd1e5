// TEST INFRASTRUCTURE ONLY -- C entry point over CUDA-MOEA's host-side
// reference-direction generators, compiled from the reference sources where
// they lie (oracle/ref/Makefile builds oracle/_ref/libmoea_ref_host.so with the
// plain host compiler, so the CPU tests can pin the oracle's and the product's
// Das-Dennis directions without a GPU).
//
//   initialize_refpts                 src/reference/nsga3_reference_generator.cu:153-182
//   initialize_refpts_by_partitions   src/reference/nsga3_reference_generator.cu:184-221
//   rvea::initialize_refpts           src/reference/rvea_reference_generator.cu:182-217
#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <tuple>
#include <vector>

#include "cuda_moea/reference/nsga3_reference_generator.cuh"
#include "cuda_moea/reference/rvea_reference_generator.cuh"

extern "C" {

// mode 0: NSGA-III auto layers for n points; 1: NSGA-III one layer of n
// partitions; 2: RVEA auto layers (clamped).  Writes the normalised
// directions (M, count) objective-major to out when capacity suffices and
// returns count (negative on a rejected request).
int ref_directions(int mode, int n, int M, float* out, size_t capacity)
{
    try {
        std::tuple<std::vector<float>, std::vector<float>, int> r;
        if (mode == 0) r = initialize_refpts(n, M);
        else if (mode == 1) r = initialize_refpts_by_partitions(n, M);
        else if (mode == 2) r = rvea::initialize_refpts(n, M);
        else return -1;
        const std::vector<float>& normalized = std::get<1>(r);
        const int count = std::get<2>(r);
        if (out && normalized.size() <= capacity)
            std::memcpy(out, normalized.data(), sizeof(float) * normalized.size());
        return count;
    } catch (const std::exception&) {
        return -2;
    }
}

}  // extern "C"
