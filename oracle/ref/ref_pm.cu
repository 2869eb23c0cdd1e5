// TEST INFRASTRUCTURE ONLY -- the reference's polynomial-mutation kernel,
// compiled in place from its source (src/reproduction/polynomial_mutation.cu,
// included through the Makefile's include path) and launched on draws the
// test supplies (polynomial_mutation.cu:20-60).
#include "reproduction/polynomial_mutation.cu"

extern "C" int ref_pm(float* d_off, const float* d_bounds, const float* d_u, float eta, float prob, int n,
                      int D)
{
    const int count = n * D;
    if (count > 0)
        cuda_moea::polynomial_mutation_kernel<<<(count + 255) / 256, 256>>>(
            reinterpret_cast<const float2*>(d_u), d_off, d_bounds, eta, prob, count, D);
    return cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 1;
}
