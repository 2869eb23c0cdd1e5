// TEST INFRASTRUCTURE ONLY -- the reference's SBX kernel, compiled in place
// from its source (src/reproduction/sbx_crossover.cu, included below through
// the Makefile's include path) so that this translation unit can launch its
// file-local kernel with draws the test supplies.  The reference fills those
// draws with cuRAND launchers whose element-to-thread mapping depends on the
// GPU model; the kernel itself (sbx_crossover.cu:20-70) is what is pinned.
#include "reproduction/sbx_crossover.cu"

extern "C" int ref_sbx(const float* d_parents, const int* d_pidx, const float* d_bounds, const float* d_u,
                       const int* d_sign, const float* d_copy, float* d_off, float eta, float prob,
                       float copy_prob, int n_off, int D)
{
    const int pairs = n_off / 2;
    const int count = pairs * D;
    if (count > 0)
        cuda_moea::sbx_kernel<<<(count + 255) / 256, 256>>>(d_parents, d_pidx, d_bounds,
                                                            reinterpret_cast<const float2*>(d_u), d_sign,
                                                            d_copy, d_off, eta, prob, copy_prob, pairs, D);
    if (n_off % 2 != 0)
        cuda_moea::copy_last_parent_kernel<<<(D + 255) / 256, 256>>>(d_parents, d_pidx, d_off, n_off - 1, D);
    return cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// The reference's host-side annealing of the distribution index
// (sbx_crossover.cu:12-18).
extern "C" float ref_annealed(float begin, float end, int generation, int total)
{
    return cuda_moea::annealed(begin, end, generation, total);
}
