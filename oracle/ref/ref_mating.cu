// TEST INFRASTRUCTURE ONLY -- the reference's tournament-winner kernel,
// compiled in place from its source (src/reproduction/mating_selection.cu,
// included through the Makefile's include path) and launched on candidate
// pairs the test supplies (mating_selection.cu:11-35).
#include "reproduction/mating_selection.cu"

extern "C" int ref_tournament(const int* d_cand, const int* d_rank, const float* d_cv, int n, int* d_winners)
{
    if (n > 0)
        cuda_moea::tournament_winner_kernel<<<(n + 255) / 256, 256>>>(reinterpret_cast<const int2*>(d_cand),
                                                                       d_rank, d_cv, d_winners, n);
    return cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 1;
}
