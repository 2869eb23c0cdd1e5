// Shared device/host helpers for the B200 generation path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "moea_b200.h"

namespace moea {

// Records a formatted message in the thread-local error slot and returns code.
int set_error(int code, const char* fmt, ...);
const char* last_error();

// Stage boundary for the per-stage profile of one generation: records a CUDA
// event on `stream` when a profile is being taken on this thread, else no-op.
void stage_mark(const char* name, cudaStream_t stream);

#define MOEA_CUDA_TRY(expr)                                                     \
    do {                                                                        \
        cudaError_t err__ = (expr);                                             \
        if (err__ != cudaSuccess)                                               \
            return ::moea::set_error(MOEA_ERR_CUDA, "%s failed: %s (%s:%d)",    \
                                     #expr, cudaGetErrorString(err__),          \
                                     __FILE__, __LINE__);                       \
    } while (0)

#define MOEA_TRY(expr)                                                          \
    do {                                                                        \
        int st__ = (expr);                                                      \
        if (st__ != MOEA_OK) return st__;                                       \
    } while (0)

constexpr int kMaxObjectives = 16;  // objectives per point handled by the kernels
constexpr int kWarp = 32;

__host__ __device__ inline uint32_t float_bits(float f)
{
    union { float f; uint32_t u; } v;
    v.f = f;
    return v.u;
}

// Order-preserving map float -> uint32 (ascending), with -0.0 folded onto +0.0
// so that the integer order agrees with IEEE comparison on non-NaN values.
__host__ __device__ inline uint32_t float_order_key(float f)
{
    uint32_t u = float_bits(f);
    if (u == 0x80000000u) u = 0u;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// ---------------------------------------------------------------------------
// Random numbers
// ---------------------------------------------------------------------------

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
__host__ __device__ inline void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                              uint32_t c3, uint32_t k0, uint32_t k1,
                                              uint32_t out[4])
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1;
        c3 = (uint32_t)p0;
        c0 = n0;
        c2 = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Draw streams of the product RNG: one Philox block per (element, generation, tag).
enum RngTag : uint32_t {
    kTagInit = 1,
    kTagMating = 2,
    kTagCrossover = 3,
    kTagMutation = 4,
    kTagCrossTest = 5,   // SBX crossover test draws (only when the crossover probability is below 1)
    kTagCopy = 6,        // SBX variable copy draws (only when the copy probability is above 0)
};

__host__ __device__ inline void rng_block(uint64_t seed, uint64_t element, uint32_t generation,
                                          uint32_t tag, uint32_t out[4])
{
    philox4x32_10((uint32_t)element, (uint32_t)(element >> 32), generation, tag,
                  (uint32_t)seed, (uint32_t)(seed >> 32), out);
}

// Uniform float in [0, 1) from the top 24 bits of a 32-bit draw.
__host__ __device__ inline float u32_to_unit(uint32_t x)
{
    return (float)(x >> 8) * (1.0f / 16777216.0f);
}

// SplitMix64 counter hash used by the niching tie-break draws
// (CUDA-MOEA nat/src/core/cuda/cuda_random.cu:1606-1613).
__host__ __device__ inline uint32_t splitmix_u32(uint64_t counter, uint64_t seed)
{
    uint64_t z = counter ^ seed;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (uint32_t)z;
}

// Seed derivation of RNDManager (nat/src/core/cuda/cuda_manager.cu:27-40, island 0).
inline uint64_t derive_seed(uint64_t seed)
{
    uint64_t x = seed;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Device status word written by kernels that wait on one another.
enum DeviceStatus : int {
    kDevOk = 0,
    kDevBarrierTimeout = 1,
    kDevPeelInconsistent = 2,
    kDevTensorTimeout = 3,      // a wait of the tensor-core association ran out
    kDevNichingSize = 4,        // a last front larger than the niching cluster holds
};

}  // namespace moea
