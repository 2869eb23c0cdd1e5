// Plugin SDK of libmoea_b200: the CUDA context handed to a problem plugin.
// The member functions are those of CUDA-MOEA's CudaContext
// (nat/include/cuda_moea/core/cuda_context.cuh).  Here one stream carries
// both evaluation and execution work (the algorithm's stream), so the two
// wait functions are no-ops, and the pools are the device's default pool.
#pragma once

#include <cuda_runtime.h>

namespace cuda_moea {

struct CudaConfig {
    int device_id = 0;
    float evaluation_pool_ratio = 0.25f;
    float execution_pool_ratio = 0.75f;
    int memory_pool_policy = 1;
    unsigned long long seed = 2887ULL;
    bool enable_warmup = true;
};

class CudaContext {
public:
    explicit CudaContext(const CudaConfig& config = {}) : config_(config) {}
    CudaContext(const CudaContext&) = delete;
    CudaContext& operator=(const CudaContext&) = delete;

    cudaStream_t evaluation_stream() const noexcept { return stream_; }
    cudaStream_t execution_stream() const noexcept { return stream_; }
    cudaMemPool_t evaluation_pool() const noexcept { return default_pool(); }
    cudaMemPool_t execution_pool() const noexcept { return default_pool(); }

    unsigned long long random_seed() const noexcept { return config_.seed; }
    unsigned long long& random_offset() noexcept { return offset_; }

    void wait_evaluation_on_execution() {}
    void wait_execution_on_evaluation() {}
    void synchronize() { cudaStreamSynchronize(stream_); }

    // Set by the library before it calls into the plugin.
    void bind(cudaStream_t stream, int device, unsigned long long seed) noexcept
    {
        stream_ = stream;
        config_.device_id = device;
        config_.seed = seed;
    }

private:
    cudaMemPool_t default_pool() const noexcept
    {
        cudaMemPool_t pool = nullptr;
        cudaDeviceGetDefaultMemPool(&pool, config_.device_id);
        return pool;
    }

    CudaConfig config_;
    cudaStream_t stream_ = nullptr;
    unsigned long long offset_ = 0;
};

}  // namespace cuda_moea
