// Snapshot writer and resume reader (snapshot.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace moea {

// Fixed description of a run, written to metadata.json.
struct SnapshotMeta {
    std::string algorithm_name, problem_name;
    int N = 0, D = 0, M = 0, H = 0, T = 0, constraint_count = 0;
    uint64_t seed = 0;
};

// One snapshot request: device buffers of the parents (valid until the
// compute stream's next work) and the host-side state.
struct SnapshotSave {
    int generation = 0;
    const float* vars = nullptr;
    const float* objs = nullptr;
    const float* cv = nullptr;
    const float* refs = nullptr;
    const int* aux = nullptr;
    int aux_count = 0;
    const int* d_active = nullptr;   // device active count, or NULL: `active`
    int active = 0;
    const float* ideal = nullptr;
    const unsigned long long* offset = nullptr;
    uint32_t epoch = 0;
    int last_prepared_target = 0;
    int ideal_ready = 0;
};

// Contents of a generation directory, read back for a resume.
struct SnapshotLoad {
    int generation = 0, active = 0, last_prepared_target = 0, ideal_ready = 0;
    uint32_t epoch = 0;
    unsigned long long niching_offset = 0;
    std::vector<float> vars, objs, cv, refs, ideal;
    std::vector<int> aux;
};

class SnapshotWriter {
public:
    SnapshotWriter();
    ~SnapshotWriter();
    SnapshotWriter(const SnapshotWriter&) = delete;
    SnapshotWriter& operator=(const SnapshotWriter&) = delete;

    // Writes the run's root files and allocates the two pinned slots.
    int open(const std::string& directory, int interval, const SnapshotMeta& meta, const std::vector<float>& lower,
             const std::vector<float>& upper, const float* d_initial_refs, cudaStream_t stream);
    bool should_save(int generation) const;
    // Queues the snapshot of `in.generation` when it is due.
    int save(const SnapshotSave& in, cudaStream_t compute);
    // Waits for every queued snapshot; the first write error since the last flush.
    int flush();

private:
    struct Slot;
    static void CUDART_CB write_slot(void* user);

    std::string root_;
    int interval_ = 1;
    SnapshotMeta meta_;
    cudaStream_t side_ = nullptr;
    cudaEvent_t ready_ = nullptr, copied_ = nullptr;
    Slot* slots_[2] = {nullptr, nullptr};
    int next_ = 0;
    std::mutex mutex_;
    std::string error_;
};

int load_snapshot_files(const std::string& directory, const SnapshotMeta& meta, bool need_aux, SnapshotLoad& out);

}  // namespace moea
