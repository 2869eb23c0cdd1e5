// Internal declarations shared by the translation units of libmoea_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>
#include <vector>

#include "common.cuh"

namespace moea {

// Events recorded at stage boundaries while a generation is being profiled.
struct StageProfile {
    std::vector<cudaEvent_t> events;
    std::vector<const char*> names;
};
StageProfile*& stage_profile();

// A population split across two buffers ("parents" a and "offspring" b) and
// addressed as one merged index space [0, n_a + n_b).  The reference copies
// both halves into merged buffers every generation
// (nat/src/selection/nsga3/kernels/nsga3_population_update.cu:7-115); here the
// kernels read through this view instead, so no merge copy exists.
struct SplitPop {
    const float* objs_a;
    const float* objs_b;
    const float* cv_a;
    const float* cv_b;
    int stride_a;  // row stride (points) of objs_a
    int stride_b;
    int n_a;
    int n;         // total points

    __device__ __forceinline__ float obj(int m, int i) const
    {
        return i < n_a ? objs_a[(size_t)m * stride_a + i]
                       : objs_b[(size_t)m * stride_b + (i - n_a)];
    }
    __device__ __forceinline__ float cvv(int i) const
    {
        return i < n_a ? cv_a[i] : cv_b[i - n_a];
    }
};

inline SplitPop merged_view(const float* objs, const float* cv, int n)
{
    return SplitPop{objs, objs, cv, cv, n, n, n, n};
}

// Device scratch for the generation path, sized once for (n_max, m_max, h_max).
struct Workspace {
    int device = 0;
    int n_max = 0;   // merged population capacity (2N)
    int m_max = 0;
    int h_max = 0;
    int words = 0;   // 32-bit words per dominance row = ceil(n_max / 32)
    size_t bytes = 0;

    // --- non-dominated sort ---
    uint32_t* rows = nullptr;       // [n_max][words] dominator bits per sorted point
    uint32_t* key32[2] = {};        // LSD pass keys
    uint64_t* key64[2] = {};        // final pass keys / niching keys (ping-pong)
    uint64_t* key0 = nullptr;       // per point: class << 32 | order key of f0 or cv
    int* perm[2] = {};              // sorted position -> point index
    float* sorted_f = nullptr;      // [(m_max-1)][n_max] objectives 1..M-1 in sorted order
    int* qinfo = nullptr;           // per sorted position: dup position | infeasible bit
    int* head = nullptr;            // run heads
    int* run_start = nullptr;       // scanned run heads
    uint32_t* chunk_keys = nullptr; // [(m_max-1)][words*32] sorted objective keys per word
    uint32_t* chunk_bits = nullptr; // [(m_max-1)][words*33] prefix position sets per word
    uint32_t* block_tables = nullptr;  // per block of 128 or 256 positions and objective: search
                                       // tree of the keys and prefix sets (nds_block_rows)
    int* blocker = nullptr;         // per sorted position: last known unassigned dominator
    int* front_sorted = nullptr;    // per sorted position: front index or -1
    int* front_list = nullptr;      // members of each peeled front, front by front
    int* counters = nullptr;        // [0] feasible count, [1] list length (batched peel),
                                    // [2] max_front, [3] assigned, [4] grid-barrier arrivals,
                                    // [6] device status, [10] class-2 count, [11] class-3 count,
                                    // [12] last feasible front, [13] long runs of equal sort keys,
                                    // [16..19] two 64-bit barrier words carrying front sizes
    int peel_grid = 0;              // co-resident CTAs of the peel kernel
    int sm_count = 0;               // SMs of the workspace's device
    int peel_owned_grid = 0;        // CTAs of the lane-owned peel (one per SM), 0 if unavailable
    int peel_smem = 0;
    bool peel_single_cta = false;   // peel with one ordinary CTA (instances of a batch)
    bool peel_general = false;      // always the general peel (moea_workspace_set_peel)
    bool word_tiles = false;        // dominance rows from per-word tables (moea_workspace_set_tiles)
    uint32_t* peel_fmask = nullptr; // [3][words] members of the last three fronts (peel)

    // --- NSGA-III stages ---
    int* fronts = nullptr;          // fronts of the merged population (point order)
    int* nds_gidx = nullptr;        // [prior; last] point indices
    int* sizes = nullptr;           // {N_prior, N_last, N_rem, N_nds}
    int* chunk_counts = nullptr;    // ordered-compaction partial counts
    float* nds_objs = nullptr;      // (m_max, n_max) translated objectives of nds points
    float* norm_part = nullptr;     // ASF / max partials
    int* norm_part_idx = nullptr;
    float* rcp_b = nullptr;         // (m_max) reciprocal intercepts
    int* extreme = nullptr;         // (m_max)
    float* ideal_tmp = nullptr;     // (m_max)
    unsigned long long* assoc_best = nullptr;  // packed (d2 bits, j) per nds point
    int* assoc_idx = nullptr;
    float* assoc_dist = nullptr;
    int* rho = nullptr;             // (h_max) niche counts of prior fronts
    int* sel_vals[2] = {};          // niching sort values
    int* rank = nullptr;
    int* selected = nullptr;        // (n_max) selection before ordering
    int* flags = nullptr;           // (n_max) survivor flags
    unsigned long long* offset_dev = nullptr;  // niching counter offset

    // --- cone tree of the directions for the pruned association ---
    // Device copy of a DirectionTreeHost; valid for the directions at
    // tree_src (M = tree_M, H = tree_H) until prepared again.
    const float* tree_src = nullptr;
    int tree_M = 0, tree_H = 0, tree_nodes = 0, tree_depth = 0;
    float tree_delta = 0.0f;
    size_t tree_cap_dirs = 0, tree_cap_nodes = 0;   // allocated capacities
    float* tree_dirs = nullptr;     // (M, H) directions in tree order
    int* tree_order = nullptr;      // (H) tree position -> direction index
    float* tree_center = nullptr;   // (M, nodes)
    float* tree_cos = nullptr;      // (nodes)
    float* tree_sin = nullptr;      // (nodes)
    int2* tree_link = nullptr;      // (nodes)
    float* dir_delta = nullptr;     // (1) max | |r|^2 - 1 | of the last scanned directions

    // --- split TF32 operand of the directions for the tensor-core association ---
    // Valid for the directions at tc_src (M = tc_M, H = tc_H) until prepared again.
    const float* tc_src = nullptr;
    int tc_M = 0, tc_H = 0;
    size_t tc_cap = 0;              // floats allocated at tc_dirs
    float* tc_dirs = nullptr;       // tiles of 128 directions in the MMA's shared-memory image,
                                    // then one float: max | |r|^2 - 1 | of the directions
    unsigned* tc_rowmax = nullptr;  // (n_max) largest |x.r_j| estimate per point (FP32 bits)
    double* scalar_d = nullptr;     // (1) FP64 result word (IGD mean)

    // --- CUB temporary storage ---
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
};

// ---- per-TU entry points -------------------------------------------------
// Non-dominated sort of the split view.  Fronts in point order into ws.fronts
// (or out_fronts when non-null), max front into ws.counters[2].
// Passes of the Philox variation: SBX and PM fused, SBX alone, PM alone (in
// place).  The draws are the same in every form.
enum VariationPass { kPassBoth = 3, kPassCrossover = 1, kPassMutation = 2 };
int run_variation_pass(int passes, const float* parents, const int* pidx, const float* bounds, float* off,
                       int n_off, int D, float sbx_eta0, float sbx_eta1, float sbx_prob, float copy_prob,
                       int mutate, float pm_eta0, float pm_eta1, float pm_prob, int total,
                       uint64_t seed, const int* d_gen, uint32_t gen, cudaStream_t stream);

int run_ndsort(Workspace& ws, const SplitPop& pop, int M, int target, int* out_fronts,
               cudaStream_t stream);

// Ordered compaction of the fronts into [prior; last] (ws.nds_gidx, ws.sizes).
int run_extract(Workspace& ws, const int* fronts, int n, const int* d_max_front, int N,
                int* nds_gidx, int* sizes, cudaStream_t stream);

// Gather translated objectives of the nds points and run the normalisation;
// leaves translated values in ws.nds_objs and reciprocal intercepts in ws.rcp_b.
int run_normalize_split(Workspace& ws, const SplitPop& pop, const int* nds_gidx,
                        const int* sizes, const float* ideal, int M, cudaStream_t stream);

// Copy of `units` 16-byte words by the threads lane = 0 .. lanes-1 of a
// group, four loads in flight per thread (a row of a large-D population is
// otherwise copied one dependent load/store pair at a time).
__device__ __forceinline__ void copy_units4(float4* __restrict__ dst, const float4* __restrict__ src, int units,
                                           int lane, int lanes)
{
    int u = lane;
    for (; u + 3 * lanes < units; u += 4 * lanes) {
        const float4 a = __ldg(src + u), b = __ldg(src + u + lanes);
        const float4 c = __ldg(src + u + 2 * lanes), d = __ldg(src + u + 3 * lanes);
        dst[u] = a;
        dst[u + lanes] = b;
        dst[u + 2 * lanes] = c;
        dst[u + 3 * lanes] = d;
    }
    for (; u < units; u += lanes) dst[u] = __ldg(src + u);
}

// Margin of the dot^2 candidate filter of the association for a point with
// |x|^2 = xx.  For directions with | |r|^2 - 1 | <= delta, the reference's
// FP32 distance (association.cu:139-170) differs from xx - dot^2 by at most
// about (4M+5) 2^-24 xx plus xx (1 + delta) delta; the filter uses
// (16M+64) 2^-24 xx + 2.5 delta xx.  Directions far from unit length
// (delta > 1e-3) and non-finite points get an infinite margin: every
// direction is re-scored.
__device__ __forceinline__ float assoc_margin(int M, float xx, float delta)
{
    const float kEps = 5.9604645e-08f;  // 2^-24
    float margin = xx * ((16.0f * M + 64.0f) * kEps + 2.5f * delta) + 1e-35f;
    if (!isfinite(xx) || !(delta <= 1e-3f)) margin = INFINITY;
    return margin;
}

// max_j | |r_j|^2 - 1 | of the directions (M,H) in FP64, rounded up to FP32.
int run_dir_delta(const float* refs, int M, int H, float* out, cudaStream_t stream);

// Packed (d2 bits, direction) minima of the association merged across
// direction ranges: reset to "none", then unpacked into idx/dist.
int run_assoc_reset(unsigned long long* best, int n_cap, cudaStream_t stream);
int run_assoc_finish(const unsigned long long* best, const int* d_n, int n_cap, int* idx, float* dist,
                     cudaStream_t stream);

// Tensor-core association (MOEA_ASSOC_TENSOR): split TF32 operand of the
// directions, built on the device; the association itself.  MOEA_ASSOC_TREE
// also takes this search for more objectives than the cone tree handles when
// there are at least kTensorMinPairs point-direction pairs (tensor_preferred)
// and the operand was prepared.
constexpr long long kTensorMinPairs = 1ll << 24;
bool tensor_preferred(int M, int n_cap, int H);
int prepare_tensor_directions(Workspace& ws, const float* d_refs, int M, int H, cudaStream_t stream);
bool tensor_directions_ready(const Workspace& ws, const float* d_refs, int M, int H);
int run_associate_tensor(Workspace& ws, const float* x, int x_stride, const float* scale, const float* refs,
                         int M, const int* d_n, int n_cap, int H, int* idx, float* dist, cudaStream_t stream);

// mode MOEA_ASSOC_TREE needs prepare_direction_tree for these refs first,
// mode MOEA_ASSOC_TENSOR prepare_tensor_directions.
int run_associate(Workspace& ws, const float* x, int x_stride, const float* scale,
                  const float* refs, int M, const int* d_n, int n_cap, int H, int* idx,
                  float* dist, int mode, cudaStream_t stream);

// Builds the cone tree of the directions on the host and uploads it into the
// workspace, tagged with the device pointer d_refs.  h_refs may be null, in
// which case the directions are read back from d_refs (synchronising stream).
int prepare_direction_tree(Workspace& ws, const float* d_refs, const float* h_refs, int M, int H,
                           cudaStream_t stream);
bool direction_tree_ready(const Workspace& ws, const float* d_refs, int M, int H);

// Niching of the last front on one 16-CTA cluster (niching_cluster.cu):
// merged populations up to niching_cluster_capacity() members.
int niching_cluster_capacity();
bool niching_cluster_ready();
int launch_niching_cluster(const int* idx, const float* dist, const int* sizes, const int* rho, int H,
                           uint64_t seed, unsigned long long* offset, const int* nds_gidx, int* selected,
                           int* status, cudaStream_t stream);
int run_niching(Workspace& ws, uint64_t seed, const int* nds_gidx, const float* dist,
                const int* idx, const int* sizes, int H, int N, int* selected,
                cudaStream_t stream);

// ideal_out[m] = fminf(prev[m], min_i objs[m][i]) (prev may be null).
int run_ideal(const float* objs, int stride, int M, int n, const float* prev, float* ideal_out,
              cudaStream_t stream);

// Survivor ordering: ascending unique indices from an unordered selection.
int run_order_selection(Workspace& ws, const int* selected, int count, int n_mix,
                        int* out_sorted, cudaStream_t stream);

// Ascending indices i < n with ws.flags[i] != 0 into out.
int run_flag_compaction(Workspace& ws, int n, int* out, cudaStream_t stream);

size_t cub_temp_bytes_needed(int n_max);

// ---- fused batch ------------------------------------------------------------
// One NSGA-III instance of a fused batch: sizes, parameters and every buffer a
// generation touches, for one parity of the slot rotation (P parents, O
// offspring, X next).  The fused generation runs each stage once for all
// instances: one CTA per instance where the stage needs a block-wide sort,
// scan or barrier (n = 2N <= kFusedMaxPoints), flattened work items elsewhere.
constexpr int kFusedMaxPoints = 8192;
constexpr int kDirTreeMaxDepth = 8;   // stack depth of the tree association kernels
constexpr int kFusedThreads = 1024;
constexpr int kFusedItems = kFusedMaxPoints / kFusedThreads;

struct BatchInst {
    int N, D, M, H, n, n_max, W, kind, tournament, mutate, T;
    float sbx_eta0, sbx_eta1, sbx_prob, sbx_copy, pm_eta0, pm_eta1, pm_prob;
    uint64_t seed;        // draws of mating and variation
    uint64_t nich_seed;   // niching tie-break hash
    const float* varsP; const float* objsP; const float* cvP; const int* rankP;
    float* varsO; float* objsO; float* cvO;
    float* varsX; float* objsX; float* cvX; int* rankX;
    const float* bounds; int* pidx; int* d_gen; float* ideal;
    uint64_t* key0; uint64_t* key64; int* perm; int* vals; float* sorted_f; int* qinfo;
    int* blocker; int* front_sorted; int* front_list; int* counters;
    uint32_t* rows; uint32_t* chunk_keys; uint32_t* chunk_bits;
    int* fronts; int* nds_gidx; int* sizes; float* nds_objs; float* rcp_b; int* extreme;
    int* assoc_idx; float* assoc_dist; int* rho; int* selected; int* flags; int* survivors;
    unsigned long long* assoc_best;  // packed (d2 bits, index) minima of a direction-split scan
    unsigned long long* offset;
    const float* t_dirs_orig;  // (M, H) directions in their own order
    const float* t_dirs; const int* t_order; const float* t_center; const float* t_cos;
    const float* t_sin; const int2* t_link; int t_nodes; float t_delta;
};

// Launch plan of one M value: instance ids and the prefix of their tile blocks.
struct FusedBucket {
    int M = 0, count = 0, max_n = 0, tile_blocks = 0;
    int shape = 0;                 // dominance tile shape (fused_tile_blocks)
    int max_H = 0;                 // most directions of an instance
    int* d_ids = nullptr;          // (count) instance indices
    int* d_tile_prefix = nullptr;  // (count + 1) first tile block of each instance
};

// A group of instances that runs the fused chain of kernels on one stream:
// its instance ids, size bounds and per-M buckets.
struct FusedGroup {
    int count = 0, max_n = 0, max_N = 0, max_D = 0, max_M = 0;
    int max_W = 0;                       // largest row stride (words) of the group's workspaces
    int* d_ids = nullptr;                // (count) instance indices
    std::vector<FusedBucket> buckets;    // per objective count
};

int fused_reproduce(const BatchInst* d_inst, const FusedGroup& g, cudaStream_t s);
int fused_evaluate(const BatchInst* d_inst, const FusedGroup& g, cudaStream_t s);
int fused_ndsort(const BatchInst* d_inst, const FusedGroup& g, cudaStream_t s);
int fused_select(const BatchInst* d_inst, const FusedGroup& g, cudaStream_t s);
int fused_tile_blocks(int M, int n, int shape);  // tile CTAs of one instance in a tile shape (0, 1)
constexpr int kTileShapes = 2;
// Kernel attributes (shared memory opt-in) of the fused stages, set once per
// device before any capture.
int fused_ndsort_configure();
int fused_select_configure();

}  // namespace moea

struct moea_workspace {
    moea::Workspace ws;
};
