// Workspace management, error reporting and the stage-level C entry points.
#include <cstdarg>
#include <cstring>
#include <new>

#include "internal.cuh"

namespace moea {

int configure_peel(Workspace& ws);
size_t block_table_words(int n_max, int m_max);
int configure_block_rows();
int selftest_barrier_timeout(Workspace& ws, int which, unsigned long long limit_ns, cudaStream_t stream);
int selftest_mbar_timeout(Workspace& ws, unsigned long long limit_ns, cudaStream_t stream);
int run_normalize_inplace(Workspace& ws, float* objs, const float* ideal, int M, int n,
                          float* rcp_out, int* extreme_out, cudaStream_t stream);
int run_nsga3_select(Workspace& ws, const SplitPop& pop, int M, int N, const float* refs, int H,
                     uint64_t seed, float* ideal_last, int* survivors, int* survivor_fronts,
                     int assoc_mode, cudaStream_t stream, const SplitPop* sort_pop);
int run_quantize_cv(const float* cv, float* out, int n, float eps, float clip, float log_alpha,
                    int bins, cudaStream_t stream);

namespace {
thread_local char g_error[1024] = "";
}

int set_error(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    return code;
}

const char* last_error() { return g_error; }

StageProfile*& stage_profile()
{
    static thread_local StageProfile* p = nullptr;
    return p;
}

void stage_mark(const char* name, cudaStream_t stream)
{
    StageProfile* p = stage_profile();
    if (!p) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, stream);
    p->events.push_back(e);
    p->names.push_back(name);
}

namespace {

template <class T>
int dalloc(Workspace& ws, T** p, size_t count)
{
    const size_t bytes = sizeof(T) * (count > 0 ? count : 1);
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(e == cudaErrorMemoryAllocation ? MOEA_ERR_OUT_OF_MEMORY : MOEA_ERR_CUDA,
                         "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    ws.bytes += bytes;
    return MOEA_OK;
}

void free_all(Workspace& ws)
{
    void* ptrs[] = {ws.rows, ws.key32[0], ws.key32[1], ws.key64[0], ws.key64[1], ws.key0,
                    ws.perm[0], ws.perm[1], ws.sorted_f, ws.qinfo, ws.head, ws.run_start,
                    ws.blocker, ws.front_sorted, ws.front_list, ws.counters, ws.fronts,
                    ws.nds_gidx, ws.sizes, ws.chunk_counts, ws.nds_objs, ws.norm_part,
                    ws.norm_part_idx, ws.rcp_b, ws.extreme, ws.ideal_tmp, ws.assoc_best,
                    ws.assoc_idx, ws.assoc_dist, ws.rho, ws.sel_vals[0], ws.sel_vals[1],
                    ws.rank, ws.selected, ws.flags, ws.offset_dev, ws.cub_tmp, ws.tree_dirs,
                    ws.tree_order, ws.tree_center, ws.dir_delta, ws.chunk_keys, ws.chunk_bits,
                    ws.block_tables, ws.scalar_d, ws.tc_dirs, ws.tc_rowmax, ws.peel_fmask};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    ws = Workspace{};
}

}  // namespace

int workspace_init(Workspace& ws, int device, int n_max, int m_max, int h_max)
{
    if (n_max < 2 || m_max < 1 || m_max > kMaxObjectives || h_max < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT,
                         "workspace: max_points=%d max_objectives=%d (1..%d) max_directions=%d",
                         n_max, m_max, kMaxObjectives, h_max);
    if (n_max > (1 << 24))
        return set_error(MOEA_ERR_UNSUPPORTED, "workspace: max_points=%d exceeds 2^24", n_max);
    MOEA_CUDA_TRY(cudaSetDevice(device));
    ws.device = device;
    ws.n_max = n_max;
    ws.m_max = m_max;
    ws.h_max = h_max;
    // row words per point, a multiple of 4 so that every row starts on a
    // 16-byte boundary (the peel copies aligned 16-byte chunks of rows)
    ws.words = 4 * ceil_div(n_max, 128);
    const size_t n = (size_t)n_max;
    const int nb = ceil_div(n_max, 256);
    int st = MOEA_OK;
#define A(p, c) if (st == MOEA_OK) st = dalloc(ws, &(p), (c))
    A(ws.rows, n * (size_t)ws.words);
    A(ws.key32[0], n); A(ws.key32[1], n);
    A(ws.key64[0], n); A(ws.key64[1], n); A(ws.key0, n);
    A(ws.perm[0], n); A(ws.perm[1], n);
    A(ws.sorted_f, n * (size_t)(m_max > 1 ? m_max - 1 : 1));
    A(ws.qinfo, n); A(ws.head, n); A(ws.run_start, n);
    A(ws.blocker, n); A(ws.front_sorted, n); A(ws.front_list, n);
    A(ws.chunk_keys, (size_t)(m_max > 1 ? m_max - 1 : 1) * ws.words * 32);
    A(ws.chunk_bits, (size_t)(m_max > 1 ? m_max - 1 : 1) * ws.words * 33);
    if (m_max > 1) A(ws.block_tables, block_table_words(n_max, m_max));
    A(ws.counters, 32);
    A(ws.fronts, n); A(ws.nds_gidx, n); A(ws.sizes, 8);
    A(ws.chunk_counts, 2 * (size_t)ceil_div(n_max, 1024) + 2);
    A(ws.nds_objs, n * (size_t)m_max);
    A(ws.norm_part, 2 * (size_t)nb * m_max);
    A(ws.norm_part_idx, (size_t)nb * m_max);
    A(ws.rcp_b, m_max); A(ws.extreme, m_max); A(ws.ideal_tmp, m_max);
    A(ws.assoc_best, n); A(ws.assoc_idx, n); A(ws.assoc_dist, n);
    A(ws.rho, (size_t)h_max);
    A(ws.sel_vals[0], n); A(ws.sel_vals[1], n);
    A(ws.rank, n); A(ws.selected, n); A(ws.flags, n);
    A(ws.offset_dev, 1);
    A(ws.dir_delta, 1);
    A(ws.scalar_d, 1);
#undef A
    if (st == MOEA_OK) {
        ws.cub_bytes = cub_temp_bytes_needed(n_max);
        st = dalloc(ws, (char**)&ws.cub_tmp, ws.cub_bytes);
    }
    if (st == MOEA_OK) {
        cudaError_t e = cudaMemset(ws.counters, 0, 32 * sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(ws.offset_dev, 0, sizeof(unsigned long long));
        if (e != cudaSuccess) st = set_error(MOEA_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    }
    if (st == MOEA_OK) st = configure_peel(ws);
    if (st == MOEA_OK) st = configure_block_rows();
    if (st == MOEA_OK) st = dalloc(ws, &ws.peel_fmask, 3 * (size_t)ws.words);
    if (st != MOEA_OK) free_all(ws);
    return st;
}

void workspace_free(Workspace& ws) { free_all(ws); }

// Reads and clears the device status word; converts it to a moea_status.
int workspace_check_status(Workspace& ws, cudaStream_t stream)
{
    int st = 0;
    MOEA_CUDA_TRY(cudaMemcpyAsync(&st, ws.counters + 6, sizeof(int), cudaMemcpyDeviceToHost, stream));
    MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
    if (st != kDevOk) {
        const int zero = 0;
        cudaMemcpy(ws.counters + 6, &zero, sizeof(int), cudaMemcpyHostToDevice);
        if (st == kDevBarrierTimeout)
            return set_error(MOEA_ERR_DEVICE_TIMEOUT, "front peeling: grid barrier timed out");
        if (st == kDevTensorTimeout)
            return set_error(MOEA_ERR_DEVICE_TIMEOUT, "association: tensor-core wait timed out");
        if (st == kDevNichingSize)
            return set_error(MOEA_ERR_UNSUPPORTED, "niching: last front exceeds the cluster's capacity");
        return set_error(MOEA_ERR_CUDA, "front peeling: inconsistent dominance relation (status %d)", st);
    }
    return MOEA_OK;
}

}  // namespace moea

using namespace moea;

namespace {
inline cudaStream_t S(void* s) { return (cudaStream_t)s; }
#define CHECK_WS(ws)                                                              \
    if (!(ws)) return set_error(MOEA_ERR_INVALID_ARGUMENT, "workspace is NULL")
}  // namespace

extern "C" {

int moea_abi_version(void) { return MOEA_ABI_VERSION; }
const char* moea_last_error(void) { return moea::last_error(); }

moea_status moea_workspace_create(int device, int max_points, int max_objectives,
                                  int max_directions, moea_workspace** out)
{
    if (!out) return set_error(MOEA_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    moea_workspace* w = new (std::nothrow) moea_workspace();
    if (!w) return set_error(MOEA_ERR_OUT_OF_MEMORY, "host allocation failed");
    const int st = workspace_init(w->ws, device, max_points, max_objectives, max_directions);
    if (st != MOEA_OK) {
        delete w;
        return st;
    }
    *out = w;
    return MOEA_OK;
}

void moea_workspace_destroy(moea_workspace* ws)
{
    if (!ws) return;
    cudaSetDevice(ws->ws.device);
    workspace_free(ws->ws);
    delete ws;
}

size_t moea_workspace_bytes(const moea_workspace* ws) { return ws ? ws->ws.bytes : 0; }

moea_status moea_workspace_set_peel(moea_workspace* w, int mode)
{
    CHECK_WS(w);
    if (mode != MOEA_PEEL_AUTO && mode != MOEA_PEEL_GENERAL)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "set_peel: mode %d", mode);
    w->ws.peel_general = mode == MOEA_PEEL_GENERAL;
    return MOEA_OK;
}

moea_status moea_workspace_set_tiles(moea_workspace* w, int mode)
{
    CHECK_WS(w);
    if (mode != MOEA_TILES_AUTO && mode != MOEA_TILES_WORD)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "set_tiles: mode %d", mode);
    w->ws.word_tiles = mode == MOEA_TILES_WORD;
    return MOEA_OK;
}

moea_status moea_ndsort(moea_workspace* w, const float* d_cv, const float* d_objs, int M, int n,
                        int target, int* d_fronts, int* h_max_front, void* stream)
{
    CHECK_WS(w);
    if (!d_cv || !d_objs || !d_fronts || n < 0)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "ndsort: null pointer or negative size");
    if (n == 0) {
        if (h_max_front) *h_max_front = 0;
        return MOEA_OK;
    }
    Workspace& ws = w->ws;
    MOEA_TRY(run_ndsort(ws, merged_view(d_objs, d_cv, n), M, target, d_fronts, S(stream)));
    int mf = 0;
    MOEA_CUDA_TRY(cudaMemcpyAsync(&mf, ws.counters + 2, sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
    MOEA_TRY(workspace_check_status(ws, S(stream)));
    if (h_max_front) *h_max_front = mf;
    return MOEA_OK;
}

moea_status moea_nds_extract(moea_workspace* w, const int* d_fronts, int n_mix,
                             const int* d_max_front, int N, int* d_nds_gidx, int* d_sizes,
                             void* stream)
{
    CHECK_WS(w);
    if (!d_fronts || !d_max_front || !d_nds_gidx || !d_sizes || n_mix <= 0 || n_mix > w->ws.n_max)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "nds_extract: bad arguments");
    return run_extract(w->ws, d_fronts, n_mix, d_max_front, N, d_nds_gidx, d_sizes, S(stream));
}

moea_status moea_ideal_point(moea_workspace* w, const float* d_objs, int M, int n, float* d_ideal,
                             void* stream)
{
    CHECK_WS(w);
    if (!d_objs || !d_ideal || M < 1 || n < 0)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "ideal_point: bad arguments");
    return run_ideal(d_objs, n, M, n, nullptr, d_ideal, S(stream));
}

moea_status moea_normalize(moea_workspace* w, float* d_objs, const float* d_ideal, int M, int n,
                           float* d_rcp_b, int* d_extreme, void* stream)
{
    CHECK_WS(w);
    if (!d_objs || !d_ideal || !d_rcp_b || n < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "normalize: bad arguments");
    return run_normalize_inplace(w->ws, d_objs, d_ideal, M, n, d_rcp_b, d_extreme, S(stream));
}

moea_status moea_associate(moea_workspace* w, const float* d_x, const float* d_refs, int M, int n,
                           int H, int* d_idx, float* d_dist, int mode, void* stream)
{
    CHECK_WS(w);
    if (!d_x || !d_refs || !d_idx || !d_dist || n < 0 || n > w->ws.n_max || M < 1 ||
        M > kMaxObjectives || H < 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "associate: bad arguments");
    if (n == 0) return MOEA_OK;
    Workspace& ws = w->ws;
    if (mode == MOEA_ASSOC_TREE) MOEA_TRY(prepare_direction_tree(ws, d_refs, nullptr, M, H, S(stream)));
    const bool tensor = mode == MOEA_ASSOC_TENSOR || (mode == MOEA_ASSOC_TREE && tensor_preferred(M, n, H));
    if (tensor) MOEA_TRY(prepare_tensor_directions(ws, d_refs, M, H, S(stream)));
    int hs[4] = {0, n, 0, n};
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.sizes + 4, &hs[3], sizeof(int), cudaMemcpyHostToDevice, S(stream)));
    MOEA_TRY(run_associate(ws, d_x, n, nullptr, d_refs, M, ws.sizes + 4, n, H, d_idx, d_dist, mode,
                           S(stream)));
    if (tensor) return workspace_check_status(ws, S(stream));
    return MOEA_OK;
}

moea_status moea_niching(moea_workspace* w, uint64_t seed, uint64_t* h_offset,
                         const int* d_nds_gidx, const float* d_dist, const int* d_idx,
                         const int* d_sizes, int H, int N, int* d_selected, void* stream)
{
    CHECK_WS(w);
    if (!h_offset || !d_nds_gidx || !d_dist || !d_idx || !d_sizes || !d_selected || N < 1 ||
        2 * N > w->ws.n_max || H < 1 || H > w->ws.h_max)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "niching: bad arguments");
    Workspace& ws = w->ws;
    unsigned long long off = *h_offset;
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.offset_dev, &off, sizeof(off), cudaMemcpyHostToDevice, S(stream)));
    MOEA_TRY(run_niching(ws, seed, d_nds_gidx, d_dist, d_idx, d_sizes, H, N, d_selected, S(stream)));
    MOEA_CUDA_TRY(cudaMemcpyAsync(&off, ws.offset_dev, sizeof(off), cudaMemcpyDeviceToHost, S(stream)));
    MOEA_CUDA_TRY(cudaStreamSynchronize(S(stream)));
    *h_offset = off;
    return MOEA_OK;
}

moea_status moea_nsga3_select(moea_workspace* w, const float* d_mix_cv, const float* d_mix_objs,
                              int M, int N, const float* d_refs, int H, uint64_t seed,
                              uint64_t* h_offset, float* d_ideal_last, int* d_survivors,
                              int* d_survivor_fronts, int* d_sizes, int assoc_mode, void* stream)
{
    CHECK_WS(w);
    Workspace& ws = w->ws;
    if (!d_mix_cv || !d_mix_objs || !d_refs || !h_offset || !d_ideal_last || !d_survivors ||
        N < 1 || 2 * N > ws.n_max || M < 1 || M > ws.m_max || H < 1 || H > ws.h_max)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "nsga3_select: bad arguments");
    if (assoc_mode == MOEA_ASSOC_TREE) MOEA_TRY(prepare_direction_tree(ws, d_refs, nullptr, M, H, S(stream)));
    if (assoc_mode == MOEA_ASSOC_TENSOR || (assoc_mode == MOEA_ASSOC_TREE && tensor_preferred(M, 2 * N, H)))
        MOEA_TRY(prepare_tensor_directions(ws, d_refs, M, H, S(stream)));
    unsigned long long off = *h_offset;
    MOEA_CUDA_TRY(cudaMemcpyAsync(ws.offset_dev, &off, sizeof(off), cudaMemcpyHostToDevice, S(stream)));
    SplitPop pop{d_mix_objs, d_mix_objs + N, d_mix_cv, d_mix_cv + N, 2 * N, 2 * N, N, 2 * N};
    MOEA_TRY(run_nsga3_select(ws, pop, M, N, d_refs, H, seed, d_ideal_last, d_survivors,
                              d_survivor_fronts, assoc_mode, S(stream), nullptr));
    if (d_sizes)
        MOEA_CUDA_TRY(cudaMemcpyAsync(d_sizes, ws.sizes, 4 * sizeof(int), cudaMemcpyDeviceToDevice,
                                      S(stream)));
    MOEA_CUDA_TRY(cudaMemcpyAsync(&off, ws.offset_dev, sizeof(off), cudaMemcpyDeviceToHost, S(stream)));
    MOEA_TRY(workspace_check_status(ws, S(stream)));
    *h_offset = off;
    return MOEA_OK;
}

moea_status moea_quantize_cv(const float* d_cv, float* d_out, int n, float eps_feas,
                             float clip_upper, float log_alpha, int bins, void* stream)
{
    if (!d_cv || !d_out || n < 0 || bins <= 0 || !(clip_upper > 0.0f) || log_alpha < 0.0f ||
        eps_feas < 0.0f)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "quantize_cv: bad arguments");
    return run_quantize_cv(d_cv, d_out, n, eps_feas, clip_upper, log_alpha, bins, S(stream));
}

moea_status moea_selftest_wait_timeout(moea_workspace* w, int which, unsigned long long limit_ns, void* stream)
{
    CHECK_WS(w);
    if (which < 0 || which > 2 || limit_ns == 0 || limit_ns > 2000000000ull)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "selftest_wait_timeout: which=%d limit_ns=%llu", which,
                         limit_ns);
    Workspace& ws = w->ws;
    MOEA_CUDA_TRY(cudaSetDevice(ws.device));
    if (which < 2) MOEA_TRY(selftest_barrier_timeout(ws, which, limit_ns, S(stream)));
    else MOEA_TRY(selftest_mbar_timeout(ws, limit_ns, S(stream)));
    return workspace_check_status(ws, S(stream));
}

}  // extern "C"
