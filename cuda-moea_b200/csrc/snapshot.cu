// Snapshots of a running algorithm in the reference's DataRecorder format
// (nat/src/algorithm/data_recorder.cu:128-292), and resumption from them.
//
// On-disk format, kept byte for byte:
//   <root>/lower_bounds.bin, upper_bounds.bin   D float32 each
//   <root>/initial_reference_directions.bin     (M,K) float32, objective-major
//   <root>/metadata.json                        run description (same keys and text)
//   <root>/generation_NNNNNN/variables.bin      (N,D) float32, row-major
//                            objectives.bin     (M,N) float32, objective-major
//                            constraints.bin    (N) float32
//                            reference_directions.bin        (M,K) float32
//                            selector_auxiliary_indices.bin  int32 (when non-empty)
//                            snapshot.json
// Saved: generation 0, every interval-th generation and the last one
// (data_recorder.cu:128-136).
//
// Unlike the reference, which synchronises and copies with cudaMemcpy, a
// snapshot here is two pinned host slots used in turn: the device-to-host
// copies run on a side stream after an event of the compute stream, the
// compute stream waits only for those copies (the next generation overwrites
// the parents' buffers), and a host function on the side stream writes the
// files.  Write errors are kept and reported by flush().
//
// resume.bin (not in the reference) holds the state a bit-identical
// continuation needs besides the files above: the generation, the reset
// epoch, the active count, the niching counter offset, the running ideal
// point and the constraint-activation bookkeeping.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "snapshot.h"

namespace moea {
namespace fs = std::filesystem;

namespace {

constexpr char kResumeMagic[8] = {'M', 'O', 'E', 'A', 'R', 'S', 'M', '1'};

std::string json_string(const std::string& value)
{
    std::ostringstream out;
    out << '"';
    for (const char c : value) {
        switch (c) {
        case '"': out << "\\\""; break;
        case '\\': out << "\\\\"; break;
        case '\b': out << "\\b"; break;
        case '\f': out << "\\f"; break;
        case '\n': out << "\\n"; break;
        case '\r': out << "\\r"; break;
        case '\t': out << "\\t"; break;
        default:
            if (static_cast<unsigned char>(c) < 0x20) {
                out << "\\u" << std::hex << std::setw(4) << std::setfill('0')
                    << static_cast<int>(static_cast<unsigned char>(c)) << std::dec << std::setfill(' ');
            } else {
                out << c;
            }
        }
    }
    out << '"';
    return out.str();
}

bool write_file(const fs::path& path, const void* data, size_t bytes, std::string& err)
{
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    if (!out) {
        err = "Cannot create data file: " + path.string();
        return false;
    }
    if (bytes) out.write(static_cast<const char*>(data), static_cast<std::streamsize>(bytes));
    if (!out) {
        err = "Failed to write data file: " + path.string();
        return false;
    }
    return true;
}

bool write_text(const fs::path& path, const std::string& text, std::string& err)
{
    return write_file(path, text.data(), text.size(), err);
}

// Exactly `bytes` bytes of the file, or false.
bool read_file(const fs::path& path, void* data, size_t bytes, std::string& err)
{
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        err = "Cannot open " + path.string();
        return false;
    }
    in.seekg(0, std::ios::end);
    const auto size = static_cast<size_t>(in.tellg());
    if (size != bytes) {
        err = path.string() + " holds " + std::to_string(size) + " bytes, expected " + std::to_string(bytes);
        return false;
    }
    in.seekg(0);
    if (bytes) in.read(static_cast<char*>(data), static_cast<std::streamsize>(bytes));
    if (!in) {
        err = "Failed to read " + path.string();
        return false;
    }
    return true;
}

fs::path generation_directory(const fs::path& root, int generation)
{
    std::ostringstream name;
    name << "generation_" << std::setw(6) << std::setfill('0') << generation;
    return root / name.str();
}

struct ResumeHeader {
    char magic[8];
    int32_t version, N, D, M, H, generation, active, last_prepared_target, ideal_ready;
    uint32_t epoch;
    uint64_t niching_offset;
};

}  // namespace

// One pinned staging area and the description of the snapshot it holds.
struct SnapshotWriter::Slot {
    SnapshotWriter* owner = nullptr;
    char* host = nullptr;             // vars | objs | cv | refs | aux | ideal | offset | active
    float *vars = nullptr, *objs = nullptr, *cv = nullptr, *refs = nullptr, *ideal = nullptr;
    int* aux = nullptr;
    unsigned long long* offset = nullptr;
    int* active = nullptr;
    cudaEvent_t done = nullptr;       // files of this slot written
    bool busy = false;
    SnapshotSave info{};
};

SnapshotWriter::SnapshotWriter() = default;

SnapshotWriter::~SnapshotWriter()
{
    flush();
    for (auto& s : slots_) {
        if (!s) continue;
        if (s->done) cudaEventDestroy(s->done);
        if (s->host) cudaFreeHost(s->host);
        delete s;
    }
    if (copied_) cudaEventDestroy(copied_);
    if (ready_) cudaEventDestroy(ready_);
    if (side_) cudaStreamDestroy(side_);
}

bool SnapshotWriter::should_save(int generation) const
{
    return generation == 0 || generation == meta_.T || generation % interval_ == 0;
}

int SnapshotWriter::open(const std::string& directory, int interval, const SnapshotMeta& meta,
                         const std::vector<float>& lower, const std::vector<float>& upper,
                         const float* d_initial_refs, cudaStream_t stream)
{
    if (directory.empty()) return set_error(MOEA_ERR_INVALID_ARGUMENT, "saveData output directory cannot be empty");
    if (interval <= 0) return set_error(MOEA_ERR_INVALID_ARGUMENT, "saveData generation interval must be positive");
    root_ = directory;
    interval_ = interval;
    meta_ = meta;
    std::error_code ec;
    fs::create_directories(root_, ec);
    if (ec)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "Cannot create data directory '%s': %s", root_.c_str(),
                         ec.message().c_str());
    std::string err;
    if (!write_file(fs::path(root_) / "lower_bounds.bin", lower.data(), sizeof(float) * lower.size(), err) ||
        !write_file(fs::path(root_) / "upper_bounds.bin", upper.data(), sizeof(float) * upper.size(), err))
        return set_error(MOEA_ERR_CUDA, "%s", err.c_str());
    const size_t nref = (size_t)meta.M * meta.H;
    if (d_initial_refs && nref > 0) {
        std::vector<float> h(nref);
        MOEA_CUDA_TRY(cudaMemcpyAsync(h.data(), d_initial_refs, sizeof(float) * nref, cudaMemcpyDeviceToHost, stream));
        MOEA_CUDA_TRY(cudaStreamSynchronize(stream));
        if (!write_file(fs::path(root_) / "initial_reference_directions.bin", h.data(), sizeof(float) * nref, err))
            return set_error(MOEA_ERR_CUDA, "%s", err.c_str());
    }
    std::ostringstream m;
    m << "{\n"
      << "  \"format_version\": 1,\n"
      << "  \"scalar_type\": \"float32\",\n"
      << "  \"index_type\": \"int32\",\n"
      << "  \"algorithm_name\": " << (meta.algorithm_name.empty() ? "null" : json_string(meta.algorithm_name)) << ",\n"
      << "  \"problem_name\": " << (meta.problem_name.empty() ? "null" : json_string(meta.problem_name)) << ",\n"
      << "  \"population_size\": " << meta.N << ",\n"
      << "  \"dimension\": " << meta.D << ",\n"
      << "  \"objective_count\": " << meta.M << ",\n"
      << "  \"constraint_count\": " << meta.constraint_count << ",\n"
      << "  \"max_generations\": " << meta.T << ",\n"
      << "  \"random_seed\": " << meta.seed << ",\n"
      << "  \"generation_interval\": " << interval << ",\n"
      << "  \"reference_direction_count\": " << meta.H << ",\n"
      << "  \"layouts\": {\n"
      << "    \"variables\": \"row-major (N,D)\",\n"
      << "    \"objectives\": \"objective-major (M,N)\",\n"
      << "    \"constraints\": \"(N)\",\n"
      << "    \"reference_directions\": \"objective-major (M,K)\",\n"
      << "    \"bounds\": \"separate lower/upper arrays (D)\"\n"
      << "  }\n"
      << "}\n";
    if (!write_text(fs::path(root_) / "metadata.json", m.str(), err)) return set_error(MOEA_ERR_CUDA, "%s", err.c_str());

    MOEA_CUDA_TRY(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
    MOEA_CUDA_TRY(cudaEventCreateWithFlags(&ready_, cudaEventDisableTiming));
    MOEA_CUDA_TRY(cudaEventCreateWithFlags(&copied_, cudaEventDisableTiming));
    const size_t N = meta.N, D = meta.D, M = meta.M, H = meta.H;
    auto r16 = [](size_t b) { return (b + 15) & ~size_t(15); };
    const size_t bytes = r16(sizeof(unsigned long long)) + r16(sizeof(float) * N * D) + r16(sizeof(float) * M * N) +
                         r16(sizeof(float) * N) + r16(sizeof(float) * M * H) + r16(sizeof(float) * M) +
                         r16(sizeof(int) * N) + r16(sizeof(int));
    for (auto& s : slots_) {
        s = new Slot();
        s->owner = this;
        MOEA_CUDA_TRY(cudaMallocHost((void**)&s->host, bytes));
        MOEA_CUDA_TRY(cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming));
        char* p = s->host;
        auto take = [&](size_t b) { char* q = p; p += r16(b); return q; };
        s->offset = reinterpret_cast<unsigned long long*>(take(sizeof(unsigned long long)));
        s->vars = reinterpret_cast<float*>(take(sizeof(float) * N * D));
        s->objs = reinterpret_cast<float*>(take(sizeof(float) * M * N));
        s->cv = reinterpret_cast<float*>(take(sizeof(float) * N));
        s->refs = reinterpret_cast<float*>(take(sizeof(float) * M * H));
        s->ideal = reinterpret_cast<float*>(take(sizeof(float) * M));
        s->aux = reinterpret_cast<int*>(take(sizeof(int) * N));
        s->active = reinterpret_cast<int*>(take(sizeof(int)));
    }
    return MOEA_OK;
}

// Runs on the side stream's host-function thread: no CUDA calls here.
void CUDART_CB SnapshotWriter::write_slot(void* user)
{
    Slot* s = static_cast<Slot*>(user);
    SnapshotWriter* w = s->owner;
    const SnapshotSave& in = s->info;
    const SnapshotMeta& meta = w->meta_;
    const size_t N = meta.N, D = meta.D, M = meta.M, H = meta.H;
    const int active = in.d_active ? *s->active : in.active;
    std::string err;
    const fs::path dir = generation_directory(w->root_, in.generation);
    std::error_code ec;
    fs::create_directories(dir, ec);
    bool ok = !ec;
    if (!ok) err = "Cannot create data directory '" + dir.string() + "': " + ec.message();
    ok = ok && write_file(dir / "variables.bin", s->vars, sizeof(float) * N * D, err);
    ok = ok && write_file(dir / "objectives.bin", s->objs, sizeof(float) * M * N, err);
    ok = ok && write_file(dir / "constraints.bin", s->cv, sizeof(float) * N, err);
    if (ok && H > 0) ok = write_file(dir / "reference_directions.bin", s->refs, sizeof(float) * M * H, err);
    if (ok && in.aux_count > 0)
        ok = write_file(dir / "selector_auxiliary_indices.bin", s->aux, sizeof(int) * (size_t)in.aux_count, err);
    if (ok) {
        std::ostringstream j;
        j << "{\n"
          << "  \"generation\": " << in.generation << ",\n"
          << "  \"population_size\": " << meta.N << ",\n"
          << "  \"dimension\": " << meta.D << ",\n"
          << "  \"objective_count\": " << meta.M << ",\n"
          << "  \"active_count\": " << active << ",\n"
          << "  \"reference_direction_count\": " << meta.H << ",\n"
          << "  \"auxiliary_index_count\": " << in.aux_count << "\n"
          << "}\n";
        ok = write_text(dir / "snapshot.json", j.str(), err);
    }
    if (ok) {
        std::vector<char> buf(sizeof(ResumeHeader) + sizeof(float) * M);
        ResumeHeader h{};
        std::memcpy(h.magic, kResumeMagic, sizeof(h.magic));
        h.version = 1;
        h.N = meta.N;
        h.D = meta.D;
        h.M = meta.M;
        h.H = meta.H;
        h.generation = in.generation;
        h.active = active;
        h.last_prepared_target = in.last_prepared_target;
        h.ideal_ready = in.ideal_ready;
        h.epoch = in.epoch;
        h.niching_offset = *s->offset;
        std::memcpy(buf.data(), &h, sizeof(h));
        std::memcpy(buf.data() + sizeof(h), s->ideal, sizeof(float) * M);
        ok = write_file(dir / "resume.bin", buf.data(), buf.size(), err);
    }
    if (!ok) {
        std::lock_guard<std::mutex> lock(w->mutex_);
        if (w->error_.empty()) w->error_ = err;
    }
}

int SnapshotWriter::save(const SnapshotSave& in, cudaStream_t compute)
{
    if (!should_save(in.generation)) return MOEA_OK;
    Slot* s = slots_[next_];
    next_ ^= 1;
    // the slot's previous snapshot must be on disk before it is reused
    if (s->busy) MOEA_CUDA_TRY(cudaEventSynchronize(s->done));
    s->info = in;
    const size_t N = meta_.N, D = meta_.D, M = meta_.M, H = meta_.H;
    MOEA_CUDA_TRY(cudaEventRecord(ready_, compute));
    MOEA_CUDA_TRY(cudaStreamWaitEvent(side_, ready_, 0));
    MOEA_CUDA_TRY(cudaMemcpyAsync(s->vars, in.vars, sizeof(float) * N * D, cudaMemcpyDeviceToHost, side_));
    MOEA_CUDA_TRY(cudaMemcpyAsync(s->objs, in.objs, sizeof(float) * M * N, cudaMemcpyDeviceToHost, side_));
    MOEA_CUDA_TRY(cudaMemcpyAsync(s->cv, in.cv, sizeof(float) * N, cudaMemcpyDeviceToHost, side_));
    if (H > 0 && in.refs)
        MOEA_CUDA_TRY(cudaMemcpyAsync(s->refs, in.refs, sizeof(float) * M * H, cudaMemcpyDeviceToHost, side_));
    if (in.aux_count > 0)
        MOEA_CUDA_TRY(cudaMemcpyAsync(s->aux, in.aux, sizeof(int) * (size_t)in.aux_count, cudaMemcpyDeviceToHost, side_));
    MOEA_CUDA_TRY(cudaMemcpyAsync(s->ideal, in.ideal, sizeof(float) * M, cudaMemcpyDeviceToHost, side_));
    MOEA_CUDA_TRY(cudaMemcpyAsync(s->offset, in.offset, sizeof(unsigned long long), cudaMemcpyDeviceToHost, side_));
    if (in.d_active) MOEA_CUDA_TRY(cudaMemcpyAsync(s->active, in.d_active, sizeof(int), cudaMemcpyDeviceToHost, side_));
    // the compute stream waits for the copies only, not for the files
    MOEA_CUDA_TRY(cudaEventRecord(copied_, side_));
    MOEA_CUDA_TRY(cudaStreamWaitEvent(compute, copied_, 0));
    MOEA_CUDA_TRY(cudaLaunchHostFunc(side_, &SnapshotWriter::write_slot, s));
    MOEA_CUDA_TRY(cudaEventRecord(s->done, side_));
    s->busy = true;
    return MOEA_OK;
}

int SnapshotWriter::flush()
{
    if (side_) MOEA_CUDA_TRY(cudaStreamSynchronize(side_));
    std::lock_guard<std::mutex> lock(mutex_);
    if (!error_.empty()) {
        const std::string e = error_;
        error_.clear();
        return set_error(MOEA_ERR_CUDA, "%s", e.c_str());
    }
    return MOEA_OK;
}

int load_snapshot_files(const std::string& directory, const SnapshotMeta& meta, bool need_aux, SnapshotLoad& out)
{
    const fs::path dir(directory);
    const size_t N = meta.N, D = meta.D, M = meta.M, H = meta.H;
    std::string err;
    std::vector<char> buf(sizeof(ResumeHeader) + sizeof(float) * M);
    if (!read_file(dir / "resume.bin", buf.data(), buf.size(), err))
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "snapshot: %s", err.c_str());
    ResumeHeader h;
    std::memcpy(&h, buf.data(), sizeof(h));
    if (std::memcmp(h.magic, kResumeMagic, sizeof(h.magic)) != 0 || h.version != 1)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "snapshot: resume.bin has an unknown format");
    if (h.N != meta.N || h.D != meta.D || h.M != meta.M || h.H != meta.H)
        return set_error(MOEA_ERR_INVALID_ARGUMENT,
                         "snapshot: saved N=%d D=%d M=%d K=%d, the algorithm has N=%d D=%d M=%d K=%d", h.N, h.D,
                         h.M, h.H, meta.N, meta.D, meta.M, meta.H);
    if (h.generation < 0 || h.generation > meta.T)
        return set_error(MOEA_ERR_INVALID_ARGUMENT, "snapshot: generation %d outside 0..%d", h.generation, meta.T);
    out.generation = h.generation;
    out.epoch = h.epoch;
    out.active = h.active;
    out.last_prepared_target = h.last_prepared_target;
    out.ideal_ready = h.ideal_ready;
    out.niching_offset = h.niching_offset;
    out.ideal.assign(reinterpret_cast<const float*>(buf.data() + sizeof(h)),
                     reinterpret_cast<const float*>(buf.data() + sizeof(h)) + M);
    out.vars.resize(N * D);
    out.objs.resize(M * N);
    out.cv.resize(N);
    out.refs.resize(M * H);
    bool ok = read_file(dir / "variables.bin", out.vars.data(), sizeof(float) * N * D, err) &&
              read_file(dir / "objectives.bin", out.objs.data(), sizeof(float) * M * N, err) &&
              read_file(dir / "constraints.bin", out.cv.data(), sizeof(float) * N, err) &&
              (H == 0 || read_file(dir / "reference_directions.bin", out.refs.data(), sizeof(float) * M * H, err));
    if (ok && need_aux) {
        out.aux.resize(N);
        ok = read_file(dir / "selector_auxiliary_indices.bin", out.aux.data(), sizeof(int) * N, err);
    }
    if (!ok) return set_error(MOEA_ERR_INVALID_ARGUMENT, "snapshot: %s", err.c_str());
    return MOEA_OK;
}

}  // namespace moea
