// Problem plugins: C++ libraries implementing IProblemEvaluator, built
// against the plugin SDK (cuda-moea_b200/sdk/include) and loaded here.
//
// The checks follow the reference's loader (python/csrc/native_problem.cpp:
// 15-37, 76-108): the registration's primitive prefix (ABI 1 and this SDK's
// build id) is checked before any C++ object of the plugin is touched;
// parameter names must be unique; a value's type is the type of the
// registered default (a float parameter also takes an integer); the
// constructed problem's ProblemInfo must repeat the requested dimension,
// objective count and bounds.  Exceptions of the plugin are caught at this
// boundary and become error messages, so no plugin-defined exception type
// outlives dlclose.
//
// The algorithm calls a plugin through its callback hooks (moea_evaluate_fn,
// moea_prepare_fn, moea_problem_reset_fn) with the handle as user pointer.
// The plugin sees a CudaContext bound to the algorithm's stream; its
// initialize() runs once, before the first evaluation.
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "cuda_moea/native/plugin.cuh"
#include "moea_b200.h"

namespace cn = cuda_moea::native;

struct moea_native_problem {
    void* handle = nullptr;
    const cn::Plugin* plugin = nullptr;
    std::unordered_map<std::string, cn::Parameter> values;  // set before create
    cuda_moea::IProblemEvaluator* instance = nullptr;
    std::unique_ptr<cuda_moea::CudaContext> cuda;
    bool initialized = false;
    int device = -1;
    cudaStream_t last_stream = nullptr;
    float* d_bounds = nullptr;  // interleaved [lb0, ub0, ...] for PopulationView::bounds
    std::vector<float> lower, upper;
};

namespace {

const char* kTypeNames[] = {"int", "float", "bool", "str", "float_list"};

std::string json_escape(const char* s)
{
    std::ostringstream out;
    out << '"';
    for (const char* c = s ? s : ""; *c; ++c) {
        switch (*c) {
        case '"': out << "\\\""; break;
        case '\\': out << "\\\\"; break;
        case '\n': out << "\\n"; break;
        case '\r': out << "\\r"; break;
        case '\t': out << "\\t"; break;
        default:
            if (static_cast<unsigned char>(*c) < 0x20) {
                char buf[8];
                std::snprintf(buf, sizeof(buf), "\\u%04x", static_cast<unsigned char>(*c));
                out << buf;
            } else {
                out << *c;
            }
        }
    }
    out << '"';
    return out.str();
}

std::string json_double(double v)
{
    if (!std::isfinite(v)) return "null";
    char buf[40];
    std::snprintf(buf, sizeof(buf), "%.17g", v);
    std::string s(buf);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";  // keep it a float in JSON
    return s;
}

std::string json_value(const cn::Parameter& p)
{
    switch (p.index()) {
    case 0: return std::to_string(std::get<std::int64_t>(p));
    case 1: return json_double(std::get<double>(p));
    case 2: return std::get<bool>(p) ? "true" : "false";
    case 3: return json_escape(std::get<std::string>(p).c_str());
    default: {
        std::string s = "[";
        const auto& v = std::get<std::vector<double>>(p);
        for (size_t i = 0; i < v.size(); ++i) s += (i ? ", " : "") + json_double(v[i]);
        return s + "]";
    }
    }
}

const cn::ParameterSpec* find_spec(const moea_native_problem* p, const char* name)
{
    if (!name) return nullptr;
    for (const auto& spec : *p->plugin->parameters)
        if (std::strcmp(spec.name, name) == 0) return &spec;
    return nullptr;
}

int set_value(moea_native_problem* p, const char* name, cn::Parameter value, int kind)
{
    if (!p || !p->plugin) return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "native problem: NULL handle");
    if (p->instance) return moea::set_error(MOEA_ERR_STATE, "native problem: parameters are fixed once created");
    const cn::ParameterSpec* spec = find_spec(p, name);
    if (!spec) return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "Unknown native problem parameter: %s", name ? name : "");
    const int want = static_cast<int>(spec->default_value.index());
    if (want == 1 && kind == 0) value = static_cast<double>(std::get<std::int64_t>(value));  // int for a float
    else if (want != kind)
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "Invalid type/value for native parameter '%s' (%s)",
                               spec->name, kTypeNames[want]);
    if (value.index() == 1 && !std::isfinite(std::get<double>(value)))
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "Invalid type/value for native parameter '%s' (not finite)",
                               spec->name);
    if (value.index() == 4)
        for (double x : std::get<std::vector<double>>(value))
            if (!std::isfinite(x))
                return moea::set_error(MOEA_ERR_INVALID_ARGUMENT,
                                       "Invalid type/value for native parameter '%s' (not finite)", spec->name);
    p->values[spec->name] = std::move(value);
    return MOEA_OK;
}

// First use on a stream: bind the context, run the plugin's initialize once
// and stage the interleaved bounds on the device.
int ensure_ready(moea_native_problem* p, cudaStream_t stream)
{
    if (!p->initialized) {
        MOEA_CUDA_TRY(cudaGetDevice(&p->device));
        const size_t D = p->lower.size();
        std::vector<float> hb(2 * D);
        for (size_t d = 0; d < D; ++d) {
            hb[2 * d] = p->lower[d];
            hb[2 * d + 1] = p->upper[d];
        }
        MOEA_CUDA_TRY(cudaMalloc((void**)&p->d_bounds, sizeof(float) * (hb.empty() ? 1 : hb.size())));
        if (!hb.empty())
            MOEA_CUDA_TRY(cudaMemcpy(p->d_bounds, hb.data(), sizeof(float) * hb.size(), cudaMemcpyHostToDevice));
        p->cuda->bind(stream, p->device, p->cuda->random_seed());
        p->instance->initialize(*p->cuda);
        p->initialized = true;
    }
    p->cuda->bind(stream, p->device, p->cuda->random_seed());
    p->last_stream = stream;
    return MOEA_OK;
}

template <class F>
int guarded(const char* what, F&& f)
{
    try {
        return f();
    } catch (const std::exception& e) {
        return moea::set_error(MOEA_ERR_CALLBACK, "native problem %s failed: %s", what, e.what());
    } catch (...) {
        return moea::set_error(MOEA_ERR_CALLBACK, "native problem %s failed with a nonstandard exception", what);
    }
}

}  // namespace

extern "C" {

moea_status moea_native_open(const char* library_path, moea_native_problem** out)
{
    if (!library_path || !out) return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "native problem: NULL argument");
    *out = nullptr;
    void* h = dlopen(library_path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return moea::set_error(MOEA_ERR_LOAD, "Cannot load native problem: %s", dlerror());
    auto entry = reinterpret_cast<cn::Entry>(dlsym(h, "cuda_moea_problem_v1"));
    if (!entry) {
        dlclose(h);
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "Missing cuda_moea_problem_v1 registration in %s",
                               library_path);
    }
    const cn::Plugin* plugin = entry();
    if (!plugin || plugin->abi != 1 || !plugin->build_id ||
        std::strcmp(plugin->build_id, CUDA_MOEA_NATIVE_BUILD_ID) != 0) {
        dlclose(h);
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT,
                               "Native problem SDK mismatch; rebuild the problem against this library's SDK (%s)",
                               CUDA_MOEA_NATIVE_BUILD_ID);
    }
    if (!plugin->name || !plugin->parameters || !plugin->create || !plugin->destroy) {
        dlclose(h);
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "Incomplete native problem registration");
    }
    std::set<std::string> names;
    for (const auto& spec : *plugin->parameters) {
        if (!spec.name || !names.insert(spec.name).second) {
            dlclose(h);
            return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "Invalid or duplicate native parameter name");
        }
    }
    auto* p = new (std::nothrow) moea_native_problem();
    if (!p) {
        dlclose(h);
        return moea::set_error(MOEA_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    p->handle = h;
    p->plugin = plugin;
    *out = p;
    return MOEA_OK;
}

void moea_native_close(moea_native_problem* p)
{
    if (!p) return;
    int previous = -1;
    if (p->initialized) {
        cudaGetDevice(&previous);
        cudaSetDevice(p->device);
        if (p->last_stream) cudaStreamSynchronize(p->last_stream);
    }
    if (p->instance) {
        try {
            p->plugin->destroy(p->instance);
        } catch (...) {
        }
    }
    // a destructor may enqueue frees: finish them before the code goes away
    if (p->initialized && p->last_stream) cudaStreamSynchronize(p->last_stream);
    if (p->d_bounds) cudaFree(p->d_bounds);
    p->cuda.reset();
    if (p->handle) dlclose(p->handle);
    if (previous >= 0) cudaSetDevice(previous);
    delete p;
}

moea_status moea_native_schema(const moea_native_problem* p, char* buf, size_t cap, size_t* needed)
{
    if (!p || !p->plugin) return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "native problem: NULL handle");
    std::ostringstream s;
    s << "{\"name\": " << json_escape(p->plugin->name) << ", \"build_id\": " << json_escape(p->plugin->build_id)
      << ", \"parameters\": {";
    bool first = true;
    for (const auto& spec : *p->plugin->parameters) {
        s << (first ? "" : ", ") << json_escape(spec.name) << ": {\"type\": \""
          << kTypeNames[spec.default_value.index()] << "\", \"default\": " << json_value(spec.default_value)
          << ", \"description\": " << json_escape(spec.description) << "}";
        first = false;
    }
    s << "}}";
    const std::string text = s.str();
    if (needed) *needed = text.size() + 1;
    if (buf && cap > 0) {
        const size_t n = text.size() < cap - 1 ? text.size() : cap - 1;
        std::memcpy(buf, text.data(), n);
        buf[n] = '\0';
        if (n < text.size()) return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "native problem: schema buffer too small");
    }
    return MOEA_OK;
}

moea_status moea_native_set_int(moea_native_problem* p, const char* name, long long value)
{
    return set_value(p, name, cn::Parameter{static_cast<std::int64_t>(value)}, 0);
}

moea_status moea_native_set_float(moea_native_problem* p, const char* name, double value)
{
    return set_value(p, name, cn::Parameter{value}, 1);
}

moea_status moea_native_set_bool(moea_native_problem* p, const char* name, int value)
{
    return set_value(p, name, cn::Parameter{value != 0}, 2);
}

moea_status moea_native_set_string(moea_native_problem* p, const char* name, const char* value)
{
    if (!value) return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "native problem: NULL string");
    return set_value(p, name, cn::Parameter{std::string(value)}, 3);
}

moea_status moea_native_set_floats(moea_native_problem* p, const char* name, const double* values, int count)
{
    if (count < 0 || (count > 0 && !values))
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "native problem: bad list");
    return set_value(p, name, cn::Parameter{std::vector<double>(values, values + count)}, 4);
}

moea_status moea_native_create(moea_native_problem* p, const char* name, int dimension, int objectives,
                               const float* h_lower, const float* h_upper)
{
    if (!p || !p->plugin) return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "native problem: NULL handle");
    if (p->instance) return moea::set_error(MOEA_ERR_STATE, "native problem: already created");
    if (!name || std::strcmp(name, p->plugin->name) != 0)
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "Library registers '%s', not '%s'", p->plugin->name,
                               name ? name : "");
    if (dimension <= 0 || objectives <= 0 || !h_lower || !h_upper)
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "native problem: dimension, objectives and bounds required");
    cn::ProblemConfig config{dimension, objectives, std::vector<float>(h_lower, h_lower + dimension),
                             std::vector<float>(h_upper, h_upper + dimension), {}};
    for (const auto& spec : *p->plugin->parameters) {
        auto it = p->values.find(spec.name);
        config.parameters.emplace(spec.name, it != p->values.end() ? it->second : spec.default_value);
    }
    // a constructor that rejects its configuration is an invalid argument
    // (python/csrc/native_problem.cpp:93-99)
    cuda_moea::IProblemEvaluator* made = nullptr;
    try {
        made = p->plugin->create(config);
    } catch (const std::exception& e) {
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "Native problem construction failed: %s", e.what());
    } catch (...) {
        return moea::set_error(MOEA_ERR_CALLBACK, "Native problem construction failed with a nonstandard exception");
    }
    if (!made) return moea::set_error(MOEA_ERR_CALLBACK, "Native problem factory returned null");
    const auto& info = made->info();
    if (info.dimension != dimension || info.objective_count != objectives || info.lower_bounds != config.lower_bounds ||
        info.upper_bounds != config.upper_bounds || info.constraint_count < 0) {
        p->plugin->destroy(made);
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT,
                               "Native ProblemInfo must match the requested dimensions and bounds");
    }
    p->instance = made;
    p->lower = config.lower_bounds;
    p->upper = config.upper_bounds;
    p->cuda.reset(new cuda_moea::CudaContext());
    return MOEA_OK;
}

moea_status moea_native_constraint_count(const moea_native_problem* p, int* out)
{
    if (!p || !p->instance || !out) return moea::set_error(MOEA_ERR_STATE, "native problem: not created");
    *out = p->instance->info().constraint_count;
    return MOEA_OK;
}

int moea_native_evaluate(void* user, const float* d_vars, float* d_objs, float* d_cv, int N, int D, int M,
                         int generation, int max_generations, void* stream)
{
    auto* p = static_cast<moea_native_problem*>(user);
    if (!p || !p->instance) return moea::set_error(MOEA_ERR_STATE, "native problem: not created");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    MOEA_TRY(guarded("initialize", [&]() -> int { return ensure_ready(p, s); }));
    cudaGetLastError();  // the plugin's launch errors only
    return guarded("evaluate", [&]() -> int {
        cuda_moea::PopulationView view{const_cast<float*>(d_vars), d_objs, d_cv, p->d_bounds, N, D, M};
        const cuda_moea::EvaluationContext context{generation, max_generations, *p->cuda};
        p->instance->evaluate(view, context, s);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return moea::set_error(MOEA_ERR_CUDA, "native problem evaluate: %s", cudaGetErrorString(e));
        return MOEA_OK;
    });
}

int moea_native_prepare(void* user, float* d_vars, float* d_objs, float* d_cv, int N, int D, int M, int generation,
                        int max_generations, void* stream, int* h_changed)
{
    auto* p = static_cast<moea_native_problem*>(user);
    if (!p || !p->instance || !h_changed) return moea::set_error(MOEA_ERR_STATE, "native problem: not created");
    *h_changed = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    MOEA_TRY(guarded("initialize", [&]() -> int { return ensure_ready(p, s); }));
    return guarded("prepare_parent", [&]() -> int {
        cuda_moea::PopulationView view{d_vars, d_objs, d_cv, p->d_bounds, N, D, M};
        const cuda_moea::EvaluationContext context{generation, max_generations, *p->cuda};
        *h_changed = p->instance->prepare_parent(view, context, s) ? 1 : 0;
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return moea::set_error(MOEA_ERR_CUDA, "native problem prepare_parent: %s", cudaGetErrorString(e));
        return MOEA_OK;
    });
}

void moea_native_reset(void* user)
{
    auto* p = static_cast<moea_native_problem*>(user);
    if (!p || !p->instance) return;
    guarded("reset", [&]() -> int {
        p->instance->reset();
        return MOEA_OK;
    });
}

}  // extern "C"
