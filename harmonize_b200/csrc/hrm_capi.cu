// hrm_capi.cu — libhrm.so: the C ABI over the B200-native runtime and its built-in specs.
//
// Each exported function catches every C++ exception and turns it into a status code plus
// a thread-local message (the original's generated shim let exceptions cross extern "C",
// harmonize/python/templates.py:3-184).
#include "../../include/harmonize.h"
#include "../../include/hrm_capi.h"
#include "specs/collatz.h"

#include <mutex>
#include <string>

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

struct DeviceFlagError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Type-erased program instance.
struct ProgramBase {
    int spec = -1;
    int type = -1;
    virtual ~ProgramBase() {}
    virtual void init(size_t groups, cudaStream_t s) = 0;
    virtual void exec(size_t groups, size_t n, cudaStream_t s) = 0;
    virtual unsigned int flags() = 0;
    virtual bool complete() = 0;
    virtual void clear_flags() = 0;
    virtual std::vector<unsigned long long> stats() = 0;
    virtual std::vector<unsigned int> overview() = 0;
};

template <typename P>
struct ProgramImpl : ProgramBase {
    typename P::Instance inst;
    ProgramImpl(size_t arena, const typename P::DeviceState& ds) : inst(arena, ds) {}
    void init(size_t groups, cudaStream_t s) override { P::launch_init(inst, groups, s); }
    void exec(size_t groups, size_t n, cudaStream_t s) override { P::launch_exec(inst, groups, n, s); }
    unsigned int flags() override { return inst.flags(); }
    bool complete() override {
        try {
            return inst.complete();
        } catch (std::runtime_error& e) {
            throw DeviceFlagError(e.what());
        }
    }
    void clear_flags() override { inst.clear_flags(); }
    std::vector<unsigned long long> stats() override { return inst.read_stats(); }
    std::vector<unsigned int> overview() override { return inst.overview(); }
};

using CollatzAsync = AsyncProgram<hrm_specs::CollatzSpec<>>;
using CollatzEvent = EventProgram<hrm_specs::CollatzSpec<>>;

static_assert(sizeof(hrm_collatz_state) == sizeof(hrm_specs::CollatzState), "collatz state layout");

template <typename STATE>
STATE state_from(const void* p, size_t n) {
    if (p == nullptr || n != sizeof(STATE)) throw std::invalid_argument("device state size mismatch");
    STATE s;
    memcpy(&s, p, sizeof(STATE));
    return s;
}

ProgramBase* make_program(int spec, int type, size_t arena, const void* state, size_t state_size) {
    ProgramBase* p = nullptr;
    switch (spec) {
        case HRM_SPEC_COLLATZ: {
            auto s = state_from<hrm_specs::CollatzState>(state, state_size);
            if (s.leap == 0) s.leap = 1;
            if (type == HRM_ASYNC) p = new ProgramImpl<CollatzAsync>(arena, s);
            else if (type == HRM_EVENT) p = new ProgramImpl<CollatzEvent>(arena, s);
            break;
        }
        default:
            break;
    }
    if (p == nullptr) throw std::invalid_argument("unknown spec or program type");
    p->spec = spec;
    p->type = type;
    return p;
}

size_t default_arena(int spec, int type) {
    if (type == HRM_EVENT) return spec == HRM_SPEC_COLLATZ ? (1u << 20) : (1u << 22);
    return 1u << 18;
}

// Runs an instance to completion: init, then exec until complete or the budget ends.
int run_to_completion(ProgramBase* p, const hrm_run_config& cfg, hrm_run_result* res) {
    cudaStream_t s = (cudaStream_t)cfg.stream;
    size_t groups = cfg.groups ? cfg.groups : (size_t)1 << 30;
    size_t n = (p->type == HRM_ASYNC) ? (cfg.cycles ? cfg.cycles : ((size_t)1 << 24)) : (cfg.chunk ? cfg.chunk : 1);
    size_t max_execs = cfg.max_execs ? cfg.max_execs : 4096;
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    ck(cudaEventRecord(e0, s), "cudaEventRecord");
    p->init(groups, s);
    ck(cudaGetLastError(), "init launch");
    size_t execs = 0;
    bool done = false;
    int status = HRM_OK;
    try {
        while (execs < max_execs) {
            p->exec(groups, n, s);
            ck(cudaGetLastError(), "exec launch");
            execs++;
            ck(cudaStreamSynchronize(s), "exec");
            if (p->complete()) {
                done = true;
                break;
            }
        }
    } catch (DeviceFlagError& e) {
        status = fail(HRM_EDEVICE, e.what());
    }
    ck(cudaEventRecord(e1, s), "cudaEventRecord");
    ck(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (res) {
        res->flags = p->flags();
        res->execs = (uint32_t)execs;
        std::vector<unsigned long long> st = p->stats();
        for (int i = 0; i < HRM_STAT_COUNT; i++) res->stats[i] = st[i];
        res->device_ms = ms;
    }
    if (status != HRM_OK) return status;
    if (!done) return fail(HRM_EINCOMPLETE, "run did not complete within max_execs exec calls");
    return HRM_OK;
}

template <typename T>
struct DeviceArray {
    T* ptr = nullptr;
    explicit DeviceArray(size_t n) {
        if (n) ck(cudaMalloc((void**)&ptr, n * sizeof(T)), "cudaMalloc");
    }
    ~DeviceArray() {
        if (ptr) cudaFree(ptr);
    }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
};

hrm_run_config config_or_default(const hrm_run_config* cfg) {
    hrm_run_config c;
    memset(&c, 0, sizeof(c));
    if (cfg) c = *cfg;
    return c;
}

int collatz_run(uint32_t start, uint32_t count, uint32_t* d_out, const hrm_run_config* cfg_in, hrm_run_result* res) {
    hrm_run_config cfg = config_or_default(cfg_in);
    if ((uint64_t)start + count > 0xFFFFFFFFull) return fail(HRM_EINVAL, "start + count exceeds 2^32");
    cudaStream_t s = (cudaStream_t)cfg.stream;
    DeviceArray<util::iter::AtomicIter<unsigned int>> it(1);
    util::iter::AtomicIter<unsigned int> host_it(start, start + count);
    ck(cudaMemcpyAsync(it.ptr, &host_it, sizeof(host_it), cudaMemcpyHostToDevice, s), "iterator upload");
    hrm_specs::CollatzState st;
    st.start = start;
    st.limit = start + count;
    st.output = d_out;
    st.iterator = it.ptr;
    st.leap = 1;
    size_t arena = cfg.arena ? cfg.arena : default_arena(HRM_SPEC_COLLATZ, cfg.program_type);
    std::unique_ptr<ProgramBase> p(make_program(HRM_SPEC_COLLATZ, cfg.program_type, arena, &st, sizeof(st)));
    return run_to_completion(p.get(), cfg, res);
}

}  // namespace

struct hrm_program {
    ProgramBase* impl;
};

#define HRM_GUARD(body)                                          \
    try {                                                        \
        body                                                     \
    } catch (std::invalid_argument & e) {                        \
        return fail(HRM_EINVAL, e.what());                       \
    } catch (DeviceFlagError & e) {                              \
        return fail(HRM_EDEVICE, e.what());                      \
    } catch (std::bad_alloc & e) {                               \
        return fail(HRM_ENOMEM, e.what());                       \
    } catch (std::exception & e) {                               \
        return fail(HRM_ECUDA, e.what());                        \
    }

extern "C" {

const char* hrm_last_error(void) { return g_last_error.c_str(); }

int hrm_set_device(int device) {
    HRM_GUARD(ck(cudaSetDevice(device), "cudaSetDevice"); return HRM_OK;)
}

int hrm_device_sync(void) {
    HRM_GUARD(ck(cudaDeviceSynchronize(), "cudaDeviceSynchronize"); return HRM_OK;)
}

int hrm_program_create(int spec, int program_type, size_t arena_or_io, const void* device_state, size_t state_size,
                       hrm_program** out) {
    if (out == nullptr) return fail(HRM_EINVAL, "out is NULL");
    HRM_GUARD({
        size_t arena = arena_or_io ? arena_or_io : default_arena(spec, program_type);
        ProgramBase* p = make_program(spec, program_type, arena, device_state, state_size);
        *out = new hrm_program{p};
        return HRM_OK;
    })
}

int hrm_program_destroy(hrm_program* prog) {
    if (prog == nullptr) return HRM_OK;
    HRM_GUARD({
        delete prog->impl;
        delete prog;
        return HRM_OK;
    })
}

int hrm_program_init(hrm_program* prog, size_t groups, void* stream) {
    if (prog == nullptr) return fail(HRM_EINVAL, "program is NULL");
    HRM_GUARD({
        prog->impl->init(groups, (cudaStream_t)stream);
        ck(cudaGetLastError(), "init launch");
        return HRM_OK;
    })
}

int hrm_program_exec(hrm_program* prog, size_t groups, size_t n, void* stream) {
    if (prog == nullptr) return fail(HRM_EINVAL, "program is NULL");
    HRM_GUARD({
        prog->impl->exec(groups, n, (cudaStream_t)stream);
        ck(cudaGetLastError(), "exec launch");
        return HRM_OK;
    })
}

int hrm_program_complete(hrm_program* prog, int* out) {
    if (prog == nullptr || out == nullptr) return fail(HRM_EINVAL, "NULL argument");
    HRM_GUARD({
        *out = prog->impl->complete() ? 1 : 0;
        return HRM_OK;
    })
}

int hrm_program_flags(hrm_program* prog, uint32_t* out) {
    if (prog == nullptr || out == nullptr) return fail(HRM_EINVAL, "NULL argument");
    HRM_GUARD({
        *out = prog->impl->flags();
        return HRM_OK;
    })
}

int hrm_program_clear_flags(hrm_program* prog) {
    if (prog == nullptr) return fail(HRM_EINVAL, "program is NULL");
    HRM_GUARD({
        prog->impl->clear_flags();
        return HRM_OK;
    })
}

int hrm_program_stats(hrm_program* prog, uint64_t* out, size_t n) {
    if (prog == nullptr || out == nullptr) return fail(HRM_EINVAL, "NULL argument");
    HRM_GUARD({
        std::vector<unsigned long long> st = prog->impl->stats();
        for (size_t i = 0; i < n && i < st.size(); i++) out[i] = st[i];
        return HRM_OK;
    })
}

int hrm_program_overview(hrm_program* prog, uint32_t* out, size_t n, size_t* written) {
    if (prog == nullptr || out == nullptr) return fail(HRM_EINVAL, "NULL argument");
    HRM_GUARD({
        std::vector<unsigned int> v = prog->impl->overview();
        size_t k = 0;
        for (; k < n && k < v.size(); k++) out[k] = v[k];
        if (written) *written = v.size();
        return HRM_OK;
    })
}

int hrm_collatz_run_device(uint32_t start, uint32_t count, uint32_t* d_out, const hrm_run_config* cfg,
                           hrm_run_result* res) {
    if (d_out == nullptr && count != 0) return fail(HRM_EINVAL, "output is NULL");
    HRM_GUARD(return collatz_run(start, count, d_out, cfg, res);)
}

int hrm_collatz_run(uint32_t start, uint32_t count, uint32_t* out, const hrm_run_config* cfg_in,
                    hrm_run_result* res) {
    if (out == nullptr && count != 0) return fail(HRM_EINVAL, "output is NULL");
    HRM_GUARD({
        hrm_run_config cfg = config_or_default(cfg_in);
        cudaStream_t s = (cudaStream_t)cfg.stream;
        DeviceArray<uint32_t> d(count);
        int rc = collatz_run(start, count, d.ptr, &cfg, res);
        if (rc != HRM_OK) return rc;
        ck(cudaMemcpyAsync(out, d.ptr, (size_t)count * 4u, cudaMemcpyDeviceToHost, s), "output download");
        ck(cudaStreamSynchronize(s), "output download");
        return HRM_OK;
    })
}

}  // extern "C"
