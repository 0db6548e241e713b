// hrm_capi.cu — libhrm.so: the C ABI over the B200-native runtime and its built-in specs.
//
// Each exported function catches every C++ exception and turns it into a status code plus
// a thread-local message (the original's generated shim let exceptions cross extern "C",
// harmonize/python/templates.py:3-184).
#include "../../include/harmonize.h"
#include "../../include/hrm_capi.h"
#include "specs/bfs.h"
#include "specs/collatz.h"
#include "specs/photon.h"

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

static_assert(sizeof(hrm_collatz_state) == sizeof(hrm_specs::CollatzState), "collatz state layout");
static_assert(sizeof(hrm_photon_state) == sizeof(hrm_specs::PhotonState), "photon state layout");
static_assert(sizeof(hrm_bfs_state) == sizeof(hrm_specs::BfsState), "bfs state layout");

template <typename STATE>
STATE state_from(const void* p, size_t n) {
    if (p == nullptr || n != sizeof(STATE)) throw std::invalid_argument("device state size mismatch");
    STATE s;
    memcpy(&s, p, sizeof(STATE));
    return s;
}

// Instantiates spec SPEC<RING, TEAMS> for the chosen program type and tuning variant.
template <template <size_t, size_t> class SPEC, typename STATE>
ProgramBase* make_variant(int type, int variant, size_t arena, const STATE& s) {
    if (type == HRM_ASYNC) {
        switch (variant) {
            case HRM_VARIANT_R2_T4: return new ProgramImpl<AsyncProgram<SPEC<2, 4>>>(arena, s);
            case HRM_VARIANT_R4_T4: return new ProgramImpl<AsyncProgram<SPEC<4, 4>>>(arena, s);
            case HRM_VARIANT_R4_T2: return new ProgramImpl<AsyncProgram<SPEC<4, 2>>>(arena, s);
            case HRM_VARIANT_R8_T2: return new ProgramImpl<AsyncProgram<SPEC<8, 2>>>(arena, s);
            case HRM_VARIANT_R2_T8: return new ProgramImpl<AsyncProgram<SPEC<2, 8>>>(arena, s);
            default: break;
        }
    } else if (type == HRM_EVENT) {
        switch (variant) {
            case HRM_VARIANT_R2_T4:
            case HRM_VARIANT_R4_T4: return new ProgramImpl<EventProgram<SPEC<2, 4>>>(arena, s);
            case HRM_VARIANT_R4_T2:
            case HRM_VARIANT_R8_T2: return new ProgramImpl<EventProgram<SPEC<2, 2>>>(arena, s);
            case HRM_VARIANT_R2_T8: return new ProgramImpl<EventProgram<SPEC<2, 8>>>(arena, s);
            default: break;
        }
    }
    return nullptr;
}

ProgramBase* make_program(int spec, int type, size_t arena, const void* state, size_t state_size, int variant = 0) {
    ProgramBase* p = nullptr;
    switch (spec) {
        case HRM_SPEC_COLLATZ: {
            auto s = state_from<hrm_specs::CollatzState>(state, state_size);
            if (s.leap == 0) s.leap = 1;
            p = make_variant<hrm_specs::CollatzSpec>(type, variant, arena, s);
            break;
        }
        case HRM_SPEC_PHOTON: {
            auto s = state_from<hrm_specs::PhotonState>(state, state_size);
            if (s.leap == 0) s.leap = 1;
            p = make_variant<hrm_specs::PhotonSpec>(type, variant, arena, s);
            break;
        }
        case HRM_SPEC_BFS: {
            auto s = state_from<hrm_specs::BfsState>(state, state_size);
            p = make_variant<hrm_specs::BfsSpec>(type, variant, arena, s);
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
    if (type == HRM_EVENT) return spec == HRM_SPEC_COLLATZ ? (1u << 20) : (1u << 24);
    return spec == HRM_SPEC_COLLATZ ? (1u << 18) : (1u << 20);
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
    std::unique_ptr<ProgramBase> p(make_program(HRM_SPEC_COLLATZ, cfg.program_type, arena, &st, sizeof(st), cfg.variant));
    return run_to_completion(p.get(), cfg, res);
}

// Photon walk with device-resident medium and tally (tally zeroed here).
int photon_run(const float* d_mu, const float* d_ab, const uint8_t* d_sp, uint32_t n, uint64_t seed, uint32_t first,
               uint32_t count, uint64_t* d_tally, const hrm_run_config* cfg_in, hrm_run_result* res) {
    hrm_run_config cfg = config_or_default(cfg_in);
    if (n < 2 || n > 1024 || (n & 1u)) return fail(HRM_EINVAL, "grid edge must be even and in [2, 1024]");
    if ((uint64_t)first + count > 0xFFFFFFFFull) return fail(HRM_EINVAL, "first + count exceeds 2^32");
    cudaStream_t s = (cudaStream_t)cfg.stream;
    const size_t slots = (size_t)n * n * n + 3u * hrm_specs::PHOTON_SPREAD;
    ck(cudaMemsetAsync(d_tally, 0, slots * sizeof(uint64_t), s), "tally clear");
    DeviceArray<util::iter::AtomicIter<unsigned int>> it(1);
    util::iter::AtomicIter<unsigned int> host_it(first, first + count);
    ck(cudaMemcpyAsync(it.ptr, &host_it, sizeof(host_it), cudaMemcpyHostToDevice, s), "iterator upload");
    hrm_specs::PhotonState st;
    st.mu_s = d_mu;
    st.absorb = d_ab;
    st.split = d_sp;
    st.tally = (unsigned long long*)d_tally;
    st.source = it.ptr;
    st.n = n;
    st.seed_lo = (uint32_t)seed;
    st.seed_hi = (uint32_t)(seed >> 32);
    st.leap = 1;
    // EventProgram launches new photons only while the move buffer is under 1/64 full:
    // splits grow a batch of photons several-fold before roulette thins it.
    st.load_limit = 0.015625f;
    size_t arena = cfg.arena ? cfg.arena : default_arena(HRM_SPEC_PHOTON, cfg.program_type);
    std::unique_ptr<ProgramBase> p(make_program(HRM_SPEC_PHOTON, cfg.program_type, arena, &st, sizeof(st), cfg.variant));
    return run_to_completion(p.get(), cfg, res);
}

// BFS over a device-resident CSR graph; levels initialised here.
int bfs_run(const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t nv, uint32_t root, uint32_t* d_levels,
            const hrm_run_config* cfg_in, hrm_run_result* res) {
    hrm_run_config cfg = config_or_default(cfg_in);
    if (root >= nv) return fail(HRM_EINVAL, "root out of range");
    cudaStream_t s = (cudaStream_t)cfg.stream;
    ck(cudaMemsetAsync(d_levels, 0xFF, (size_t)nv * 4u, s), "levels init");
    DeviceArray<util::iter::AtomicIter<unsigned int>> it(1);
    util::iter::AtomicIter<unsigned int> host_it(0, 1);
    ck(cudaMemcpyAsync(it.ptr, &host_it, sizeof(host_it), cudaMemcpyHostToDevice, s), "iterator upload");
    hrm_specs::BfsState st;
    st.rowptr = d_rowptr;
    st.col = d_col;
    st.levels = d_levels;
    st.roots = it.ptr;
    st.root = root;
    st.nv = nv;
    size_t arena = cfg.arena ? cfg.arena : default_arena(HRM_SPEC_BFS, cfg.program_type);
    std::unique_ptr<ProgramBase> p(make_program(HRM_SPEC_BFS, cfg.program_type, arena, &st, sizeof(st), cfg.variant));
    return run_to_completion(p.get(), cfg, res);
}

}  // namespace

struct hrm_program {
    ProgramBase* impl;
};

#define HRM_GUARD(...)                                           \
    try {                                                        \
        __VA_ARGS__                                              \
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

int hrm_program_create_variant(int spec, int program_type, int variant, size_t arena_or_io, const void* device_state,
                               size_t state_size, hrm_program** out) {
    if (out == nullptr) return fail(HRM_EINVAL, "out is NULL");
    HRM_GUARD({
        size_t arena = arena_or_io ? arena_or_io : default_arena(spec, program_type);
        ProgramBase* p = make_program(spec, program_type, arena, device_state, state_size, variant);
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

int hrm_photon_run_device(const float* d_mu_s, const float* d_absorb, const uint8_t* d_split, uint32_t n,
                          uint64_t seed, uint32_t first, uint32_t count, uint64_t* d_tally,
                          const hrm_run_config* cfg, hrm_run_result* res) {
    if (!d_mu_s || !d_absorb || !d_split || !d_tally) return fail(HRM_EINVAL, "NULL buffer");
    HRM_GUARD(return photon_run(d_mu_s, d_absorb, d_split, n, seed, first, count, d_tally, cfg, res);)
}

int hrm_photon_run(const float* mu_s, const float* absorb, const uint8_t* split, uint32_t n, uint64_t seed,
                   uint32_t first, uint32_t count, uint64_t* tally, const hrm_run_config* cfg_in,
                   hrm_run_result* res) {
    if (!mu_s || !absorb || !split || !tally) return fail(HRM_EINVAL, "NULL buffer");
    if (n < 2 || n > 1024) return fail(HRM_EINVAL, "grid edge out of range");
    HRM_GUARD({
        hrm_run_config cfg = config_or_default(cfg_in);
        cudaStream_t s = (cudaStream_t)cfg.stream;
        const size_t nvox = (size_t)n * n * n;
        const size_t slots = nvox + 3u * hrm_specs::PHOTON_SPREAD;
        DeviceArray<float> dm(nvox), da(nvox);
        DeviceArray<uint8_t> dsp(nvox);
        DeviceArray<uint64_t> dt(slots);
        ck(cudaMemcpyAsync(dm.ptr, mu_s, nvox * 4u, cudaMemcpyHostToDevice, s), "medium upload");
        ck(cudaMemcpyAsync(da.ptr, absorb, nvox * 4u, cudaMemcpyHostToDevice, s), "medium upload");
        ck(cudaMemcpyAsync(dsp.ptr, split, nvox, cudaMemcpyHostToDevice, s), "medium upload");
        int rc = photon_run(dm.ptr, da.ptr, dsp.ptr, n, seed, first, count, dt.ptr, &cfg, res);
        if (rc != HRM_OK) return rc;
        ck(cudaMemcpyAsync(tally, dt.ptr, slots * 8u, cudaMemcpyDeviceToHost, s), "tally download");
        ck(cudaStreamSynchronize(s), "tally download");
        return HRM_OK;
    })
}

int hrm_bfs_run_device(const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t nv, uint32_t root,
                       uint32_t* d_levels, const hrm_run_config* cfg, hrm_run_result* res) {
    if (!d_rowptr || !d_col || !d_levels) return fail(HRM_EINVAL, "NULL buffer");
    HRM_GUARD(return bfs_run(d_rowptr, d_col, nv, root, d_levels, cfg, res);)
}

int hrm_bfs_run(const uint32_t* rowptr, const uint32_t* col, uint32_t nv, uint32_t root, uint32_t* levels,
                const hrm_run_config* cfg_in, hrm_run_result* res) {
    if (!rowptr || !col || !levels) return fail(HRM_EINVAL, "NULL buffer");
    if (nv == 0) return fail(HRM_EINVAL, "empty graph");
    HRM_GUARD({
        hrm_run_config cfg = config_or_default(cfg_in);
        cudaStream_t s = (cudaStream_t)cfg.stream;
        const size_t ne = rowptr[nv];
        DeviceArray<uint32_t> drp((size_t)nv + 1), dcol(ne ? ne : 1), dlev(nv);
        ck(cudaMemcpyAsync(drp.ptr, rowptr, ((size_t)nv + 1) * 4u, cudaMemcpyHostToDevice, s), "graph upload");
        if (ne) ck(cudaMemcpyAsync(dcol.ptr, col, ne * 4u, cudaMemcpyHostToDevice, s), "graph upload");
        int rc = bfs_run(drp.ptr, dcol.ptr, nv, root, dlev.ptr, &cfg, res);
        if (rc != HRM_OK) return rc;
        ck(cudaMemcpyAsync(levels, dlev.ptr, (size_t)nv * 4u, cudaMemcpyDeviceToHost, s), "levels download");
        ck(cudaStreamSynchronize(s), "levels download");
        return HRM_OK;
    })
}

}  // extern "C"
