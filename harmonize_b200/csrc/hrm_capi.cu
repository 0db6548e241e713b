// hrm_capi.cu — libhrm.so: the C ABI over the B200-native runtime and its built-in specs.
//
// Each exported function catches every C++ exception and turns it into a status code plus
// a thread-local message (the original's generated shim let exceptions cross extern "C",
// harmonize/python/templates.py:3-184).
#include "../../include/harmonize.h"
#include "../../include/hrm_capi.h"
#include "capi_internal.h"
#include "specs/barrier_demo.h"
#include "specs/bfs.h"
#include "specs/collatz.h"
#include "specs/photon.h"

#include <chrono>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>

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
    virtual void set_state(const void* state, size_t size) = 0;
    virtual void set_tuning(unsigned int patience, unsigned int fill_links) = 0;
    // Teams of an AsyncProgram exec that fit on the device at once (0 for EventProgram).
    virtual size_t resident_teams() = 0;
    // Device scratch of the whole-run helpers (the start-value / source iterator), kept with
    // the instance so that cached runs allocate nothing.
    util::host::DevBuf<util::iter::AtomicIter<unsigned int>> iterator{(size_t)1};
    std::mutex run_lock;  // one whole run at a time per cached instance
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
    void set_state(const void* state, size_t size) override {
        if (size != sizeof(typename P::DeviceState)) throw std::invalid_argument("device state size mismatch");
        memcpy((void*)&inst.device_state, state, size);
    }
    size_t resident_teams() override {
        if constexpr (hrm_capi::is_async_program<P>::value) {
            return (size_t)P::resident_ctas() * P::TEAMS_PER_CTA;
        } else {
            return 0;
        }
    }
    void set_tuning(unsigned int patience, unsigned int fill_links) override {
        if constexpr (hrm_capi::is_async_program<P>::value) {
            inst.patience = patience;
            inst.fill_links = fill_links;
        }
    }
};

static_assert(sizeof(hrm_collatz_state) == sizeof(hrm_specs::CollatzState), "collatz state layout");
static_assert(sizeof(hrm_photon_state) == sizeof(hrm_specs::PhotonState), "photon state layout");
static_assert(sizeof(hrm_bfs_state) == sizeof(hrm_specs::BfsState), "bfs state layout");
static_assert(sizeof(hrm_barrier_demo_state) == sizeof(hrm_specs::BarrierDemoState), "barrier demo state layout");

template <typename STATE>
STATE state_from(const void* p, size_t n) {
    if (p == nullptr || n != sizeof(STATE)) throw std::invalid_argument("device state size mismatch");
    STATE s;
    memcpy(&s, p, sizeof(STATE));
    return s;
}

// Tuning adapter of the "lean" variants: the spec's first async function keeps rings of BIG
// links, every other function gets SMALL links, and the kernel is compiled for at least
// MIN_CTAS resident CTAs per SM (__launch_bounds__). Smaller rings for the functions that a
// batch of the first one feeds leave shared memory for more teams per SM.
template <class BASE, size_t BIG, size_t SMALL, size_t MIN_CTAS>
struct LeanRings : BASE {
    static const size_t MIN_CTAS_PER_SM = MIN_CTAS;
    template <typename Op>
    struct RING_LINKS_OF {
        static const size_t value = std::is_same<Op, typename OpAt<0, typename BASE::OpSet>::type>::value ? BIG : SMALL;
    };
};

using hrm_capi::MinCtas;

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
            case HRM_VARIANT_LEAN_T2_M10: return new ProgramImpl<AsyncProgram<LeanRings<SPEC<4, 2>, 4, 2, 10>>>(arena, s);
            case HRM_VARIANT_LEAN_T2_M11: return new ProgramImpl<AsyncProgram<LeanRings<SPEC<4, 2>, 4, 2, 11>>>(arena, s);
            case HRM_VARIANT_R4_T2_M11: return new ProgramImpl<AsyncProgram<MinCtas<SPEC<4, 2>, 11>>>(arena, s);
            case HRM_VARIANT_R4_T4_M5: return new ProgramImpl<AsyncProgram<MinCtas<SPEC<4, 4>, 5>>>(arena, s);
            case HRM_VARIANT_R3_T2_M14: return new ProgramImpl<AsyncProgram<MinCtas<SPEC<3, 2>, 14>>>(arena, s);
            default: break;
        }
    } else if (type == HRM_EVENT) {
        switch (variant) {
            case HRM_VARIANT_R2_T4:
            case HRM_VARIANT_R4_T4: return new ProgramImpl<EventProgram<SPEC<2, 4>>>(arena, s);
            case HRM_VARIANT_R4_T2:
            case HRM_VARIANT_R8_T2:
            case HRM_VARIANT_LEAN_T2_M10:
            case HRM_VARIANT_LEAN_T2_M11:
            case HRM_VARIANT_R4_T2_M11:
            case HRM_VARIANT_R3_T2_M14: return new ProgramImpl<EventProgram<SPEC<2, 2>>>(arena, s);
            case HRM_VARIANT_R4_T4_M5: return new ProgramImpl<EventProgram<SPEC<2, 4>>>(arena, s);
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
        case HRM_SPEC_BARRIER_DEMO: {
            // Barriers hold promises in the AsyncProgram arena: no EventProgram form.
            if (type != HRM_ASYNC) throw std::invalid_argument("the barrier demo runs on AsyncProgram only");
            auto s = state_from<hrm_specs::BarrierDemoState>(state, state_size);
            if (s.barrier_count == 0) throw std::invalid_argument("barrier_count must be >= 1");
            switch (variant) {
                case HRM_VARIANT_R2_T4: p = new ProgramImpl<AsyncProgram<hrm_specs::BarrierDemoSpec<2, 4>>>(arena, s); break;
                case HRM_VARIANT_R4_T4: p = new ProgramImpl<AsyncProgram<hrm_specs::BarrierDemoSpec<4, 4>>>(arena, s); break;
                default: throw std::invalid_argument("the barrier demo is built for variants R2/T4 and R4/T4");
            }
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
    hrm_capi::EventPair ev;
    ck(cudaEventRecord(ev.start, s), "cudaEventRecord");
    p->set_tuning(cfg.patience, cfg.fill_links);
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
    ck(cudaEventRecord(ev.stop, s), "cudaEventRecord");
    const float ms = ev.elapsed_ms();
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

// Device copies of the inputs and outputs of the host-buffer whole runs (hrm_*_run), kept per
// device and grown on demand, so that repeated runs allocate nothing: allocating and freeing
// tens of MB per call cost up to a second of host time in measurement. A host-buffer run
// holds its device's staging lock from upload to download.
struct Staging {
    std::mutex lock;
    std::vector<std::pair<void*, size_t>> bufs;  // slot -> (device pointer, bytes)
    template <typename T>
    T* get(size_t slot, size_t count) {
        const size_t bytes = count * sizeof(T) ? count * sizeof(T) : 16;
        if (bufs.size() <= slot) bufs.resize(slot + 1, {nullptr, 0});
        auto& b = bufs[slot];
        if (b.second < bytes) {
            if (b.first) ck(cudaFree(b.first), "cudaFree");
            b = {nullptr, 0};
            ck(cudaMalloc(&b.first, bytes), "cudaMalloc");
            b.second = bytes;
        }
        return (T*)b.first;
    }
    ~Staging() {
        for (auto& b : bufs)
            if (b.first) cudaFree(b.first);
    }
};
std::mutex g_staging_mutex;
std::map<int, std::shared_ptr<Staging>> g_staging;

// Shared ownership: hrm_release_cache drops the map's reference, and a run in progress keeps
// its staging alive until it ends.
std::shared_ptr<Staging> staging() {
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(g_staging_mutex);
    auto& s = g_staging[dev];
    if (!s) s = std::make_shared<Staging>();
    return s;
}

// Program instances of the whole-run helpers, kept per (device, spec, type, variant,
// arena) and re-initialised by every run, so that repeated runs allocate nothing.
struct CacheKey {
    int dev, spec, type, variant;
    size_t arena;
    unsigned int lane;  // concurrent runs of one configuration use instances of different lanes
    bool operator<(const CacheKey& o) const {
        return std::tie(dev, spec, type, variant, arena, lane) <
               std::tie(o.dev, o.spec, o.type, o.variant, o.arena, o.lane);
    }
};
std::mutex g_cache_mutex;
std::map<CacheKey, std::shared_ptr<ProgramBase>> g_cache;

// Shared ownership, as for staging: a run holds its instance until it ends, even if
// hrm_release_cache drops the cache's reference meanwhile.
template <typename STATE>
std::shared_ptr<ProgramBase> cached_program(int spec, int type, int variant, size_t arena, const STATE& st,
                                            unsigned int lane = 0) {
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    CacheKey key{dev, spec, type, variant, arena, lane};
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    auto it = g_cache.find(key);
    if (it == g_cache.end()) {
        it = g_cache.emplace(key, std::shared_ptr<ProgramBase>(make_program(spec, type, arena, &st, sizeof(st),
                                                                            variant))).first;
    }
    return it->second;
}

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
    hrm_specs::CollatzState st;
    st.start = start;
    st.limit = start + count;
    st.output = d_out;
    st.iterator = nullptr;
    st.leap = 1;
    size_t arena = cfg.arena ? cfg.arena : default_arena(HRM_SPEC_COLLATZ, cfg.program_type);
    std::shared_ptr<ProgramBase> p = cached_program(HRM_SPEC_COLLATZ, cfg.program_type, cfg.variant, arena, st);
    std::lock_guard<std::mutex> run(p->run_lock);
    util::iter::AtomicIter<unsigned int> host_it(start, start + count);
    ck(cudaMemcpyAsync(p->iterator.data(), &host_it, sizeof(host_it), cudaMemcpyHostToDevice, s), "iterator upload");
    st.iterator = p->iterator.data();
    p->set_state(&st, sizeof(st));
    return run_to_completion(p.get(), cfg, res);
}

// Photon walk with device-resident medium and tally (tally zeroed here), on the cached
// instance of `lane` (concurrent walks of one configuration use different lanes).
int photon_run_lane(unsigned int lane, const float* d_mu, const float* d_ab, const uint8_t* d_sp, uint32_t n,
                    uint64_t seed, uint32_t first, uint32_t count, uint64_t* d_tally, const hrm_run_config* cfg_in,
                    hrm_run_result* res) {
    hrm_run_config cfg = config_or_default(cfg_in);
    if (n < 2 || n > 1024 || (n & 1u)) return fail(HRM_EINVAL, "grid edge must be even and in [2, 1024]");
    if ((uint64_t)first + count > 0xFFFFFFFFull) return fail(HRM_EINVAL, "first + count exceeds 2^32");
    cudaStream_t s = (cudaStream_t)cfg.stream;
    const size_t slots = (size_t)n * n * n + 3u * hrm_specs::PHOTON_SPREAD;
    ck(cudaMemsetAsync(d_tally, 0, slots * sizeof(uint64_t), s), "tally clear");
    hrm_specs::PhotonState st;
    st.mu_s = d_mu;
    st.absorb = d_ab;
    st.split = d_sp;
    st.tally = (unsigned long long*)d_tally;
    st.source = nullptr;
    st.n = n;
    st.seed_lo = (uint32_t)seed;
    st.seed_hi = (uint32_t)(seed >> 32);
    st.leap = 1;
    // EventProgram launches new photons only while the move buffer is under 1/64 full:
    // splits grow a batch of photons several-fold before roulette thins it.
    st.load_limit = 0.015625f;
    size_t arena = cfg.arena ? cfg.arena : default_arena(HRM_SPEC_PHOTON, cfg.program_type);
    std::shared_ptr<ProgramBase> p = cached_program(HRM_SPEC_PHOTON, cfg.program_type, cfg.variant, arena, st, lane);
    std::lock_guard<std::mutex> run(p->run_lock);
    util::iter::AtomicIter<unsigned int> host_it(first, first + count);
    ck(cudaMemcpyAsync(p->iterator.data(), &host_it, sizeof(host_it), cudaMemcpyHostToDevice, s), "iterator upload");
    st.source = p->iterator.data();
    p->set_state(&st, sizeof(st));
    return run_to_completion(p.get(), cfg, res);
}

int photon_run(const float* d_mu, const float* d_ab, const uint8_t* d_sp, uint32_t n, uint64_t seed, uint32_t first,
               uint32_t count, uint64_t* d_tally, const hrm_run_config* cfg_in, hrm_run_result* res) {
    return photon_run_lane(0, d_mu, d_ab, d_sp, n, seed, first, count, d_tally, cfg_in, res);
}

// BFS over a device-resident CSR graph; levels initialised here.
int bfs_run(const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t nv, uint32_t root, uint32_t* d_levels,
            const hrm_run_config* cfg_in, hrm_run_result* res) {
    hrm_run_config cfg = config_or_default(cfg_in);
    if (root >= nv) return fail(HRM_EINVAL, "root out of range");
    cudaStream_t s = (cudaStream_t)cfg.stream;
    ck(cudaMemsetAsync(d_levels, 0xFF, (size_t)nv * 4u, s), "levels init");
    hrm_specs::BfsState st;
    st.rowptr = d_rowptr;
    st.col = d_col;
    st.levels = d_levels;
    st.roots = nullptr;
    st.root = root;
    st.nv = nv;
    size_t arena = cfg.arena ? cfg.arena : default_arena(HRM_SPEC_BFS, cfg.program_type);
    std::shared_ptr<ProgramBase> p = cached_program(HRM_SPEC_BFS, cfg.program_type, cfg.variant, arena, st);
    std::lock_guard<std::mutex> run(p->run_lock);
    util::iter::AtomicIter<unsigned int> host_it(0, 1);
    ck(cudaMemcpyAsync(p->iterator.data(), &host_it, sizeof(host_it), cudaMemcpyHostToDevice, s), "iterator upload");
    st.roots = p->iterator.data();
    p->set_state(&st, sizeof(st));
    return run_to_completion(p.get(), cfg, res);
}

// Remapping-barrier workload; counters and barriers are set up here, results copied out.
int barrier_demo_run(uint32_t dep, uint32_t ndep, uint32_t bar, uint32_t* counter, uint32_t* released,
                     const hrm_run_config* cfg_in, hrm_run_result* res) {
    hrm_run_config cfg = config_or_default(cfg_in);
    if (bar == 0) return fail(HRM_EINVAL, "barrier_count must be >= 1");
    if ((uint64_t)dep + ndep >= hrm_specs::BARRIER_FINAL) return fail(HRM_EINVAL, "dep + ndep too large");
    if (cfg.program_type != HRM_ASYNC) return fail(HRM_EINVAL, "the barrier demo runs on AsyncProgram only");
    cudaStream_t s = (cudaStream_t)cfg.stream;
    using Barrier = RemappingBarrier<hrm_specs::BarrierOps>;
    using Unit = UnitBarrier<hrm_specs::BarrierOps>;
    // Barrier b waits for the dependent ids congruent to b (demo.cpp:163-170).
    std::vector<Barrier> bars(bar);
    for (uint32_t b = 0; b < bar; b++) bars[b] = Barrier::blank(dep / bar + ((dep % bar) > b ? 1u : 0u));
    Unit unit(PromiseEnum<hrm_specs::BarrierOps>(Promise<hrm_specs::BarrierStep>(hrm_specs::BARRIER_FINAL)), ndep);
    DeviceArray<Barrier> dbars(bar);
    DeviceArray<Unit> dunit(1);
    DeviceArray<uint32_t> dcount(4), drel(bar);
    ck(cudaMemcpyAsync(dbars.ptr, bars.data(), sizeof(Barrier) * bar, cudaMemcpyHostToDevice, s), "barrier upload");
    ck(cudaMemcpyAsync(dunit.ptr, &unit, sizeof(Unit), cudaMemcpyHostToDevice, s), "barrier upload");
    ck(cudaMemsetAsync(dcount.ptr, 0, 16, s), "counter clear");
    ck(cudaMemsetAsync(drel.ptr, 0, (size_t)bar * 4u, s), "counter clear");
    hrm_specs::BarrierDemoState st;
    st.dep_count = dep;
    st.non_dep_count = ndep;
    st.barrier_count = bar;
    st.pad = 0;
    st.source = nullptr;
    st.counter = dcount.ptr;
    st.released = drel.ptr;
    st.barriers = dbars.ptr;
    st.unit = dunit.ptr;
    size_t arena = cfg.arena ? cfg.arena : ((size_t)1 << 18);
    std::shared_ptr<ProgramBase> p = cached_program(HRM_SPEC_BARRIER_DEMO, HRM_ASYNC, cfg.variant, arena, st);
    std::lock_guard<std::mutex> run(p->run_lock);
    util::iter::AtomicIter<unsigned int> host_it(0, dep + ndep);
    ck(cudaMemcpyAsync(p->iterator.data(), &host_it, sizeof(host_it), cudaMemcpyHostToDevice, s), "iterator upload");
    st.source = p->iterator.data();
    p->set_state(&st, sizeof(st));
    int rc = run_to_completion(p.get(), cfg, res);
    if (rc != HRM_OK) return rc;
    ck(cudaMemcpyAsync(counter, dcount.ptr, 16, cudaMemcpyDeviceToHost, s), "counter download");
    ck(cudaMemcpyAsync(released, drel.ptr, (size_t)bar * 4u, cudaMemcpyDeviceToHost, s), "counter download");
    ck(cudaStreamSynchronize(s), "counter download");
    return HRM_OK;
}

}  // namespace

struct hrm_program {
    ProgramBase* impl;
};

int hrm_capi::set_error(int code, const std::string& msg) { return fail(code, msg); }

hrm_capi::CtaFootprint hrm_capi::photon_cta_footprint(int variant) {
    if (variant != HRM_VARIANT_R4_T4_M5) throw std::invalid_argument("photon_cta_footprint: variant not supported");
    using P = AsyncProgram<MinCtas<hrm_specs::PhotonSpec<4, 4>, 5>>;
    P::resident_ctas();  // opts the kernel into its dynamic shared memory
    cudaFuncAttributes fa;
    ck(cudaFuncGetAttributes(&fa, hrm_rt::async_exec_kernel<P>), "kernel attributes");
    CtaFootprint f;
    f.regs_per_thread = (unsigned int)fa.numRegs;
    f.threads = P::CTA_THREADS;
    f.smem = fa.sharedSizeBytes + P::SMEM_BYTES;
    return f;
}

unsigned int hrm_capi::ctas_beside(const CtaFootprint& a, unsigned int a_ctas, const CtaFootprint& b) {
    int dev = 0, smem_sm = 0, reserved = 0, regs_sm = 0, threads_sm = 0, blocks_sm = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev), "attribute");
    ck(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev), "attribute");
    ck(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev), "attribute");
    ck(cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev), "attribute");
    ck(cudaDeviceGetAttribute(&blocks_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev), "attribute");
    SmLimits sm;
    sm.smem = (size_t)smem_sm;
    sm.reserved = (size_t)reserved;
    sm.regs = (size_t)regs_sm;
    sm.threads = (size_t)threads_sm;
    sm.blocks = (unsigned int)blocks_sm;
    return ctas_beside(a, a_ctas, b, sm);
}

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

// Forgets the kept device addresses of the no-allocation scratch area (defined below).
void noalloc_forget_addresses();

int hrm_capi::photon_walk_lane(unsigned int lane, const float* d_mu_s, const float* d_absorb, const uint8_t* d_split,
                               uint32_t n, uint64_t seed, uint32_t first, uint32_t count, uint64_t* d_tally,
                               const hrm_run_config* cfg, hrm_run_result* res) {
    if (!d_mu_s || !d_absorb || !d_split || !d_tally) return fail(HRM_EINVAL, "NULL buffer");
    HRM_GUARD(return photon_run_lane(lane, d_mu_s, d_absorb, d_split, n, seed, first, count, d_tally, cfg, res);)
}

size_t hrm_capi::photon_resident_teams(int variant) {
    hrm_specs::PhotonState st;
    memset(&st, 0, sizeof(st));
    std::shared_ptr<ProgramBase> p =
        cached_program(HRM_SPEC_PHOTON, HRM_ASYNC, variant, default_arena(HRM_SPEC_PHOTON, HRM_ASYNC), st);
    return p->resident_teams();
}

extern "C" {

const char* hrm_last_error(void) { return g_last_error.c_str(); }

int hrm_set_device(int device) {
    HRM_GUARD(ck(cudaSetDevice(device), "cudaSetDevice"); return HRM_OK;)
}

int hrm_device_sync(void) {
    HRM_GUARD(ck(cudaDeviceSynchronize(), "cudaDeviceSynchronize"); return HRM_OK;)
}

int hrm_release_cache(void) {
    HRM_GUARD({
        noalloc_forget_addresses();
        {
            std::lock_guard<std::mutex> lock(g_cache_mutex);
            g_cache.clear();
        }
        std::lock_guard<std::mutex> lock(g_staging_mutex);
        g_staging.clear();
        return HRM_OK;
    })
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

int hrm_program_set_state(hrm_program* prog, const void* device_state, size_t state_size) {
    if (prog == nullptr || device_state == nullptr) return fail(HRM_EINVAL, "program or state is NULL");
    HRM_GUARD({
        prog->impl->set_state(device_state, state_size);
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
        std::shared_ptr<Staging> st_ref = staging();
        Staging& st = *st_ref;
        std::lock_guard<std::mutex> staged(st.lock);
        uint32_t* d = st.get<uint32_t>(0, count);
        int rc = collatz_run(start, count, d, &cfg, res);
        if (rc != HRM_OK) return rc;
        ck(cudaMemcpyAsync(out, d, (size_t)count * 4u, cudaMemcpyDeviceToHost, s), "output download");
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
        std::shared_ptr<Staging> st_ref = staging();
        Staging& st = *st_ref;
        std::lock_guard<std::mutex> staged(st.lock);
        float* dm = st.get<float>(0, nvox);
        float* da = st.get<float>(1, nvox);
        uint8_t* dsp = st.get<uint8_t>(2, nvox);
        uint64_t* dt = st.get<uint64_t>(3, slots);
        ck(cudaMemcpyAsync(dm, mu_s, nvox * 4u, cudaMemcpyHostToDevice, s), "medium upload");
        ck(cudaMemcpyAsync(da, absorb, nvox * 4u, cudaMemcpyHostToDevice, s), "medium upload");
        ck(cudaMemcpyAsync(dsp, split, nvox, cudaMemcpyHostToDevice, s), "medium upload");
        int rc = photon_run(dm, da, dsp, n, seed, first, count, dt, &cfg, res);
        if (rc != HRM_OK) return rc;
        ck(cudaMemcpyAsync(tally, dt, slots * 8u, cudaMemcpyDeviceToHost, s), "tally download");
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
        std::shared_ptr<Staging> st_ref = staging();
        Staging& st = *st_ref;
        std::lock_guard<std::mutex> staged(st.lock);
        uint32_t* drp = st.get<uint32_t>(0, (size_t)nv + 1);
        uint32_t* dcol = st.get<uint32_t>(1, ne ? ne : 1);
        uint32_t* dlev = st.get<uint32_t>(2, nv);
        ck(cudaMemcpyAsync(drp, rowptr, ((size_t)nv + 1) * 4u, cudaMemcpyHostToDevice, s), "graph upload");
        if (ne) ck(cudaMemcpyAsync(dcol, col, ne * 4u, cudaMemcpyHostToDevice, s), "graph upload");
        int rc = bfs_run(drp, dcol, nv, root, dlev, &cfg, res);
        if (rc != HRM_OK) return rc;
        ck(cudaMemcpyAsync(levels, dlev, (size_t)nv * 4u, cudaMemcpyDeviceToHost, s), "levels download");
        ck(cudaStreamSynchronize(s), "levels download");
        return HRM_OK;
    })
}

int hrm_barrier_demo_run(uint32_t dep_count, uint32_t non_dep_count, uint32_t barrier_count, uint32_t* counter,
                         uint32_t* released, const hrm_run_config* cfg, hrm_run_result* res) {
    if (!counter || !released) return fail(HRM_EINVAL, "NULL buffer");
    HRM_GUARD(return barrier_demo_run(dep_count, non_dep_count, barrier_count, counter, released, cfg, res);)
}

}  // extern "C"

// =======================================================================================
// hrm_collatz_run_device_noalloc: a Collatz whole run that allocates no device memory.
//
// Why it exists: some callers cannot call cudaMalloc at the moment they want to run the
// program. Examples: plug-in hosts that hand out only buffers registered ahead of time, and
// services that forbid allocation after start-up to keep their memory use fixed. Every
// other entry point here builds a program instance with cudaMalloc (arena, queues, control
// block); this one runs the same AsyncProgram<CollatzSpec<2,4>> kernels over a scratch
// area compiled into the library.
//
// The scratch area is the file-scope array g_noalloc_scratch (about 2.2 MiB); every GPU
// that loads this library holds it until the process exits. It caps the runtime arena at
// HRM_NOALLOC_MAX_ARENA_LINKS links of 32 promises: larger requests are rejected, and a run
// whose promises in flight outgrow it stops with ARENA_EXHAUSTED (HRM_EDEVICE).
//
// In host code the name g_noalloc_scratch is a host-side stand-in, not a device address:
// a kernel handed it would fault or, where the GPU can reach host memory, silently use the
// wrong memory. So the first call on each device, with that device current, looks up the
// device address once with cudaGetSymbolAddress and keeps it; make that first call before
// any stream capture starts. A device reset unloads the module and so invalidates the kept
// address: hrm_release_cache() forgets it, and the next call looks it up again. The run
// itself waits on the host for each exec (it reads the flags back to decide whether to
// launch another) and reads the statistics back with a synchronous copy at the end.
//
// All calls share the one array, which keeps the previous call's contents; each call
// rewrites everything the run needs initialised. Calls that overlap on the GPU (several host
// threads, or several streams) use the same scratch and race: serialise them.
// =======================================================================================
namespace {

using NoAllocProgram = AsyncProgram<hrm_specs::CollatzSpec<2, 4>>;

constexpr size_t NA_LINKS = HRM_NOALLOC_MAX_ARENA_LINKS;  // a power of two: also the ring capacity
static_assert((NA_LINKS & (NA_LINKS - 1)) == 0, "no-allocation arena must be a power of two");
constexpr size_t NA_FN = NoAllocProgram::FN;
constexpr size_t NA_LINK_WORDS = NoAllocProgram::LINK_WORDS;

// Layout of the scratch area: byte offsets, each 256-byte aligned.
constexpr size_t na_align(size_t x) { return (x + 255u) & ~(size_t)255u; }
constexpr size_t NA_OFF_CONTROL = 0;
constexpr size_t NA_OFF_HEADS = na_align(NA_OFF_CONTROL + sizeof(hrm_rt::RuntimeControl));
constexpr size_t NA_OFF_STATS = na_align(NA_OFF_HEADS + sizeof(hrm_rt::RingHead) * (NA_FN + 1));
constexpr size_t NA_OFF_ITER = na_align(NA_OFF_STATS + sizeof(unsigned long long) * hrm_rt::STAT_COUNT);
constexpr size_t NA_OFF_SLOTS = na_align(NA_OFF_ITER + sizeof(util::iter::AtomicIter<unsigned int>));
constexpr size_t NA_OFF_META = na_align(NA_OFF_SLOTS + sizeof(unsigned long long) * (NA_FN + 1) * NA_LINKS);
constexpr size_t NA_OFF_WORDS = na_align(NA_OFF_META + sizeof(unsigned int) * 2u * NA_LINKS);
constexpr size_t NA_SCRATCH_BYTES = na_align(NA_OFF_WORDS + sizeof(unsigned int) * NA_LINK_WORDS * 32u * NA_LINKS);

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

// Device address of g_noalloc_scratch, looked up once per device.
constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
unsigned char* g_na_address[NA_MAX_DEVICES] = {};

unsigned char* noalloc_scratch_address() {
    int dev = -1;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= NA_MAX_DEVICES) throw std::invalid_argument("device index beyond the supported 64");
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (g_na_address[dev] == nullptr) {
        void* p = nullptr;
        ck(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-allocation scratch)");
        if (p == nullptr) throw std::runtime_error("cudaGetSymbolAddress returned NULL for the scratch area");
        g_na_address[dev] = (unsigned char*)p;
    }
    return g_na_address[dev];
}

}  // namespace

void noalloc_forget_addresses() {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    for (auto& a : g_na_address) a = nullptr;
}

namespace {

// Sets the start-value iterator that lives in the scratch area.
__global__ void noalloc_iterator_kernel(util::iter::AtomicIter<unsigned int>* it, unsigned int start,
                                        unsigned int limit) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        it->value = start;
        it->limit = limit;
    }
}

int collatz_run_noalloc(uint32_t start, uint32_t count, uint32_t* d_out, const hrm_run_config* cfg_in,
                        hrm_run_result* res) {
    hrm_run_config cfg = config_or_default(cfg_in);
    if ((uint64_t)start + count > 0xFFFFFFFFull) return fail(HRM_EINVAL, "start + count exceeds 2^32");
    if (cfg.program_type != HRM_ASYNC) return fail(HRM_EINVAL, "the no-allocation entry point runs AsyncProgram only");
    if (cfg.variant != 0) return fail(HRM_EINVAL, "the no-allocation entry point runs tuning variant 0 only");
    size_t arena = cfg.arena ? cfg.arena : NA_LINKS;
    if (arena > NA_LINKS) {
        return fail(HRM_EINVAL, "requested arena of " + std::to_string(arena) +
                                    " links exceeds the no-allocation maximum of " + std::to_string(NA_LINKS) +
                                    " links");
    }
    unsigned char* base = noalloc_scratch_address();
    cudaStream_t s = (cudaStream_t)cfg.stream;

    NoAllocProgram::DeviceContext ctx;
    ctx.ctl = (hrm_rt::RuntimeControl*)(base + NA_OFF_CONTROL);
    ctx.rings.heads = (hrm_rt::RingHead*)(base + NA_OFF_HEADS);
    ctx.rings.slots = (unsigned long long*)(base + NA_OFF_SLOTS);
    ctx.rings.mask = (unsigned int)NA_LINKS - 1u;
    ctx.link_words = (unsigned int*)(base + NA_OFF_WORDS);
    ctx.link_meta = (unsigned int*)(base + NA_OFF_META);
    ctx.stats = (unsigned long long*)(base + NA_OFF_STATS);
    ctx.arena_links = (unsigned int)arena;
    NoAllocProgram::set_tunables(ctx, cfg.patience, cfg.fill_links);
    auto* it = (util::iter::AtomicIter<unsigned int>*)(base + NA_OFF_ITER);

    hrm_specs::CollatzState st;
    st.start = start;
    st.limit = start + count;
    st.output = d_out;
    st.iterator = it;
    st.leap = 1;

    size_t groups = cfg.groups ? cfg.groups : (size_t)1 << 30;
    size_t cycles = cfg.cycles ? cfg.cycles : ((size_t)1 << 24);
    size_t max_execs = cfg.max_execs ? cfg.max_execs : 4096;
    unsigned int ctas = NoAllocProgram::ctas_for(groups);
    unsigned int cyc = cycles > 0xFFFFFFFFull ? 0xFFFFFFFFu : (unsigned int)cycles;

    auto t0 = std::chrono::steady_clock::now();
    // The init kernel rewrites every ring slot, ring head, control word and statistic, so
    // nothing the previous call left behind reaches this run.
    noalloc_iterator_kernel<<<1, 32, 0, s>>>(it, start, start + count);
    ck(cudaGetLastError(), "iterator launch");
    hrm_rt::async_init_kernel<NoAllocProgram><<<148, 256, 0, s>>>(ctx);
    ck(cudaGetLastError(), "init launch");
    size_t execs = 0;
    bool done = false;
    unsigned int flags = 0;
    while (execs < max_execs) {
        hrm_rt::async_prep_kernel<NoAllocProgram><<<1, 32, 0, s>>>(ctx, ctas * NoAllocProgram::TEAMS_PER_CTA);
        hrm_rt::async_exec_kernel<NoAllocProgram>
            <<<ctas, NoAllocProgram::CTA_THREADS, NoAllocProgram::SMEM_BYTES, s>>>(ctx, st, cyc);
        ck(cudaGetLastError(), "exec launch");
        execs++;
        ck(cudaMemcpyAsync(&flags, &ctx.ctl->flags, sizeof(flags), cudaMemcpyDeviceToHost, s), "flags read");
        ck(cudaStreamSynchronize(s), "exec");
        if (flags & hrm_rt::ERROR_MASK) break;
        if (flags & hrm_rt::COMPLETION_FLAG) {
            done = true;
            break;
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    if (res) {
        unsigned long long st_host[hrm_rt::STAT_COUNT];
        ck(cudaMemcpy(st_host, ctx.stats, sizeof(st_host), cudaMemcpyDeviceToHost), "stats read");
        res->flags = flags;
        res->execs = (uint32_t)execs;
        for (int i = 0; i < HRM_STAT_COUNT; i++) res->stats[i] = st_host[i];
        res->device_ms = (float)std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    if (flags & hrm_rt::ERROR_MASK) {
        try {
            hrm_rt::throw_flags(flags);
        } catch (std::runtime_error& e) {
            return fail(HRM_EDEVICE, e.what());
        }
    }
    if (!done) return fail(HRM_EINCOMPLETE, "run did not complete within max_execs exec calls");
    return HRM_OK;
}

}  // namespace

extern "C" int hrm_collatz_run_device_noalloc(uint32_t start, uint32_t count, uint32_t* d_out_steps,
                                              const hrm_run_config* cfg, hrm_run_result* res) {
    if (d_out_steps == nullptr && count != 0) return fail(HRM_EINVAL, "output is NULL");
    HRM_GUARD(return collatz_run_noalloc(start, count, d_out_steps, cfg, res);)
}
