// hrm_batch.cu — batched and plain execution of many independent jobs (libhrm.so).
//
//  * hrm_batch_run: every job of a mixed batch (Collatz ranges, photon batches, BFS) in ONE
//    persistent AsyncProgram launch over the job-multiplexing spec (specs/mix.h). The
//    launch sequence (timestamp, output preparation, init, exec) is captured once into a
//    CUDA graph per cached batch context and replayed; jobs share the per-function queues,
//    so small jobs fill warp-full batches together.
//  * hrm_plain_run: the baseline — one launch per job of a plain kernel (one thread per
//    Collatz start value, one thread per source photon walking its descendants, one CTA per
//    BFS), round-robin over a set of streams.
// Both record each job's completion time relative to the start of the call.
#include "../../include/harmonize.h"
#include "../../include/hrm_capi.h"
#include "capi_internal.h"
#include "specs/mix.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstddef>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using hrm_specs::JobRecord;
using hrm_specs::MixState;

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------------------
// Job table construction (host).
// ---------------------------------------------------------------------------------------
size_t job_sources(const hrm_job& j) { return j.kind == HRM_JOB_BFS ? 1u : j.count; }

void validate(const hrm_job& j) {
    if (j.kind > HRM_JOB_BFS) throw std::invalid_argument("unknown job kind");
    if (j.out == nullptr) throw std::invalid_argument("job output is NULL");
    if (j.kind == HRM_JOB_PHOTON && (j.a == nullptr || j.b == nullptr || j.c == nullptr || j.n < 2 || (j.n & 1u)))
        throw std::invalid_argument("photon job needs a medium and an even grid edge");
    if (j.kind == HRM_JOB_BFS && (j.a == nullptr || j.b == nullptr || j.first >= j.n))
        throw std::invalid_argument("bfs job needs a graph and a root below its vertex count");
    if (j.kind != HRM_JOB_BFS && (uint64_t)j.first + j.count > 0xFFFFFFFFull)
        throw std::invalid_argument("first + count exceeds 2^32");
}

// Rough work of a job in async calls, from its size (measured means on the built-in specs:
// about 1600 calls per photon on the 32^3 media, 130 steps per Collatz start below 2^21, two
// calls per edge of a BFS). Jobs of LARGE_JOB_CALLS or more (photon jobs of 2^15 photons and
// up) fill the GPU on their own.
double estimated_calls(const hrm_job& j) {
    if (j.kind == HRM_JOB_PHOTON) return 1600.0 * j.count;
    if (j.kind == HRM_JOB_COLLATZ) return 130.0 * j.count;
    return 32.0 * j.n;
}
const double LARGE_JOB_CALLS = 1600.0 * 32768.0;

JobRecord make_record(const hrm_job& j, JobRecord* d_slot) {
    JobRecord r;
    memset(&r, 0, sizeof(r));
    r.kind = j.kind;
    auto* src = reinterpret_cast<util::iter::AtomicIter<unsigned int>*>(reinterpret_cast<char*>(d_slot) +
                                                                         offsetof(JobRecord, source));
    if (j.kind == HRM_JOB_COLLATZ) {
        r.source = util::iter::AtomicIter<unsigned int>(j.first, j.first + j.count);
        r.s.c.start = j.first;
        r.s.c.limit = j.first + j.count;
        r.s.c.output = (unsigned int*)j.out;
        r.s.c.iterator = src;
        r.s.c.leap = 1;
    } else if (j.kind == HRM_JOB_PHOTON) {
        r.source = util::iter::AtomicIter<unsigned int>(j.first, j.first + j.count);
        r.s.p.mu_s = (const float*)j.a;
        r.s.p.absorb = (const float*)j.b;
        r.s.p.split = (const unsigned char*)j.c;
        r.s.p.tally = (unsigned long long*)j.out;
        r.s.p.source = src;
        r.s.p.n = j.n;
        r.s.p.seed_lo = (unsigned int)j.seed;
        r.s.p.seed_hi = (unsigned int)(j.seed >> 32);
        r.s.p.leap = 1;
        r.s.p.load_limit = 2.0f;
    } else {
        r.source = util::iter::AtomicIter<unsigned int>(0, 1);
        r.s.b.rowptr = (const unsigned int*)j.a;
        r.s.b.col = (const unsigned int*)j.b;
        r.s.b.levels = (unsigned int*)j.out;
        r.s.b.roots = src;
        r.s.b.root = j.first;
        r.s.b.nv = j.n;
    }
    if (job_sources(j) == 0) {
        r.done = 1;
        r.source_closed = 1;
    }
    r.large = estimated_calls(j) >= LARGE_JOB_CALLS ? 1u : 0u;
    return r;
}

// Clears each job's outputs on the device: photon tallies to 0, BFS levels to unreached.
__global__ void mix_prepare_kernel(JobRecord* jobs, const unsigned int* admitted) {
    const unsigned int n = *admitted;
    for (unsigned int j = blockIdx.x; j < n; j += gridDim.x) {
        JobRecord& r = jobs[j];
        if (r.kind == hrm_specs::JOB_PHOTON) {
            size_t slots = (size_t)r.s.p.n * r.s.p.n * r.s.p.n + 3u * hrm_specs::PHOTON_SPREAD;
            for (size_t i = threadIdx.x; i < slots; i += blockDim.x) r.s.p.tally[i] = 0ull;
        } else if (r.kind == hrm_specs::JOB_BFS) {
            for (size_t i = threadIdx.x; i < r.s.b.nv; i += blockDim.x) r.s.b.levels[i] = 0xFFFFFFFFu;
        }
    }
}

__global__ void stamp_kernel(unsigned long long* t) {
    if (threadIdx.x == 0) *t = hrm_specs::global_ns();
}

// The order in which make_work serves jobs (hrm_run_config.job_order).
unsigned int job_order_of(const hrm_run_config& cfg) {
    switch (cfg.job_order) {
        case HRM_JOB_ORDER_ROUND_ROBIN: return hrm_specs::JOB_ORDER_ROUND_ROBIN;
        case HRM_JOB_ORDER_ADMISSION: return hrm_specs::JOB_ORDER_ADMISSION;
        case HRM_JOB_ORDER_SMALL_FIRST: return hrm_specs::JOB_ORDER_SMALL_FIRST;
        default: throw std::invalid_argument("unknown job_order");
    }
}

// ---------------------------------------------------------------------------------------
// Batch contexts: program instance + job table + counters, cached per (device, variant,
// capacity, arena), with the launch sequence captured in a CUDA graph.
// ---------------------------------------------------------------------------------------
struct BatchBase {
    virtual ~BatchBase() {}
    virtual JobRecord* table() = 0;  // device job table that job records point into
    virtual void run(const std::vector<JobRecord>& recs, unsigned int closed0, const hrm_run_config& cfg,
                     hrm_run_result* res, uint64_t* done_ns) = 0;
};

template <typename P>
struct Batch : BatchBase {
    typename P::Instance inst;
    util::host::DevBuf<JobRecord> jobs;
    util::host::DevBuf<unsigned int> counters;      // admitted, cursor, open, completed, closed
    util::host::DevBuf<unsigned long long> t0;
    unsigned int capacity;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    size_t graph_groups = 0, graph_cycles = 0;
    std::mutex lock;

    static MixState state_for(JobRecord* j, unsigned int* c, unsigned int cap) {
        MixState s;
        s.jobs = j;
        s.admitted = c + 0;
        s.cursor = c + 1;
        s.open = c + 2;
        s.completed = c + 3;
        s.closed = c + 4;
        s.low = c + 5;
        s.started = c + 6;
        s.max_active = 256;
        s.job_order = hrm_specs::JOB_ORDER_ROUND_ROBIN;
        s.done_host = nullptr;
        s.njobs = cap;
        return s;
    }

    Batch(unsigned int cap, size_t arena)
        : inst((typename P::AdrType)arena, MixState{}), jobs((size_t)cap), counters((size_t)8), t0((size_t)1),
          capacity(cap) {
        inst.device_state = state_for(jobs.data(), counters.data(), cap);
        ck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
    }
    ~Batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
    }
    JobRecord* table() override { return jobs.data(); }

    // Captures: timestamp, output preparation, init<P>, exec<P> (the launches bake in the
    // instance's tunables, so a change of them re-captures).
    void capture(size_t groups, size_t cycles, unsigned int patience, unsigned int fill_links, unsigned int order) {
        if (graph && groups == graph_groups && cycles == graph_cycles && patience == inst.patience &&
            fill_links == inst.fill_links && order == inst.device_state.job_order)
            return;
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        inst.patience = patience;
        inst.fill_links = fill_links;
        inst.device_state.job_order = order;
        P::resident_ctas();  // sets the kernel's shared-memory attribute outside the capture
        cudaGraph_t g;
        ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        stamp_kernel<<<1, 32, 0, stream>>>(t0.data());
        mix_prepare_kernel<<<1184, 256, 0, stream>>>(jobs.data(), counters.data());
        P::launch_init(inst, groups, stream);
        P::launch_exec(inst, groups, cycles, stream);
        ck(cudaStreamEndCapture(stream, &g), "end capture");
        ck(cudaGraphInstantiate(&graph, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
        graph_groups = groups;
        graph_cycles = cycles;
    }

    void run(const std::vector<JobRecord>& recs, unsigned int closed0, const hrm_run_config& cfg, hrm_run_result* res,
             uint64_t* done_ns) override {
        std::lock_guard<std::mutex> g(lock);
        const unsigned int n = (unsigned int)recs.size();
        size_t groups = cfg.groups ? cfg.groups : (size_t)1 << 30;
        size_t cycles = cfg.cycles ? cfg.cycles : ((size_t)1 << 24);
        size_t max_execs = cfg.max_execs ? cfg.max_execs : 4096;
        capture(groups, cycles, cfg.patience, cfg.fill_links, job_order_of(cfg));
        unsigned int ctr[8] = {n, 0u, 0u, 0u, closed0, 0u, 0u, 0u};
        ck(cudaMemcpyAsync(jobs.data(), recs.data(), sizeof(JobRecord) * n, cudaMemcpyHostToDevice, stream), "jobs");
        ck(cudaMemcpyAsync(counters.data(), ctr, sizeof(ctr), cudaMemcpyHostToDevice, stream), "counters");
        hrm_capi::EventPair ev;
        ck(cudaEventRecord(ev.start, stream), "event");
        ck(cudaGraphLaunch(graph, stream), "graph launch");
        size_t execs = 1;
        ck(cudaStreamSynchronize(stream), "batch exec");
        bool done = inst.complete();
        while (!done && execs < max_execs) {
            P::launch_exec(inst, groups, cycles, stream);
            execs++;
            ck(cudaStreamSynchronize(stream), "batch exec");
            done = inst.complete();
        }
        ck(cudaEventRecord(ev.stop, stream), "event");
        const float ms = ev.elapsed_ms();
        std::vector<JobRecord> out(n);
        unsigned long long start = 0;
        ck(cudaMemcpy(out.data(), jobs.data(), sizeof(JobRecord) * n, cudaMemcpyDeviceToHost), "jobs back");
        ck(cudaMemcpy(&start, t0.data(), sizeof(start), cudaMemcpyDeviceToHost), "t0");
        unsigned int not_done = 0;
        for (unsigned int j = 0; j < n; j++) {
            if (!out[j].done) not_done++;
            if (done_ns) done_ns[j] = out[j].done ? (out[j].t_done > start ? out[j].t_done - start : 0ull) : ~0ull;
        }
        if (res) {
            res->flags = inst.flags();
            res->execs = (uint32_t)execs;
            std::vector<unsigned long long> st = inst.read_stats();
            for (int i = 0; i < HRM_STAT_COUNT; i++) res->stats[i] = st[i];
            res->device_ms = ms;
        }
        if (!done) throw std::runtime_error("batch did not complete within max_execs exec calls");
        if (not_done) throw std::runtime_error(std::to_string(not_done) + " jobs did not complete");
    }
};

template <size_t R, size_t T>
using MixAsync = AsyncProgram<hrm_specs::MixSpec<R, T>>;
template <size_t R, size_t T, size_t M>
using MixAsyncMin = AsyncProgram<hrm_capi::MinCtas<hrm_specs::MixSpec<R, T>, M>>;

struct BatchKey {
    int dev, variant;
    unsigned int capacity;
    size_t arena;
    bool operator<(const BatchKey& o) const {
        if (dev != o.dev) return dev < o.dev;
        if (variant != o.variant) return variant < o.variant;
        if (capacity != o.capacity) return capacity < o.capacity;
        return arena < o.arena;
    }
};
std::mutex g_batch_mutex;
std::map<BatchKey, std::unique_ptr<BatchBase>> g_batches;

BatchBase* batch_for(int variant, unsigned int njobs, size_t arena) {
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    unsigned int cap = 1024;
    while (cap < njobs) cap <<= 1;
    BatchKey key{dev, variant, cap, arena};
    std::lock_guard<std::mutex> g(g_batch_mutex);
    auto it = g_batches.find(key);
    if (it != g_batches.end()) return it->second.get();
    BatchBase* b = nullptr;
    switch (variant) {
        case HRM_VARIANT_R2_T4: b = new Batch<MixAsync<2, 4>>(cap, arena); break;
        case HRM_VARIANT_R4_T4: b = new Batch<MixAsync<4, 4>>(cap, arena); break;
        case HRM_VARIANT_R4_T2: b = new Batch<MixAsync<4, 2>>(cap, arena); break;
        case HRM_VARIANT_R4_T2_M11: b = new Batch<MixAsyncMin<4, 2, 11>>(cap, arena); break;
        case HRM_VARIANT_R4_T4_M5: b = new Batch<MixAsyncMin<4, 4, 5>>(cap, arena); break;
        default: throw std::invalid_argument("batched runs support variants R2/T4, R4/T4, R4/T2, R4/T2 M11 and R4/T4 M5");
    }
    g_batches.emplace(key, std::unique_ptr<BatchBase>(b));
    return b;
}

// ---------------------------------------------------------------------------------------
// Plain one-launch-per-job kernels (baseline).
// ---------------------------------------------------------------------------------------
__global__ void collatz_plain_kernel(unsigned int first, unsigned int count, unsigned int* out) {
    unsigned int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    unsigned long long v = (unsigned long long)first + i;
    unsigned int steps = 0;
    while (v > 1ull) {
        v = (v % 2ull == 0ull) ? v / 2ull : 3ull * v + 1ull;
        steps++;
    }
    out[i] = steps;
}

__global__ void photon_plain_kernel(hrm_specs::PhotonState s, unsigned int first, unsigned int count,
                                    unsigned int* overflow) {
    unsigned int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    if (!hrm_specs::photon_walk_thread<48>(s, first + i, nullptr)) atomicOr(overflow, 1u);
}

// One CTA: level-synchronous BFS with two frontiers in global memory.
__global__ void __launch_bounds__(1024) bfs_plain_block_kernel(const unsigned int* rowptr, const unsigned int* col,
                                                                unsigned int nv, unsigned int root,
                                                                unsigned int* levels, unsigned int* fa,
                                                                unsigned int* fb) {
    __shared__ unsigned int n_next;
    for (unsigned int v = threadIdx.x; v < nv; v += blockDim.x) levels[v] = 0xFFFFFFFFu;
    __syncthreads();
    if (threadIdx.x == 0) {
        levels[root] = 0;
        fa[0] = root;
    }
    unsigned int n_cur = 1, level = 0;
    __syncthreads();
    while (n_cur > 0) {
        if (threadIdx.x == 0) n_next = 0;
        __syncthreads();
        for (unsigned int i = threadIdx.x; i < n_cur; i += blockDim.x) {
            unsigned int v = fa[i];
            for (unsigned int e = rowptr[v]; e < rowptr[v + 1]; e++) {
                unsigned int u = col[e];
                if (levels[u] == 0xFFFFFFFFu && atomicCAS(&levels[u], 0xFFFFFFFFu, level + 1u) == 0xFFFFFFFFu) {
                    fb[atomicAdd(&n_next, 1u)] = u;
                }
            }
        }
        __syncthreads();
        n_cur = n_next;
        level++;
        unsigned int* t = fa;
        fa = fb;
        fb = t;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Serving: a resident runtime that admits jobs while it runs.
// ---------------------------------------------------------------------------------------
// Session trace: with HRM_SERVE_TRACE set in the environment, a serving session writes one
// line per event (exec launched and ended, solo job started and ended, halt requested,
// admission held back) to stderr, stamped in milliseconds since the session opened.
struct SessionTrace {
    const bool on = std::getenv("HRM_SERVE_TRACE") != nullptr;
    const std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::mutex lock;
    void operator()(const char* fmt, ...) {
        if (!on) return;
        const double ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::lock_guard<std::mutex> g(lock);
        std::fprintf(stderr, "[hrm serve %10.3f ms] ", ms);
        va_list ap;
        va_start(ap, fmt);
        std::vfprintf(stderr, fmt, ap);
        va_end(ap);
        std::fputc('\n', stderr);
    }
};

struct ServerBase {
    SessionTrace trace;
    virtual ~ServerBase() {}
    virtual unsigned int submit(const hrm_job* jobs, unsigned int n) = 0;  // returns first index
    virtual unsigned int poll(uint64_t* done_ns, unsigned int max) = 0;    // returns completed count
    virtual void close(unsigned int timeout_ms) = 0;
    virtual size_t arena_bytes() const = 0;
    // Free arena bytes as the device sees them now: links never handed out plus links on the
    // free-link ring, read from the running instance's control block and ring head.
    virtual size_t observed_free_bytes() = 0;
    virtual std::string describe_unfinished() = 0;
    virtual volatile unsigned long long* done_flags() = 0;
    virtual std::string error() = 0;
};

template <typename P>
struct Server : ServerBase {
    typename P::Instance inst;
    util::host::DevBuf<JobRecord> jobs;
    util::host::DevBuf<unsigned int> counters;  // admitted, cursor, open, completed, closed
    unsigned long long* done_host = nullptr;    // mapped: %globaltimer of completion per job
    JobRecord* staging = nullptr;               // pinned staging for job records
    unsigned int* pinned_ctr = nullptr;         // pinned staging for counter writes; [6] = 1, [7] = 0
    // Pinned fill patterns (all zero bytes, all 0xFF bytes) that the copy engine writes over a
    // submitted job's outputs: while the persistent kernel holds every SM, a kernel launched
    // to clear them would wait for the exec to end.
    static const size_t PATTERN_BYTES = (size_t)1 << 20;
    unsigned char* zeros = nullptr;
    unsigned char* ones = nullptr;
    long long clock_offset_ns = 0;              // %globaltimer - host steady clock, at set-up
    unsigned int capacity;
    std::atomic<unsigned int> submitted{0};  // written by submit, read by poll and close
    size_t groups, cycles;
    cudaStream_t exec_s = nullptr, submit_s = nullptr;
    std::thread runner;
    std::atomic<bool> host_open{true};
    std::atomic<bool> stop{false};
    std::mutex err_lock;
    std::string err;
    std::mutex submit_lock;
    size_t arena_links;
    // Solo lane, partitioned residency: photon jobs of at least solo_photons photons fill the
    // GPU on their own and run at about half speed inside the multiplexing kernel, so the
    // session serves them through the single-spec runtime, BESIDE the resident kernel: while
    // a solo job is queued or running, the resident kernel is launched with a quarter of its
    // CTAs per SM (shared_groups) and the solo job's kernel with as many CTAs per SM as fit beside
    // them (solo_groups; shared memory, threads, and registers per SM sub-partition), so both
    // are resident at once and the small jobs keep flowing. With no solo work the resident
    // kernel runs with all its teams. submit queues a solo job and, if the resident
    // exec on the GPU holds every team, halts it (teams spill their work and leave within a
    // few scheduling rounds) so that the runner relaunches it with its share; the solo runner
    // halts the shared exec once the queue drains, so that it comes back with all teams.
    // A solo job's record is a placeholder with an empty source, which the kernel closes and
    // never works on; its completion is stamped by the solo runner.
    unsigned int solo_photons;
    // The solo lane's photon kernel: 4 teams per CTA (one warp per SM sub-partition).
    static const int SOLO_VARIANT = HRM_VARIANT_R4_T4_M5;
    // Solo jobs run on SOLO_LANES lanes at once (a runner thread, a stream and a program
    // instance each), every lane with its share of the solo lane's teams, so that one job's
    // tail of dependent calls overlaps the other's work.
    static const unsigned int SOLO_LANES = 2;
    std::mutex solo_lock;                                     // guards the fields below
    std::condition_variable solo_cv;
    std::deque<std::pair<unsigned int, hrm_job>> solo_queue;  // (job index, job)
    unsigned int solo_active = 0;                             // solo jobs on the GPU
    bool exec_shared = false;                                 // the exec on the GPU holds its share beside the solo lane
    bool exec_on_gpu = false;                                 // a resident exec is launched
    unsigned int solo_alone = 0;                              // solo jobs that keep the resident kernel off the GPU
    bool solo_exit = false;                                   // the solo runners should stop
    unsigned int solo_submitted = 0, solo_done = 0;           // solo jobs queued / stamped so far
    unsigned long long exec_epoch = 0;                         // resident execs launched so far
    unsigned long long halted_epoch = ~0ull;                   // the exec the solo runner last halted
    // Teams of a solo job beside the resident kernel / with it off the GPU: the whole share
    // for a job that runs by itself, a lane's share while several run.
    size_t shared_groups = 0, solo_groups = 0, alone_groups = 0, solo_groups_lane = 0, alone_groups_lane = 0;
    cudaStream_t solo_s[SOLO_LANES] = {};
    std::vector<std::thread> solo_runners;
    unsigned long long* done_dev = nullptr;                    // device alias of done_host

    Server(unsigned int cap, const hrm_run_config& cfg)
        : inst((typename P::AdrType)(cfg.arena ? cfg.arena : ((size_t)1 << 21)), MixState{}),
          jobs((size_t)cap),
          counters((size_t)8),
          capacity(cap),
          groups(cfg.groups ? cfg.groups : (size_t)1 << 30),
          cycles(cfg.cycles ? cfg.cycles : ((size_t)1 << 20)),
          arena_links(cfg.arena ? cfg.arena : ((size_t)1 << 21)),
          solo_photons(cfg.solo_photons) {
        try {
            set_up(cap, cfg);
        } catch (...) {
            release_host_resources();  // the destructor does not run for a failed constructor
            throw;
        }
        runner = std::thread([this] { loop(); });
        if (solo_photons) {
            for (unsigned int lane = 0; lane < SOLO_LANES; lane++) solo_runners.emplace_back([this, lane] { solo_loop(lane); });
        }
    }

    void set_up(unsigned int cap, const hrm_run_config& cfg) {
        ck(cudaHostAlloc((void**)&done_host, sizeof(unsigned long long) * cap, cudaHostAllocMapped), "done flags");
        memset(done_host, 0, sizeof(unsigned long long) * cap);
        ck(cudaHostGetDevicePointer((void**)&done_dev, done_host, 0), "done flags device alias");
        ck(cudaHostAlloc((void**)&staging, sizeof(JobRecord) * 4096, cudaHostAllocDefault), "staging");
        ck(cudaHostAlloc((void**)&pinned_ctr, sizeof(unsigned int) * 8, cudaHostAllocDefault), "staging");
        memset(pinned_ctr, 0, sizeof(unsigned int) * 8);
        pinned_ctr[6] = 1u;
        ck(cudaHostAlloc((void**)&zeros, PATTERN_BYTES, cudaHostAllocDefault), "fill pattern");
        ck(cudaHostAlloc((void**)&ones, PATTERN_BYTES, cudaHostAllocDefault), "fill pattern");
        memset(zeros, 0, PATTERN_BYTES);
        memset(ones, 0xFF, PATTERN_BYTES);
        ck(cudaStreamCreateWithFlags(&exec_s, cudaStreamNonBlocking), "stream");
        ck(cudaStreamCreateWithFlags(&submit_s, cudaStreamNonBlocking), "stream");
        MixState st = Batch<P>::state_for(jobs.data(), counters.data(), cap);
        st.done_host = done_dev;
        inst.device_state = st;
        inst.patience = cfg.patience;
        inst.fill_links = cfg.fill_links;
        inst.device_state.job_order = job_order_of(cfg);
        unsigned int ctr[8] = {0u, 0u, 1u, 0u, 0u, 0u, 0u, 0u};
        ck(cudaMemcpy(counters.data(), ctr, sizeof(ctr), cudaMemcpyHostToDevice), "counters");
        P::launch_init(inst, groups, exec_s);
        ck(cudaStreamSynchronize(exec_s), "init");
        // While the persistent kernel runs, the session launches no kernel of its own (a
        // kernel needs room on an SM, which the persistent kernel may leave none of): job
        // outputs are cleared and halts requested by copies, and solo completions stamped by
        // the host in %globaltimer units through this offset (one probe, before the session).
        {
            util::host::DevBuf<unsigned long long> probe((size_t)1);
            const auto h0 = std::chrono::steady_clock::now();
            stamp_kernel<<<1, 32, 0, submit_s>>>(probe.data());
            ck(cudaGetLastError(), "clock probe");
            ck(cudaStreamSynchronize(submit_s), "clock probe");
            const auto h1 = std::chrono::steady_clock::now();
            unsigned long long g = 0;
            ck(cudaMemcpy(&g, probe.data(), sizeof(g), cudaMemcpyDeviceToHost), "clock probe");
            const long long mid = std::chrono::duration_cast<std::chrono::nanoseconds>(
                                      (h0 + (h1 - h0) / 2).time_since_epoch()).count();
            clock_offset_ns = (long long)g - mid;
        }
        if (solo_photons) {
            for (auto& st : solo_s) ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
            int dev = 0, sms = 1;
            ck(cudaGetDevice(&dev), "cudaGetDevice");
            ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
            // A quarter of the resident kernel's CTAs per SM, and as many CTAs of the solo photon
            // kernel (4 teams per CTA, so that each CTA puts one warp on each SM sub-partition)
            // as fit beside them; fewer resident CTAs if none fit. Large photon jobs carry most
            // of the mix's work, so the solo lane gets the larger share: with half each, the
            // lane saturated at 0.75 of the plain kernels' job rate.
            const unsigned int mix_ctas_per_sm = P::resident_ctas() / (unsigned int)sms;
            cudaFuncAttributes mf;
            ck(cudaFuncGetAttributes(&mf, hrm_rt::async_exec_kernel<P>), "kernel attributes");
            hrm_capi::CtaFootprint mix_cta;
            mix_cta.regs_per_thread = (unsigned int)mf.numRegs;
            mix_cta.threads = P::CTA_THREADS;
            mix_cta.smem = mf.sharedSizeBytes + P::SMEM_BYTES;
            const hrm_capi::CtaFootprint solo_cta = hrm_capi::photon_cta_footprint(SOLO_VARIANT);
            unsigned int m = std::max(1u, mix_ctas_per_sm / 4u), s = 0;
            while (m > 0 && (s = hrm_capi::ctas_beside(mix_cta, m, solo_cta)) == 0) m--;
            if (m == 0 || s == 0) throw std::runtime_error("solo lane: the photon kernel fits beside no resident CTA");
            shared_groups = (size_t)m * (size_t)sms * P::TEAMS_PER_CTA;
            const size_t cta_teams = solo_cta.threads / 32u;
            auto per_lane = [&](size_t teams) {  // one lane's share, in whole CTAs, at least one CTA
                const size_t g = teams / SOLO_LANES / cta_teams * cta_teams;
                return g > cta_teams ? g : cta_teams;
            };
            solo_groups = (size_t)s * (size_t)sms * cta_teams;
            alone_groups = hrm_capi::photon_resident_teams(SOLO_VARIANT);
            solo_groups_lane = per_lane(solo_groups);
            alone_groups_lane = per_lane(alone_groups);
            trace("solo lane: resident %u of %u CTAs per SM (%u regs, %zu B), solo photon %u CTAs per SM "
                  "(%u regs, %zu B): shared_groups %zu; solo teams beside it %zu (a lane's share %zu), alone %zu "
                  "(%zu)", m, mix_ctas_per_sm, mix_cta.regs_per_thread, mix_cta.smem, s, solo_cta.regs_per_thread,
                  solo_cta.smem, shared_groups, solo_groups, solo_groups_lane, alone_groups, alone_groups_lane);
            // The solo job's kernel must start before the shared exec may be counted on:
            // load it now (lazy loading would hold it back until a running kernel ends).
            // Every lane's program instance is made now too (it allocates its arena).
            util::host::DevBuf<float> mu((size_t)8);
            util::host::DevBuf<unsigned char> sp((size_t)8);
            util::host::DevBuf<unsigned long long> t((size_t)(8 + 3 * hrm_specs::PHOTON_SPREAD));
            ck(cudaMemset(mu.data(), 0, 8 * sizeof(float)), "warm-up medium");
            ck(cudaMemset(sp.data(), 0, 8), "warm-up medium");
            for (unsigned int lane = 0; lane < SOLO_LANES; lane++) {
                hrm_run_config c;
                memset(&c, 0, sizeof(c));
                c.program_type = HRM_ASYNC;
                c.variant = SOLO_VARIANT;
                c.stream = solo_s[lane];
                c.groups = solo_groups_lane;
                hrm_run_result r;
                if (hrm_capi::photon_walk_lane(lane, mu.data(), mu.data(), sp.data(), 2, 1, 0, 0, (uint64_t*)t.data(),
                                               &c, &r) != HRM_OK)
                    throw std::runtime_error(std::string("solo lane warm-up: ") + hrm_last_error());
            }
        }
    }

    void release_host_resources() {
        if (exec_s) cudaStreamDestroy(exec_s);
        if (submit_s) cudaStreamDestroy(submit_s);
        for (auto& st : solo_s) {
            if (st) cudaStreamDestroy(st);
            st = nullptr;
        }
        if (done_host) cudaFreeHost(done_host);
        if (staging) cudaFreeHost(staging);
        if (pinned_ctr) cudaFreeHost(pinned_ctr);
        if (zeros) cudaFreeHost(zeros);
        if (ones) cudaFreeHost(ones);
        exec_s = submit_s = nullptr;
        done_host = nullptr;
        staging = nullptr;
        pinned_ctr = nullptr;
        zeros = ones = nullptr;
    }

    // Teardown is bounded: the session is closed, the running exec is asked to halt (teams
    // leave within a few scheduling rounds, spilling their work), and the runner stops after
    // that exec whether or not every job finished.
    ~Server() {
        host_open = false;
        stop = true;
        {
            std::lock_guard<std::mutex> g(solo_lock);  // wakes a resident loop waiting on a solo job
        }
        solo_cv.notify_all();
        if (runner.joinable()) {
            pinned_ctr[2] = 0;
            cudaMemcpyAsync(counters.data() + 2, pinned_ctr + 2, 4, cudaMemcpyHostToDevice, submit_s);
            cudaMemcpyAsync(&inst.control.data()->halt_request, pinned_ctr + 6, 4, cudaMemcpyHostToDevice, submit_s);
            cudaStreamSynchronize(submit_s);
            runner.join();
        }
        stop_solo_runner();
        release_host_resources();
    }

    void stop_solo_runner() {
        {
            std::lock_guard<std::mutex> g(solo_lock);
            solo_exit = true;
        }
        solo_cv.notify_all();
        for (auto& t : solo_runners)
            if (t.joinable()) t.join();
        solo_runners.clear();
    }

    void halt_resident() {
        trace("halt requested");
        ck(cudaMemcpyAsync(&inst.control.data()->halt_request, pinned_ctr + 6, 4, cudaMemcpyHostToDevice, submit_s),
           "halt");
        ck(cudaStreamSynchronize(submit_s), "halt");
    }

    // One solo job on lane `lane`: beside the shared resident exec or with the resident kernel
    // off the GPU, with the whole share (`whole`: no other solo job is running or waiting) or
    // a lane's share.
    void run_solo(unsigned int lane, unsigned int j, const hrm_job& jb, bool alone, bool whole) {
        hrm_run_config c;
        memset(&c, 0, sizeof(c));
        c.program_type = HRM_ASYNC;
        c.variant = SOLO_VARIANT;
        c.stream = solo_s[lane];
        c.groups = alone ? (whole ? alone_groups : alone_groups_lane) : (whole ? solo_groups : solo_groups_lane);
        hrm_run_result r;
        trace("solo job %u (%u photons) starts on lane %u %s, %zu teams", j, jb.count, lane,
              alone ? "with the resident kernel off the GPU" : "beside the resident kernel", (size_t)c.groups);
        if (hrm_capi::photon_walk_lane(lane, (const float*)jb.a, (const float*)jb.b, (const uint8_t*)jb.c, jb.n,
                                       jb.seed, jb.first, jb.count, (uint64_t*)jb.out, &c, &r) != HRM_OK)
            throw std::runtime_error(std::string("solo photon job: ") + hrm_last_error());
        trace("solo job %u ends: %.3f ms on the device, %u execs", j, r.device_ms, r.execs);
        // The run above synchronised with its stream: stamp the completion from the host.
        const long long now = std::chrono::duration_cast<std::chrono::nanoseconds>(
                                  std::chrono::steady_clock::now().time_since_epoch()).count();
        const unsigned long long stamp = (unsigned long long)(now + clock_offset_ns);
        ((volatile unsigned long long*)done_host)[j] = stamp ? stamp : 1ull;
    }

    // Jobs admitted to the resident kernel and not finished yet (solo_lock held).
    unsigned int resident_in_flight() {
        const unsigned int total = submitted.load();
        unsigned int done = 0;
        for (unsigned int j = 0; j < total; j++) done += ((volatile unsigned long long*)done_host)[j] != 0ull;
        const unsigned int resident_done = done - std::min(done, solo_done);
        const unsigned int resident_jobs = total - std::min(total, solo_submitted);
        return resident_jobs > resident_done ? resident_jobs - resident_done : 0u;
    }

    // A solo runner (one per lane): serves the solo queue in submission order, one job at a
    // time per lane. With no job in flight in the resident kernel, a job runs with the resident
    // kernel off the GPU (the resident exec is halted and not relaunched while such a job
    // runs; jobs submitted meanwhile wait in the table); otherwise beside the resident exec
    // once that holds only its share.
    void solo_loop(unsigned int lane) {
        try {
            while (true) {
                std::pair<unsigned int, hrm_job> sj;
                bool alone = false, halt = false, whole = false;
                {
                    std::unique_lock<std::mutex> g(solo_lock);
                    solo_cv.wait_for(g, std::chrono::milliseconds(2),
                                     [this] { return solo_exit || !solo_queue.empty(); });
                    if (solo_exit) break;
                    if (solo_queue.empty()) continue;
                    alone = resident_in_flight() == 0u;
                    if (!alone && exec_on_gpu && !exec_shared) {
                        // An exec holding every team: ask it once to come back with its share.
                        halt = halted_epoch != exec_epoch;
                        halted_epoch = exec_epoch;
                    }
                }
                if (halt) halt_resident();
                {
                    std::unique_lock<std::mutex> g(solo_lock);
                    if (solo_queue.empty()) continue;
                    alone = resident_in_flight() == 0u;
                    if (!alone && !(exec_shared || !exec_on_gpu)) continue;  // wait for the shared exec
                    sj = solo_queue.front();
                    solo_queue.pop_front();
                    // By itself: the whole share. (A job that starts later with a lane's share
                    // waits for room until this one ends.)
                    whole = solo_active == 0 && solo_queue.empty();
                    solo_active++;
                    if (alone) solo_alone++;
                }
                if (alone) {
                    bool running;
                    {
                        std::lock_guard<std::mutex> g(solo_lock);
                        running = exec_on_gpu;
                    }
                    if (running) halt_resident();
                    std::unique_lock<std::mutex> g(solo_lock);
                    solo_cv.wait(g, [this] { return !exec_on_gpu || solo_exit; });
                    if (solo_exit) {
                        solo_alone--;
                        solo_active--;
                        break;
                    }
                }
                run_solo(lane, sj.first, sj.second, alone, whole);
                bool drained;
                {
                    std::lock_guard<std::mutex> g(solo_lock);
                    solo_active--;
                    if (alone) solo_alone--;
                    solo_done++;
                    drained = solo_queue.empty() && solo_active == 0 && exec_on_gpu && exec_shared;
                }
                solo_cv.notify_all();
                // Nothing left for the solo lanes: give the resident exec all its teams back.
                if (drained) halt_resident();
            }
        } catch (std::exception& e) {
            {
                std::lock_guard<std::mutex> g(err_lock);
                err = e.what();
            }
            std::lock_guard<std::mutex> g(solo_lock);
            solo_alone = 0;  // never leave the resident loop waiting
            solo_cv.notify_all();
        }
    }

    // Relaunches the persistent kernel until the session is closed and every job is done.
    void loop() {
        try {
            while (true) {
                if (stop) break;
                // Clear a served halt request, then look at the solo lane: submit queues a job
                // before it requests the halt, so a job queued after this look comes with a
                // halt that lands after this clear and stops the exec launched below.
                ck(cudaMemcpyAsync(&inst.control.data()->flags, pinned_ctr + 7, 4, cudaMemcpyHostToDevice, exec_s),
                   "clear flags");
                ck(cudaMemcpyAsync(&inst.control.data()->halt_request, pinned_ctr + 7, 4, cudaMemcpyHostToDevice,
                                   exec_s), "clear halt request");
                ck(cudaStreamSynchronize(exec_s), "clear flags");
                bool shared;
                {
                    // A solo job that holds the whole GPU keeps the resident kernel off it.
                    std::unique_lock<std::mutex> g(solo_lock);
                    solo_cv.wait(g, [this] { return solo_alone == 0 || stop; });
                    if (stop) break;
                    shared = solo_photons && (!solo_queue.empty() || solo_active > 0);
                    exec_shared = shared;
                    exec_on_gpu = true;
                    exec_epoch++;
                }
                solo_cv.notify_all();
                // A shared exec runs a short cycle budget: should the solo job's CTAs not all
                // find room beside it, the job waits for this exec's end, not for a whole one.
                const size_t exec_cycles = shared ? std::max<size_t>(cycles / 64u, 4096u) : cycles;
                trace("exec launched: %s, %zu groups, %zu cycles", shared ? "shared" : "full", shared ? shared_groups : groups,
                      exec_cycles);
                P::launch_exec(inst, shared ? shared_groups : groups, exec_cycles, exec_s);
                cudaError_t le = cudaStreamSynchronize(exec_s);
                trace("exec ended");
                {
                    std::lock_guard<std::mutex> g(solo_lock);
                    exec_on_gpu = false;
                }
                solo_cv.notify_all();
                ck(le, "serving exec");
                unsigned int f = inst.flags();
                if (f & hrm_rt::ERROR_MASK) hrm_rt::throw_flags(f);
                if (stop) break;
                bool solo_left;
                {
                    std::lock_guard<std::mutex> g(solo_lock);
                    solo_left = !solo_queue.empty() || solo_active > 0;
                }
                if (!host_open && (f & hrm_rt::COMPLETION_FLAG) && !solo_left) break;
            }
        } catch (std::exception& e) {
            {
                std::lock_guard<std::mutex> g(err_lock);
                err = e.what();
            }
            std::lock_guard<std::mutex> g(solo_lock);
            exec_on_gpu = false;  // never leave the solo runner waiting for this loop
            solo_cv.notify_all();
        }
    }

    unsigned int submit(const hrm_job* in, unsigned int n) override {
        std::lock_guard<std::mutex> one_at_a_time(submit_lock);  // submissions from several threads
        if (submitted + n > capacity) throw std::invalid_argument("server job table is full");
        unsigned int first = submitted;
        std::vector<std::pair<unsigned int, hrm_job>> solo;
        for (unsigned int done = 0; done < n;) {
            unsigned int k = std::min(n - done, 4096u);
            for (unsigned int i = 0; i < k; i++) {
                const hrm_job& jb = in[done + i];
                if (job_sources(jb) == 0) throw std::invalid_argument("a served job needs work to do");
                validate(jb);
                staging[i] = make_record(jb, jobs.data() + first + done + i);
                if (solo_photons && jb.kind == HRM_JOB_PHOTON && jb.count >= solo_photons) {
                    // Placeholder: an empty source, already done; the kernel closes it.
                    staging[i].source = util::iter::AtomicIter<unsigned int>(jb.first, jb.first);
                    staging[i].done = 1;
                    solo.emplace_back(first + done + i, jb);
                }
            }
            ck(cudaMemcpyAsync(jobs.data() + first + done, staging, sizeof(JobRecord) * k, cudaMemcpyHostToDevice,
                               submit_s), "job records");
            ck(cudaStreamSynchronize(submit_s), "job records");
            done += k;
        }
        // Clear the outputs (photon tallies to zero, BFS levels to unreached) with the copy
        // engine, on the stream that then publishes the jobs.
        for (unsigned int i = 0; i < n; i++) {
            const hrm_job& jb = in[i];
            if (solo_photons && jb.kind == HRM_JOB_PHOTON && jb.count >= solo_photons) continue;  // cleared by its run
            size_t bytes = 0;
            const unsigned char* pattern = zeros;
            if (jb.kind == HRM_JOB_PHOTON) {
                bytes = ((size_t)jb.n * jb.n * jb.n + 3u * hrm_specs::PHOTON_SPREAD) * sizeof(unsigned long long);
            } else if (jb.kind == HRM_JOB_BFS) {
                bytes = (size_t)jb.n * sizeof(unsigned int);
                pattern = ones;
            }
            for (size_t off = 0; off < bytes; off += PATTERN_BYTES) {
                ck(cudaMemcpyAsync((unsigned char*)jb.out + off, pattern, std::min(PATTERN_BYTES, bytes - off),
                                   cudaMemcpyHostToDevice, submit_s), "output preparation");
            }
        }
        pinned_ctr[0] = first + n;
        // Published after the records (same stream): teams never see a job before its record.
        ck(cudaMemcpyAsync(counters.data(), pinned_ctr, 4, cudaMemcpyHostToDevice, submit_s), "admit");
        ck(cudaStreamSynchronize(submit_s), "admit");
        submitted = first + n;
        if (!solo.empty()) {
            bool full_on_gpu;
            {
                std::lock_guard<std::mutex> g(solo_lock);
                for (auto& s : solo) solo_queue.push_back(s);
                solo_submitted += (unsigned int)solo.size();
                // With jobs in flight the solo lane will share the GPU: the exec holding every
                // team must come back with its share. (With none, the solo runner halts it and
                // takes the whole GPU.)
                full_on_gpu = exec_on_gpu && !exec_shared && resident_in_flight() > 0u;
            }
            solo_cv.notify_all();
            // Queued first, then the halt (see loop()).
            if (full_on_gpu) halt_resident();
        }
        return first;
    }

    unsigned int poll(uint64_t* done_ns, unsigned int max) override {
        unsigned int c = 0;
        unsigned int m = std::min(max, submitted.load());
        for (unsigned int j = 0; j < m; j++) {
            unsigned long long t = ((volatile unsigned long long*)done_host)[j];
            if (done_ns) done_ns[j] = t;
            c += (t != 0ull);
        }
        return c;
    }

    void close(unsigned int timeout_ms) override {
        host_open = false;
        pinned_ctr[1] = 0;
        ck(cudaMemcpyAsync(counters.data() + 2, pinned_ctr + 1, 4, cudaMemcpyHostToDevice, submit_s), "close");
        ck(cudaStreamSynchronize(submit_s), "close");
        auto t0 = std::chrono::steady_clock::now();
        const unsigned int total = submitted.load();
        while (poll(nullptr, total) < total) {
            if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms)) {
                throw std::runtime_error("serving session did not finish within the close timeout");
            }
            std::this_thread::sleep_for(std::chrono::microseconds(200));
            std::string e = error();
            if (!e.empty()) throw std::runtime_error(e);
        }
        if (runner.joinable()) runner.join();
        stop_solo_runner();
        std::string e = error();
        if (!e.empty()) throw std::runtime_error(e);
    }

    // Device-side state of up to 8 unfinished jobs, for error messages.
    std::string describe_unfinished() override {
        const unsigned int total = submitted.load();
        std::vector<JobRecord> recs(total);
        if (total == 0 || cudaMemcpy(recs.data(), jobs.data(), sizeof(JobRecord) * total,
                                         cudaMemcpyDeviceToHost) != cudaSuccess)
            return "";
        unsigned int ctr[8] = {};
        cudaMemcpy(ctr, counters.data(), sizeof(ctr), cudaMemcpyDeviceToHost);
        std::string s = " [admitted " + std::to_string(ctr[0]) + " completed " + std::to_string(ctr[3]) + " closed " +
                        std::to_string(ctr[4]) + " low " + std::to_string(ctr[5]) + " flags " +
                        std::to_string(inst.flags()) + "]";
        int shown = 0;
        for (unsigned int j = 0; j < total && shown < 8; j++) {
            const JobRecord& r = recs[j];
            if (r.done) continue;
            s += " job " + std::to_string(j) + ": kind " + std::to_string(r.kind) + " pending " +
                 std::to_string(r.pending) + " source " + std::to_string(r.source.value) + "/" +
                 std::to_string(r.source.limit) + " closed " + std::to_string(r.source_closed) + ";";
            shown++;
        }
        return s;
    }

    size_t arena_bytes() const override { return arena_links * P::LINK_WORDS * 128u; }
    size_t observed_free_bytes() override {
        // Two 4-byte reads on the submit stream; the copy engine reads them through L2 while
        // the persistent kernel runs.
        ck(cudaMemcpyAsync(pinned_ctr + 4, &inst.control.data()->bump, 4, cudaMemcpyDeviceToHost, submit_s), "bump");
        ck(cudaMemcpyAsync(pinned_ctr + 5, &inst.heads.data()[P::FN].avail, 4, cudaMemcpyDeviceToHost, submit_s),
           "free links");
        ck(cudaStreamSynchronize(submit_s), "free arena read");
        const size_t bump = std::min<size_t>(pinned_ctr[4], arena_links);
        const int on_ring = (int)pinned_ctr[5];
        const size_t free_links = (arena_links - bump) + (size_t)(on_ring > 0 ? on_ring : 0);
        return free_links * P::LINK_WORDS * 128u;
    }
    volatile unsigned long long* done_flags() override { return done_host; }
    std::string error() override {
        std::lock_guard<std::mutex> g(err_lock);
        return err;
    }
};

ServerBase* make_server(unsigned int cap, const hrm_run_config& cfg) {
    switch (cfg.variant) {
        case HRM_VARIANT_R2_T4: return new Server<MixAsync<2, 4>>(cap, cfg);
        case HRM_VARIANT_R4_T4: return new Server<MixAsync<4, 4>>(cap, cfg);
        case HRM_VARIANT_R4_T2: return new Server<MixAsync<4, 2>>(cap, cfg);
        case HRM_VARIANT_R4_T2_M11: return new Server<MixAsyncMin<4, 2, 11>>(cap, cfg);
        case HRM_VARIANT_R4_T4_M5: return new Server<MixAsyncMin<4, 4, 5>>(cap, cfg);
        default: throw std::invalid_argument("serving supports variants R2/T4, R4/T4, R4/T2, R4/T2 M11 and R4/T4 M5");
    }
}

// Estimated arena bytes a job may occupy while in flight (admission control).
size_t job_footprint(const hrm_job& j) {
    size_t per = j.kind == HRM_JOB_PHOTON ? 48u : (j.kind == HRM_JOB_BFS ? 16u : 16u);
    size_t items = j.kind == HRM_JOB_BFS ? ((size_t)j.n * 4u) : (size_t)j.count;
    size_t b = items * per;
    return b < ((size_t)64 << 20) ? b : ((size_t)64 << 20);
}

}  // namespace

struct hrm_server {
    ServerBase* impl;
};

extern "C" {

int hrm_server_open(uint32_t capacity, const hrm_run_config* cfg_in, hrm_server** out) {
    if (out == nullptr || capacity == 0) return hrm_capi::set_error(HRM_EINVAL, "bad server arguments");
    try {
        hrm_run_config cfg;
        memset(&cfg, 0, sizeof(cfg));
        if (cfg_in) cfg = *cfg_in;
        *out = new hrm_server{make_server(capacity, cfg)};
        return HRM_OK;
    } catch (std::invalid_argument& e) {
        return hrm_capi::set_error(HRM_EINVAL, e.what());
    } catch (std::exception& e) {
        return hrm_capi::set_error(HRM_ECUDA, e.what());
    }
}

int hrm_server_submit(hrm_server* srv, const hrm_job* jobs, uint32_t n, uint32_t* first_index) {
    if (srv == nullptr || (jobs == nullptr && n)) return hrm_capi::set_error(HRM_EINVAL, "bad submit arguments");
    try {
        uint32_t f = srv->impl->submit(jobs, n);
        if (first_index) *first_index = f;
        return HRM_OK;
    } catch (std::invalid_argument& e) {
        return hrm_capi::set_error(HRM_EINVAL, e.what());
    } catch (std::exception& e) {
        return hrm_capi::set_error(HRM_ECUDA, e.what());
    }
}

int hrm_server_poll(hrm_server* srv, uint64_t* done_ns, uint32_t max, uint32_t* completed) {
    if (srv == nullptr) return hrm_capi::set_error(HRM_EINVAL, "server is NULL");
    uint32_t c = srv->impl->poll(done_ns, max);
    if (completed) *completed = c;
    std::string e = srv->impl->error();
    if (!e.empty()) return hrm_capi::set_error(HRM_EDEVICE, e);
    return HRM_OK;
}

int hrm_server_close(hrm_server* srv, uint32_t timeout_ms) {
    if (srv == nullptr) return hrm_capi::set_error(HRM_EINVAL, "server is NULL");
    try {
        srv->impl->close(timeout_ms);
        return HRM_OK;
    } catch (std::exception& e) {
        return hrm_capi::set_error(HRM_EDEVICE, e.what());
    }
}

int hrm_server_destroy(hrm_server* srv) {
    if (srv == nullptr) return HRM_OK;
    delete srv->impl;
    delete srv;
    return HRM_OK;
}

// Replays an arrival schedule: arrival_ns[j] (non-decreasing, from the start of the call).
// mode 0: the resident runtime (a server session, jobs admitted FIFO while the device reports
// at least a quarter of the arena free and their estimated arena bytes fit half of it); mode 1: one plain launch per job at its arrival, on
// nstreams streams. latency_ns[j] = host-observed completion - arrival.
int hrm_serve_replay(const hrm_job* jobs, uint32_t njobs, const uint64_t* arrival_ns, int mode, uint32_t nstreams,
                     const hrm_run_config* cfg_in, uint64_t* latency_ns, float* makespan_ms) {
    if ((jobs == nullptr || arrival_ns == nullptr || latency_ns == nullptr) && njobs)
        return hrm_capi::set_error(HRM_EINVAL, "bad replay arguments");
    using clk = std::chrono::steady_clock;
    auto ns_since = [](clk::time_point t0) {
        return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(clk::now() - t0).count();
    };
    try {
        hrm_run_config cfg;
        memset(&cfg, 0, sizeof(cfg));
        if (cfg_in) cfg = *cfg_in;
        for (uint32_t j = 0; j < njobs; j++) validate(jobs[j]);
        // Every replay ends: at the latest two minutes after the last arrival.
        const uint64_t deadline_ns = (njobs ? arrival_ns[njobs - 1] : 0ull) + 120000000000ull;
        if (mode == 0) {
            std::unique_ptr<ServerBase> srv(make_server(njobs ? njobs : 1, cfg));
            const size_t budget = srv->arena_bytes() / 2;
            // Admission by free arena bytes: a job is admitted while the arena the device
            // reports free stays above a quarter of it, and while the estimated footprints of
            // the jobs in flight fit half of it (the estimate covers jobs admitted since the
            // last read, whose promises the device has not counted yet).
            const size_t free_floor = srv->arena_bytes() / 4;
            volatile unsigned long long* done = srv->done_flags();
            std::vector<uint32_t> inflight;
            size_t used = 0;
            uint32_t admitted = 0, finished = 0;
            std::vector<hrm_job> batch;
            bool held_back = false;
            auto t0 = clk::now();
            while (finished < njobs) {
                uint64_t now = ns_since(t0);
                if (now > deadline_ns) {
                    throw std::runtime_error("replay did not finish before its deadline; " + std::to_string(finished) +
                                             " of " + std::to_string(njobs) + " done" + srv->describe_unfinished());
                }
                batch.clear();
                const bool arrivals = admitted < njobs && arrival_ns[admitted] <= now;
                const size_t free_now = arrivals ? srv->observed_free_bytes() : 0;
                while (admitted < njobs && arrival_ns[admitted] <= now) {
                    size_t fp = job_footprint(jobs[admitted]);
                    if ((used + fp > budget || free_now < free_floor) && !inflight.empty()) {
                        if (!held_back) {
                            srv->trace("admission held back: %zu B free (floor %zu), %zu B estimated in flight "
                                       "(budget %zu), %zu jobs in flight", free_now, free_floor, used, budget,
                                       inflight.size());
                        }
                        held_back = true;
                        break;
                    }
                    held_back = false;
                    used += fp;
                    batch.push_back(jobs[admitted]);
                    inflight.push_back(admitted);
                    admitted++;
                }
                if (!batch.empty()) srv->submit(batch.data(), (unsigned int)batch.size());
                for (size_t k = 0; k < inflight.size();) {
                    uint32_t j = inflight[k];
                    if (done[j] != 0ull) {
                        latency_ns[j] = ns_since(t0) - arrival_ns[j];
                        if (latency_ns[j] > 100000000ull)
                            srv->trace("job %u (kind %u, %u items) done after %.1f ms", j, jobs[j].kind,
                                       (unsigned int)job_sources(jobs[j]), latency_ns[j] / 1e6);
                        used -= job_footprint(jobs[j]);
                        inflight[k] = inflight.back();
                        inflight.pop_back();
                        finished++;
                    } else {
                        k++;
                    }
                }
                std::string e = srv->error();
                if (!e.empty()) throw std::runtime_error(e);
            }
            if (makespan_ms) *makespan_ms = (float)(ns_since(t0) / 1e6);
            srv->close(60000);
        } else {
            if (nstreams == 0) nstreams = 16;
            std::vector<cudaStream_t> streams(nstreams, nullptr);
            std::vector<cudaEvent_t> ev(njobs, nullptr);
            unsigned int* d_ovf = nullptr;
            unsigned int* d_fr = nullptr;
            auto release = hrm_capi::on_scope_exit([&] {  // also when a launch or the deadline throws
                for (auto& s : streams)
                    if (s) cudaStreamDestroy(s);
                for (auto& e : ev)
                    if (e) cudaEventDestroy(e);
                if (d_ovf) cudaFree(d_ovf);
                if (d_fr) cudaFree(d_fr);
            });
            for (auto& s : streams) ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
            for (auto& e : ev) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
            size_t max_nv = 0;
            for (uint32_t j = 0; j < njobs; j++)
                if (jobs[j].kind == HRM_JOB_BFS && jobs[j].n > max_nv) max_nv = jobs[j].n;
            ck(cudaMalloc((void**)&d_ovf, 4), "overflow flag");
            ck(cudaMemset(d_ovf, 0, 4), "overflow flag");
            if (max_nv) ck(cudaMalloc((void**)&d_fr, max_nv * 2 * 4 * nstreams), "frontiers");
            ck(cudaDeviceSynchronize(), "sync");
            std::vector<uint32_t> inflight;
            uint32_t launched = 0, finished = 0;
            auto t0 = clk::now();
            while (finished < njobs) {
                uint64_t now = ns_since(t0);
                if (now > deadline_ns) throw std::runtime_error("replay did not finish before its deadline");
                while (launched < njobs && arrival_ns[launched] <= now) {
                    const hrm_job& jb = jobs[launched];
                    cudaStream_t s = streams[launched % nstreams];
                    if (jb.kind == HRM_JOB_COLLATZ) {
                        collatz_plain_kernel<<<(jb.count + 127) / 128, 128, 0, s>>>(jb.first, jb.count,
                                                                                 (unsigned int*)jb.out);
                    } else if (jb.kind == HRM_JOB_PHOTON) {
                        size_t slots = (size_t)jb.n * jb.n * jb.n + 3u * hrm_specs::PHOTON_SPREAD;
                        ck(cudaMemsetAsync(jb.out, 0, slots * 8u, s), "tally clear");
                        hrm_specs::PhotonState st;
                        memset(&st, 0, sizeof(st));
                        st.mu_s = (const float*)jb.a;
                        st.absorb = (const float*)jb.b;
                        st.split = (const unsigned char*)jb.c;
                        st.tally = (unsigned long long*)jb.out;
                        st.n = jb.n;
                        st.seed_lo = (unsigned int)jb.seed;
                        st.seed_hi = (unsigned int)(jb.seed >> 32);
                        photon_plain_kernel<<<(jb.count + 127) / 128, 128, 0, s>>>(st, jb.first, jb.count, d_ovf);
                    } else {
                        unsigned int* fr = d_fr + (size_t)(launched % nstreams) * max_nv * 2;
                        bfs_plain_block_kernel<<<1, 1024, 0, s>>>((const unsigned int*)jb.a, (const unsigned int*)jb.b,
                                                                  jb.n, jb.first, (unsigned int*)jb.out, fr,
                                                                  fr + max_nv);
                    }
                    ck(cudaGetLastError(), "plain launch");
                    ck(cudaEventRecord(ev[launched], s), "event");
                    inflight.push_back(launched);
                    launched++;
                }
                for (size_t k = 0; k < inflight.size();) {
                    uint32_t j = inflight[k];
                    cudaError_t q = cudaEventQuery(ev[j]);
                    if (q == cudaSuccess) {
                        latency_ns[j] = ns_since(t0) - arrival_ns[j];
                        inflight[k] = inflight.back();
                        inflight.pop_back();
                        finished++;
                    } else if (q == cudaErrorNotReady) {
                        k++;
                    } else {
                        ck(q, "plain job");
                    }
                }
            }
            if (makespan_ms) *makespan_ms = (float)(ns_since(t0) / 1e6);
        }
        return HRM_OK;
    } catch (std::invalid_argument& e) {
        return hrm_capi::set_error(HRM_EINVAL, e.what());
    } catch (std::exception& e) {
        return hrm_capi::set_error(HRM_EDEVICE, e.what());
    }
}

int hrm_serve_replay_runtime(const hrm_job* jobs, uint32_t njobs, const uint64_t* arrival_ns, int program_type,
                             const int* variants, uint64_t* latency_ns, float* makespan_ms) {
    if ((jobs == nullptr || arrival_ns == nullptr || latency_ns == nullptr) && njobs)
        return hrm_capi::set_error(HRM_EINVAL, "bad replay arguments");
    using clk = std::chrono::steady_clock;
    try {
        for (uint32_t j = 0; j < njobs; j++) validate(jobs[j]);
        ck(cudaDeviceSynchronize(), "sync");
        auto t0 = clk::now();
        auto ns_since = [&]() {
            return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(clk::now() - t0).count();
        };
        for (uint32_t j = 0; j < njobs; j++) {
            while (ns_since() < arrival_ns[j]) std::this_thread::yield();  // FIFO: one job at a time
            int rc = hrm_runtime_run(&jobs[j], 1, program_type, variants, nullptr, nullptr);
            if (rc != HRM_OK) return rc;
            latency_ns[j] = ns_since() - arrival_ns[j];
        }
        if (makespan_ms) *makespan_ms = (float)(ns_since() / 1e6);
        return HRM_OK;
    } catch (std::invalid_argument& e) {
        return hrm_capi::set_error(HRM_EINVAL, e.what());
    } catch (std::exception& e) {
        return hrm_capi::set_error(HRM_EDEVICE, e.what());
    }
}

int hrm_batch_run(const hrm_job* jobs, uint32_t njobs, const hrm_run_config* cfg_in, hrm_run_result* res,
                  uint64_t* done_ns) {
    if (jobs == nullptr && njobs != 0) return hrm_capi::set_error(HRM_EINVAL, "jobs is NULL");
    try {
        hrm_run_config cfg;
        memset(&cfg, 0, sizeof(cfg));
        if (cfg_in) cfg = *cfg_in;
        if (cfg.program_type != HRM_ASYNC) throw std::invalid_argument("batched runs use AsyncProgram");
        for (uint32_t j = 0; j < njobs; j++) validate(jobs[j]);
        // Default arena: 2^23 links (about 12 GB for the mixed spec). Thousands of BFS jobs
        // fan out millions of relaxations at once and none of that can be throttled.
        size_t arena = cfg.arena ? cfg.arena : ((size_t)1 << 23);
        BatchBase* b = batch_for(cfg.variant, njobs ? njobs : 1, arena);
        JobRecord* d_table = b->table();  // records point into the cached context's job table
        std::vector<JobRecord> recs(njobs);
        unsigned int closed0 = 0;
        for (uint32_t j = 0; j < njobs; j++) {
            recs[j] = make_record(jobs[j], d_table + j);
            if (recs[j].source_closed) closed0++;
        }
        b->run(recs, closed0, cfg, res, done_ns);
        return HRM_OK;
    } catch (std::invalid_argument& e) {
        return hrm_capi::set_error(HRM_EINVAL, e.what());
    } catch (std::exception& e) {
        return hrm_capi::set_error(HRM_EDEVICE, e.what());
    }
}

int hrm_runtime_run(const hrm_job* jobs, uint32_t njobs, int program_type, const int* variants, uint64_t* done_ns,
                    float* total_ms) {
    if (jobs == nullptr && njobs != 0) return hrm_capi::set_error(HRM_EINVAL, "jobs is NULL");
    try {
        for (uint32_t j = 0; j < njobs; j++) validate(jobs[j]);
        ck(cudaDeviceSynchronize(), "sync");
        auto t0 = std::chrono::steady_clock::now();
        for (uint32_t j = 0; j < njobs; j++) {
            const hrm_job& jb = jobs[j];
            hrm_run_config cfg;
            memset(&cfg, 0, sizeof(cfg));
            cfg.program_type = program_type;
            cfg.variant = variants ? variants[jb.kind] : 0;
            hrm_run_result res;
            int rc = HRM_OK;
            if (jb.kind == HRM_JOB_COLLATZ) {
                rc = hrm_collatz_run_device(jb.first, jb.count, (uint32_t*)jb.out, &cfg, &res);
            } else if (jb.kind == HRM_JOB_PHOTON) {
                rc = hrm_photon_run_device((const float*)jb.a, (const float*)jb.b, (const uint8_t*)jb.c, jb.n, jb.seed,
                                           jb.first, jb.count, (uint64_t*)jb.out, &cfg, &res);
            } else {
                rc = hrm_bfs_run_device((const uint32_t*)jb.a, (const uint32_t*)jb.b, jb.n, jb.first,
                                        (uint32_t*)jb.out, &cfg, &res);
            }
            if (rc != HRM_OK) return rc;  // message already set by the whole-run call
            if (done_ns) {
                done_ns[j] = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                                 std::chrono::steady_clock::now() - t0)
                                 .count();
            }
        }
        if (total_ms) {
            *total_ms = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        return HRM_OK;
    } catch (std::invalid_argument& e) {
        return hrm_capi::set_error(HRM_EINVAL, e.what());
    } catch (std::exception& e) {
        return hrm_capi::set_error(HRM_ECUDA, e.what());
    }
}

int hrm_solo_run(const hrm_job* jobs, uint32_t njobs, int variant, uint32_t nlanes, uint64_t* done_ns,
                 float* total_ms) {
    if (jobs == nullptr && njobs != 0) return hrm_capi::set_error(HRM_EINVAL, "jobs is NULL");
    if (nlanes == 0 || nlanes > 8) return hrm_capi::set_error(HRM_EINVAL, "nlanes must be 1..8");
    try {
        for (uint32_t j = 0; j < njobs; j++) {
            validate(jobs[j]);
            if (jobs[j].kind != HRM_JOB_PHOTON) throw std::invalid_argument("hrm_solo_run takes photon jobs only");
        }
        if (njobs == 0) {
            if (total_ms) *total_ms = 0.0f;
            return HRM_OK;
        }
        int dev = 0;
        ck(cudaGetDevice(&dev), "cudaGetDevice");
        const size_t teams = hrm_capi::photon_resident_teams(variant);
        const size_t lane_groups = std::max<size_t>(2, (teams / nlanes) & ~(size_t)1);
        std::vector<cudaStream_t> streams(nlanes, nullptr);
        auto release = hrm_capi::on_scope_exit([&] {
            for (auto& st : streams)
                if (st) cudaStreamDestroy(st);
        });
        for (auto& st : streams) ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
        ck(cudaDeviceSynchronize(), "sync");
        std::atomic<uint32_t> next{0};
        std::atomic<bool> failed{false};
        std::mutex err_lock;
        int err_code = HRM_OK;
        std::string err_msg;
        const auto t0 = std::chrono::steady_clock::now();
        auto lane_main = [&](unsigned int lane) {
            if (cudaSetDevice(dev) != cudaSuccess) {
                failed = true;
                return;
            }
            hrm_run_config cfg;
            memset(&cfg, 0, sizeof(cfg));
            cfg.program_type = HRM_ASYNC;
            cfg.variant = variant;
            cfg.stream = streams[lane];
            cfg.groups = nlanes > 1 ? lane_groups : 0;
            while (!failed) {
                const uint32_t j = next++;
                if (j >= njobs) break;
                const hrm_job& jb = jobs[j];
                hrm_run_result res;
                const int rc = hrm_capi::photon_walk_lane(lane, (const float*)jb.a, (const float*)jb.b,
                                                          (const uint8_t*)jb.c, jb.n, jb.seed, jb.first, jb.count,
                                                          (uint64_t*)jb.out, &cfg, &res);
                if (rc != HRM_OK) {
                    std::lock_guard<std::mutex> g(err_lock);
                    if (err_code == HRM_OK) {
                        err_code = rc;
                        err_msg = hrm_last_error();
                    }
                    failed = true;
                    break;
                }
                if (done_ns) {
                    done_ns[j] = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                                     std::chrono::steady_clock::now() - t0)
                                     .count();
                }
            }
        };
        std::vector<std::thread> threads;
        for (unsigned int lane = 1; lane < nlanes; lane++) threads.emplace_back(lane_main, lane);
        lane_main(0);
        for (auto& t : threads) t.join();
        if (total_ms) {
            *total_ms = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        if (err_code != HRM_OK) return hrm_capi::set_error(err_code, err_msg);
        if (failed) return hrm_capi::set_error(HRM_ECUDA, "cudaSetDevice failed on a lane thread");
        return HRM_OK;
    } catch (std::invalid_argument& e) {
        return hrm_capi::set_error(HRM_EINVAL, e.what());
    } catch (std::exception& e) {
        return hrm_capi::set_error(HRM_ECUDA, e.what());
    }
}

int hrm_plain_run(const hrm_job* jobs, uint32_t njobs, uint32_t nstreams, uint64_t* done_ns, float* total_ms) {
    if (jobs == nullptr && njobs != 0) return hrm_capi::set_error(HRM_EINVAL, "jobs is NULL");
    if (nstreams == 0) nstreams = 1;
    std::vector<cudaStream_t> streams(nstreams, nullptr);
    std::vector<cudaEvent_t> ev(njobs, nullptr);
    cudaEvent_t e0 = nullptr;
    unsigned int* d_overflow = nullptr;
    unsigned int* d_frontiers = nullptr;
    try {
        size_t max_nv = 0;
        for (uint32_t j = 0; j < njobs; j++) {
            validate(jobs[j]);
            if (jobs[j].kind == HRM_JOB_BFS && jobs[j].n > max_nv) max_nv = jobs[j].n;
        }
        for (auto& s : streams) ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        for (auto& e : ev) ck(cudaEventCreate(&e), "event");
        ck(cudaEventCreate(&e0), "event");
        ck(cudaMalloc((void**)&d_overflow, 4), "overflow flag");
        ck(cudaMemset(d_overflow, 0, 4), "overflow flag");
        if (max_nv) ck(cudaMalloc((void**)&d_frontiers, max_nv * 2 * 4 * nstreams), "frontiers");
        ck(cudaDeviceSynchronize(), "sync");
        ck(cudaEventRecord(e0, 0), "event");
        for (uint32_t j = 0; j < njobs; j++) {
            cudaStream_t s = streams[j % nstreams];
            ck(cudaStreamWaitEvent(s, e0, 0), "wait");
            const hrm_job& jb = jobs[j];
            if (jb.kind == HRM_JOB_COLLATZ) {
                if (jb.count) collatz_plain_kernel<<<(jb.count + 127) / 128, 128, 0, s>>>(jb.first, jb.count,
                                                                                       (unsigned int*)jb.out);
            } else if (jb.kind == HRM_JOB_PHOTON) {
                size_t slots = (size_t)jb.n * jb.n * jb.n + 3u * hrm_specs::PHOTON_SPREAD;
                ck(cudaMemsetAsync(jb.out, 0, slots * 8u, s), "tally clear");
                hrm_specs::PhotonState st;
                st.mu_s = (const float*)jb.a;
                st.absorb = (const float*)jb.b;
                st.split = (const unsigned char*)jb.c;
                st.tally = (unsigned long long*)jb.out;
                st.source = nullptr;
                st.n = jb.n;
                st.seed_lo = (unsigned int)jb.seed;
                st.seed_hi = (unsigned int)(jb.seed >> 32);
                st.leap = 1;
                st.load_limit = 2.0f;
                if (jb.count) photon_plain_kernel<<<(jb.count + 127) / 128, 128, 0, s>>>(st, jb.first, jb.count,
                                                                                      d_overflow);
            } else {
                unsigned int* fr = d_frontiers + (size_t)(j % nstreams) * max_nv * 2;
                bfs_plain_block_kernel<<<1, 1024, 0, s>>>((const unsigned int*)jb.a, (const unsigned int*)jb.b, jb.n,
                                                          jb.first, (unsigned int*)jb.out, fr, fr + max_nv);
            }
            ck(cudaGetLastError(), "plain launch");
            ck(cudaEventRecord(ev[j], s), "event");
        }
        ck(cudaDeviceSynchronize(), "plain run");
        float last = 0;
        for (uint32_t j = 0; j < njobs; j++) {
            float ms = 0;
            ck(cudaEventElapsedTime(&ms, e0, ev[j]), "elapsed");
            if (done_ns) done_ns[j] = (uint64_t)((double)ms * 1e6);
            if (ms > last) last = ms;
        }
        if (total_ms) *total_ms = last;
        unsigned int ovf = 0;
        ck(cudaMemcpy(&ovf, d_overflow, 4, cudaMemcpyDeviceToHost), "overflow flag");
        for (auto& s : streams) cudaStreamDestroy(s);
        for (auto& e : ev) cudaEventDestroy(e);
        cudaEventDestroy(e0);
        cudaFree(d_overflow);
        if (d_frontiers) cudaFree(d_frontiers);
        if (ovf) return hrm_capi::set_error(HRM_EDEVICE, "a plain photon walk overflowed its per-thread stack");
        return HRM_OK;
    } catch (std::invalid_argument& e) {
        return hrm_capi::set_error(HRM_EINVAL, e.what());
    } catch (std::exception& e) {
        for (auto& s : streams) if (s) cudaStreamDestroy(s);
        for (auto& e2 : ev) if (e2) cudaEventDestroy(e2);
        if (e0) cudaEventDestroy(e0);
        if (d_overflow) cudaFree(d_overflow);
        if (d_frontiers) cudaFree(d_frontiers);
        return hrm_capi::set_error(HRM_ECUDA, e.what());
    }
}

}  // extern "C"
