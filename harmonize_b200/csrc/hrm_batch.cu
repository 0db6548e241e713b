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

#include <cstddef>
#include <map>
#include <memory>
#include <mutex>
#include <string>
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

    // Captures: timestamp, output preparation, init<P>, exec<P>.
    void capture(size_t groups, size_t cycles) {
        if (graph && groups == graph_groups && cycles == graph_cycles) return;
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
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
        capture(groups, cycles);
        unsigned int ctr[8] = {n, 0u, 0u, 0u, closed0, 0u, 0u, 0u};
        ck(cudaMemcpyAsync(jobs.data(), recs.data(), sizeof(JobRecord) * n, cudaMemcpyHostToDevice, stream), "jobs");
        ck(cudaMemcpyAsync(counters.data(), ctr, sizeof(ctr), cudaMemcpyHostToDevice, stream), "counters");
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        ck(cudaEventRecord(e0, stream), "event");
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
        ck(cudaEventRecord(e1, stream), "event");
        ck(cudaEventSynchronize(e1), "event");
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
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
        default: throw std::invalid_argument("batched runs support variants R2/T4, R4/T4 and R4/T2");
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

}  // namespace

extern "C" {

int hrm_batch_run(const hrm_job* jobs, uint32_t njobs, const hrm_run_config* cfg_in, hrm_run_result* res,
                  uint64_t* done_ns) {
    if (jobs == nullptr && njobs != 0) return hrm_capi::set_error(HRM_EINVAL, "jobs is NULL");
    try {
        hrm_run_config cfg;
        memset(&cfg, 0, sizeof(cfg));
        if (cfg_in) cfg = *cfg_in;
        if (cfg.program_type != HRM_ASYNC) throw std::invalid_argument("batched runs use AsyncProgram");
        for (uint32_t j = 0; j < njobs; j++) validate(jobs[j]);
        size_t arena = cfg.arena ? cfg.arena : ((size_t)1 << 21);
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
