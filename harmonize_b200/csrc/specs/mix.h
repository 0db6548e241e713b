// mix.h — many independent program instances ("jobs") of mixed specs in one program.
//
// Batched and serving runs of this runtime (no counterpart in Harmonize, which runs one
// program instance per launch). Every async function F of the Collatz, photon-walk and BFS
// specs appears once as Job<F>, whose promises carry the job id in front of F's own
// arguments. The inner spec code is unchanged: its evals receive a JobProgram whose
// `device` is the job's own state and whose async<G>(...) becomes async<Job<G>>(job, ...).
// So the jobs share the runtime's per-function queues and coalescing: Collatz steps of
// different jobs fill one warp-full batch together, which is what makes thousands of small
// instances efficient in one persistent launch.
//
// Per job: its spec state (with a source iterator embedded in the job record), a count of
// pending work `pending` (promises alive, plus one token per make_work in progress),
// admission and completion timestamps (%globaltimer, ns) and a done flag. A job is done
// when `pending` returns to zero with its source exhausted; every change of `pending` is
// one atomicAdd per (warp, job) after __match_any_sync grouping.
//
// Serving: the host appends job records and then raises `admitted` (device memory, written
// while the persistent kernel runs); make_work picks jobs among [0, admitted) that still
// have sources, and keeps returning true while the session is open, so teams poll for new
// jobs instead of terminating; completions are also written to a host-mapped array.
#ifndef HRM_SPECS_MIX_H
#define HRM_SPECS_MIX_H

#include "bfs.h"
#include "collatz.h"
#include "photon.h"

namespace hrm_specs {

enum JobKind : unsigned int { JOB_COLLATZ = 0u, JOB_PHOTON = 1u, JOB_BFS = 2u };

// One job per 128-byte-aligned record: records never share a cache line, so a team that
// reads an admitted record cannot pull a not-yet-written neighbour into its SM's L1 (records
// are written by the host while the serving kernel runs).
struct alignas(128) JobRecord {
    unsigned int kind;
    int pending;                                 // promises alive + make_work tokens
    unsigned int done;                           // 1 once complete
    unsigned int source_closed;                  // 1 once a make_work saw the source exhausted
    unsigned long long t_admit;                  // %globaltimer when first worked on
    unsigned long long t_done;                   // %globaltimer at completion
    util::iter::AtomicIter<unsigned int> source; // the job's start values / photon ids / root
    unsigned int pad[2];
    union State {
        CollatzState c;
        PhotonState p;
        BfsState b;
    } s;
};

struct MixState {
    JobRecord* jobs;
    unsigned int* admitted;        // jobs [0, *admitted) may be worked on
    unsigned int* cursor;          // round-robin job cursor of make_work
    unsigned int* open;            // 1 while more jobs may still be admitted (serving)
    unsigned int* completed;       // number of completed jobs
    unsigned int* closed;          // number of jobs whose source is exhausted (host closes
                                   // jobs with no source at all when it admits them)
    unsigned int* low;             // every job below this index has an exhausted source
    unsigned long long* done_host; // host-mapped: t_done of each job (0 = not done), or null
    unsigned int njobs;            // capacity of the job table
};

// The state type of an inner async function.
template <typename F>
struct JobStateOf;
template <>
struct JobStateOf<CollatzEven> {
    using type = CollatzState;
    HRM_HD static CollatzState& get(JobRecord& r) { return r.s.c; }
};
template <>
struct JobStateOf<CollatzOdd> : JobStateOf<CollatzEven> {};
template <>
struct JobStateOf<PhotonMove> {
    using type = PhotonState;
    HRM_HD static PhotonState& get(JobRecord& r) { return r.s.p; }
};
template <>
struct JobStateOf<PhotonCollide> : JobStateOf<PhotonMove> {};
template <>
struct JobStateOf<PhotonTally> : JobStateOf<PhotonMove> {};
template <>
struct JobStateOf<BfsRelax> {
    using type = BfsState;
    HRM_HD static BfsState& get(JobRecord& r) { return r.s.b; }
};
template <>
struct JobStateOf<BfsExpand> : JobStateOf<BfsRelax> {};

template <typename F>
struct Job;

// Function pointer type with the job id prepended.
template <typename T>
struct PrependJob;
template <typename R, typename... A>
struct PrependJob<R (*)(A...)> {
    using type = R (*)(unsigned int, A...);
};

HRM_DEV HRM_FI unsigned long long global_ns() {
#if defined(__CUDA_ARCH__)
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
#else
    return 0ull;
#endif
}

// Marks job j complete (once) and publishes the completion.
HRM_DEV HRM_FI void job_complete(const MixState& st, unsigned int j) {
#if defined(__CUDA_ARCH__)
    JobRecord& r = st.jobs[j];
    if (atomicCAS(&r.done, 0u, 1u) == 0u) {
        unsigned long long t = global_ns();
        r.t_done = t;
        __threadfence();
        atomicAdd(st.completed, 1u);
        if (st.done_host != nullptr) {
            volatile unsigned long long* h = st.done_host;
            h[j] = t;
            __threadfence_system();
        }
    }
#endif
}

// Adds `delta` to job j's pending count, one atomic per group of lanes with the same job;
// completes the job when the count returns to zero with its source exhausted.
HRM_DEV HRM_FI void job_settle(const MixState& st, unsigned int j, int delta) {
#if defined(__CUDA_ARCH__)
    unsigned int mask = __activemask();
    unsigned int grp = __match_any_sync(mask, j);
    int sum = (int)__reduce_add_sync(grp, (unsigned int)delta);
    unsigned int lane;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(lane));
    if (lane == (unsigned int)(__ffs(grp) - 1) && sum != 0) {
        __threadfence();
        int old = atomicAdd(&st.jobs[j].pending, sum);
        if (old + sum == 0 && st.jobs[j].source.done()) job_complete(st, j);
    }
#endif
}

// The program handed to an inner spec's code: the job's state, asyncs tagged with the job id.
template <typename OUTER, typename STATE>
struct JobProgram {
    OUTER outer;
    STATE& device;
    unsigned int job;
    int* delta;

    template <typename F, typename... A>
    HRM_DEV HRM_FI void async(A... a) {
        outer.template async<Job<F>>(job, a...);
        *delta += 1;
    }
    template <typename F, typename... A>
    HRM_DEV HRM_FI void sync(A... a) {
        Promise<F>(a...)(*this);
    }
    template <typename F>
    HRM_DEV HRM_FI float load_fraction() {
        return outer.template load_fraction<Job<F>>();
    }
    HRM_DEV HRM_FI void halt_early() {}
};

template <typename F>
struct Job {
    using Type = typename PrependJob<typename F::Type>::type;
    using Inner = F;
    template <typename PROGRAM, typename... A>
    HRM_DEV static void eval(PROGRAM prog, unsigned int job, A... a) {
        using S = typename JobStateOf<F>::type;
        const MixState& st = prog.device;
        S& inner_state = JobStateOf<F>::get(st.jobs[job]);
        int delta = -1;
        JobProgram<PROGRAM, S> jp{prog, inner_state, job, &delta};
        F::template eval<JobProgram<PROGRAM, S>>(jp, a...);
        job_settle(st, job, delta);
    }
};

// Starts work of job j for the calling lane: its share of the job's sources.
template <typename PROGRAM>
HRM_DEV HRM_FI int job_make_work(PROGRAM prog, const MixState& st, unsigned int j) {
    JobRecord& r = st.jobs[j];
    int delta = 0;
    const unsigned int kind = *(volatile unsigned int*)&r.kind;
    if (kind == JOB_COLLATZ) {
        JobProgram<PROGRAM, CollatzState> jp{prog, r.s.c, j, &delta};
        CollatzSpec<>::template make_work<JobProgram<PROGRAM, CollatzState>>(jp);
    } else if (kind == JOB_PHOTON) {
        JobProgram<PROGRAM, PhotonState> jp{prog, r.s.p, j, &delta};
        PhotonSpec<>::template make_work<JobProgram<PROGRAM, PhotonState>>(jp);
    } else {
        JobProgram<PROGRAM, BfsState> jp{prog, r.s.b, j, &delta};
        BfsSpec<>::template make_work<JobProgram<PROGRAM, BfsState>>(jp);
    }
    return delta;
}

template <size_t RING = 4, size_t TEAMS = 4>
struct MixSpec {
    typedef OpUnion<Job<CollatzEven>, Job<CollatzOdd>, Job<PhotonMove>, Job<PhotonCollide>, Job<PhotonTally>,
                    Job<BfsRelax>, Job<BfsExpand>>
        OpSet;
    typedef MixState DeviceState;

    static const size_t STASH_SIZE = 16;
    static const size_t RING_LINKS = RING;
    static const size_t TEAMS_PER_CTA = TEAMS;

    template <typename PROGRAM>
    HRM_DEV static void initialize(PROGRAM) {}
    template <typename PROGRAM>
    HRM_DEV static void finalize(PROGRAM) {}

    // Called by a whole team: picks one job that still has sources (round robin over the
    // admitted jobs), takes a token on it, makes its share of work, settles the count.
    template <typename PROGRAM>
    HRM_DEV static bool make_work(PROGRAM prog) {
#if defined(__CUDA_ARCH__)
        const MixState& st = prog.device;
        unsigned int lane;
        asm volatile("mov.u32 %0, %%laneid;" : "=r"(lane));
        unsigned int admitted = *(volatile unsigned int*)st.admitted;
        unsigned int j = 0xFFFFFFFFu;
        if (lane == 0 && admitted > 0) {
            // Advance the low watermark past jobs whose sources are exhausted, then probe
            // round robin among [low, admitted).
            unsigned int low = *(volatile unsigned int*)st.low;
            while (low < admitted && *(volatile unsigned int*)&st.jobs[low].source_closed) {
                low = atomicCAS(st.low, low, low + 1u) == low ? low + 1u : *(volatile unsigned int*)st.low;
            }
            unsigned int span = admitted > low ? admitted - low : 1u;
            for (unsigned int tries = 0; tries < 64u; tries++) {
                unsigned int c = low + atomicAdd(st.cursor, 1u) % span;
                if (c >= admitted) break;
                JobRecord& r = st.jobs[c];
                if (!r.source.done() && *(volatile unsigned int*)&r.done == 0u) {
                    j = c;
                    atomicAdd(&r.pending, 1);  // token: the job cannot complete mid make_work
                    if (r.t_admit == 0ull) r.t_admit = global_ns();
                    break;
                }
            }
        }
        j = __shfl_sync(0xFFFFFFFFu, j, 0);
        if (j == 0xFFFFFFFFu) {
            // No job found in this probe. Keep making work while any admitted job still has
            // sources, and while the session is open (serving teams poll for new jobs).
            unsigned int closed = *(volatile unsigned int*)st.closed;
            bool open = *(volatile unsigned int*)st.open != 0u;
            bool left = closed < *(volatile unsigned int*)st.admitted;
            if (!left && open) __nanosleep(2000);
            return open || left;
        }
        int delta = job_make_work(prog, st, j);
        __syncwarp();
        delta = (int)__reduce_add_sync(0xFFFFFFFFu, (unsigned int)delta);
        if (lane == 0) {
            JobRecord& r = st.jobs[j];
            if (r.source.done() && atomicCAS(&r.source_closed, 0u, 1u) == 0u) atomicAdd(st.closed, 1u);
            __threadfence();
            int old = atomicAdd(&r.pending, delta - 1);
            if (old + delta - 1 == 0 && r.source.done()) job_complete(st, j);
        }
        return true;
#else
        (void)prog;
        return false;
#endif
    }
};

}  // namespace hrm_specs

#endif
