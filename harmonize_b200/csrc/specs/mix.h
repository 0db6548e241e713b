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
// when `pending` returns to zero with its source exhausted; changes of `pending` are
// grouped per (warp, job) with __match_any_sync and collected in a per-team table that is
// published in batches (see the bookkeeping notes below).
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
enum JobOrder : unsigned int { JOB_ORDER_ROUND_ROBIN = 0u, JOB_ORDER_ADMISSION = 1u, JOB_ORDER_SMALL_FIRST = 2u };

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
    unsigned int large;                          // 1: large job, served last by JOB_ORDER_SMALL_FIRST
    unsigned int pad;
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
    unsigned int* started;         // jobs that have received their first make_work
    unsigned int max_active;       // a job starts only while started - completed < max_active
    unsigned int job_order;        // JOB_ORDER_ROUND_ROBIN or JOB_ORDER_ADMISSION (make_work)
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

// Pending-count bookkeeping (the mix spec's GroupState, in shared memory).
//
// Each evaluation records, in its lane's slot, its job and its change of that job's count
// (promises created minus the one consumed). After the batch the whole team settles the
// slots together (after_batch): lanes are grouped by job and each group's net change is
// added to a small per-team table keyed by job. Increases in the table are published
// (relaxed atomics) before any promise of the team becomes visible to other teams
// (before_publish: spills, overflow links held during a step) and when evicted; decreases
// (one fence per flush, with the completion check) when evicted, every FLUSH_EVERY batches,
// and whenever the team runs out of work (make_work, on_idle, finalize).
//
// Why this is safe. Let D_t be team t's unpublished net change of a job. If D_t > 0, look at
// the last moment t published promises (or the entry's creation): D_t was <= 0 then, so
// since then t made more promises than it consumed; those promises are all still in t's
// rings or were consumed by t (nothing was published since), and t made them by consuming
// older promises, so D_t is at most (the job's promises alive in t's rings) - 1. The
// published count is (promises alive) - sum of D_t, which is therefore at least one while
// any promise is alive and never below zero; it reaches zero only when no promise is alive
// and nothing is held: a job is declared complete exactly when it is.
struct MixTeam {
    static const unsigned int SLOTS = 16;
    static const unsigned int FLUSH_EVERY = 64;
    static const unsigned int EMPTY = 0xFFFFFFFFu;
    unsigned int lane_job[32];  // job of the lane's evaluation in this batch, or EMPTY
    int lane_delta[32];
    unsigned int job[SLOTS];
    int delta[SLOTS];
    unsigned int settles;
    unsigned int used;  // bit s set while job[s] holds an entry
};

// One lane: publishes a decrease of job j's count, completing the job at zero with its
// source exhausted. The fence orders this team's writes of the job's results before the count.
HRM_DEV HRM_FI void job_publish(const MixState& st, unsigned int j, int d) {
#if defined(__CUDA_ARCH__)
    __threadfence();
    int old = atomicAdd(&st.jobs[j].pending, d);
    if (old + d == 0 && st.jobs[j].source.done()) job_complete(st, j);
#endif
}

// Publishing a net increase never completes a job (the published count is never below
// zero, so it rises from zero or more) and orders nothing: a relaxed atomic, no fence.
HRM_DEV HRM_FI void job_raise(const MixState& st, unsigned int j, int d) {
#if defined(__CUDA_ARCH__)
    atomicAdd(&st.jobs[j].pending, d);
#endif
}

// One lane: publishes the team table's increases (negatives = false) or every entry.
HRM_DEV HRM_FI void team_flush(const MixState& st, MixTeam& t, bool negatives) {
#if defined(__CUDA_ARCH__)
    unsigned int used = t.used;
    bool fenced = false;
    while (used) {
        const unsigned int s = __ffs(used) - 1;
        used &= used - 1;
        const int d = t.delta[s];
        if (d < 0 && !negatives) continue;
        if (d > 0) {
            job_raise(st, t.job[s], d);
        } else if (d < 0) {
            if (!fenced) {
                __threadfence();  // this team's writes of job results before the counts
                fenced = true;
            }
            const int old = atomicAdd(&st.jobs[t.job[s]].pending, d);
            if (old + d == 0 && st.jobs[t.job[s]].source.done()) job_complete(st, t.job[s]);
        }
        t.job[s] = MixTeam::EMPTY;
        t.used &= ~(1u << s);
    }
    if (negatives) t.settles = 0u;
#endif
}

// One lane: adds a change of job j's count to the team table.
HRM_DEV HRM_FI void team_defer(const MixState& st, MixTeam& t, unsigned int j, int d) {
    const unsigned int s = j & (MixTeam::SLOTS - 1u);
    const unsigned int bit = 1u << s;
    if ((t.used & bit) != 0u && t.job[s] == j) {
        t.delta[s] += d;
        return;
    }
    if ((t.used & bit) != 0u) {  // evict the other job
        const int e = t.delta[s];
        if (e > 0) job_raise(st, t.job[s], e);
        else if (e < 0) job_publish(st, t.job[s], e);
    }
    t.job[s] = j;
    t.delta[s] = d;
    t.used |= bit;
}

// Whole team, converged: settles the lane slots of the batch just evaluated.
HRM_DEV HRM_FI void team_settle(const MixState& st, MixTeam& t) {
#if defined(__CUDA_ARCH__)
    unsigned int lane;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(lane));
    const unsigned int j = t.lane_job[lane];
    const int delta = t.lane_delta[lane];
    t.lane_job[lane] = MixTeam::EMPTY;
    const unsigned int grp = __match_any_sync(0xFFFFFFFFu, j);
    const int sum = (int)__reduce_add_sync(grp, (unsigned int)delta);
    const bool leader = j != MixTeam::EMPTY && lane == (unsigned int)(__ffs(grp) - 1);
    unsigned int defer = __ballot_sync(0xFFFFFFFFu, leader && sum != 0);
    // One lane at a time updates the table (it belongs to this team alone).
    while (defer) {
        const unsigned int src = __ffs(defer) - 1;
        defer &= defer - 1;
        if (lane == src) team_defer(st, t, j, sum);
        __syncwarp();
    }
    if (lane == 0 && ++t.settles >= MixTeam::FLUSH_EVERY) team_flush(st, t, true);
    __syncwarp();
#endif
}

// Whole team: publishes the table's increases, or (negatives) every entry.
HRM_DEV HRM_FI void team_flush_all(const MixState& st, MixTeam& t, bool negatives = true) {
#if defined(__CUDA_ARCH__)
    __syncwarp();
    unsigned int lane;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(lane));
    if (lane == 0) team_flush(st, t, negatives);
    __syncwarp();
#endif
}

// The program handed to an inner spec's code: the job's state, asyncs tagged with the job id.
template <typename OUTER, typename STATE>
struct JobProgram {
    OUTER outer;
    STATE& device;
    unsigned int job;
    int* delta;  // promises made by this lane for its job (settled by the team later)

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
        // A copy in registers: the inner evals only read their state (the pointers in it
        // lead to the job's buffers), and a register copy saves re-loading the job record
        // after every store the eval makes.
        S inner_state = JobStateOf<F>::get(st.jobs[job]);
        int delta = -1;  // the consumed promise
        JobProgram<PROGRAM, S> jp{prog, inner_state, job, &delta};
        F::template eval<JobProgram<PROGRAM, S>>(jp, a...);
        // Settled by the whole team after the batch (after_batch).
        MixTeam& t = prog.group;
        const unsigned int lane = util::lane_id();
        t.lane_job[lane] = job;
        t.lane_delta[lane] = delta;
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

// The functions of each job kind form one ring group (RING_GROUP_OF): a kind never calls
// another kind's functions, so a team holds promises of one kind at a time and the three
// kinds' rings share one stash, as large as the photon rings alone. RING: ring links of the
// photon functions (a move carries a whole photon, 12 words with the job id, a collide 9;
// every collide batch feeds a batch of tallies, so each needs room for several batches;
// collides get half); the Collatz and BFS functions, with 5 words or fewer, get 2*RING links.
template <size_t RING = 4, size_t TEAMS = 4>
struct MixSpec {
    typedef OpUnion<Job<CollatzEven>, Job<CollatzOdd>, Job<PhotonMove>, Job<PhotonCollide>, Job<PhotonTally>,
                    Job<BfsRelax>, Job<BfsExpand>>
        OpSet;
    typedef MixState DeviceState;
    typedef MixTeam GroupState;

    static const size_t STASH_SIZE = 16;
    static const size_t RING_LINKS = 2;
    static const size_t TEAMS_PER_CTA = TEAMS;
    template <typename Op>
    struct RING_GROUP_OF {
        static const unsigned int value =
            (std::is_same<Op, Job<CollatzEven>>::value || std::is_same<Op, Job<CollatzOdd>>::value) ? JOB_COLLATZ
            : (std::is_same<Op, Job<BfsRelax>>::value || std::is_same<Op, Job<BfsExpand>>::value)  ? JOB_BFS
                                                                                                      : JOB_PHOTON;
    };
    // Photon collides get half the photon ring (at least 2 links): a batch of moves makes at
    // most one collide per lane.
    template <typename Op>
    struct RING_LINKS_OF {
        static const size_t value =
            std::is_same<Op, Job<PhotonCollide>>::value ? (RING / 2 < 2 ? 2 : RING / 2)
            : RING_GROUP_OF<Op>::value == JOB_PHOTON    ? RING
                                                        : 2 * RING;
    };
    // BFS jobs take their teams' oldest calls first, as the BFS spec does on its own.
    template <typename Op>
    struct OLDEST_FIRST_OF {
        static const bool value = RING_GROUP_OF<Op>::value == JOB_BFS;
    };

    template <typename PROGRAM>
    HRM_DEV static void initialize(PROGRAM prog) {
        MixTeam& t = prog.group;
        const unsigned int lane = util::lane_id();
        t.lane_job[lane] = MixTeam::EMPTY;
        t.lane_delta[lane] = 0;
        if (lane < MixTeam::SLOTS) t.job[lane] = MixTeam::EMPTY;
        if (lane == 0) {
            t.settles = 0;
            t.used = 0;
        }
        __syncwarp();
    }
    template <typename PROGRAM>
    HRM_DEV static void finalize(PROGRAM prog) {
        team_flush_all(prog.device, prog.group);
    }
    template <typename PROGRAM>
    HRM_DEV static void on_idle(PROGRAM prog) {
        team_flush_all(prog.device, prog.group);
    }
    template <typename PROGRAM>
    HRM_DEV static void after_batch(PROGRAM prog) {
        team_settle(prog.device, prog.group);
    }
    template <typename PROGRAM>
    HRM_DEV static void before_publish(PROGRAM prog) {
        team_flush_all(prog.device, prog.group, false);  // increases only: decreases may wait
    }

    // Called by a whole team: picks one job that still has sources (round robin over the
    // admitted jobs), takes a token on it, makes its share of work, settles the count.
    template <typename PROGRAM>
    HRM_DEV static bool make_work(PROGRAM prog) {
#if defined(__CUDA_ARCH__)
        const MixState& st = prog.device;
        team_flush_all(st, prog.group);
        unsigned int lane;
        asm volatile("mov.u32 %0, %%laneid;" : "=r"(lane));
        unsigned int admitted = *(volatile unsigned int*)st.admitted;
        unsigned int j = 0xFFFFFFFFu;
        if (lane == 0 && admitted > 0) {
            // Advance the low watermark past jobs whose sources are exhausted, then probe
            // round robin among [low, admitted).
            unsigned int low = *(volatile unsigned int*)st.low;
            while (low < admitted) {
                JobRecord& lr = st.jobs[low];
                if (*(volatile unsigned int*)&lr.source_closed == 0u) {
                    // A job whose source is exhausted but that no make_work closed yet (one
                    // the host serves outside this kernel arrives that way) is closed here.
                    if (!lr.source.done()) break;
                    if (atomicCAS(&lr.source_closed, 0u, 1u) == 0u) atomicAdd(st.closed, 1u);
                }
                low = atomicCAS(st.low, low, low + 1u) == low ? low + 1u : *(volatile unsigned int*)st.low;
            }
            unsigned int span = admitted > low ? admitted - low : 1u;
            // Round robin spreads the teams over all jobs in progress (they share the GPU);
            // admission order gives the oldest job with work left every team that asks, so
            // jobs finish nearly one after another, each at nearly full speed; small first
            // does the same among the small jobs, and serves large ones when no small job has
            // work left to start.
            const bool rr = st.job_order == JOB_ORDER_ROUND_ROBIN;
            const unsigned int passes = st.job_order == JOB_ORDER_SMALL_FIRST ? 2u : 1u;
            for (unsigned int tries = 0; tries < 64u * passes && j == 0xFFFFFFFFu; tries++) {
                const bool small_only = passes == 2u && tries < 64u;
                unsigned int c = rr ? low + atomicAdd(st.cursor, 1u) % span : low + (tries & 63u);
                if (c >= admitted) {
                    if (small_only) {
                        tries = 63u;  // on to the second pass
                        continue;
                    }
                    break;
                }
                JobRecord& r = st.jobs[c];
                if (small_only && r.large) continue;
                if (!r.source.done() && *(volatile unsigned int*)&r.done == 0u) {
                    if (*(volatile unsigned long long*)&r.t_admit == 0ull) {
                        // Not started yet: start it only while fewer than max_active jobs
                        // are in progress (bounds the promises in flight).
                        unsigned int active = *(volatile unsigned int*)st.started -
                                              *(volatile unsigned int*)st.completed;
                        if (active >= st.max_active) continue;
                        if (atomicCAS(&r.t_admit, 0ull, global_ns()) == 0ull) atomicAdd(st.started, 1u);
                    }
                    j = c;
                    atomicAdd(&r.pending, 1);  // token: the job cannot complete mid make_work
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
            // Publish the promises made and return the token (the runtime publishes the
            // promises that overflowed to the arena only after make_work returns).
            JobRecord& r = st.jobs[j];
            if (r.source.done() && atomicCAS(&r.source_closed, 0u, 1u) == 0u) atomicAdd(st.closed, 1u);
            job_publish(st, j, delta - 1);
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
