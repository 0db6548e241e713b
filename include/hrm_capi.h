/* hrm_capi.h — C ABI of the B200-native Harmonize runtime (libhrm.so).
 *
 * The original exposes each specialised program to foreign callers through a generated
 * C shim per spec (harmonize/python/templates.py:3-184, bound by
 * harmonize/python/runtime.py:1324-1408): alloc_program_S, init_program_S,
 * exec_program_S, complete_S, clear_flags_S, free_program_S, set_device_S. This library
 * exports the same life cycle for its built-in specs behind one set of entry points that
 * take the spec as an enum, with these differences:
 *   - every call returns an int status (HRM_OK or an HRM_E* code) instead of throwing
 *     through extern "C"; hrm_last_error() returns the message of the last failure on
 *     the calling thread;
 *   - launches take an optional CUDA stream (NULL = legacy default stream) and do not
 *     synchronise unless the call says so;
 *   - whole-run helpers (hrm_*_run) take HOST buffers, copy in, run to completion and
 *     copy out: the call an application makes.
 * No signature uses a C++ or torch type.
 */
#ifndef HRM_CAPI_H
#define HRM_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define HRM_OK 0
#define HRM_EINVAL 1        /* bad argument */
#define HRM_ECUDA 2         /* a CUDA runtime call failed */
#define HRM_EDEVICE 3       /* the device raised an error flag (see hrm_program_flags) */
#define HRM_EINCOMPLETE 4   /* the run did not complete within its exec budget */
#define HRM_ENOMEM 5        /* allocation failed */

/* Program types (one-line swappable in C++: AsyncProgram / EventProgram). */
#define HRM_ASYNC 0
#define HRM_EVENT 1

/* Built-in program specifications. */
#define HRM_SPEC_COLLATZ 0
#define HRM_SPEC_PHOTON 1
#define HRM_SPEC_BFS 2
#define HRM_SPEC_BARRIER_DEMO 3

/* Device status flags (same bit values as the original runtime where they exist). */
#define HRM_FLAG_BAD_FUNC_ID 0x00000001u
#define HRM_FLAG_STASH_FAIL 0x00000002u
#define HRM_FLAG_ARENA_EXHAUSTED 0x00000004u
#define HRM_FLAG_QUEUE_OVERFLOW 0x00000008u
#define HRM_FLAG_WAIT_TIMEOUT 0x00000010u
#define HRM_FLAG_EARLY_HALT 0x40000000u
#define HRM_FLAG_COMPLETION 0x80000000u

/* Runtime statistics, indices into the array filled by hrm_program_stats. */
#define HRM_STAT_EVALS 0
#define HRM_STAT_BATCHES 1
#define HRM_STAT_FULL_BATCHES 2
#define HRM_STAT_SPILL_LINKS 3
#define HRM_STAT_FILL_LINKS 4
#define HRM_STAT_MAKE_WORK 5
#define HRM_STAT_IDLE_POLLS 6
#define HRM_STAT_GENERATIONS 7
#define HRM_STAT_FN_EVALS 8   /* HRM_STAT_FN_EVALS + f: evaluations of async function f (f < 16) */
#define HRM_STAT_COUNT 24

typedef struct hrm_program hrm_program; /* opaque: one program instance on one device */

/* Execution parameters of a whole run. Zero fields take defaults. */
typedef struct hrm_run_config {
    int program_type;          /* HRM_ASYNC or HRM_EVENT */
    size_t groups;             /* 32-lane work groups; 0 = all that can be resident */
    size_t cycles;             /* AsyncProgram cycle budget per exec; 0 = 2^24 */
    size_t chunk;              /* EventProgram promises per lane per grab; 0 = 1 */
    size_t arena;              /* AsyncProgram arena links / EventProgram io_size; 0 = default */
    size_t max_execs;          /* exec calls before giving up with HRM_EINCOMPLETE; 0 = 4096 */
    void* stream;              /* cudaStream_t, NULL = default stream */
    int variant;               /* compiled tuning variant (see HRM_VARIANT_*), 0 = default */
    uint32_t patience;         /* AsyncProgram coalescing threshold: scheduling steps a partial
                                  batch may wait without growing before it runs; 0 = 16 */
    uint32_t fill_links;       /* AsyncProgram links one fill takes from the arena; 0 = 2 */
    uint32_t job_order;        /* batched and serving runs: HRM_JOB_ORDER_* (which job make_work serves) */
    uint32_t solo_photons;     /* serving sessions: photon jobs of at least this many photons run
                                  alone through the single-spec runtime (the resident kernel
                                  pauses meanwhile); 0 = never */
} hrm_run_config;

/* Job orders of batched and serving runs: round robin over the jobs in progress (they share
 * the GPU), admission order (the oldest job with work left gets every team that asks), or
 * small first (admission order among the jobs estimated to need fewer than about 5e7 async
 * calls, then among all). */
#define HRM_JOB_ORDER_ROUND_ROBIN 0u
#define HRM_JOB_ORDER_ADMISSION 1u
#define HRM_JOB_ORDER_SMALL_FIRST 2u

/* Compiled tuning variants: shared-memory ring per async function (in 32-promise links)
 * and 32-lane teams per CTA. EventProgram uses only the team count. */
#define HRM_VARIANT_R2_T4 0
#define HRM_VARIANT_R4_T4 1
#define HRM_VARIANT_R4_T2 2
#define HRM_VARIANT_R8_T2 3
#define HRM_VARIANT_R2_T8 4
/* Lean rings: the spec's first async function 4 links, the others 2, 2 teams per CTA, compiled
 * for at least 10 (M10) or 11 (M11) resident CTAs per SM (more teams per SM, fewer registers). */
#define HRM_VARIANT_LEAN_T2_M10 5
#define HRM_VARIANT_LEAN_T2_M11 6
/* 4-link rings, 2 teams per CTA, compiled for at least 11 resident CTAs per SM; 4-link rings,
 * 4 teams per CTA, at least 5 CTAs per SM (register caps that leave shared memory the only
 * limit on teams per SM). */
#define HRM_VARIANT_R4_T2_M11 7
#define HRM_VARIANT_R4_T4_M5 8
/* 3-link rings (the photon walk's Collide 2), 2 teams per CTA, compiled for at least 14 resident
 * CTAs per SM: a stash small enough for 14 CTAs of 2 teams in an SM's shared memory, and at most
 * 72 registers a thread so that 7 teams fit each SM sub-partition (28 warps per SM). */
#define HRM_VARIANT_R3_T2_M14 9
#define HRM_VARIANT_COUNT 10

/* What a whole run reports back. */
typedef struct hrm_run_result {
    uint32_t flags;            /* device flags after the last exec */
    uint32_t execs;            /* exec calls made */
    uint64_t stats[HRM_STAT_COUNT];
    float device_ms;           /* CUDA-event time of init + all execs */
} hrm_run_result;

const char* hrm_last_error(void);
int hrm_set_device(int device);
int hrm_device_sync(void);
/* The whole-run helpers (hrm_*_run*) keep one program instance per device, spec, program
 * type, variant and arena size, re-initialised by each run, so repeated runs allocate no
 * device memory; concurrent runs on the same cached instance are serialised. The host-buffer
 * runs (hrm_collatz_run, hrm_photon_run, hrm_bfs_run) likewise keep their device copies of
 * inputs and outputs per device, grown on demand, and run one at a time per device. This
 * frees both; what a run in progress on another thread uses is freed when that run ends. */
int hrm_release_cache(void);

/* ---- program life cycle (templates.py:3-184 counterparts) ------------------------------
 * hrm_program_create: spec + type + arena/io size + a copy of the spec's device state
 *   (the struct layouts are given by hrm_*_state below);
 * hrm_program_init: reset queues and flags (init<P>); hrm_program_exec: one exec<P>;
 * hrm_program_complete: *out = 1 when the last exec completed (throws nothing: an error
 *   flag returns HRM_EDEVICE). */
int hrm_program_create(int spec, int program_type, size_t arena_or_io, const void* device_state,
                       size_t state_size, hrm_program** out);
/* Same, choosing a compiled tuning variant (HRM_VARIANT_*). */
int hrm_program_create_variant(int spec, int program_type, int variant, size_t arena_or_io,
                               const void* device_state, size_t state_size, hrm_program** out);
int hrm_program_destroy(hrm_program* prog);
/* Replaces the instance's copy of the spec's device state (the next init / exec launch sees
 * it); the original passes its DeviceState by value into every launch (program/mod.h:66), so
 * a caller may change it between launches. */
int hrm_program_set_state(hrm_program* prog, const void* device_state, size_t state_size);
int hrm_program_init(hrm_program* prog, size_t groups, void* stream);
int hrm_program_exec(hrm_program* prog, size_t groups, size_t cycles_or_chunk, void* stream);
int hrm_program_complete(hrm_program* prog, int* out);
int hrm_program_flags(hrm_program* prog, uint32_t* out);
int hrm_program_clear_flags(hrm_program* prog);
int hrm_program_stats(hrm_program* prog, uint64_t* out, size_t n);
/* Host-side structure check (the role of runtime_overview in the original, async.h:2766):
 * AsyncProgram: out[0] links handed out, out[1] links on the free list, out[2+f] links queued
 * for function f, then tail-head of each ring; EventProgram: out[f] promises waiting for f.
 * *written receives the full length. */
int hrm_program_overview(hrm_program* prog, uint32_t* out, size_t n, size_t* written);

/* ---- built-in spec device states ------------------------------------------------------ */
typedef struct hrm_collatz_state {
    uint32_t start;            /* first start value */
    uint32_t limit;            /* one past the last start value */
    uint32_t* output;          /* device pointer: output[n - start] = stopping time of n */
    void* iterator;            /* device pointer to an AtomicIter<uint32> {value, limit} */
    uint32_t leap;             /* start values per lane per make_work call (0 = 1) */
} hrm_collatz_state;

typedef struct hrm_photon_state {
    const float* mu_s;         /* device: scattering coefficient per voxel (n^3) */
    const float* absorb;       /* device: absorbed fraction per collision per voxel */
    const uint8_t* split;      /* device: 1 = photons entering the voxel split in two */
    uint64_t* tally;           /* device: n^3 voxel tallies + 3*1024 escape/kill/gain slots,
                                  2^-32 fixed point */
    void* source;              /* device pointer to an AtomicIter<uint32> over photon ids */
    uint32_t n;                /* grid edge in voxels (even) */
    uint32_t seed_lo, seed_hi; /* Philox counter words 2 and 3 */
    uint32_t leap;             /* photons per lane per make_work call (0 = 1) */
    float load_limit;          /* EventProgram: launch no photons above this move-buffer load */
} hrm_photon_state;

typedef struct hrm_bfs_state {
    const uint32_t* rowptr;    /* device CSR row offsets (nv + 1) */
    const uint32_t* col;       /* device CSR targets */
    uint32_t* levels;          /* device, nv entries, pre-filled with 0xFFFFFFFF */
    void* roots;               /* device pointer to an AtomicIter<uint32> over [0, 1) */
    uint32_t root;
    uint32_t nv;
} hrm_bfs_state;

/* ---- whole runs (host buffers in and out) --------------------------------------------- */

/* Collatz stopping times of n = start .. start+count-1 into out_steps[count] (host). */
int hrm_collatz_run(uint32_t start, uint32_t count, uint32_t* out_steps, const hrm_run_config* cfg,
                    hrm_run_result* res);
/* Same, with a device output buffer (no host copies). */
int hrm_collatz_run_device(uint32_t start, uint32_t count, uint32_t* d_out_steps, const hrm_run_config* cfg,
                           hrm_run_result* res);

/* Photon walk of photons [first, first+count) over an n^3 medium (host arrays of n^3);
 * tally receives n^3 + 3*1024 uint64 slots (voxels, then escaped, roulette-killed and
 * roulette-gained weight, each spread over 1024 slots), in units of 2^-32. */
int hrm_photon_run(const float* mu_s, const float* absorb, const uint8_t* split, uint32_t n, uint64_t seed,
                   uint32_t first, uint32_t count, uint64_t* tally, const hrm_run_config* cfg,
                   hrm_run_result* res);
int hrm_photon_run_device(const float* d_mu_s, const float* d_absorb, const uint8_t* d_split, uint32_t n,
                          uint64_t seed, uint32_t first, uint32_t count, uint64_t* d_tally,
                          const hrm_run_config* cfg, hrm_run_result* res);

/* Breadth-first levels from `root` over a CSR graph (host arrays); unreached = 0xFFFFFFFF. */
int hrm_bfs_run(const uint32_t* rowptr, const uint32_t* col, uint32_t nv, uint32_t root, uint32_t* levels,
                const hrm_run_config* cfg, hrm_run_result* res);
int hrm_bfs_run_device(const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t nv, uint32_t root,
                       uint32_t* d_levels, const hrm_run_config* cfg, hrm_run_result* res);

/* Remapping-barrier workload (harmonize examples/cpp/barrier_demo/demo.cpp:20-86, which the
 * original runs as `demo dep=.. ndep=.. bar=..`): ids [0, dep+ndep) each run one Step; the
 * dependent ones (id < dep) hold a follow-up Step on RemappingBarrier id % bar and then
 * decrement it, each barrier starting at the number of dependent ids mapped to it; a
 * UnitBarrier armed with ndep releases one final Step after the non-dependent Steps.
 * counter[4] (host) receives: Steps run (2*dep + ndep + (ndep > 0)), non-dependent Steps,
 * final Steps, and violations (a follow-up that ran before its barrier released, or a final
 * Step that ran early; always 0). released[bar] (host) receives the follow-ups run per
 * barrier. AsyncProgram only (barriers keep held promises in the arena); bar >= 1. */
int hrm_barrier_demo_run(uint32_t dep_count, uint32_t non_dep_count, uint32_t barrier_count, uint32_t* counter,
                         uint32_t* released, const hrm_run_config* cfg, hrm_run_result* res);

/* Device state of HRM_SPEC_BARRIER_DEMO for hrm_program_create (device pointers). */
typedef struct hrm_barrier_demo_state {
    uint32_t dep_count, non_dep_count, barrier_count, pad;
    void* source;              /* AtomicIter<uint32> over [0, dep + ndep) */
    uint32_t* counter;         /* 4 counters, zeroed */
    uint32_t* released;        /* barrier_count counters, zeroed */
    void* barriers;            /* barrier_count RemappingBarrier values made by blank(wait count) */
    void* unit;                /* one UnitBarrier */
} hrm_barrier_demo_state;

/* ---- many independent jobs --------------------------------------------------------------
 * No counterpart in the original (one program instance per launch there). A job is one
 * instance of a built-in spec; all pointers are device pointers owned by the caller. */
#define HRM_JOB_COLLATZ 0
#define HRM_JOB_PHOTON 1
#define HRM_JOB_BFS 2
typedef struct hrm_job {
    uint32_t kind;      /* HRM_JOB_* */
    uint32_t first;     /* collatz: first start value; photon: first photon id; bfs: root */
    uint32_t count;     /* collatz: start values; photon: photons; bfs: unused */
    uint32_t n;         /* photon: grid edge (even); bfs: vertex count */
    uint64_t seed;      /* photon: Philox seed */
    const void* a;      /* photon: float mu_s[n^3]; bfs: uint32 rowptr[n+1] */
    const void* b;      /* photon: float absorb[n^3]; bfs: uint32 col[] */
    const void* c;      /* photon: uint8 split[n^3] */
    void* out;          /* collatz: uint32 steps[count]; photon: uint64 tally[n^3 + 3*1024];
                           bfs: uint32 levels[n] */
} hrm_job;

/* All jobs in ONE persistent AsyncProgram launch (job-multiplexing spec; the launch sequence
 * is a CUDA graph replayed per call). done_ns (host, njobs entries, may be NULL) receives each
 * job's completion time in ns after the start of the device work. cfg->variant: R2/T4, R4/T4,
 * R4/T2, R4/T2 M11 or R4/T4 M5. Outputs equal those of one run per job, bit for bit. The batch context (instance,
 * job table and graph, per device, variant, job capacity rounded up to a power of two and
 * arena) is kept for the next call until the process exits; calls on one context are
 * serialised. */
int hrm_batch_run(const hrm_job* jobs, uint32_t njobs, const hrm_run_config* cfg, hrm_run_result* res,
                  uint64_t* done_ns);
/* Baseline: one launch of a plain kernel per job (one thread per Collatz start value, one
 * thread per source photon with its descendants, one CTA per BFS), jobs round-robin over
 * nstreams streams. done_ns as above; *total_ms = time until the last job completed. */
int hrm_plain_run(const hrm_job* jobs, uint32_t njobs, uint32_t nstreams, uint64_t* done_ns, float* total_ms);
/* Baseline: plain execution of the runtime itself, one job at a time, as a program built on
 * the original would run them: for each job, one whole run of the single-spec program
 * (hrm_collatz/photon/bfs_run_device: init, exec until complete, synchronised). variants
 * (NULL = variant 0 for all) gives the compiled variant per job kind (HRM_JOB_*). done_ns
 * (host clock, ns from the first job's start) and *total_ms as above. */
int hrm_runtime_run(const hrm_job* jobs, uint32_t njobs, int program_type, const int* variants, uint64_t* done_ns,
                    float* total_ms);
/* Large photon jobs through the single-spec AsyncProgram (no counterpart in the original): the
 * jobs (all HRM_JOB_PHOTON) run in order over nlanes lanes (1..8), each lane a host thread
 * with its own stream and program instance and 1/nlanes of the teams that fit on the device,
 * so that one job's tail of dependent calls overlaps the others' work. variant: the compiled
 * photon variant. done_ns (host clock, ns from the start of the call) and *total_ms as above.
 * Outputs equal one run per job, bit for bit. */
int hrm_solo_run(const hrm_job* jobs, uint32_t njobs, int variant, uint32_t nlanes, uint64_t* done_ns,
                 float* total_ms);

/* ---- serving: a resident runtime admitting jobs while it runs ---------------------------
 * No counterpart in the original. hrm_server_open starts a persistent AsyncProgram over the
 * job-multiplexing spec (a host thread relaunches its kernel while the session is open; queue
 * state stays on the device between launches). hrm_server_submit appends jobs (each needs
 * count >= 1) and publishes them to the running kernel; indices are in submission order.
 * hrm_server_poll copies the completion stamps (%globaltimer ns, 0 = not done) of the first
 * `max` jobs and counts completions. hrm_server_close stops admissions and waits for every
 * submitted job. Capacity bounds the number of jobs per session. */
typedef struct hrm_server hrm_server;
int hrm_server_open(uint32_t capacity, const hrm_run_config* cfg, hrm_server** out);
int hrm_server_submit(hrm_server* srv, const hrm_job* jobs, uint32_t n, uint32_t* first_index);
int hrm_server_poll(hrm_server* srv, uint64_t* done_ns, uint32_t max, uint32_t* completed);
int hrm_server_close(hrm_server* srv, uint32_t timeout_ms);
int hrm_server_destroy(hrm_server* srv);
/* Replays an arrival schedule (arrival_ns[j], non-decreasing, from the start of the call):
 * mode 0 = the resident runtime (jobs admitted FIFO while the free arena the device reports
 * stays above a quarter of the arena and their estimated arena bytes fit in half of it), mode 1 = one plain launch per job at its arrival on nstreams streams.
 * latency_ns[j] = host-observed completion minus arrival; *makespan_ms = time to the last. */
int hrm_serve_replay(const hrm_job* jobs, uint32_t njobs, const uint64_t* arrival_ns, int mode, uint32_t nstreams,
                     const hrm_run_config* cfg, uint64_t* latency_ns, float* makespan_ms);
/* The same replay against plain execution of the runtime itself: jobs served one at a time in
 * arrival order, each by one whole single-spec run (as hrm_runtime_run; variants per job kind,
 * NULL = 0). */
int hrm_serve_replay_runtime(const hrm_job* jobs, uint32_t njobs, const uint64_t* arrival_ns, int program_type,
                             const int* variants, uint64_t* latency_ns, float* makespan_ms);

/* ---- run without device allocation ------------------------------------------------------
 * No counterpart in the original Harmonize (every original program instance allocates its
 * buffers). For callers that cannot call cudaMalloc when they run a program: plug-in hosts
 * that only hand out buffers registered ahead of time, and services that forbid allocation
 * after start-up to keep their memory use fixed.
 * Same result as hrm_collatz_run_device with AsyncProgram and variant 0, but the runtime's
 * arena, queues and control block live in a scratch area compiled into the library (about
 * 2.2 MiB, held on every GPU that loads the library until the process exits). The caller
 * still passes the output buffer. Limits: cfg->arena may not exceed
 * HRM_NOALLOC_MAX_ARENA_LINKS (0 means that maximum; larger is rejected with HRM_EINVAL), and
 * a run whose promises in flight outgrow it stops with HRM_EDEVICE (ARENA_EXHAUSTED);
 * program_type must be HRM_ASYNC and variant 0. The first call on each device looks up the
 * scratch area's device address (cudaGetSymbolAddress) and keeps it, so make that first call
 * before any stream capture begins; after cudaDeviceReset on a device, call
 * hrm_release_cache() before the next call so that the address is looked up again. The call
 * waits for every exec it launches (it reads the device flags back after each one), and reads
 * the statistics back before it returns. All calls share the scratch area and each call
 * re-initialises it; calls that overlap on the GPU race, so serialise them. res->device_ms is
 * host wall time for this entry point. */
#define HRM_NOALLOC_MAX_ARENA_LINKS 4096
int hrm_collatz_run_device_noalloc(uint32_t start, uint32_t count, uint32_t* d_out_steps,
                                   const hrm_run_config* cfg, hrm_run_result* res);

/* ---- seeded synthetic inputs (host) ---------------------------------------------------- */

/* R-MAT graph with 2^scale vertices and edge_factor * 2^scale edges, quadrant
 * probabilities (a, b, c, 1-a-b-c), as CSR sorted by (source, target):
 * rowptr[2^scale + 1], col[edge_factor * 2^scale]. Returns 0, or 1 on bad arguments. */
int hrm_rmat_csr(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                 uint32_t* rowptr, uint32_t* col);
/* Photon medium: mu_s ~ lognormal(0, 0.5), absorb ~ U[0.02, 0.2], split with p = 0.1. */
int hrm_photon_medium(uint32_t n, uint64_t seed, float* mu_s, float* absorb, uint8_t* split);

#ifdef __cplusplus
}
#endif

#endif
