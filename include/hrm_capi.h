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
#define HRM_STAT_COUNT 8

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
} hrm_run_config;

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

/* ---- program life cycle (templates.py:3-184 counterparts) ------------------------------
 * hrm_program_create: spec + type + arena/io size + a copy of the spec's device state
 *   (the struct layouts are given by hrm_*_state below);
 * hrm_program_init: reset queues and flags (init<P>); hrm_program_exec: one exec<P>;
 * hrm_program_complete: *out = 1 when the last exec completed (throws nothing: an error
 *   flag returns HRM_EDEVICE). */
int hrm_program_create(int spec, int program_type, size_t arena_or_io, const void* device_state,
                       size_t state_size, hrm_program** out);
int hrm_program_destroy(hrm_program* prog);
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

/* ---- whole runs (host buffers in and out) --------------------------------------------- */

/* Collatz stopping times of n = start .. start+count-1 into out_steps[count] (host). */
int hrm_collatz_run(uint32_t start, uint32_t count, uint32_t* out_steps, const hrm_run_config* cfg,
                    hrm_run_result* res);
/* Same, with a device output buffer (no host copies). */
int hrm_collatz_run_device(uint32_t start, uint32_t count, uint32_t* d_out_steps, const hrm_run_config* cfg,
                           hrm_run_result* res);

#ifdef __cplusplus
}
#endif

#endif
