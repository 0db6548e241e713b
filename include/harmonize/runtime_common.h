// runtime_common.h — pieces shared by AsyncProgram and EventProgram:
//  * detection of optional program-specification members with their defaults (the role of
//    MEMBER_SWITCH / CONST_SWITCH in harmonize/cpp/program/async.h:26-36,101-131);
//  * status flags (async.h:151-155, event.h:80-82) plus this runtime's error flags;
//  * bounded waits: every spin in this runtime gives up after a fixed number of polls,
//    sets WAIT_TIMEOUT_FLAG and returns, so that no kernel can hang the GPU;
//  * the lock-free link ring used for promise queues and the free-link list.
#ifndef HARMONIZE_B200_RUNTIME_COMMON_H
#define HARMONIZE_B200_RUNTIME_COMMON_H

#include "promise.h"

namespace hrm_rt {

// ---------------------------------------------------------------------------------------
// Specification members: type members, constants, and the three hooks.
// ---------------------------------------------------------------------------------------
#define HRM_SPEC_TYPE(NAME, DEFAULT)                                                   \
    template <class S, class = void>                                                   \
    struct spec_##NAME {                                                               \
        using type = DEFAULT;                                                          \
    };                                                                                 \
    template <class S>                                                                 \
    struct spec_##NAME<S, std::void_t<typename S::NAME>> {                             \
        using type = typename S::NAME;                                                 \
    };

#define HRM_SPEC_CONST(NAME, DEFAULT)                                                  \
    template <class S, class = void>                                                   \
    struct spec_##NAME : std::integral_constant<size_t, (DEFAULT)> {};                 \
    template <class S>                                                                 \
    struct spec_##NAME<S, std::void_t<decltype(S::NAME)>>                              \
        : std::integral_constant<size_t, (size_t)(S::NAME)> {};

HRM_SPEC_TYPE(AdrType, unsigned int)
HRM_SPEC_TYPE(OpSet, OpUnion<>)
HRM_SPEC_TYPE(DeviceState, VoidState)
HRM_SPEC_TYPE(GroupState, VoidState)
HRM_SPEC_TYPE(ThreadState, VoidState)

HRM_SPEC_CONST(STASH_SIZE, 16)
HRM_SPEC_CONST(FRAME_SIZE, 32)
HRM_SPEC_CONST(POOL_SIZE, 32)
HRM_SPEC_CONST(STACK_SIZE, 0)
HRM_SPEC_CONST(GROUP_SIZE, 32)
// Tunables of this runtime (a spec may pin them; the autotuner passes them as template
// arguments through the built-in specs).
HRM_SPEC_CONST(RING_LINKS, 2)      // per-function shared-memory ring, in 32-promise links
HRM_SPEC_CONST(TEAMS_PER_CTA, 4)   // 32-lane teams (work groups) per CTA
HRM_SPEC_CONST(MIN_CTAS_PER_SM, 1) // occupancy hint for __launch_bounds__
// Coalescing threshold: a function whose partial batch (1-31 promises) has not grown for
// this many scheduling steps of its team (full batches of other functions, arena fills,
// make_work calls) is run as a partial batch, so that no promise waits behind an endless
// supply of other work, while partial batches that are still filling are left to fill.
HRM_SPEC_CONST(COALESCE_PATIENCE, 16)
// Full batches of one function a team runs back to back before it schedules again, while the
// function still holds a full batch and every other ring keeps room for a batch's calls
// (1 = schedule every batch). The batches run through the one evaluation site of the loop:
// a second inlined copy of every eval doubled the kernel's code and cost 1.8x on the photon
// walk; this form saves 2% there.
HRM_SPEC_CONST(BURST, 4)
// Order in which a team takes a function's promises from its shared-memory ring: newest
// first (0, the default: depth first, which keeps the set of live promises small when calls
// fan out) or oldest first (1: breadth first, for label-correcting searches, where an older
// promise carries a smaller label and evaluating it first saves re-expansions).
HRM_SPEC_CONST(OLDEST_FIRST, 0)

#undef HRM_SPEC_TYPE
#undef HRM_SPEC_CONST

// Per-function ring size: a spec may give functions rings of different sizes by defining
//   template <typename Op> struct RING_LINKS_OF { static const size_t value = ...; };
// (at least 2 for each Op); otherwise every function gets RING_LINKS.
template <class S, class Op, class = void>
struct fn_RING_LINKS : spec_RING_LINKS<S> {};
template <class S, class Op>
struct fn_RING_LINKS<S, Op, std::void_t<decltype(S::template RING_LINKS_OF<Op>::value)>>
    : std::integral_constant<size_t, (size_t)(S::template RING_LINKS_OF<Op>::value)> {};

// Ring groups: a spec whose functions fall into groups that never call one another (for
// example the functions of independent programs multiplexed in one launch) may define
//   template <typename Op> struct RING_GROUP_OF { static const unsigned int value = ...; };
// The rings of different groups then share the same shared memory: a team holds promises of
// one group at a time and changes group only when its rings are empty. A push of another
// group's promise goes to the arena. Default: one group.
template <class S, class Op, class = void>
struct fn_RING_GROUP : std::integral_constant<unsigned int, 0u> {};
template <class S, class Op>
struct fn_RING_GROUP<S, Op, std::void_t<decltype(S::template RING_GROUP_OF<Op>::value)>>
    : std::integral_constant<unsigned int, (unsigned int)(S::template RING_GROUP_OF<Op>::value)> {};

// Pop order per function: a spec may define
//   template <typename Op> struct OLDEST_FIRST_OF { static const bool value = ...; };
// to choose OLDEST_FIRST function by function (e.g. only for the search functions of a spec
// that multiplexes several programs); otherwise every function follows OLDEST_FIRST.
template <class S, class Op, class = void>
struct fn_OLDEST_FIRST : std::integral_constant<bool, spec_OLDEST_FIRST<S>::value != 0> {};
template <class S, class Op>
struct fn_OLDEST_FIRST<S, Op, std::void_t<decltype(S::template OLDEST_FIRST_OF<Op>::value)>>
    : std::integral_constant<bool, (bool)(S::template OLDEST_FIRST_OF<Op>::value)> {};

template <class S, class P, class = void>
struct has_initialize : std::false_type {};
template <class S, class P>
struct has_initialize<S, P, std::void_t<decltype(S::template initialize<P>(std::declval<P>()))>>
    : std::true_type {};

template <class S, class P, class = void>
struct has_finalize : std::false_type {};
template <class S, class P>
struct has_finalize<S, P, std::void_t<decltype(S::template finalize<P>(std::declval<P>()))>>
    : std::true_type {};

template <class S, class P, class = void>
struct has_make_work : std::false_type {};
template <class S, class P>
struct has_make_work<S, P, std::void_t<decltype(S::template make_work<P>(std::declval<P>()))>>
    : std::true_type {};

template <class S, class P>
__device__ __forceinline__ void call_initialize(P prog) {
    if constexpr (has_initialize<S, P>::value) S::template initialize<P>(prog);
}
template <class S, class P>
__device__ __forceinline__ void call_finalize(P prog) {
    if constexpr (has_finalize<S, P>::value) S::template finalize<P>(prog);
}
template <class S, class P>
__device__ __forceinline__ bool call_make_work(P prog) {
    if constexpr (has_make_work<S, P>::value) {
        return S::template make_work<P>(prog);
    } else {
        return false;
    }
}

// Optional hooks of this runtime's AsyncProgram (no counterpart in the original API), for
// specs that keep per-team bookkeeping in their GroupState:
//   template <class P> __device__ static void after_batch(P prog);
//     called by the whole team, converged, right after the evaluations of each batch;
//   template <class P> __device__ static void on_idle(P prog);
//     called by the whole team when it finds no work at all, before it waits, so that
//     bookkeeping held by the team is published before the team sleeps.
template <class S, class P, class = void>
struct has_on_idle : std::false_type {};
template <class S, class P>
struct has_on_idle<S, P, std::void_t<decltype(S::template on_idle<P>(std::declval<P>()))>> : std::true_type {};
template <class S, class P>
__device__ __forceinline__ void call_on_idle(P prog) {
    if constexpr (has_on_idle<S, P>::value) S::template on_idle<P>(prog);
}
//   template <class P> __device__ static void before_publish(P prog);
//     called by the whole team, converged, right before promises of the team become visible
//     to other teams (spills, overflow links held during a step), so that bookkeeping about
//     them can be published first.
template <class S, class P, class = void>
struct has_before_publish : std::false_type {};
template <class S, class P>
struct has_before_publish<S, P, std::void_t<decltype(S::template before_publish<P>(std::declval<P>()))>>
    : std::true_type {};
template <class S, class P>
__device__ __forceinline__ void call_before_publish(P prog) {
    if constexpr (has_before_publish<S, P>::value) S::template before_publish<P>(prog);
}
template <class S, class P, class = void>
struct has_after_batch : std::false_type {};
template <class S, class P>
struct has_after_batch<S, P, std::void_t<decltype(S::template after_batch<P>(std::declval<P>()))>>
    : std::true_type {};
template <class S, class P>
__device__ __forceinline__ void call_after_batch(P prog) {
    if constexpr (has_after_batch<S, P>::value) S::template after_batch<P>(prog);
}

// ---------------------------------------------------------------------------------------
// Status flags. The first four keep the values of the original runtime.
// ---------------------------------------------------------------------------------------
static const unsigned int BAD_FUNC_ID_FLAG = 0x00000001u;
static const unsigned int STASH_FAIL_FLAG = 0x00000002u;
static const unsigned int ARENA_EXHAUSTED_FLAG = 0x00000004u;  // a spill found no free link
static const unsigned int QUEUE_OVERFLOW_FLAG = 0x00000008u;   // an event buffer overflowed
static const unsigned int WAIT_TIMEOUT_FLAG = 0x00000010u;     // a bounded wait gave up
static const unsigned int LAUNCH_FLAG = 0x00000020u;           // co-residency not possible
static const unsigned int ERROR_MASK = 0x000000FFu;
static const unsigned int EARLY_HALT_FLAG = 0x40000000u;
static const unsigned int COMPLETION_FLAG = 0x80000000u;

// Host side: turns error flags into an exception with a readable message.
static inline void throw_flags(unsigned int f) {
    std::string m = "harmonize device error flags 0x";
    char buf[16];
    snprintf(buf, sizeof(buf), "%08x", f);
    m += buf;
    if (f & BAD_FUNC_ID_FLAG) m += " BAD_FUNC_ID";
    if (f & STASH_FAIL_FLAG) m += " STASH_FAIL";
    if (f & ARENA_EXHAUSTED_FLAG) m += " ARENA_EXHAUSTED";
    if (f & QUEUE_OVERFLOW_FLAG) m += " QUEUE_OVERFLOW";
    if (f & WAIT_TIMEOUT_FLAG) m += " WAIT_TIMEOUT";
    if (f & LAUNCH_FLAG) m += " LAUNCH";
    throw std::runtime_error(m);
}

// Upper bound on polls of any wait. With the back-off below a wait gives up after roughly
// 2^20 * 200 ns = 0.2 s.
static const unsigned int SPIN_LIMIT = 1u << 20;

// ---------------------------------------------------------------------------------------
// Memory access helpers (PTX memory-model operations at GPU scope).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
// Acquire-release fence at GPU scope (lighter than __threadfence's sequentially consistent one).
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ unsigned int ld_relaxed(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ---------------------------------------------------------------------------------------
// Device-wide control block of one program instance.
// ---------------------------------------------------------------------------------------
struct alignas(128) RuntimeControl {
    unsigned int flags;        // status flags (persist between exec calls)
    unsigned int checkout;     // teams that finished the current exec
    unsigned int done;         // quiescence detected during the current exec
    unsigned int total_teams;  // teams launched by the current exec
    unsigned int bump;         // arena links handed out lazily so far
    unsigned int arena_links;  // number of links in the arena
    unsigned int generation;   // EventProgram: completed generations
    // Nonzero: the host asks the running AsyncProgram exec to stop (as halt_early() does). The
    // host writes it with a copy, so that no kernel launch is needed while a persistent
    // kernel occupies every SM; the host clears it before the next exec.
    unsigned int halt_request;
    // [63:40] teams that are busy (not idle, not exited); [39:0] wake-up epoch.
    alignas(128) unsigned long long busy_epoch;
};

static const unsigned long long BUSY_ONE = 1ull << 40;

// Per-instance statistics, summed over teams at the end of each exec.
enum StatIndex : unsigned int {
    STAT_EVALS = 0,       // promises evaluated
    STAT_BATCHES = 1,     // warp batches executed
    STAT_FULL_BATCHES = 2,// batches with all 32 lanes active
    STAT_SPILL_LINKS = 3, // links written to the arena
    STAT_FILL_LINKS = 4,  // links read back from the arena
    STAT_MAKE_WORK = 5,   // make_work calls (per team)
    STAT_IDLE_POLLS = 6,  // polls made while idle
    STAT_GENERATIONS = 7, // EventProgram generations
    STAT_FN_EVALS = 8,    // STAT_FN_EVALS + f: promises of function f evaluated (f < 16)
    STAT_COUNT = 24
};

// ---------------------------------------------------------------------------------------
// Link ring: a bounded multi-producer multi-consumer queue of 32-bit entries, one 64-bit
// slot per position holding {sequence (hi 32), entry (lo 32)}. A producer owning position
// t waits for sequence t, writes {t+1, entry}; a consumer owning position t waits for
// sequence t+1 and writes {t+capacity, 0}. Positions are handed out in batches by one
// atomicAdd per warp. `avail` counts published, unclaimed entries; a consumer first
// reserves entries from `avail` (atomicSub, see ring_reserve), then positions from `head`.
// ---------------------------------------------------------------------------------------
struct alignas(128) RingHead {
    unsigned int head;
    unsigned int tail;
    unsigned int avail;
    unsigned int pad;
};

struct RingSet {
    RingHead* heads;              // one per ring
    unsigned long long* slots;    // ring r uses slots[r * capacity ... (r+1) * capacity)
    unsigned int mask;            // capacity - 1 (capacity is a power of two)
};

// Sets WAIT_TIMEOUT_FLAG; called by the lane whose wait ran out.
__device__ __forceinline__ void raise_flag(RuntimeControl* ctl, unsigned int f) { atomicOr(&ctl->flags, f); }

// Lane-cooperative publish: lanes with `j < n` (j = rank among `mask`) push entry `e` to
// ring `r`. Returns false if a wait timed out (the flag is raised).
__device__ __forceinline__ bool ring_push(RingSet rs, RuntimeControl* ctl, unsigned int r, unsigned int e,
                                          unsigned int j, unsigned int n, unsigned int mask) {
    const unsigned int leader = __ffs(mask) - 1;
    unsigned int t = 0;
    if (j == 0 && n > 0) t = atomicAdd(&rs.heads[r].tail, n);
    t = __shfl_sync(mask, t, leader);
    bool ok = true;
    if (j < n) {
        unsigned int pos = t + j;
        unsigned long long* slot = rs.slots + (size_t)r * (rs.mask + 1) + (pos & rs.mask);
        unsigned int spins = 0;
        while ((unsigned int)(ld_acquire64(slot) >> 32) != pos) {
            if (++spins > SPIN_LIMIT) { ok = false; raise_flag(ctl, WAIT_TIMEOUT_FLAG); break; }
            __nanosleep(128);
        }
        if (ok) st_release64(slot, ((unsigned long long)(pos + 1) << 32) | e);
    }
    __syncwarp(mask);
    if (j == 0 && n > 0) {
        // The slots above before the count that announces them (a consumer that sees the
        // count still waits for each slot's sequence: this orders progress, not data).
        fence_acq_rel();
        atomicAdd(&rs.heads[r].avail, n);
    }
    return __all_sync(mask, ok);
}

// Reserves up to `want` published entries of ring r (called by one lane). Returns the
// number reserved and the first position in `pos`.
// `avail` is decremented optimistically with atomicSub (it may dip below zero for an
// instant while an over-claim is handed back), so contention never makes a reservation
// fail while entries are available; a reader that sees a value <= 0 treats the ring as
// momentarily empty.
__device__ __forceinline__ unsigned int ring_reserve(RingSet rs, unsigned int r, unsigned int want, unsigned int& pos) {
    unsigned int* avail = &rs.heads[r].avail;
    int a = (int)ld_relaxed(avail);
    if (a <= 0 || want == 0) return 0;
    unsigned int take = (unsigned int)a < want ? (unsigned int)a : want;
    int old = (int)atomicSub(avail, take);
    unsigned int got = old >= (int)take ? take : (old > 0 ? (unsigned int)old : 0u);
    if (got < take) atomicAdd(avail, take - got);
    if (got > 0) pos = atomicAdd(&rs.heads[r].head, got);
    return got;
}

// True if ring r appears to hold published entries.
__device__ __forceinline__ bool ring_nonempty(RingSet rs, unsigned int r) {
    return (int)ld_relaxed(&rs.heads[r].avail) > 0;
}

// Lane-cooperative take: lanes with j < n consume position pos + j of ring r and return its
// entry (0 if the wait timed out).
__device__ __forceinline__ unsigned int ring_take(RingSet rs, RuntimeControl* ctl, unsigned int r, unsigned int pos0,
                                                  unsigned int j, unsigned int n) {
    if (j >= n) return 0u;
    unsigned int pos = pos0 + j;
    unsigned long long* slot = rs.slots + (size_t)r * (rs.mask + 1) + (pos & rs.mask);
    unsigned long long v;
    unsigned int spins = 0;
    while (true) {
        v = ld_acquire64(slot);
        if ((unsigned int)(v >> 32) == pos + 1) break;
        if (++spins > SPIN_LIMIT) { raise_flag(ctl, WAIT_TIMEOUT_FLAG); return 0u; }
        __nanosleep(128);
    }
    unsigned int e = (unsigned int)v;
    st_relaxed64(slot, (unsigned long long)(pos + rs.mask + 1) << 32);
    return e;
}

// Initialises every slot of `rings` rings: slot i holds sequence i.
__device__ __forceinline__ void ring_init_slots(RingSet rs, unsigned int rings, size_t tid, size_t nthreads) {
    size_t cap = (size_t)rs.mask + 1;
    for (size_t i = tid; i < cap * rings; i += nthreads) {
        rs.slots[i] = (unsigned long long)(unsigned int)(i & rs.mask) << 32;
    }
    for (size_t i = tid; i < rings; i += nthreads) {
        rs.heads[i].head = 0;
        rs.heads[i].tail = 0;
        rs.heads[i].avail = 0;
        rs.heads[i].pad = 0;
    }
}

// Link entry encoding: bits [31:5] link index + 1, bits [4:0] promise count - 1.
__device__ __forceinline__ unsigned int encode_link(unsigned int link, unsigned int count) {
    return ((link + 1u) << 5) | ((count - 1u) & 31u);
}
__device__ __forceinline__ unsigned int entry_link(unsigned int e) { return (e >> 5) - 1u; }
__device__ __forceinline__ unsigned int entry_count(unsigned int e) { return (e & 31u) + 1u; }

static inline unsigned int next_pow2(unsigned long long v) {
    unsigned long long p = 1;
    while (p < v) p <<= 1;
    return (unsigned int)p;
}

// Number of CTAs of `kernel` that can be resident at once on the current device.
template <typename KERNEL>
static inline unsigned int max_resident_ctas(KERNEL kernel, int threads, size_t dyn_smem) {
    int dev = 0;
    cudaGetDevice(&dev);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, dyn_smem);
    return (unsigned int)(per_sm * sms);
}

// ---------------------------------------------------------------------------------------
// LazyLoad arguments of prog.async<F> (AsyncProgram copies them asynchronously).
// ---------------------------------------------------------------------------------------
template <typename T>
struct is_lazy_load : std::false_type {};
template <typename T>
struct is_lazy_load<LazyLoad<T>> : std::true_type {};

// The value an argument contributes to the promise built at the call: a LazyLoad argument
// contributes zero (its words are filled by the copy), any other argument itself.
template <typename T>
__device__ __forceinline__ T lazy_placeholder(T v) {
    return v;
}
template <typename T>
__device__ __forceinline__ T lazy_placeholder(LazyLoad<T>) {
    static_assert(sizeof(T) % 4 == 0 && alignof(T) >= 4,
                  "LazyLoad arguments are copied as 32-bit words: their type must be a multiple of "
                  "4 bytes and 4-byte aligned");
    return T{};
}

// Marks the promise words of argument I onwards that come from LazyLoad arguments, with the
// address each word is copied from.
template <typename ARGS, size_t I>
__device__ __forceinline__ void mark_lazy_words(ARGS&, bool*, const unsigned int**) {}

template <typename ARGS, size_t I, typename HEAD, typename... TAIL>
__device__ __forceinline__ void mark_lazy_words(ARGS& tuple, bool* lazy, const unsigned int** src, HEAD head,
                                                TAIL... tail) {
    if constexpr (is_lazy_load<HEAD>::value) {
        using T = typename HEAD::Type;
        constexpr unsigned int off = ArgWordOffset<I, ARGS>::value;  // packed word of argument I
        const unsigned int* from = (const unsigned int*)&head.reference;
        (void)tuple;
#pragma unroll
        for (unsigned int j = 0; j < sizeof(T) / 4u; j++) {
            lazy[off + j] = true;
            src[off + j] = from + j;
        }
    }
    mark_lazy_words<ARGS, I + 1>(tuple, lazy, src, tail...);
}

}  // namespace hrm_rt

#endif
