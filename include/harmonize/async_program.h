// async_program.h — AsyncProgram<Spec>: the persistent work-coalescing runtime.
//
// Source-level contract kept from harmonize/cpp/program/async.h:
//  * the spec members and defaults (async.h:101-131), Instance(arena_links, DeviceState)
//    with complete() / clear_flags() (async.h:302-384), init<P>/exec<P>;
//  * prog.async<F>(args...), prog.sync<F>(args...), prog.load_fraction<F>() (NaN here, as in
//    async.h:2902-2906), prog.halt_early(), prog.device / prog.group / prog.thread;
//  * exec(cycles) runs at most `cycles` scheduling rounds per team, then leaves every
//    pending promise in device memory so that the next exec resumes it (async.h:2625-2668);
//  * completion: COMPLETION_FLAG is set only when every team found no work anywhere and
//    every team's make_work returned false (async.h:2323-2393); a team that stops while
//    make_work still wanted to run, or a halt_early() call, leaves the run incomplete.
//
// Internals (the B200 design, not a translation):
//  * a "team" is one warp; a CTA holds TEAMS_PER_CTA teams. Each team owns, in shared
//    memory, one ring per async function of RING_LINKS*32 promise slots (a spec may size
//    functions' rings apart with RING_LINKS_OF<Op>), stored as structure-of-arrays 32-bit
//    words (conflict-free for 32 consecutive slots).
//  * prog.async<F>: the lanes active at the call site reserve slots with ONE shared-memory
//    atomicAdd issued by the lowest lane (__activemask / popc rank / __shfl_sync), then each
//    lane writes its own words. Promises of one function therefore land contiguously, and
//    the scheduler evaluates them 32 at a time: every batch is warp-full while work lasts.
//  * when a ring passes its high-water mark the team spills its oldest promises as whole
//    links to the HBM arena: one atomicAdd claims all links needed, each lane stores one
//    32-bit word per promise word (every store instruction covers 128 contiguous bytes),
//    and one atomicAdd publishes all links to the function's lock-free ring.
//  * an idle team fills from the arena the function closest to a full batch; teams count
//    themselves busy/idle in one 64-bit word with a wake-up epoch, and quiescence is
//    declared only when "all idle" and "all queues empty" hold across an unchanged epoch.
//  * every wait is bounded (WAIT_TIMEOUT_FLAG), arena exhaustion is flagged
//    (ARENA_EXHAUSTED_FLAG) and never silent.
#ifndef HARMONIZE_B200_ASYNC_PROGRAM_H
#define HARMONIZE_B200_ASYNC_PROGRAM_H

#include "runtime_common.h"

template <typename PROGRAM_SPEC>
class AsyncProgram;

namespace hrm_rt {
template <typename PROG>
__global__ void async_init_kernel(typename PROG::DeviceContext ctx);
template <typename PROG>
__global__ void async_prep_kernel(typename PROG::DeviceContext ctx, unsigned int total_teams);
template <typename PROG>
__global__ void __launch_bounds__(PROG::CTA_THREADS, PROG::MIN_CTAS_PER_SM)
    async_exec_kernel(typename PROG::DeviceContext ctx, typename PROG::DeviceState device, unsigned int cycles);
}  // namespace hrm_rt

template <typename PROGRAM_SPEC>
class AsyncProgram {
   public:
    typedef AsyncProgram<PROGRAM_SPEC> ProgramType;
    typedef PROGRAM_SPEC Spec;

    using AdrType = typename hrm_rt::spec_AdrType<PROGRAM_SPEC>::type;
    using OpSet = typename hrm_rt::spec_OpSet<PROGRAM_SPEC>::type;
    using DeviceState = typename hrm_rt::spec_DeviceState<PROGRAM_SPEC>::type;
    using GroupState = typename hrm_rt::spec_GroupState<PROGRAM_SPEC>::type;
    using ThreadState = typename hrm_rt::spec_ThreadState<PROGRAM_SPEC>::type;

    typedef PromiseUnion<OpSet> PromiseUnionType;
    typedef PromiseEnum<OpSet> PromiseEnumType;

    template <typename TYPE>
    struct Lookup {
        typedef typename PromiseUnionType::template Lookup<TYPE>::type type;
    };

    static const size_t STASH_SIZE = hrm_rt::spec_STASH_SIZE<PROGRAM_SPEC>::value;
    static const size_t FRAME_SIZE = hrm_rt::spec_FRAME_SIZE<PROGRAM_SPEC>::value;
    static const size_t POOL_SIZE = hrm_rt::spec_POOL_SIZE<PROGRAM_SPEC>::value;
    static const size_t STACK_SIZE = hrm_rt::spec_STACK_SIZE<PROGRAM_SPEC>::value;
    static const size_t GROUP_SIZE = hrm_rt::spec_GROUP_SIZE<PROGRAM_SPEC>::value;
    static const size_t WORK_GROUP_SIZE = GROUP_SIZE;
    static_assert(GROUP_SIZE == 32, "work groups are 32-lane warps");

    static const unsigned int RING_LINKS = (unsigned int)hrm_rt::spec_RING_LINKS<PROGRAM_SPEC>::value;
    static const unsigned int RING = RING_LINKS * 32u;
    static_assert(RING_LINKS >= 2, "RING_LINKS must be at least 2");
    static const unsigned int TEAMS_PER_CTA = (unsigned int)hrm_rt::spec_TEAMS_PER_CTA<PROGRAM_SPEC>::value;
    static const unsigned int CTA_THREADS = TEAMS_PER_CTA * 32u;
    static const unsigned int MIN_CTAS_PER_SM = (unsigned int)hrm_rt::spec_MIN_CTAS_PER_SM<PROGRAM_SPEC>::value;
    static const unsigned int COALESCE_PATIENCE =
        (unsigned int)hrm_rt::spec_COALESCE_PATIENCE<PROGRAM_SPEC>::value;
    static const unsigned int BURST = (unsigned int)hrm_rt::spec_BURST<PROGRAM_SPEC>::value;
    static_assert(BURST >= 1, "BURST must be at least 1");

    static const unsigned int BAD_FUNC_ID_FLAG = hrm_rt::BAD_FUNC_ID_FLAG;
    static const unsigned int STASH_FAIL_FLAG = hrm_rt::STASH_FAIL_FLAG;
    static const unsigned int COMPLETION_FLAG = hrm_rt::COMPLETION_FLAG;
    static const unsigned int EARLY_HALT_FLAG = hrm_rt::EARLY_HALT_FLAG;

    static const unsigned char FN_ID_COUNT = (unsigned char)PromiseUnionType::Info::COUNT;
    static const unsigned int FN = FN_ID_COUNT;
    static_assert(FN >= 1 && FN <= 16, "an operation set holds 1 to 16 async functions");

    using Layout = OpLayout<OpSet>;
    static const unsigned int TOTAL_WORDS = Layout::TOTAL_WORDS;
    static const unsigned int LINK_WORDS = Layout::MAX_WORDS;  // words per promise in a link

    // Ring geometry: function F's ring holds ring_slots<F>() promises (RING_LINKS, or the
    // spec's RING_LINKS_OF<Op>, links of 32), and word i of its slot s is stored at
    // words[ring_base<F>() + i * ring_slots<F>() + s] of the team's stash. Functions of
    // different ring groups (RING_GROUP_OF) overlay one another: each group's rings start at
    // word 0, and the stash is as large as the largest group.
    template <unsigned int F>
    __host__ __device__ static constexpr unsigned int ring_slots() {
        using Op = typename OpAt<F, OpSet>::type;
        return (unsigned int)hrm_rt::fn_RING_LINKS<PROGRAM_SPEC, Op>::value * 32u;
    }
    template <unsigned int F>
    __host__ __device__ static constexpr unsigned int group_of() {
        using Op = typename OpAt<F, OpSet>::type;
        return hrm_rt::fn_RING_GROUP<PROGRAM_SPEC, Op>::value;
    }
    template <unsigned int F>
    __host__ __device__ static constexpr unsigned int ring_words() {
        using Op = typename OpAt<F, OpSet>::type;
        return Promise<Op>::WORDS * ring_slots<F>();
    }
    // Words used by the functions of group G before function F.
    template <unsigned int G, unsigned int F>
    __host__ __device__ static constexpr unsigned int group_words_before() {
        if constexpr (F == 0) {
            return 0u;
        } else {
            return group_words_before<G, F - 1>() + (group_of<F - 1>() == G ? ring_words<F - 1>() : 0u);
        }
    }
    template <unsigned int F>
    __host__ __device__ static constexpr unsigned int ring_base() {
        return group_words_before<group_of<F>(), F>();
    }
    template <unsigned int I>
    __host__ __device__ static constexpr unsigned int max_group() {
        if constexpr (I < FN) {
            return group_of<I>() > max_group<I + 1>() ? group_of<I>() : max_group<I + 1>();
        } else {
            return 0u;
        }
    }
    static const unsigned int RING_GROUPS = max_group<0>() + 1u;
    template <unsigned int G>
    __host__ __device__ static constexpr unsigned int max_group_words() {
        if constexpr (G < RING_GROUPS) {
            constexpr unsigned int w = group_words_before<G, FN>();
            constexpr unsigned int rest = max_group_words<G + 1>();
            return w > rest ? w : rest;
        } else {
            return 0u;
        }
    }
    static const unsigned int NO_GROUP = 0xFFFFFFFFu;
    template <unsigned int I>
    __host__ __device__ static constexpr bool rings_valid() {
        if constexpr (I < FN) {
            constexpr unsigned int s = ring_slots<I>();
            return s >= 64u && s % 32u == 0u && rings_valid<I + 1>();
        } else {
            return true;
        }
    }
    static_assert(rings_valid<0>(), "rings hold at least 2 links");
    static const unsigned int RING_WORDS = max_group_words<0>();
    // Ring index a (a < 2 * SLOTS: a ring position < SLOTS plus an offset <= SLOTS) reduced
    // to a slot. A mask for power-of-two rings, one compare and subtract for the others
    // (e.g. 3 links, so that a team's stash is smaller and more teams fit on an SM).
    template <unsigned int SLOTS>
    __host__ __device__ static constexpr unsigned int wrap_slot(unsigned int a) {
        if constexpr ((SLOTS & (SLOTS - 1u)) == 0u) {
            return a & (SLOTS - 1u);
        } else {
            return a >= SLOTS ? a - SLOTS : a;
        }
    }
    // Ring size and ring group of function f (run-time f).
    template <unsigned int I = 0>
    __device__ static __forceinline__ unsigned int ring_slots_of(unsigned int f) {
        if constexpr (I < FN) {
            return f == I ? ring_slots<I>() : ring_slots_of<I + 1>(f);
        } else {
            return 0u;
        }
    }
    template <unsigned int I = 0>
    __device__ static __forceinline__ unsigned int group_of_fn(unsigned int f) {
        if constexpr (I < FN) {
            return f == I ? group_of<I>() : group_of_fn<I + 1>(f);
        } else {
            return NO_GROUP;
        }
    }

    // -----------------------------------------------------------------------------------
    // Contexts (the names of async.h:181-262; contents are this runtime's).
    // -----------------------------------------------------------------------------------
    struct ThreadContext {
        unsigned int thread_id;
        unsigned int rand_state;
    };

    // One team's shared-memory stash: one ring of promise slots per function.
    // Arena links written by pushes that did not fit in the stash during one scheduling step
    // are published when the step ends (after the batch's after_batch hook, after make_work):
    // a spec that settles per batch (after_batch) sees its bookkeeping done before any
    // promise of the batch can reach another team. Beyond HELD_MAX a link is published at once.
    static const unsigned int HELD_MAX = 32;

    struct GroupContext {
        unsigned int count[FN];    // promises held per function (may exceed the ring briefly)
        unsigned int bottom[FN];   // ring index of the oldest promise per function
        unsigned int active;       // ring group whose promises the stash holds, or NO_GROUP
        unsigned int held_n;       // overflow links written and not yet published
        unsigned int loads_pending;  // a lane issued cp.async copies of LazyLoad arguments
        unsigned int overflowed;   // a push went past a ring since the last settle_overflow
        unsigned int held_e[HELD_MAX];  // their queue entries
        unsigned int held_f[HELD_MAX];  // their functions
        // The team's statistics of this exec, kept here rather than in registers (lane 0
        // updates them) and added to the device counters when the team leaves.
        // Evaluations are counted per function in fn_evals; partial batches and their evaluations
        // in n_partial and partial_evals, so full batches are (evals - partial_evals) / 32.
        unsigned long long partial_evals, n_partial, n_spill, n_fill, n_mw, n_idle;
        unsigned long long fn_evals[FN];
        unsigned int words[RING_WORDS];
    };

    struct DeviceContext {
        typedef ProgramType ParentProgramType;
        hrm_rt::RuntimeControl* ctl;
        hrm_rt::RingSet rings;        // rings [0, FN) = per-function queues, ring FN = free links
        unsigned int* link_words;     // arena: link l, word w, lane i at ((l*LINK_WORDS+w)*32+i)
        unsigned int* link_meta;      // per link {next + 1, promise count}; used by barriers
        unsigned long long* stats;    // hrm_rt::STAT_COUNT counters
        unsigned int arena_links;
        unsigned int patience;        // coalescing threshold in force (COALESCE_PATIENCE by default)
        unsigned int fill_links;      // links one fill may take from a queue (2 by default)
    };

    // Sets a context's run-time tunables (0 = the spec's defaults; both end up >= 1). Every
    // DeviceContext passed to a launch must go through here.
    __host__ static void set_tunables(DeviceContext& c, unsigned int patience, unsigned int fill_links) {
        c.patience = patience ? patience : (COALESCE_PATIENCE ? COALESCE_PATIENCE : 1u);
        c.fill_links = fill_links ? (fill_links < 32u ? fill_links : 32u) : 2u;
    }

    // -----------------------------------------------------------------------------------
    // Host-side instance: owns the device memory of one program instance.
    // -----------------------------------------------------------------------------------
    struct Instance {
        AdrType arena_size;
        util::host::DevBuf<hrm_rt::RuntimeControl> control;
        util::host::DevBuf<hrm_rt::RingHead> heads;
        util::host::DevBuf<unsigned long long> slots;
        util::host::DevBuf<unsigned int> link_words;
        util::host::DevBuf<unsigned int> link_meta;
        util::host::DevBuf<unsigned long long> stats;
        unsigned int ring_capacity;
        DeviceState device_state;
        cudaStream_t stream = nullptr;
        // Run-time tunables (0 = the spec's default): see DeviceContext.
        unsigned int patience = 0;
        unsigned int fill_links = 0;

        __host__ Instance(AdrType arsize, DeviceState ds)
            : arena_size(arsize),
              control((size_t)1),
              heads((size_t)(FN + 1)),
              slots((size_t)(FN + 1) * hrm_rt::next_pow2(arsize < 32 ? 32 : (unsigned long long)arsize)),
              link_words((size_t)arsize * LINK_WORDS * 32u),
              link_meta((size_t)arsize * 2u),
              stats((size_t)hrm_rt::STAT_COUNT),
              ring_capacity(hrm_rt::next_pow2(arsize < 32 ? 32 : (unsigned long long)arsize)),
              device_state(ds) {
            if ((unsigned long long)arsize >= (1ull << 27) - 2) {
                throw std::runtime_error("AsyncProgram arena holds at most 2^27 - 2 links");
            }
            util::host::auto_throw(cudaMemset(control.data(), 0, sizeof(hrm_rt::RuntimeControl)));
            util::host::auto_throw(cudaMemset(stats.data(), 0, sizeof(unsigned long long) * hrm_rt::STAT_COUNT));
        }

        __host__ DeviceContext to_context() {
            DeviceContext c;
            c.ctl = control.data();
            c.rings.heads = heads.data();
            c.rings.slots = slots.data();
            c.rings.mask = ring_capacity - 1;
            c.link_words = link_words.data();
            c.link_meta = link_meta.data();
            c.stats = stats.data();
            c.arena_links = (unsigned int)arena_size;
            set_tunables(c, patience, fill_links);
            return c;
        }

        __host__ unsigned int flags() {
            unsigned int f = 0;
            util::host::auto_throw(cudaMemcpy(&f, &control.data()->flags, sizeof(f), cudaMemcpyDeviceToHost));
            return f;
        }
        // True once an exec found no work anywhere and make_work exhausted everywhere.
        // Throws if the device raised an error flag, so that host loops end.
        __host__ bool complete() {
            unsigned int f = flags();
            if (f & hrm_rt::ERROR_MASK) hrm_rt::throw_flags(f);
            return (f & COMPLETION_FLAG) != 0;
        }
        __host__ void clear_flags() {
            util::host::auto_throw(cudaMemset(&control.data()->flags, 0, sizeof(unsigned int)));
        }
        // Host-side view of the arena (the role of runtime_overview, async.h:2766-2883):
        // out[0] = links handed out lazily (capped at the arena size), out[1] = links on the
        // free ring, out[2 + f] = links queued for function f, out[2 + FN + r] = tail - head
        // of ring r. A quiescent instance has out[0] == out[1] and every queue empty.
        __host__ std::vector<unsigned int> overview() {
            hrm_rt::RuntimeControl c;
            std::vector<hrm_rt::RingHead> h(FN + 1);
            util::host::auto_throw(cudaMemcpy(&c, control.data(), sizeof(c), cudaMemcpyDeviceToHost));
            util::host::auto_throw(
                cudaMemcpy(h.data(), heads.data(), sizeof(hrm_rt::RingHead) * (FN + 1), cudaMemcpyDeviceToHost));
            std::vector<unsigned int> out;
            out.push_back(c.bump < (unsigned int)arena_size ? c.bump : (unsigned int)arena_size);
            out.push_back(h[FN].avail);
            for (unsigned int f = 0; f < FN; f++) out.push_back(h[f].avail);
            for (unsigned int r = 0; r <= FN; r++) out.push_back(h[r].tail - h[r].head);
            return out;
        }

        __host__ std::vector<unsigned long long> read_stats() {
            std::vector<unsigned long long> v(hrm_rt::STAT_COUNT);
            util::host::auto_throw(cudaMemcpy(v.data(), stats.data(), sizeof(unsigned long long) * hrm_rt::STAT_COUNT,
                                              cudaMemcpyDeviceToHost));
            return v;
        }
    };

    // -----------------------------------------------------------------------------------
    // The program object handed to eval / make_work: references to the contexts.
    // -----------------------------------------------------------------------------------
    DeviceContext& _dev_ctx;
    GroupContext& _grp_ctx;
    ThreadContext& _thd_ctx;
    DeviceState& device;
    GroupState& group;
    ThreadState& thread;

    __device__ AsyncProgram(DeviceContext& d_c, GroupContext& g_c, ThreadContext& t_c, DeviceState& d,
                            GroupState& g, ThreadState& t)
        : _dev_ctx(d_c), _grp_ctx(g_c), _thd_ctx(t_c), device(d), group(g), thread(t) {}

    // ===================================================================================
    // Public device API used by specs.
    // ===================================================================================
    // An argument given as LazyLoad<T>(ref) (promise.h:208-240 of the original, its
    // ASYNC_LOADS form) is not read at the call: each lane whose promise lands in the team's
    // shared-memory ring starts an asynchronous copy (cp.async, 4 bytes per argument word)
    // from `ref` straight into the promise's slot, and the team waits for its copies only
    // when it next reads its rings (to run or spill a batch), so the load overlaps the rest
    // of the current batch. A promise that overflows to the arena reads the value at the call.
    // The referenced memory must not change until the promise first runs.
    template <typename TYPE, typename... ARGS>
    __device__ __forceinline__ void async(ARGS... args) {
        if constexpr ((hrm_rt::is_lazy_load<ARGS>::value || ...)) {
            push_lazy<TYPE>(args...);
        } else {
            push_promise<TYPE>(Promise<TYPE>(args...));
        }
    }
    template <typename TYPE>
    __device__ __forceinline__ void async_call(Promise<TYPE> promise) {
        push_promise<TYPE>(promise);
    }
    // Runtime-discriminant form (used by barriers): lanes are grouped by discriminant
    // with __match_any_sync and each group is pushed as one coalesced call.
    __device__ void async_call(PromiseEnumType promise) { push_enum<0>(promise.disc, promise.data); }
    __device__ void async_call(OpDisc disc, int, PromiseUnionType& promise) { push_enum<0>(disc, promise); }

    template <typename TYPE, typename... ARGS>
    __device__ __forceinline__ void sync(ARGS... args) {
        Promise<TYPE>(args...)(*this);
    }
    template <typename TYPE>
    __device__ __forceinline__ void sync_call(Promise<TYPE> promise) {
        promise(*this);
    }
    template <typename TYPE>
    __device__ float load_fraction() {
        return NAN;
    }
    __device__ void halt_early() { atomicOr(&_dev_ctx.ctl->flags, EARLY_HALT_FLAG); }

    // ===================================================================================
    // Promise placement.
    // ===================================================================================
    template <typename TYPE>
    __host__ __device__ static constexpr unsigned int disc_of() {
        static_assert(OpUnionLookup<TYPE, OpSet>::CONTAINED, "async function is not in the spec's OpSet");
        return OpUnionLookup<TYPE, OpSet>::DISC;
    }

    // Allocates `n` links for this lane (n <= 32, called by one lane). Returns how many
    // were obtained; link j goes to *first + j for bump links, or is popped from the free ring.
    // The lane-cooperative variant below is used instead wherever the whole warp is present.
    __device__ unsigned int alloc_links_coop(unsigned int n, unsigned int j, unsigned int mask, unsigned int& link) {
        // Lazy bump allocation first, then the free-link ring.
        const unsigned int leader = __ffs(mask) - 1;
        hrm_rt::RuntimeControl* ctl = _dev_ctx.ctl;
        unsigned int base = 0, from_bump = 0;
        if (j == 0) {
            unsigned int cur = hrm_rt::ld_relaxed(&ctl->bump);
            if (cur < _dev_ctx.arena_links) {
                base = atomicAdd(&ctl->bump, n);
                if (base < _dev_ctx.arena_links) {
                    from_bump = min(n, _dev_ctx.arena_links - base);
                }
            }
        }
        base = __shfl_sync(mask, base, leader);
        from_bump = __shfl_sync(mask, from_bump, leader);
        unsigned int need = n - from_bump;
        unsigned int got_free = 0, pos = 0;
        if (need > 0) {
            if (j == 0) {
                // Links on the free ring may be in the middle of being returned: retry a
                // bounded number of times before reporting the arena as exhausted.
                for (unsigned int attempt = 0; attempt < 64u; attempt++) {
                    got_free = hrm_rt::ring_reserve(_dev_ctx.rings, FN, need, pos);
                    if (got_free > 0) break;
                    __nanosleep(256);
                }
            }
            got_free = __shfl_sync(mask, got_free, leader);
            pos = __shfl_sync(mask, pos, leader);
        }
        link = 0xFFFFFFFFu;
        if (j < from_bump) {
            link = base + j;
        }
        unsigned int fe = 0;
        if (got_free > 0) {
            unsigned int jj = j - from_bump;
            fe = hrm_rt::ring_take(_dev_ctx.rings, _dev_ctx.ctl, FN, pos, (j >= from_bump) ? jj : 0xFFFFFFFFu, got_free);
            if (j >= from_bump && jj < got_free) link = fe ? hrm_rt::entry_link(fe) : 0xFFFFFFFFu;
        }
        return from_bump + got_free;
    }

    // Lane-cooperative: lanes j < n return link `link` to the free ring.
    __device__ void free_links_coop(unsigned int link, unsigned int j, unsigned int n, unsigned int mask) {
        hrm_rt::ring_push(_dev_ctx.rings, _dev_ctx.ctl, FN, hrm_rt::encode_link(link, 1), j, n, mask);
    }

    __device__ __forceinline__ unsigned int* link_word_ptr(unsigned int link, unsigned int w, unsigned int lane) {
        return _dev_ctx.link_words + ((size_t)link * LINK_WORDS + w) * 32u + lane;
    }

    // prog.async<F>: coalesce the active lanes' calls into F's ring.
    template <typename TYPE>
    __device__ __forceinline__ void push_promise(const Promise<TYPE>& p) {
        constexpr unsigned int F = disc_of<TYPE>();
        constexpr unsigned int W = Promise<TYPE>::WORDS;
        constexpr unsigned int SLOTS = ring_slots<F>();
        constexpr unsigned int BASE = ring_base<F>();
        unsigned int w[W];
        p.to_words(w);
        const unsigned int mask = __activemask();
        const unsigned int rank = __popc(mask & util::lanemask_lt());
        const unsigned int leader = __ffs(mask) - 1;
        GroupContext& g = _grp_ctx;
        if constexpr (RING_GROUPS > 1) {
            // The stash holds one ring group at a time: claim it if empty; a promise of
            // another group goes to the arena, where a team of that group will take it.
            constexpr unsigned int G = group_of<F>();
            unsigned int mine = 1u;
            if (rank == 0) {
                unsigned int a = *(volatile unsigned int*)&g.active;
                if (a == NO_GROUP) a = atomicCAS(&g.active, NO_GROUP, G);
                mine = (a == NO_GROUP || a == G) ? 1u : 0u;
            }
            if (__shfl_sync(mask, mine, leader) == 0u) {
                unsigned int spill_w[W];  // the out-of-line path takes a copy (see below)
#pragma unroll
                for (unsigned int i = 0; i < W; i++) spill_w[i] = w[i];
                overflow_to_arena<TYPE>(spill_w, mask);
                return;
            }
        }
        unsigned int base = 0;
        if (rank == 0) base = atomicAdd(&g.count[F], (unsigned int)__popc(mask));
        base = __shfl_sync(mask, base, leader);
        const unsigned int idx = base + rank;
        const unsigned int over = __ballot_sync(mask, idx >= SLOTS);
        if (idx < SLOTS) {
            const unsigned int slot = wrap_slot<SLOTS>(g.bottom[F] + idx);
#pragma unroll
            for (unsigned int i = 0; i < W; i++) g.words[BASE + i * SLOTS + slot] = w[i];
        }
        if (over != 0 && idx >= SLOTS) {
            unsigned int spill_w[W];
#pragma unroll
            for (unsigned int i = 0; i < W; i++) spill_w[i] = w[i];
            overflow_to_arena<TYPE>(spill_w, over);
        }
    }

    // Whole team: waits for the lanes' outstanding LazyLoad copies into the rings (each lane
    // waits for its own, then the warp synchronises so every lane sees every slot).
    __device__ __forceinline__ void settle_loads() {
        if (*(volatile unsigned int*)&_grp_ctx.loads_pending) {
            asm volatile("cp.async.wait_all;\n" ::: "memory");
            __syncwarp();
            if (util::lane_id() == 0) _grp_ctx.loads_pending = 0;
            __syncwarp();
        }
    }

    // prog.async<F> with LazyLoad arguments (see async above).
    template <typename TYPE, typename... ARGS>
    __device__ __forceinline__ void push_lazy(ARGS... args) {
        using Args = typename Promise<TYPE>::Args;
        constexpr unsigned int F = disc_of<TYPE>();
        constexpr unsigned int W = Promise<TYPE>::WORDS;
        constexpr unsigned int SLOTS = ring_slots<F>();
        constexpr unsigned int BASE = ring_base<F>();
        static_assert(sizeof...(ARGS) == Promise<TYPE>::ARITY, "async: wrong number of arguments");
        // The promise with every lazy argument left zero, and which of its words are lazy.
        Promise<TYPE> p(hrm_rt::lazy_placeholder(args)...);
        unsigned int w[W];
        p.to_words(w);
        bool lazy_word[W];
        const unsigned int* lazy_src[W];
#pragma unroll
        for (unsigned int i = 0; i < W; i++) {
            lazy_word[i] = false;
            lazy_src[i] = nullptr;
        }
        hrm_rt::mark_lazy_words<Args, 0>(p.args, lazy_word, lazy_src, args...);
        const unsigned int mask = __activemask();
        const unsigned int rank = __popc(mask & util::lanemask_lt());
        const unsigned int leader = __ffs(mask) - 1;
        GroupContext& g = _grp_ctx;
        unsigned int fits = 1u;
        if constexpr (RING_GROUPS > 1) {
            constexpr unsigned int G = group_of<F>();
            if (rank == 0) {
                unsigned int a = *(volatile unsigned int*)&g.active;
                if (a == NO_GROUP) a = atomicCAS(&g.active, NO_GROUP, G);
                fits = (a == NO_GROUP || a == G) ? 1u : 0u;
            }
            fits = __shfl_sync(mask, fits, leader);
        }
        unsigned int idx = SLOTS;
        if (fits) {
            unsigned int base = 0;
            if (rank == 0) base = atomicAdd(&g.count[F], (unsigned int)__popc(mask));
            base = __shfl_sync(mask, base, leader);
            idx = base + rank;
        }
        const unsigned int over = __ballot_sync(mask, idx >= SLOTS);
        if (idx < SLOTS) {
            const unsigned int slot = wrap_slot<SLOTS>(g.bottom[F] + idx);
#pragma unroll
            for (unsigned int i = 0; i < W; i++) {
                unsigned int* dst = &g.words[BASE + i * SLOTS + slot];
                if (lazy_word[i]) {
                    const unsigned int sa = (unsigned int)__cvta_generic_to_shared(dst);
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(lazy_src[i]) : "memory");
                } else {
                    *dst = w[i];
                }
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
            g.loads_pending = 1u;
        }
        if (over != 0 && idx >= SLOTS) {
            unsigned int spill_w[W];
#pragma unroll
            for (unsigned int i = 0; i < W; i++) spill_w[i] = lazy_word[i] ? __ldcg(lazy_src[i]) : w[i];
            overflow_to_arena<TYPE>(spill_w, over);
        }
    }

    // Lanes in `over` could not fit in shared memory: write them straight to one arena link
    // and publish it to the function's queue. Out of line, so that every push site stays
    // small (the instruction cache is the first limit of a kernel with many async functions);
    // callers pass a copy of the words made only on this rare path, so that the words of
    // ordinary pushes stay in registers instead of going through the stack.
    template <typename TYPE>
    __device__ __noinline__ void overflow_to_arena(const unsigned int (&w)[Promise<TYPE>::WORDS], unsigned int over) {
        constexpr unsigned int F = disc_of<TYPE>();
        constexpr unsigned int W = Promise<TYPE>::WORDS;
        const unsigned int r = __popc(over & util::lanemask_lt());
        const unsigned int n = __popc(over);
        if (r == 0) _grp_ctx.overflowed = 1u;
        unsigned int link = 0xFFFFFFFFu;
        unsigned int got = alloc_links_coop(1, r, over, link);
        link = __shfl_sync(over, link, __ffs(over) - 1);
        if (got == 0 || link == 0xFFFFFFFFu) {
            // No shared-memory slot and no arena link: the promises cannot be kept.
            if (r == 0) hrm_rt::raise_flag(_dev_ctx.ctl, hrm_rt::ARENA_EXHAUSTED_FLAG);
            return;
        }
#pragma unroll
        for (unsigned int i = 0; i < W; i++) __stcg(link_word_ptr(link, i, r), w[i]);
        // No fence: the barrier orders every lane's link stores before the release store that
        // publishes the link (see "Publishing a link" above spill_typed).
        __syncwarp(over);
        if (r == 0) {
            const unsigned int e = hrm_rt::encode_link(link, n);
            const unsigned int slot = atomicAdd(&_grp_ctx.held_n, 1u);
            if (slot < HELD_MAX) {
                _grp_ctx.held_e[slot] = e;
                _grp_ctx.held_f[slot] = F;
            } else {
                hrm_rt::ring_push(_dev_ctx.rings, _dev_ctx.ctl, F, e, 0, 1, 1u << util::lane_id());
            }
        }
        __syncwarp(over);
    }

    // Whole team: publishes the overflow links held during this step.
    __device__ __forceinline__ void publish_held() {
        __syncwarp();
        const unsigned int n = min(_grp_ctx.held_n, HELD_MAX);
        if (n == 0) return;
        hrm_rt::call_before_publish<PROGRAM_SPEC>(*this);
        __syncwarp();
        const unsigned int lane = util::lane_id();
        if (lane < n) {
            hrm_rt::ring_push(_dev_ctx.rings, _dev_ctx.ctl, _grp_ctx.held_f[lane], _grp_ctx.held_e[lane], 0, 1,
                              1u << lane);
        }
        __syncwarp();
        if (lane == 0) _grp_ctx.held_n = 0;
        __syncwarp();
    }

    // -----------------------------------------------------------------------------------
    // Arena links held outside the queues (remapping barriers).
    // -----------------------------------------------------------------------------------
    static const unsigned int NULL_LINK = 0xFFFFFFFFu;

    // One lane: a fresh arena link with its written-count word cleared, or NULL_LINK if the
    // arena is exhausted (ARENA_EXHAUSTED_FLAG raised).
    __device__ unsigned int alloc_held_link() {
        unsigned int link = NULL_LINK;
        const unsigned int got = alloc_links_coop(1, 0, 1u << util::lane_id(), link);
        if (got == 0 || link == NULL_LINK) {
            hrm_rt::raise_flag(_dev_ctx.ctl, hrm_rt::ARENA_EXHAUSTED_FLAG);
            return NULL_LINK;
        }
        _dev_ctx.link_meta[2u * link + 1u] = 0u;
        return link;
    }
    // One lane: returns an unused link to the free ring.
    __device__ void free_held_link(unsigned int link) { free_links_coop(link, 0, 1, 1u << util::lane_id()); }

    // Stores promise p into slot `slot` (< 32) of arena link `link`.
    template <typename TYPE>
    __device__ __forceinline__ void store_in_link(const Promise<TYPE>& p, unsigned int link, unsigned int slot) {
        constexpr unsigned int W = Promise<TYPE>::WORDS;
        unsigned int w[W];
        p.to_words(w);
#pragma unroll
        for (unsigned int i = 0; i < W; i++) __stcg(link_word_ptr(link, i, slot), w[i]);
    }

    // Per held link: `next` word (the barrier's stack) and the number of promises written.
    __device__ __forceinline__ unsigned int* link_next_ptr(unsigned int link) { return &_dev_ctx.link_meta[2u * link]; }
    __device__ __forceinline__ unsigned int* link_written_ptr(unsigned int link) {
        return &_dev_ctx.link_meta[2u * link + 1u];
    }

    // One lane: publishes a held link of function f to its queue.
    __device__ void publish_link(unsigned int f, unsigned int link, unsigned int count) {
        const unsigned int me = 1u << util::lane_id();
        hrm_rt::ring_push(_dev_ctx.rings, _dev_ctx.ctl, f, hrm_rt::encode_link(link, count), 0, 1, me);
    }

    template <unsigned int I>
    __device__ __forceinline__ void push_enum(OpDisc disc, PromiseUnionType& u) {
        if constexpr (I < FN) {
            using Op = typename OpAt<I, OpSet>::type;
            if (disc == I) {
                push_promise<Op>(u.template cast<Op>());
            } else {
                push_enum<I + 1>(disc, u);
            }
        } else {
            atomicOr(&_dev_ctx.ctl->flags, BAD_FUNC_ID_FLAG);
        }
    }

    // ===================================================================================
    // Scheduler (whole team converged).
    // ===================================================================================

    // Publishing a link. The lanes of a team write a link's words (one word of one promise
    // each), meet at __syncwarp, and one lane publishes the link's entry with a release store
    // to its queue slot (ring_push); a consumer's lane reads the slot with an acquire load
    // (ring_take), its team meets at __syncwarp, and every lane reads the words. __syncwarp
    // orders memory among the lanes that take part in it, and release/acquire is
    // cumulative, so each write is ordered before each read in the PTX memory model's
    // causality order without a fence on either side. Reuse is ordered the same way: a
    // consumer's reads of a link precede (barrier, then release of the free-link entry) the
    // next producer's acquire of that entry and its writes. Measured: dropping the three
    // fences these paths had took the R-MAT 2^22 search from 3.5 to 3.2 ms, outputs unchanged.
    //
    // spill_typed: moves the oldest min(count, nlinks*32) promises of function f to the arena;
    // returns the links written. Out of line: it is reached from several places of the scheduler.
    template <unsigned int F>
    __device__ __noinline__ unsigned int spill_typed(unsigned int nlinks) {
        using Op = typename OpAt<F, OpSet>::type;
        constexpr unsigned int W = Promise<Op>::WORDS;
        constexpr unsigned int SLOTS = ring_slots<F>();
        constexpr unsigned int BASE = ring_base<F>();
        GroupContext& g = _grp_ctx;
        const unsigned int lane = util::lane_id();
        settle_loads();
        unsigned int cnt = g.count[F];
        unsigned int n = min(cnt, nlinks * 32u);
        if (n == 0) return 0u;
        unsigned int nl = (n + 31u) / 32u;
        unsigned int link = 0xFFFFFFFFu;
        unsigned int got = alloc_links_coop(nl, lane, 0xFFFFFFFFu, link);
        if (got < nl) {
            // Return what we obtained and keep the promises in shared memory.
            if (got > 0) free_links_coop(link, lane, got, 0xFFFFFFFFu);
            return 0u;
        }
        const unsigned int bottom = g.bottom[F];
        for (unsigned int l = 0; l < nl; l++) {
            unsigned int dst = __shfl_sync(0xFFFFFFFFu, link, l);
            unsigned int k = l * 32u + lane;
            if (k < n) {
                unsigned int slot = wrap_slot<SLOTS>(bottom + k);
#pragma unroll
                for (unsigned int i = 0; i < W; i++) __stcg(link_word_ptr(dst, i, lane), g.words[BASE + i * SLOTS + slot]);
            }
        }
        __syncwarp();
        unsigned int cnt_l = (lane < nl) ? min(32u, n - lane * 32u) : 1u;
        hrm_rt::ring_push(_dev_ctx.rings, _dev_ctx.ctl, F, hrm_rt::encode_link(link, cnt_l), lane, nl, 0xFFFFFFFFu);
        __syncwarp();
        if (lane == 0) {
            g.bottom[F] = wrap_slot<SLOTS>(bottom + n);
            g.count[F] = cnt - n;
        }
        __syncwarp();
        return nl;
    }

    // Spills up to `nlinks` links of function f and counts them in the team's statistics.
    template <unsigned int I>
    __device__ __forceinline__ void spill_fn(unsigned int f, unsigned int nlinks) {
        if constexpr (I < FN) {
            if (f == I) {
                const unsigned int nl = spill_typed<I>(nlinks);
                if (util::lane_id() == 0) _grp_ctx.n_spill += nl;
            } else {
                spill_fn<I + 1>(f, nlinks);
            }
        }
    }

    // Pulls links of function F from the arena until the ring holds >= 32 promises or the
    // queue is empty. Returns the number of links taken.
    template <unsigned int F>
    __device__ unsigned int fill_typed() {
        using Op = typename OpAt<F, OpSet>::type;
        constexpr unsigned int W = Promise<Op>::WORDS;
        constexpr unsigned int SLOTS = ring_slots<F>();
        constexpr unsigned int BASE = ring_base<F>();
        GroupContext& g = _grp_ctx;
        const unsigned int lane = util::lane_id();
        unsigned int cnt = g.count[F];
        unsigned int room = (SLOTS - cnt) / 32u;   // links that surely fit
        unsigned int want = min(room, _dev_ctx.fill_links);
        if (want == 0) return 0;
        unsigned int pos = 0, take = 0;
        if (lane == 0) take = hrm_rt::ring_reserve(_dev_ctx.rings, F, want, pos);
        take = __shfl_sync(0xFFFFFFFFu, take, 0);
        if (take == 0) return 0;
        pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
        unsigned int e = hrm_rt::ring_take(_dev_ctx.rings, _dev_ctx.ctl, F, pos, lane, take);
        // No fence: each entry was read with an acquire load, and the barrier orders those
        // loads before every lane's reads of the links' words.
        __syncwarp();
        const unsigned int bottom = g.bottom[F];
        for (unsigned int l = 0; l < take; l++) {
            unsigned int el = __shfl_sync(0xFFFFFFFFu, e, l);
            if (el == 0) continue;  // timed-out take: flag raised
            unsigned int src = hrm_rt::entry_link(el);
            unsigned int k = hrm_rt::entry_count(el);
            if (lane < k) {
                unsigned int slot = wrap_slot<SLOTS>(bottom + cnt + lane);
#pragma unroll
                for (unsigned int i = 0; i < W; i++) g.words[BASE + i * SLOTS + slot] = __ldcg(link_word_ptr(src, i, lane));
            }
            cnt += k;
        }
        __syncwarp();
        if (lane == 0) g.count[F] = cnt;
        // Give the links back to the free ring. (After a timed-out take the link is unknown
        // and stays out of circulation; the error flag is already raised.)
        bool all_valid = __all_sync(0xFFFFFFFFu, lane >= take || e != 0);
        if (all_valid) free_links_coop(lane < take ? hrm_rt::entry_link(e) : 0u, lane, take, 0xFFFFFFFFu);
        __syncwarp();
        return take;
    }

    template <unsigned int I>
    __device__ unsigned int fill_fn(unsigned int f) {
        if constexpr (I < FN) {
            if (f == I) return fill_typed<I>();
            return fill_fn<I + 1>(f);
        } else {
            return 0;
        }
    }

    // Pops the newest k promises of function F and evaluates them, one per lane. `cnt` is F's
    // count as the scheduler read it (every lane read it before the warp-wide steps that chose
    // the batch, so lane 0 may overwrite it without another barrier); lane 0 also counts the
    // batch in the team's statistics.
    template <unsigned int F>
    __device__ __forceinline__ void run_typed(unsigned int k, unsigned int cnt) {
        using Op = typename OpAt<F, OpSet>::type;
        constexpr unsigned int W = Promise<Op>::WORDS;
        constexpr unsigned int SLOTS = ring_slots<F>();
        constexpr unsigned int BASE = ring_base<F>();
        constexpr bool OLDEST_FIRST = hrm_rt::fn_OLDEST_FIRST<PROGRAM_SPEC, Op>::value;
        GroupContext& g = _grp_ctx;
        const unsigned int lane = util::lane_id();
        settle_loads();
        const unsigned int bottom = g.bottom[F];
        Promise<Op> p;
        if (lane < k) {
            unsigned int w[W];
            // The k newest promises (top of the ring), or the k oldest (bottom) for functions
            // whose spec asks for OLDEST_FIRST; the batch's calls are appended at the top.
            unsigned int slot = wrap_slot<SLOTS>((OLDEST_FIRST ? bottom : bottom + cnt - k) + lane);
#pragma unroll
            for (unsigned int i = 0; i < W; i++) w[i] = g.words[BASE + i * SLOTS + slot];
            p.from_words(w);
        }
        if constexpr (OLDEST_FIRST) __syncwarp();  // every lane has read bottom before lane 0 moves it
        if (lane == 0) {
            g.count[F] = cnt - k;
            if (OLDEST_FIRST) g.bottom[F] = wrap_slot<SLOTS>(bottom + k);
            g.fn_evals[F] += k;
            if (k < 32u) {
                g.n_partial += 1ull;
                g.partial_evals += k;
            }
        }
        __syncwarp();
        if (lane < k) {
            p(*this);
        }
        __syncwarp();
    }

    template <unsigned int I>
    __device__ __forceinline__ void run_fn(unsigned int f, unsigned int k, unsigned int cnt) {
        if constexpr (I < FN) {
            if (f == I) run_typed<I>(k, cnt);
            else run_fn<I + 1>(f, k, cnt);
        }
    }

    // Whole team, after a batch: publishes the arena links of the promises that did not fit in
    // the rings during the batch and clamps the counts. When no push overflowed (the common
    // case) this is one shared-memory read.
    template <bool SYNCED = false>
    __device__ __forceinline__ void settle_overflow() {
        if constexpr (!SYNCED) __syncwarp();
        if (*(volatile unsigned int*)&_grp_ctx.overflowed == 0u) return;
        __syncwarp();
        if (util::lane_id() == 0) _grp_ctx.overflowed = 0u;
        publish_held();
        clamp_counts();
    }

    // Counts above the ring size mean the excess went to the arena: clamp.
    __device__ __forceinline__ void clamp_counts() {
        __syncwarp();
        const unsigned int lane = util::lane_id();
        if (lane < FN) {
            const unsigned int slots = ring_slots_of(lane);
            unsigned int c = _grp_ctx.count[lane];
            if (c > slots) _grp_ctx.count[lane] = slots;
        }
        __syncwarp();
    }

    // Busy/idle accounting and quiescence detection (lane 0 only).
    // Returns 2 = quiescent (or another team declared it), 1 = work may be available, 0 = idle.
    __device__ unsigned int idle_poll(bool& counted_idle, unsigned int& backoff) {
        hrm_rt::RuntimeControl* ctl = _dev_ctx.ctl;
        if (!counted_idle) {
            __threadfence();
            atomicAdd(&ctl->busy_epoch, (unsigned long long)(-(long long)hrm_rt::BUSY_ONE));
            counted_idle = true;
        }
        if (hrm_rt::ld_acquire(&ctl->done) != 0) return 2;
        unsigned long long s1 = hrm_rt::ld_acquire64(&ctl->busy_epoch);
        bool any = false;
        for (unsigned int f = 0; f < FN; f++) {
            if (hrm_rt::ld_acquire(&_dev_ctx.rings.heads[f].avail) != 0) any = true;
        }
        if (any) {
            atomicAdd(&ctl->busy_epoch, hrm_rt::BUSY_ONE + 1ull);
            counted_idle = false;
            backoff = 32;
            return 1;
        }
        if ((s1 >> 40) == 0) {
            unsigned long long s2 = hrm_rt::ld_acquire64(&ctl->busy_epoch);
            if (s2 == s1) {
                atomicExch(&ctl->done, 1u);
                return 2;
            }
        }
        __nanosleep(backoff);
        if (backoff < 2048) backoff <<= 1;
        return 0;
    }

    __device__ void init_team() {
        const unsigned int lane = util::lane_id();
        if (lane < FN) {
            _grp_ctx.count[lane] = 0;
            _grp_ctx.bottom[lane] = 0;
            _grp_ctx.fn_evals[lane] = 0;
        }
        if (lane == 0) {
            _grp_ctx.active = NO_GROUP;
            _grp_ctx.held_n = 0;
            _grp_ctx.loads_pending = 0;
            _grp_ctx.overflowed = 0;
            _grp_ctx.partial_evals = 0;
            _grp_ctx.n_partial = 0;
            _grp_ctx.n_spill = 0;
            _grp_ctx.n_fill = 0;
            _grp_ctx.n_mw = 0;
            _grp_ctx.n_idle = 0;
        }
        __syncwarp();
    }

    // The persistent scheduling loop of one team (async.h:2625-2668 / :2155-2319).
    __device__ void exec(unsigned int cycle_count) {
        const unsigned int lane = util::lane_id();
        _thd_ctx.thread_id = blockIdx.x * blockDim.x + threadIdx.x;
        _thd_ctx.rand_state = _thd_ctx.thread_id;
        init_team();
        hrm_rt::call_initialize<PROGRAM_SPEC>(*this);
        __syncwarp();
        publish_held();
        clamp_counts();  // pushes past a ring went to the arena

        GroupContext& g = _grp_ctx;
        hrm_rt::RuntimeControl* ctl = _dev_ctx.ctl;
        bool can_make_work = true;
        bool counted_idle = false;
        unsigned int backoff = 32;
        unsigned int prev_c = 0;          // lane f: f's count at the previous step
        unsigned int age = 0;             // lane f: steps f has held a partial batch that did not grow
        unsigned int rotate = 0;          // next function to favour for a forced partial batch
        unsigned int quiet = 0;           // partial batches left to run without looking at the arena
        bool quiescent = false;
        const unsigned int my_ring = (lane < FN) ? ring_slots_of(lane) : 0u;  // lane f: f's ring size
        const unsigned int my_group = (lane < FN) ? group_of_fn(lane) : NO_GROUP;  // lane f: f's ring group

        for (unsigned int cycle = 0; cycle < cycle_count; cycle++) {
            // Stop on a halt request (halt_early, or the host's halt_request) or an error flag.
            if ((cycle & 31u) == 0) {
                unsigned int fl = 0;
                if (lane == 0) {
                    fl = hrm_rt::ld_relaxed(&ctl->flags);
                    if (hrm_rt::ld_relaxed(&ctl->halt_request) != 0u && !(fl & EARLY_HALT_FLAG)) {
                        atomicOr(&ctl->flags, EARLY_HALT_FLAG);
                        fl |= EARLY_HALT_FLAG;
                    }
                }
                fl = __shfl_sync(0xFFFFFFFFu, fl, 0);
                if (fl & (EARLY_HALT_FLAG | hrm_rt::ERROR_MASK)) break;
            }

            // Pick the fullest function, except that a function past its high-water mark
            // (fewer than 32 free slots) runs first: it always holds a full batch (rings have
            // at least 64 slots), and running it makes the room that running another
            // function would otherwise have to make by spilling it to the arena.
            unsigned int c = (lane < FN) ? g.count[lane] : 0u;
            if constexpr (RING_GROUPS > 1) {
                // An empty stash belongs to no ring group.
                if (__all_sync(0xFFFFFFFFu, lane >= FN || c == 0u) && lane == 0) g.active = NO_GROUP;
                __syncwarp();
            }
            unsigned int key = (lane < FN) ? ((min(c, 0xFFFFu) << 5) | lane) : 0u;
            const unsigned int over = (lane < FN && c > my_ring - 32u) ? c - (my_ring - 32u) : 0u;
            const unsigned int okey = over ? ((min(over, 0xFFFFu) << 5) | lane) : 0u;
            const unsigned int obest = __reduce_max_sync(0xFFFFFFFFu, okey);
            unsigned int best = obest ? ((min(__shfl_sync(0xFFFFFFFFu, c, obest & 31u), 0xFFFFu) << 5) | (obest & 31u))
                                      : __reduce_max_sync(0xFFFFFFFFu, key);
            unsigned int bf = best & 31u, bc = best >> 5;

            // A partial batch that stops growing is starving: other work (full batches of
            // other functions, fills, make_work) keeps the team busy and nothing will top it
            // up. After `patience` such steps run it anyway, starving functions taken
            // in turn, so that no promise waits without bound (e.g. the last Collatz steps of
            // a small job among photon jobs). A partial batch that keeps growing (photon
            // tallies fed by every collide batch) is left to fill up.
            if (lane < FN) {
                age = (c > 0u && c < 32u && c <= prev_c) ? age + 1u : 0u;
                prev_c = c;
            }
            bool forced = false;
            const unsigned int starving = __ballot_sync(0xFFFFFFFFu, lane < FN && age >= _dev_ctx.patience);
            if (starving != 0u) {
                rotate = (rotate + 1u) % FN;
                const unsigned int upper = starving >> rotate;
                bf = upper ? rotate + (unsigned int)(__ffs(upper) - 1) : (unsigned int)(__ffs(starving) - 1);
                bc = __shfl_sync(0xFFFFFFFFu, c, bf);
                if (lane == bf) age = 0;
                forced = true;
            }
            // A tail: the last look found the arena empty and make_work done, so the next few
            // partial batches run without another look (each look is a round trip to L2):
            // Collatz 1..2^20 1.83 -> 1.75 ms, R-MAT 2^22 2.80 -> 2.72 ms, same outputs.
            const bool tail = bc > 0u && quiet > 0u && !can_make_work;
            if (tail) quiet--;
            if (bc < 32u && !forced && !tail) {
                // No full batch locally: try the arena for the function closest to full.
                unsigned int av = 0;
                if (lane < FN) av = hrm_rt::ld_relaxed(&_dev_ctx.rings.heads[lane].avail);
                // With ring groups, only the active group's queues (any, if the stash is empty).
                const unsigned int act = (RING_GROUPS > 1) ? g.active : 0u;
                const bool own = lane < FN && (RING_GROUPS == 1 || act == NO_GROUP || my_group == act);
                unsigned int fkey = (own && (int)av > 0) ? (((min(c, 0xFFFFu) + 1u) << 5) | lane) : 0u;
                unsigned int fbest = __reduce_max_sync(0xFFFFFFFFu, fkey);
                if constexpr (RING_GROUPS > 1) {
                    // Work of another group waits in the arena and this team has no full batch
                    // nor queued work of its own: hand its partial work to the arena and change
                    // group, instead of making more work of its own group.
                    if (fbest == 0 && act != NO_GROUP &&
                        __any_sync(0xFFFFFFFFu, lane < FN && my_group != act && (int)av > 0)) {
                        hrm_rt::call_before_publish<PROGRAM_SPEC>(*this);
                        __syncwarp();
                        for (unsigned int f = 0; f < FN; f++) {
                            unsigned int cf = g.count[f];
                            if (cf > 0) spill_fn<0>(f, (cf + 31u) / 32u);
                        }
                        if (__all_sync(0xFFFFFFFFu, lane >= FN || g.count[lane] == 0u)) continue;
                        // A full arena kept some promises here: go on with the counts as they are.
                        c = (lane < FN) ? g.count[lane] : 0u;
                        bc = __shfl_sync(0xFFFFFFFFu, c, bf);
                    }
                }
                if (fbest != 0) {
                    unsigned int ff = fbest & 31u;
                    if (counted_idle) {
                        if (lane == 0) atomicAdd(&ctl->busy_epoch, hrm_rt::BUSY_ONE + 1ull);
                        counted_idle = false;
                    }
                    if constexpr (RING_GROUPS > 1) {
                        if (act == NO_GROUP && lane == 0) g.active = group_of_fn(ff);
                        __syncwarp();
                    }
                    unsigned int took = fill_fn<0>(ff);
                    if (lane == 0) g.n_fill += took;
                    if (took > 0) continue;
                    // Another team won the race for that work. Never make new work while
                    // the arena holds a backlog: run what is local, or look again.
                    if (bc == 0) {
                        __nanosleep(64);
                        continue;
                    }
                } else if (can_make_work) {
                    if (counted_idle) {
                        if (lane == 0) atomicAdd(&ctl->busy_epoch, hrm_rt::BUSY_ONE + 1ull);
                        counted_idle = false;
                    }
                    const unsigned int before = __reduce_add_sync(0xFFFFFFFFu, c);
                    bool more = hrm_rt::call_make_work<PROGRAM_SPEC>(*this);
                    publish_held();
                    can_make_work = __any_sync(0xFFFFFFFFu, more);
                    if (lane == 0) g.n_mw++;
                    clamp_counts();
                    const unsigned int after = __reduce_add_sync(0xFFFFFFFFu, (lane < FN) ? g.count[lane] : 0u);
                    // New local work: plan again. Nothing local at all: keep asking. Otherwise
                    // make_work added nothing, so run the partial batch held here instead of
                    // waiting (a make_work that keeps returning true, e.g. a serving loop
                    // polling for jobs, must not starve promises already in the stash).
                    if (after != before || bc == 0) continue;
                }
                if (fbest == 0 && !can_make_work) quiet = 3;
                if (bc == 0) {
                    // Nothing local, nothing in the arena, nothing to make: idle.
                    hrm_rt::call_on_idle<PROGRAM_SPEC>(*this);
                    __syncwarp();
                    unsigned int st = 0;
                    if (lane == 0) st = idle_poll(counted_idle, backoff);
                    st = __shfl_sync(0xFFFFFFFFu, st, 0);
                    counted_idle = __shfl_sync(0xFFFFFFFFu, (unsigned int)counted_idle, 0) != 0;
                    if (lane == 0) g.n_idle++;
                    if (st == 2) { quiescent = true; break; }
                    continue;
                }
            }

            // Evaluate one batch (full when possible).
            if (counted_idle) {
                if (lane == 0) atomicAdd(&ctl->busy_epoch, hrm_rt::BUSY_ONE + 1ull);
                counted_idle = false;
            }
            unsigned int k = min(bc, 32u);
            // Every other ring needs one link of headroom for the calls this batch makes
            // (the batch's own ring frees k slots when it is popped).
            unsigned int hi = __ballot_sync(0xFFFFFFFFu, lane < FN && lane != bf && c > my_ring - 32u);
            if (hi) {
                hrm_rt::call_before_publish<PROGRAM_SPEC>(*this);
                __syncwarp();
            }
            while (hi) {
                unsigned int f = __ffs(hi) - 1;
                hi &= hi - 1;
                unsigned int cf = __shfl_sync(0xFFFFFFFFu, c, f);
                unsigned int rf = __shfl_sync(0xFFFFFFFFu, my_ring, f);
                spill_fn<0>(f, (cf - (rf - 32u) + 31u) / 32u);
            }
            // Evaluate; then, while the function still holds a full batch and every other ring
            // keeps a batch's worth of room, up to BURST - 1 more batches of it without a
            // scheduling step (one evaluation site, so the kernel holds one copy of each eval).
            for (unsigned int rep = 0;; rep++) {
                run_fn<0>(bf, k, bc);
                if constexpr (hrm_rt::has_after_batch<PROGRAM_SPEC, ProgramType>::value) {
                    hrm_rt::call_after_batch<PROGRAM_SPEC>(*this);
                    settle_overflow();
                } else {
                    settle_overflow<true>();  // run_fn ended with a barrier
                }
                if (k < 32u || forced || rep + 1u >= BURST) break;
                const unsigned int cn = (lane < FN) ? g.count[lane] : 0u;
                bc = __shfl_sync(0xFFFFFFFFu, cn, bf);
                if (bc < 32u) break;
                if (__any_sync(0xFFFFFFFFu, lane < FN && lane != bf && cn + 32u > my_ring)) break;
            }
        }

        hrm_rt::call_finalize<PROGRAM_SPEC>(*this);
        __syncwarp();
        publish_held();
        clamp_counts();  // pushes past a ring went to the arena
        hrm_rt::call_before_publish<PROGRAM_SPEC>(*this);
        __syncwarp();

        // Leave nothing in shared memory: spill every pending promise.
        for (unsigned int f = 0; f < FN; f++) {
            unsigned int cf = g.count[f];
            if (cf > 0) spill_fn<0>(f, (cf + 31u) / 32u);
        }
        __syncwarp();
        const unsigned long long my_evals = (lane < FN) ? g.fn_evals[lane] : 0ull;
        if (my_evals != 0) atomicAdd(&_dev_ctx.stats[hrm_rt::STAT_FN_EVALS + lane], my_evals);
        unsigned long long n_evals = my_evals;
#pragma unroll
        for (unsigned int o = 16; o > 0; o >>= 1) n_evals += __shfl_xor_sync(0xFFFFFFFFu, n_evals, o);
        if (lane == 0) {
            if (can_make_work) atomicOr(&ctl->flags, EARLY_HALT_FLAG);
            for (unsigned int f = 0; f < FN; f++) {
                if (g.count[f] != 0) atomicOr(&ctl->flags, hrm_rt::ARENA_EXHAUSTED_FLAG);
            }
            if (!counted_idle) {
                __threadfence();
                atomicAdd(&ctl->busy_epoch, (unsigned long long)(-(long long)hrm_rt::BUSY_ONE));
            }
            unsigned long long* st = _dev_ctx.stats;
            atomicAdd(&st[hrm_rt::STAT_EVALS], n_evals);
            const unsigned long long full = (n_evals - g.partial_evals) / 32ull;
            atomicAdd(&st[hrm_rt::STAT_BATCHES], full + g.n_partial);
            atomicAdd(&st[hrm_rt::STAT_FULL_BATCHES], full);
            atomicAdd(&st[hrm_rt::STAT_SPILL_LINKS], g.n_spill);
            atomicAdd(&st[hrm_rt::STAT_FILL_LINKS], g.n_fill);
            atomicAdd(&st[hrm_rt::STAT_MAKE_WORK], g.n_mw);
            atomicAdd(&st[hrm_rt::STAT_IDLE_POLLS], g.n_idle);
            (void)quiescent;
            __threadfence();
            unsigned int out = atomicAdd(&ctl->checkout, 1u);
            if (out == ctl->total_teams - 1u) {
                // Last team out decides completion.
                __threadfence();
                unsigned int old = atomicAnd(&ctl->flags, ~EARLY_HALT_FLAG);
                unsigned int done = hrm_rt::ld_acquire(&ctl->done);
                bool left = false;
                for (unsigned int f = 0; f < FN; f++) {
                    if (hrm_rt::ld_acquire(&_dev_ctx.rings.heads[f].avail) != 0) left = true;
                }
                if (done && !left && !(old & (EARLY_HALT_FLAG | hrm_rt::ERROR_MASK))) {
                    atomicOr(&ctl->flags, COMPLETION_FLAG);
                }
            }
        }
    }

    // Device side of init<P>: reset queues, arena and control block (async.h:2405-2516).
    __device__ static void init_program(DeviceContext ctx) {
        size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
        size_t nthreads = (size_t)gridDim.x * blockDim.x;
        hrm_rt::ring_init_slots(ctx.rings, FN + 1, tid, nthreads);
        if (tid == 0) {
            ctx.ctl->flags = 0;
            ctx.ctl->checkout = 0;
            ctx.ctl->done = 0;
            ctx.ctl->halt_request = 0;
            ctx.ctl->bump = 0;
            ctx.ctl->arena_links = ctx.arena_links;
            ctx.ctl->busy_epoch = 0;
        }
        if (tid < hrm_rt::STAT_COUNT) ctx.stats[tid] = 0;
    }

    // ===================================================================================
    // Host launch helpers used by init<P> and exec<P>.
    // ===================================================================================
    // Team stashes live in dynamic shared memory: TEAMS_PER_CTA contexts, then as many
    // GroupStates, each rounded up to 16 bytes.
    static constexpr size_t align16(size_t x) { return (x + 15u) & ~(size_t)15u; }
    static const size_t CTX_BYTES = align16(sizeof(GroupContext));
    static const size_t STATE_BYTES = align16(sizeof(GroupState));
    static const size_t SMEM_BYTES = TEAMS_PER_CTA * (CTX_BYTES + STATE_BYTES);
    static_assert(SMEM_BYTES <= 227u * 1024u, "team stashes exceed 227 KB of shared memory per CTA");

    // Opts the exec kernel into more than 48 KB of dynamic shared memory (once per device)
    // and returns how many of its CTAs can be resident at once.
    static unsigned int resident_ctas() {
        static int cached_dev = -1;
        static unsigned int cached = 0;
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev != cached_dev) {
            util::host::auto_throw(cudaFuncSetAttribute(hrm_rt::async_exec_kernel<ProgramType>,
                                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        (int)SMEM_BYTES));
            cached = hrm_rt::max_resident_ctas(hrm_rt::async_exec_kernel<ProgramType>, (int)CTA_THREADS, SMEM_BYTES);
            cached_dev = dev;
        }
        return cached;
    }

    // Number of CTAs exec<P> launches for `group_count` work groups.
    static unsigned int ctas_for(size_t group_count) {
        size_t want = (group_count + TEAMS_PER_CTA - 1) / TEAMS_PER_CTA;
        if (want == 0) want = 1;
        unsigned int cap = resident_ctas();
        if (cap == 0) cap = 1;
        return (unsigned int)(want < cap ? want : cap);
    }

    static void launch_init(Instance& inst, size_t, cudaStream_t stream) {
        hrm_rt::async_init_kernel<ProgramType><<<148, 256, 0, stream>>>(inst.to_context());
    }

    static void launch_exec(Instance& inst, size_t group_count, size_t cycle_count, cudaStream_t stream) {
        unsigned int ctas = ctas_for(group_count);
        unsigned int cycles = cycle_count > 0xFFFFFFFFull ? 0xFFFFFFFFu : (unsigned int)cycle_count;
        DeviceContext ctx = inst.to_context();
        hrm_rt::async_prep_kernel<ProgramType><<<1, 32, 0, stream>>>(ctx, ctas * TEAMS_PER_CTA);
        hrm_rt::async_exec_kernel<ProgramType><<<ctas, CTA_THREADS, SMEM_BYTES, stream>>>(ctx, inst.device_state,
                                                                                           cycles);
    }
};

namespace hrm_rt {

template <typename PROG>
__global__ void async_init_kernel(typename PROG::DeviceContext ctx) {
    PROG::init_program(ctx);
}

// Resets the per-exec counters before the persistent kernel starts.
template <typename PROG>
__global__ void async_prep_kernel(typename PROG::DeviceContext ctx, unsigned int total_teams) {
    if (threadIdx.x == 0) {
        ctx.ctl->checkout = 0;
        ctx.ctl->done = 0;
        ctx.ctl->total_teams = total_teams;
        ctx.ctl->busy_epoch = (unsigned long long)total_teams << 40;
        atomicAnd(&ctx.ctl->flags, ~COMPLETION_FLAG);
        __threadfence();
    }
}

template <typename PROG>
__global__ void __launch_bounds__(PROG::CTA_THREADS, PROG::MIN_CTAS_PER_SM)
    async_exec_kernel(typename PROG::DeviceContext ctx, typename PROG::DeviceState device, unsigned int cycles) {
    extern __shared__ __align__(16) unsigned char hrm_team_smem[];
    const unsigned int team = threadIdx.x >> 5;
    auto* grp_ctx = reinterpret_cast<typename PROG::GroupContext*>(hrm_team_smem + team * PROG::CTX_BYTES);
    auto* grp_state = reinterpret_cast<typename PROG::GroupState*>(
        hrm_team_smem + PROG::TEAMS_PER_CTA * PROG::CTX_BYTES + team * PROG::STATE_BYTES);
    typename PROG::ThreadContext thd_ctx;
    typename PROG::ThreadState thd_state;
    PROG prog(ctx, *grp_ctx, thd_ctx, device, *grp_state, thd_state);
    prog.exec(cycles);
}

}  // namespace hrm_rt

#endif
