// barrier.h — RemappingBarrier and UnitBarrier.
//
// Contract kept from harmonize/cpp/sync/barrier.h:
//  * RemappingBarrier<OpSet>::blank(n) makes a barrier whose semaphore starts at n
//    (barrier.h:60-70); it lives in device memory (host code copies blank() values there);
//  * barrier.await(prog, Promise<F>(...)) holds the promise while the semaphore is non-zero
//    and passes it straight to prog.async if the barrier is already released
//    (barrier.h:460-609); union_await does the same for a runtime discriminant;
//  * add_semaphore / sub_semaphore change the semaphore and release every held promise when
//    it reaches zero; release() forces it to zero (barrier.h:614-639);
//  * UnitBarrier holds one promise and calls it on release (barrier.h:648-699).
//
// Design (B200): held promises live in arena links, packed across warps. Per function the
// barrier keeps one partial link, described by one 64-bit word {tag, slots reserved, link};
// the lanes of a warp that await the same barrier at one call site (grouped by
// __match_any_sync on the barrier address) reserve their slots in it with ONE
// compare-and-swap made by their leader, then each lane writes its promise into its slot and
// the leader adds the group's size to the link's written count. A group that does not fit
// installs a fresh link as the partial one (same compare-and-swap) and pushes the link it
// replaced on the function's stack of retired links (a compare-and-swap on a 32-bit head),
// whose `next` word also records how many slots were reserved in it. So held promises of
// different warps share links, as the original's partial_table does (barrier.h:40-600), and
// a released barrier publishes links of up to 32 promises, which teams merge into warp-full
// batches: promises are regrouped by their next function. Releasing detaches the partial
// word and the stack with one exchange each, waits (bounded) until every reserved slot of a
// link is written, and publishes the link to its function's queue. An awaiter re-checks the
// semaphore after its write (with a sequentially consistent fence on both sides) and sweeps
// itself if the barrier was released meanwhile, so no promise is stranded. The tag makes a
// stale compare-and-swap fail even when a link is reused. Barriers need the AsyncProgram arena.
#ifndef HARMONIZE_B200_BARRIER_H
#define HARMONIZE_B200_BARRIER_H

#include "async_program.h"

namespace hrm_rt {
__device__ __forceinline__ void fence_sc() { asm volatile("fence.sc.gpu;" ::: "memory"); }

// Partial-link word of a RemappingBarrier: bits 0-31 link + 1 (0 = none), 32-39 slots
// reserved, 40-63 tag (advanced by every change).
__host__ __device__ __forceinline__ unsigned long long partial_word(unsigned long long tag, unsigned int reserved,
                                                                    unsigned int link_plus_1) {
    return ((tag & 0xFFFFFFull) << 40) | ((unsigned long long)(reserved & 0xFFu) << 32) | link_plus_1;
}
__device__ __forceinline__ unsigned int partial_link1(unsigned long long w) { return (unsigned int)w; }
__device__ __forceinline__ unsigned int partial_reserved(unsigned long long w) { return (unsigned int)(w >> 32) & 0xFFu; }
__device__ __forceinline__ unsigned long long partial_tag(unsigned long long w) { return w >> 40; }

// Stack `next` word of a retired held link: bits 0-26 next link + 1 (0 = end), 27-31 slots
// reserved - 1 (a retired link holds 1..32 promises; arena links number below 2^27).
__device__ __forceinline__ unsigned int held_next_word(unsigned int next1, unsigned int reserved) {
    return ((reserved - 1u) << 27) | next1;
}
}  // namespace hrm_rt

template <typename OP_SET, typename ADR_TYPE>
struct RemappingBarrier {
    using AdrType = ADR_TYPE;
    using UnionType = PromiseUnion<OP_SET>;
    static const size_t TYPE_COUNT = UnionType::Info::COUNT;

    TaggedSemaphore semaphore;
    unsigned int count;                          // promises currently held
    unsigned int heads[TYPE_COUNT];              // per function: retired link + 1, or 0
    unsigned long long partial[TYPE_COUNT];      // per function: partial-link word

    RemappingBarrier() = default;
    // Same as blank(sem_val) (the original's Future builds its barrier from a semaphore value,
    // async/future.h:20-22).
    __host__ __device__ explicit RemappingBarrier(unsigned int sem_val) : RemappingBarrier(blank(sem_val)) {}

    static __host__ __device__ RemappingBarrier<OP_SET, ADR_TYPE> blank(unsigned int sem_val) {
        RemappingBarrier<OP_SET, ADR_TYPE> r;
        r.semaphore = TaggedSemaphore(sem_val, 1);
        r.count = 0u;
        for (size_t i = 0; i < TYPE_COUNT; i++) {
            r.heads[i] = 0u;
            r.partial[i] = 0ull;
        }
        return r;
    }

    // One lane: waits (bounded) until the `reserved` slots of held link `link` are written,
    // then publishes it to function f's queue. False if the wait timed out (flag raised).
    template <typename PROGRAM>
    __device__ bool publish_held(PROGRAM program, unsigned int f, unsigned int link, unsigned int reserved) {
        unsigned int spins = 0;
        while (hrm_rt::ld_acquire(program.link_written_ptr(link)) < reserved) {
            if (++spins > hrm_rt::SPIN_LIMIT) {
                hrm_rt::raise_flag(program._dev_ctx.ctl, hrm_rt::WAIT_TIMEOUT_FLAG);
                return false;
            }
            __nanosleep(64);
        }
        atomicSub(&count, reserved);
        program.publish_link(f, link, reserved);
        return true;
    }

    // Detaches every held link and hands it to the program's queues (one lane).
    template <typename PROGRAM>
    __device__ void release_sweep(PROGRAM program) {
        for (unsigned int f = 0; f < TYPE_COUNT; f++) {
            // The partial link: swap in "none" (with the next tag).
            unsigned long long w = hrm_rt::ld_acquire64(&partial[f]);
            bool detached = false;
            for (unsigned int tries = 0; tries < hrm_rt::SPIN_LIMIT && !detached; tries++) {
                if (hrm_rt::partial_link1(w) == 0u) break;  // nothing to detach
                const unsigned long long none = hrm_rt::partial_word(hrm_rt::partial_tag(w) + 1ull, 0u, 0u);
                const unsigned long long prev = atomicCAS(&partial[f], w, none);
                if (prev == w) detached = true;
                else w = prev;
            }
            if (detached) {
                __threadfence();  // after observing the word: the link's state written before it
                publish_held(program, f, hrm_rt::partial_link1(w) - 1u, hrm_rt::partial_reserved(w));
            } else if (hrm_rt::partial_link1(w) != 0u) {
                hrm_rt::raise_flag(program._dev_ctx.ctl, hrm_rt::WAIT_TIMEOUT_FLAG);
            }
            // The retired links.
            unsigned int h = atomicExch(&heads[f], 0u);
            __threadfence();  // the `next` words stored before each push are visible
            // A stack holds at most every link of the arena; stop at the first failed wait.
            unsigned int guard = 0;
            while (h != 0u && guard++ < program._dev_ctx.arena_links) {
                const unsigned int link = h - 1u;
                const unsigned int nw = hrm_rt::ld_relaxed(program.link_next_ptr(link));
                if (!publish_held(program, f, link, (nw >> 27) + 1u)) break;
                h = nw & 0x07FFFFFFu;
            }
        }
    }

    // Leader of a group of m lanes: reserves m consecutive slots in function f's partial link
    // (or in a fresh link that becomes the partial one). Returns the link (NULL_LINK if the
    // arena is exhausted or the reservation timed out) and the first slot in `base`.
    template <typename PROGRAM>
    __device__ unsigned int reserve(PROGRAM program, unsigned int f, unsigned int m, unsigned int& base) {
        unsigned int fresh = PROGRAM::NULL_LINK;
        unsigned int dst = PROGRAM::NULL_LINK;
        bool settled = false;  // reserved, or gave up because the arena is exhausted
        unsigned long long w = hrm_rt::ld_acquire64(&partial[f]);
        for (unsigned int tries = 0; tries < hrm_rt::SPIN_LIMIT && !settled; tries++) {
            const unsigned int l1 = hrm_rt::partial_link1(w);
            const unsigned int c = hrm_rt::partial_reserved(w);
            const unsigned long long tag = hrm_rt::partial_tag(w) + 1ull;
            if (l1 != 0u && c + m <= 32u) {
                const unsigned long long prev = atomicCAS(&partial[f], w, hrm_rt::partial_word(tag, c + m, l1));
                if (prev == w) {
                    dst = l1 - 1u;
                    base = c;
                    settled = true;
                } else {
                    w = prev;
                }
                continue;
            }
            if (fresh == PROGRAM::NULL_LINK) {
                fresh = program.alloc_held_link();  // raises ARENA_EXHAUSTED when it fails
                if (fresh == PROGRAM::NULL_LINK) {
                    settled = true;
                    continue;
                }
                __threadfence();  // its cleared written count before it can be seen
            }
            const unsigned long long prev = atomicCAS(&partial[f], w, hrm_rt::partial_word(tag, m, fresh + 1u));
            if (prev == w) {
                dst = fresh;
                base = 0u;
                fresh = PROGRAM::NULL_LINK;
                settled = true;
                if (l1 != 0u) retire(program, f, l1 - 1u, c);
            } else {
                w = prev;
            }
        }
        if (fresh != PROGRAM::NULL_LINK) program.free_held_link(fresh);
        if (!settled) hrm_rt::raise_flag(program._dev_ctx.ctl, hrm_rt::WAIT_TIMEOUT_FLAG);
        return dst;
    }

    // One lane: pushes a link that is no longer the partial one on function f's stack.
    template <typename PROGRAM>
    __device__ void retire(PROGRAM program, unsigned int f, unsigned int link, unsigned int reserved) {
        unsigned int old = hrm_rt::ld_relaxed(&heads[f]);
        for (unsigned int tries = 0; tries < hrm_rt::SPIN_LIMIT; tries++) {
            *program.link_next_ptr(link) = hrm_rt::held_next_word(old, reserved);
            __threadfence();
            const unsigned int prev = atomicCAS(&heads[f], old, link + 1u);
            if (prev == old) return;
            old = prev;
        }
        hrm_rt::raise_flag(program._dev_ctx.ctl, hrm_rt::WAIT_TIMEOUT_FLAG);
    }

    template <bool CAN_RELEASE = true, typename PROGRAM, typename OP_TYPE>
    __device__ void await(PROGRAM program, Promise<OP_TYPE> promise) {
        static_assert(UnionType::template Lookup<OP_TYPE>::type::CONTAINED,
                      "TYPE ERROR: Remapping work queue cannot queue promises of this type.");
        constexpr unsigned int F = UnionType::template Lookup<OP_TYPE>::type::DISC;
        if (CAN_RELEASE && hrm_rt::ld_relaxed(&semaphore.sem) == 0u) {
            program.async_call(promise);
            return;
        }
        const unsigned int active = __activemask();
        const unsigned int group = __match_any_sync(active, (unsigned long long)(uintptr_t)this);
        const unsigned int r = __popc(group & util::lanemask_lt());
        const unsigned int m = __popc(group);
        const unsigned int leader = __ffs(group) - 1;
        unsigned int link = PROGRAM::NULL_LINK, base = 0u;
        if (r == 0) {
            atomicAdd(&count, m);
            link = reserve(program, F, m, base);
        }
        link = __shfl_sync(group, link, leader);
        base = __shfl_sync(group, base, leader);
        if (link != PROGRAM::NULL_LINK) program.store_in_link(promise, link, base + r);  // base + m <= 32
        __threadfence();
        __syncwarp(group);
        if (r == 0 && link != PROGRAM::NULL_LINK) {
            atomicAdd(program.link_written_ptr(link), m);
            hrm_rt::fence_sc();
            if (CAN_RELEASE && hrm_rt::ld_relaxed(&semaphore.sem) == 0u) release_sweep(program);
        }
        __syncwarp(group);
    }

    template <bool CAN_RELEASE = true, typename PROGRAM>
    __device__ void union_await(PROGRAM program, OpDisc disc, typename PROGRAM::PromiseUnionType promise_union) {
        union_await_at<CAN_RELEASE, 0>(program, disc, promise_union);
    }

    template <bool CAN_RELEASE, unsigned int I, typename PROGRAM>
    __device__ void union_await_at(PROGRAM program, OpDisc disc, typename PROGRAM::PromiseUnionType& u) {
        if constexpr (I < TYPE_COUNT) {
            using Op = typename OpAt<I, OP_SET>::type;
            if (disc == I) await<CAN_RELEASE>(program, u.template cast<Op>());
            else union_await_at<CAN_RELEASE, I + 1>(program, disc, u);
        }
    }

    template <typename PROGRAM>
    __device__ void release(PROGRAM program) {
        unsigned int now = atomicExch(&semaphore.sem, 0u);
        hrm_rt::fence_sc();
        if (now != 0u) release_sweep(program);
    }

    template <typename PROGRAM>
    __device__ void add_semaphore(PROGRAM program, unsigned int delta) {
        unsigned int now = atomicAdd(&semaphore.sem, delta);
        hrm_rt::fence_sc();
        if (now + delta == 0u) release_sweep(program);
    }

    template <typename PROGRAM>
    __device__ void sub_semaphore(PROGRAM program, unsigned int delta) {
        unsigned int now = atomicAdd(&semaphore.sem, (unsigned int)(0u - delta));
        hrm_rt::fence_sc();
        if (now - delta == 0u) release_sweep(program);
    }
};

template <typename OP_SET, typename ADR_TYPE>
struct UnitBarrier {
    using AdrType = ADR_TYPE;
    TaggedSemaphore semaphore;
    PromiseEnum<OP_SET> promise;

    UnitBarrier() = default;
    __host__ __device__ UnitBarrier(PromiseEnum<OP_SET> p, unsigned int sem_val) : semaphore(sem_val, 0), promise(p) {}

    template <typename PROGRAM>
    __device__ void release(PROGRAM program) {
        if (atomicExch(&semaphore.sem, 0u) != 0u) program.async_call(promise);
    }
    template <typename PROGRAM>
    __device__ void add_semaphore(PROGRAM program, unsigned int delta) {
        unsigned int old = atomicAdd(&semaphore.sem, delta);
        if (old + delta == 0u && old != 0u) program.async_call(promise);
    }
    template <typename PROGRAM>
    __device__ void sub_semaphore(PROGRAM program, unsigned int delta) {
        unsigned int old = atomicAdd(&semaphore.sem, (unsigned int)(0u - delta));
        if (old - delta == 0u && old != 0u) program.async_call(promise);
    }
};

// A value tied to a barrier (async/future.h:6-33 of the original). Continuations that need
// the value wait on the barrier with `await(prog, Promise<F>(...))`; each producer stores its
// part and calls `fulfill(prog)`, which takes one off the barrier's semaphore, so the held
// continuations are released once every expected producer has fulfilled (the semaphore value
// given at construction). `set` stores the value and fulfills; `get` reads it from L2, so a
// continuation that runs on another SM never sees a stale copy. (The original's ReturnOp,
// future.h:37-61, which was to fill futures from returning calls, is not instantiable there;
// producers store their results themselves.) Futures live in device memory, like barriers.
template <typename TYPE, typename BARRIER>
struct Future {
    using BarrierType = BARRIER;
    using Type = TYPE;
    static_assert(sizeof(TYPE) % 4 == 0, "Future values are read as 32-bit words");

    BarrierType barrier;
    Type data;

    Future() = default;
    __host__ __device__ Future(unsigned int semaphore_value) : barrier(semaphore_value) {}

    template <typename PROGRAM, typename OP_TYPE>
    __device__ void await(PROGRAM program, Promise<OP_TYPE> promise) {
        barrier.await(program, promise);
    }

    template <typename PROGRAM>
    __device__ void fulfill(PROGRAM program) {
        __threadfence();
        barrier.sub_semaphore(program, 1u);
    }

    template <typename PROGRAM>
    __device__ void set(PROGRAM program, const TYPE& value) {
        data = value;
        fulfill(program);
    }

    __device__ TYPE get() const {
        TYPE v;
        const unsigned int* src = (const unsigned int*)&data;
        unsigned int* dst = (unsigned int*)&v;
#pragma unroll
        for (unsigned int i = 0; i < sizeof(TYPE) / 4u; i++) dst[i] = __ldcg(src + i);
        return v;
    }
};

#endif
