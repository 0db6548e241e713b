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
// Design (B200): the lanes of a warp that await the same barrier at the same call site
// (grouped by __match_any_sync on the barrier address) write their promises into ONE
// arena link with one allocation, and the link is pushed on the barrier's per-function
// lock-free stack (compare-and-swap on a 32-bit head). Releasing detaches each function's
// stack with one exchange and publishes its links to that function's queue, where teams
// merge them into warp-full batches: promises are regrouped by their next function.
// An awaiter re-checks the semaphore after its push (with a sequentially consistent
// fence on both sides), and sweeps itself if the barrier was released meanwhile, so no
// promise is stranded. Barriers need the AsyncProgram arena.
#ifndef HARMONIZE_B200_BARRIER_H
#define HARMONIZE_B200_BARRIER_H

#include "async_program.h"

namespace hrm_rt {
__device__ __forceinline__ void fence_sc() { asm volatile("fence.sc.gpu;" ::: "memory"); }
}  // namespace hrm_rt

template <typename OP_SET, typename ADR_TYPE>
struct RemappingBarrier {
    using AdrType = ADR_TYPE;
    using UnionType = PromiseUnion<OP_SET>;
    static const size_t TYPE_COUNT = UnionType::Info::COUNT;

    TaggedSemaphore semaphore;
    unsigned int count;                // promises currently held
    unsigned int heads[TYPE_COUNT];    // per function: held link + 1, or 0

    RemappingBarrier() = default;

    static __host__ __device__ RemappingBarrier<OP_SET, ADR_TYPE> blank(unsigned int sem_val) {
        RemappingBarrier<OP_SET, ADR_TYPE> r;
        r.semaphore = TaggedSemaphore(sem_val, 1);
        r.count = 0u;
        for (size_t i = 0; i < TYPE_COUNT; i++) r.heads[i] = 0u;
        return r;
    }

    // Detaches every held link and hands it to the program's queues (one lane).
    template <typename PROGRAM>
    __device__ void release_sweep(PROGRAM program) {
        for (unsigned int f = 0; f < TYPE_COUNT; f++) {
            unsigned int h = atomicExch(&heads[f], 0u);
            unsigned int guard = 0;
            while (h != 0u && guard++ < (1u << 27)) {
                unsigned int link = h - 1u;
                unsigned int next = hrm_rt::ld_relaxed(program.link_next_ptr(link));
                unsigned int n = program.link_count(link);
                atomicSub(&count, n);
                program.publish_link(f, link, n);
                h = next;
            }
        }
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
        unsigned int link = program.template hold_in_link<OP_TYPE>(promise, group);
        if (r == 0 && link != PROGRAM::NULL_LINK) {
            atomicAdd(&count, (unsigned int)__popc(group));
            unsigned int old = hrm_rt::ld_relaxed(&heads[F]);
            for (unsigned int tries = 0; tries < hrm_rt::SPIN_LIMIT; tries++) {
                *program.link_next_ptr(link) = old;
                __threadfence();
                unsigned int prev = atomicCAS(&heads[F], old, link + 1u);
                if (prev == old) break;
                old = prev;
            }
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

#endif
