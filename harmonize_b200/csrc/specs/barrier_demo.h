// barrier_demo.h — a remapping-barrier workload with checkable results.
//
// The behaviour of harmonize examples/cpp/barrier_demo/demo.cpp:20-86: ids
// [0, dep + ndep) each run one Step (make_work, through prog.sync); a dependent step
// (id < dep) holds a follow-up Step on barrier id % bar (RemappingBarrier::await) and then
// decrements that barrier's semaphore by one; barrier b starts at the number of dependent
// ids mapped to it (demo.cpp:163-170), so it releases when its last dependent step has run,
// and its held follow-ups run after that. Every Step counts itself (counter[0]); the
// original expects 2*dep + ndep Steps (demo.cpp:216).
//
// Added so that a run checks itself: a follow-up carries FOLLOW + b, counts itself in
// released[b] and counts a violation if barrier b's semaphore is not zero when it runs;
// barriers with odd b are awaited through union_await (runtime discriminant); and a
// UnitBarrier armed with ndep releases one FINAL Step after every non-dependent step has
// decremented it, which counts itself in counter[2] and checks counter[1] == ndep.
#ifndef HRM_SPECS_BARRIER_DEMO_H
#define HRM_SPECS_BARRIER_DEMO_H

#include "../../../include/harmonize.h"

namespace hrm_specs {

struct BarrierStep;
typedef OpUnion<BarrierStep> BarrierOps;

// counter[0]: Steps run; counter[1]: non-dependent Steps; counter[2]: FINAL Steps;
// counter[3]: violations (a follow-up ran before its barrier released, or FINAL ran early).
struct BarrierDemoState {
    unsigned int dep_count;
    unsigned int non_dep_count;
    unsigned int barrier_count;
    unsigned int pad;
    util::iter::AtomicIter<unsigned int>* source;
    unsigned int* counter;
    unsigned int* released;                       // per barrier: follow-ups run
    RemappingBarrier<BarrierOps>* barriers;       // barrier_count barriers
    UnitBarrier<BarrierOps>* unit;                // armed with non_dep_count
};

static const unsigned int BARRIER_FOLLOW = 0x80000000u;  // follow-up of barrier b: FOLLOW + b
static const unsigned int BARRIER_FINAL = 0x7FFFFFFFu;

struct BarrierStep {
    using Type = void (*)(unsigned int);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, unsigned int arg) {
        const BarrierDemoState& st = prog.device;
        atomicAdd(&st.counter[0], 1u);
        if (arg >= BARRIER_FOLLOW) {
            const unsigned int b = arg - BARRIER_FOLLOW;
            atomicAdd(&st.released[b], 1u);
            if (hrm_rt::ld_relaxed(&st.barriers[b].semaphore.sem) != 0u) atomicAdd(&st.counter[3], 1u);
        } else if (arg == BARRIER_FINAL) {
            atomicAdd(&st.counter[2], 1u);
            if (atomicAdd(&st.counter[1], 0u) != st.non_dep_count) atomicAdd(&st.counter[3], 1u);
        } else if (arg < st.dep_count) {
            const unsigned int b = arg % st.barrier_count;
            RemappingBarrier<BarrierOps>& bar = st.barriers[b];
            if (b & 1u) {
                typename PROGRAM::PromiseUnionType u(Promise<BarrierStep>(BARRIER_FOLLOW + b));
                bar.union_await(prog, (OpDisc)0, u);
            } else {
                bar.await(prog, Promise<BarrierStep>(BARRIER_FOLLOW + b));
            }
            bar.add_semaphore(prog, (unsigned int)-1);
        } else {
            atomicAdd(&st.counter[1], 1u);
            __threadfence();  // the count above is visible before the unit barrier can release
            st.unit->sub_semaphore(prog, 1u);
        }
    }
};

template <size_t RING = 2, size_t TEAMS = 4>
struct BarrierDemoSpec {
    typedef BarrierOps OpSet;
    typedef BarrierDemoState DeviceState;
    static const size_t STASH_SIZE = 8;
    static const size_t FRAME_SIZE = 8191;
    static const size_t POOL_SIZE = 8191;
    static const size_t RING_LINKS = RING;
    static const size_t TEAMS_PER_CTA = TEAMS;

    template <typename PROGRAM>
    HRM_DEV static void initialize(PROGRAM) {}
    template <typename PROGRAM>
    HRM_DEV static void finalize(PROGRAM) {}

    // demo.cpp:66-84: one id per lane per call, run in place.
    template <typename PROGRAM>
    HRM_DEV static bool make_work(PROGRAM prog) {
        util::iter::Iter<unsigned int> it = prog.device.source->leap(1);
        unsigned int id;
        while (it.step(id)) prog.template sync<BarrierStep>(id);
        return !prog.device.source->done();
    }
};

}  // namespace hrm_specs

#endif
