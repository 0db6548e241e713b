// collatz.h — Collatz stopping times as a two-function async program.
//
// The same program as harmonize examples/cpp/collaz/collaz_hrm.cpp:9-61 (Even/Odd async
// functions re-enqueueing themselves until the value reaches 1, the step count written
// to output[original]) and :127-144 (make_work claims start values from a shared
// AtomicIter), written so that one source compiles against this runtime, against the
// original Harmonize headers and against the host executors in oracle/:
//  * evals are HRM_DEV (device-only under nvcc, plain functions under g++);
//  * start values are uint64 and the iterator runs over [start, limit) as uint32.
//
// Requires, before inclusion: OpUnion and util::iter::{Iter, AtomicIter} from one of
// the three environments.
#ifndef HRM_SPECS_COLLATZ_H
#define HRM_SPECS_COLLATZ_H

#include "../../../include/harmonize/spec_support.h"

namespace hrm_specs {

struct CollatzState {
    unsigned int start;
    unsigned int limit;
    unsigned int* output;                               // output[n - start] = steps of n
    util::iter::AtomicIter<unsigned int>* iterator;     // over [start, limit)
    unsigned int leap;                                  // start values per lane per make_work
};

struct CollatzEven;
struct CollatzOdd;

template <typename PROGRAM>
HRM_DEV HRM_FI void collatz_next(PROGRAM prog, unsigned long long val, unsigned int step, unsigned int original) {
    if ((val % 2ull) == 0ull) {
        prog.template async<CollatzEven>(val, step, original);
    } else {
        prog.template async<CollatzOdd>(val, step, original);
    }
}

struct CollatzEven {
    using Type = void (*)(unsigned long long, unsigned int, unsigned int);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, unsigned long long val, unsigned int step, unsigned int original) {
        if (val <= 1ull) {
            prog.device.output[original - prog.device.start] = step;
            return;
        }
        collatz_next(prog, val / 2ull, step + 1u, original);
    }
};

struct CollatzOdd {
    using Type = void (*)(unsigned long long, unsigned int, unsigned int);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, unsigned long long val, unsigned int step, unsigned int original) {
        if (val <= 1ull) {
            prog.device.output[original - prog.device.start] = step;
            return;
        }
        collatz_next(prog, val * 3ull + 1ull, step + 1u, original);
    }
};

template <size_t RING = 2, size_t TEAMS = 4>
struct CollatzSpec {
    typedef OpUnion<CollatzEven, CollatzOdd> OpSet;
    typedef CollatzState DeviceState;

    static const size_t STASH_SIZE = 16;
    static const size_t FRAME_SIZE = 8191;
    static const size_t POOL_SIZE = 8191;
    static const size_t RING_LINKS = RING;
    static const size_t TEAMS_PER_CTA = TEAMS;

    template <typename PROGRAM>
    HRM_DEV static void initialize(PROGRAM) {}
    template <typename PROGRAM>
    HRM_DEV static void finalize(PROGRAM) {}

    template <typename PROGRAM>
    HRM_DEV static bool make_work(PROGRAM prog) {
        util::iter::Iter<unsigned int> it = prog.device.iterator->leap(prog.device.leap);
        unsigned int index;
        while (it.step(index)) {
            collatz_next(prog, (unsigned long long)index, 0u, index);
        }
        return !prog.device.iterator->done();
    }
};

}  // namespace hrm_specs

#endif
