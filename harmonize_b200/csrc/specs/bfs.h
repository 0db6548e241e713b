// bfs.h — label-correcting breadth-first search as a two-function async program.
//
// Workload (no counterpart file in Harmonize): levels[v] = hop distance from the root over
// a CSR graph (rowptr[nv+1], col[E], uint32), unreached = 0xFFFFFFFF.
//  * Relax(v, l): atomicMin(levels[v], l); if that lowered the level, expand v's edges at
//    level l+1. A vertex can be relaxed more than once (label correcting); the final
//    levels equal the serial BFS distances whatever the order of evaluation.
//  * Expand(l, begin, end): ranges longer than BFS_CHUNK edges are halved into two Expand
//    calls (so high-degree vertices spread over many lanes); shorter ranges call Relax once
//    per edge whose target currently holds a level above l (one async call per edge
//    relaxation; the read is a filter only, atomicMin decides).
#ifndef HRM_SPECS_BFS_H
#define HRM_SPECS_BFS_H

#include "../../../include/harmonize/spec_support.h"

namespace hrm_specs {

static const unsigned int BFS_UNREACHED = 0xFFFFFFFFu;
static const unsigned int BFS_CHUNK = 16u;

struct BfsState {
    const unsigned int* rowptr;
    const unsigned int* col;
    unsigned int* levels;
    util::iter::AtomicIter<unsigned int>* roots;  // [0, 1): claims the single root launch
    unsigned int root;
    unsigned int nv;
};

struct BfsRelax;
struct BfsExpand;

struct BfsExpand {
    using Type = void (*)(unsigned int, unsigned int, unsigned int);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, unsigned int level, unsigned int begin, unsigned int end) {
        if (end - begin > BFS_CHUNK) {
            unsigned int mid = begin + (end - begin) / 2u;
            prog.template async<BfsExpand>(level, begin, mid);
            prog.template async<BfsExpand>(level, mid, end);
            return;
        }
        for (unsigned int e = begin; e < end; e++) {
            unsigned int u = prog.device.col[e];
            if (hrm::load_relaxed_u32(&prog.device.levels[u]) > level) {
                prog.template async<BfsRelax>(u, level);
            }
        }
    }
};

struct BfsRelax {
    using Type = void (*)(unsigned int, unsigned int);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, unsigned int v, unsigned int level) {
        unsigned int old = hrm::atomic_min_u32(&prog.device.levels[v], level);
        if (level < old) {
            unsigned int b = prog.device.rowptr[v], e = prog.device.rowptr[v + 1u];
            if (e > b) prog.template async<BfsExpand>(level + 1u, b, e);
        }
    }
};

template <size_t RING = 2, size_t TEAMS = 4>
struct BfsSpec {
    typedef OpUnion<BfsRelax, BfsExpand> OpSet;
    typedef BfsState DeviceState;

    static const size_t STASH_SIZE = 16;
    static const size_t FRAME_SIZE = 8191;
    static const size_t POOL_SIZE = 8191;
    static const size_t RING_LINKS = RING;
    static const size_t TEAMS_PER_CTA = TEAMS;
    // Relax calls with smaller levels first: fewer vertices are expanded more than once.
    static const size_t OLDEST_FIRST = 1;

    template <typename PROGRAM>
    HRM_DEV static void initialize(PROGRAM) {}
    template <typename PROGRAM>
    HRM_DEV static void finalize(PROGRAM) {}

    template <typename PROGRAM>
    HRM_DEV static bool make_work(PROGRAM prog) {
        util::iter::Iter<unsigned int> it = prog.device.roots->leap(1u);
        unsigned int i;
        while (it.step(i)) {
            prog.template async<BfsRelax>(prog.device.root, 0u);
        }
        return false;
    }
};

}  // namespace hrm_specs

#endif
