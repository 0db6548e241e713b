// bfs.h — label-correcting breadth-first search as a two-function async program.
//
// Workload (no counterpart file in Harmonize): levels[v] = hop distance from the root over
// a CSR graph (rowptr[nv+1], col[E], uint32), unreached = 0xFFFFFFFF.
//  * Relax(v, l): atomicMin(levels[v], l); if that lowered the level, expand v's edges at
//    level l+1. A vertex can be relaxed more than once (label correcting); the final
//    levels equal the serial BFS distances whatever the order of evaluation.
//  * Expand(l, begin, end, v): the edges [begin, end) of vertex v at level l. If v's level
//    has dropped below l - 1 since (a smaller level reached it and a newer Expand covers the
//    same edges with a smaller level), the call is stale and does nothing. Otherwise ranges
//    longer than BFS_CHUNK edges are halved into two Expand calls (so high-degree vertices
//    spread over many lanes); shorter ranges call Relax once per edge whose target currently
//    holds a level above l (one async call per edge relaxation; the read is a filter only,
//    atomicMin decides).
//    On the GPU the lanes of a batch that evaluate Expand together walk their short ranges
//    as one flattened edge list: lane L takes edge L, L+k, ... of the concatenation (k =
//    lanes in the batch), so the col reads of a warp are consecutive addresses and the
//    level reads of 32 edges are in flight at once, instead of each lane walking its own
//    range with one dependent load after another. The calls made are the same as lane by
//    lane (one Relax per edge whose target level is above l when read).
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
    using Type = void (*)(unsigned int, unsigned int, unsigned int, unsigned int);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, unsigned int level, unsigned int begin, unsigned int end, unsigned int v) {
        // Stale: v holds a level below level - 1, so its newer Expand relaxes these edges with
        // a smaller level (this one would only make corrections that the newer one undoes).
        if (hrm::load_relaxed_u32(&prog.device.levels[v]) + 1u < level) end = begin;
#if defined(__CUDA_ARCH__)
        // The runtimes evaluate a batch as `if (lane < k) eval(...)`: the active lanes are
        // 0 .. k-1, which the flattened walk below relies on. The lanes must also share one
        // search (a batch of the job-multiplexing runtime can hold Expand calls of several
        // jobs, each with its own graph, levels and queues): any other batch walks lane by lane.
        const unsigned int mask = __activemask();
        const bool split = end - begin > BFS_CHUNK;
        if (split) {
            unsigned int mid = begin + (end - begin) / 2u;
            prog.template async<BfsExpand>(level, begin, mid, v);
            prog.template async<BfsExpand>(level, mid, end, v);
        }
        __syncwarp(mask);
        // (One search = one graph and one levels array: every job writes its own levels.)
        int same_col = 0, same_levels = 0;
        __match_all_sync(mask, (unsigned long long)(uintptr_t)prog.device.col, &same_col);
        __match_all_sync(mask, (unsigned long long)(uintptr_t)prog.device.levels, &same_levels);
        if ((mask & (mask + 1u)) == 0u && same_col && same_levels) {
            expand_flat(prog, mask, level, begin, split ? 0u : end - begin);
            return;
        }
        if (split) return;
#else
        if (end - begin > BFS_CHUNK) {
            unsigned int mid = begin + (end - begin) / 2u;
            prog.template async<BfsExpand>(level, begin, mid, v);
            prog.template async<BfsExpand>(level, mid, end, v);
            return;
        }
#endif
        for (unsigned int e = begin; e < end; e++) {
            unsigned int u = prog.device.col[e];
            if (hrm::load_relaxed_u32(&prog.device.levels[u]) > level) {
                prog.template async<BfsRelax>(u, level);
            }
        }
    }

#if defined(__CUDA_ARCH__)
    // Lanes 0 .. k-1 (mask = 2^k - 1) each hold a range of `len` edges from `begin` at
    // `level`; together they relax the concatenation of the ranges, k edges per round.
    template <typename PROGRAM>
    HRM_DEV static void expand_flat(PROGRAM prog, unsigned int mask, unsigned int level, unsigned int begin,
                                    unsigned int len) {
        const unsigned int lane = threadIdx.x & 31u;
        const unsigned int k = 32u - __clz(mask);
        // Inclusive prefix sum of the range lengths over lanes 0 .. k-1.
        unsigned int incl = len;
#pragma unroll
        for (unsigned int d = 1; d < 32u; d <<= 1) {
            unsigned int up = __shfl_up_sync(mask, incl, d);
            if (lane >= d) incl += up;
        }
        const unsigned int total = __shfl_sync(mask, incl, k - 1u);
        for (unsigned int base = 0; base < total; base += k) {
            const unsigned int p = base + lane;
            // Owner of edge p: the first lane whose inclusive sum exceeds p (binary search
            // over lanes 0 .. k-1; every probe reads a lane of the batch).
            unsigned int lo = 0, hi = k - 1u;
#pragma unroll
            for (unsigned int step = 0; step < 5u; step++) {
                unsigned int mid = (lo + hi) >> 1;
                unsigned int v = __shfl_sync(mask, incl, mid);
                if (v > p) hi = mid;
                else lo = (mid + 1u < hi) ? mid + 1u : hi;
            }
            const unsigned int o_incl = __shfl_sync(mask, incl, lo);
            const unsigned int o_len = __shfl_sync(mask, len, lo);
            const unsigned int o_begin = __shfl_sync(mask, begin, lo);
            const unsigned int o_level = __shfl_sync(mask, level, lo);
            if (p < total) {
                const unsigned int e = o_begin + (p - (o_incl - o_len));
                const unsigned int u = prog.device.col[e];
                if (hrm::load_relaxed_u32(&prog.device.levels[u]) > o_level) {
                    prog.template async<BfsRelax>(u, o_level);
                }
            }
        }
    }
#endif
};

struct BfsRelax {
    using Type = void (*)(unsigned int, unsigned int);
    template <typename PROGRAM>
    HRM_DEV static void eval(PROGRAM prog, unsigned int v, unsigned int level) {
        unsigned int old = hrm::atomic_min_u32(&prog.device.levels[v], level);
        if (level < old) {
            unsigned int b = prog.device.rowptr[v], e = prog.device.rowptr[v + 1u];
            if (e > b) prog.template async<BfsExpand>(level + 1u, b, e, v);
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
