// A spec that passes values back up a call tree through Futures (async/future.h of the
// original): Sum(node) over a complete binary tree of 2^LEVELS leaves. A leaf stores its value
// in its own future and fulfills its parent's; an inner node holds a Combine continuation on
// its own future (semaphore 2), starts both children, and Combine adds the children's values
// once both have fulfilled. AsyncProgram only (held continuations live in its arena).
//
//     futures LEVELS OUT_FILE     writes the 2^(LEVELS+1)-1 node sums (uint32, heap order)
#include "harmonize.h"

#include <cstdio>
#include <cstdlib>
#include <vector>

struct Sum;
struct Combine;
typedef OpUnion<Sum, Combine> TreeOps;
typedef Future<unsigned int, RemappingBarrier<TreeOps>> NodeFuture;

struct TreeState {
    NodeFuture* futures;   // one per node, heap order (children of n: 2n+1, 2n+2)
    unsigned int leaves;   // 2^LEVELS
    util::iter::AtomicIter<unsigned int>* root;
};

__host__ __device__ inline unsigned int leaf_value(unsigned int i) { return (i * 2654435761u) >> 7; }

template <typename PROGRAM>
__device__ void finish(PROGRAM prog, unsigned int node, unsigned int value) {
    NodeFuture* f = prog.device.futures;
    f[node].data = value;
    if (node != 0u) f[(node - 1u) / 2u].fulfill(prog);
}

struct Combine {
    using Type = void (*)(unsigned int);
    template <typename PROGRAM>
    __device__ static void eval(PROGRAM prog, unsigned int node) {
        NodeFuture* f = prog.device.futures;
        finish(prog, node, f[2u * node + 1u].get() + f[2u * node + 2u].get());
    }
};

struct Sum {
    using Type = void (*)(unsigned int);
    template <typename PROGRAM>
    __device__ static void eval(PROGRAM prog, unsigned int node) {
        const unsigned int first_leaf = prog.device.leaves - 1u;
        if (node >= first_leaf) {
            finish(prog, node, leaf_value(node - first_leaf));
            return;
        }
        prog.device.futures[node].await(prog, Promise<Combine>(node));
        prog.template async<Sum>(2u * node + 1u);
        prog.template async<Sum>(2u * node + 2u);
    }
};

struct TreeSpec {
    typedef TreeOps OpSet;
    typedef TreeState DeviceState;

    template <typename PROGRAM>
    __device__ static void initialize(PROGRAM) {}
    template <typename PROGRAM>
    __device__ static void finalize(PROGRAM) {}

    template <typename PROGRAM>
    __device__ static bool make_work(PROGRAM prog) {
        util::iter::Iter<unsigned int> it = prog.device.root->leap(1u);
        unsigned int i;
        while (it.step(i)) prog.template async<Sum>(0u);
        return false;
    }
};

using ProgType = AsyncProgram<TreeSpec>;

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s LEVELS OUT_FILE\n", argv[0]);
        return 2;
    }
    const unsigned int levels = (unsigned int)std::strtoul(argv[1], nullptr, 0);
    const unsigned int leaves = 1u << levels;
    const unsigned int nodes = 2u * leaves - 1u;
    std::vector<NodeFuture> host_f(nodes);
    for (unsigned int n = 0; n < nodes; n++) host_f[n] = NodeFuture(n < leaves - 1u ? 2u : 0u);
    util::host::DevBuf<NodeFuture> futures((size_t)nodes);
    futures << host_f;
    util::host::DevBuf<util::iter::AtomicIter<unsigned int>> root;
    root << util::iter::AtomicIter<unsigned int>(0u, 1u);
    TreeState state{futures.data(), leaves, root.data()};

    ProgType::Instance instance((size_t)1 << 18, state);
    const size_t groups = 4096;
    init<ProgType>(instance, groups);
    unsigned int execs = 0;
    do {
        exec<ProgType>(instance, groups, (size_t)1 << 20);
        util::host::check_error();
        execs++;
    } while (!instance.complete() && execs < 10000u);
    if (!instance.complete()) {
        std::fprintf(stderr, "no completion after %u execs\n", execs);
        return 1;
    }
    futures >> host_f;
    std::vector<unsigned int> sums(nodes), expect(nodes);
    for (unsigned int n = 0; n < nodes; n++) sums[n] = host_f[n].data;
    for (unsigned int n = nodes; n-- > 0;) {
        expect[n] = n >= leaves - 1u ? leaf_value(n - (leaves - 1u)) : expect[2 * n + 1] + expect[2 * n + 2];
    }
    unsigned int bad = 0;
    for (unsigned int n = 0; n < nodes; n++) {
        if (sums[n] != expect[n] && bad++ < 5) std::fprintf(stderr, "node %u: %u, expected %u\n", n, sums[n], expect[n]);
    }
    FILE* f = std::fopen(argv[2], "wb");
    if (f == nullptr || std::fwrite(sums.data(), sizeof(unsigned int), nodes, f) != nodes) return 1;
    std::fclose(f);
    std::printf("execs %u mismatches %u\n", execs, bad);
    return bad == 0 ? 0 : 3;
}
