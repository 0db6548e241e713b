// A spec whose async calls take LazyLoad arguments (promise.h:208-240 of the original): each
// call of Walk names the table entries of its next step by reference, and the runtime fills
// them in (AsyncProgram: an asynchronous copy into the promise's shared-memory slot, or a read
// at the call for a promise that overflows to the arena; EventProgram: a read at the call).
// The program type is one line (PROGRAM_TYPE); LEAP start values per lane per make_work call
// (4 overflows the two-link rings of this spec, so both AsyncProgram paths run).
//
//     lazy_load COUNT STEPS OUT_FILE     writes COUNT uint32 results
#include "harmonize.h"

#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <vector>

#ifndef LEAP
#define LEAP 1
#endif

struct Pair {
    unsigned int a, b;
};

struct LazyState {
    const unsigned int* table;    // TABLE_N words
    const Pair* pairs;            // PAIRS_N pairs
    unsigned int* out;            // out[i] = result of walk i
    unsigned int steps;           // Walk steps per start value
    util::iter::AtomicIter<unsigned int>* starts;
};

static const unsigned int TABLE_N = 1u << 20;
static const unsigned int PAIRS_N = 1u << 16;

__host__ __device__ inline unsigned int table_index(unsigned int i, unsigned int k) {
    return (i * 2654435761u + k * 40503u) & (TABLE_N - 1u);
}
__host__ __device__ inline unsigned int pair_index(unsigned int i, unsigned int k) {
    return (i ^ (k * 2246822519u)) & (PAIRS_N - 1u);
}
__host__ __device__ inline unsigned int mix(unsigned int acc, unsigned int k, unsigned int v, Pair q) {
    return acc * 31u + v + q.a * 7u + (q.b ^ k);
}

struct Walk {
    using Type = void (*)(unsigned int, unsigned int, unsigned int, unsigned int, Pair);
    template <typename PROGRAM>
    __device__ static void eval(PROGRAM prog, unsigned int i, unsigned int k, unsigned int acc, unsigned int v,
                                Pair q) {
        const LazyState& s = prog.device;
        unsigned int next = mix(acc, k, v, q);
        if (k + 1u < s.steps) {
            prog.template async<Walk>(i, k + 1u, next, LazyLoad<unsigned int>(*(unsigned int*)&s.table[table_index(i, k + 1u)]),
                                      LazyLoad<Pair>(*(Pair*)&s.pairs[pair_index(i, k + 1u)]));
        } else {
            s.out[i] = next;
        }
    }
};

struct LazySpec {
    typedef OpUnion<Walk> OpSet;
    typedef LazyState DeviceState;
    static const size_t RING_LINKS = 2;
    static const size_t TEAMS_PER_CTA = 4;

    template <typename PROGRAM>
    __device__ static void initialize(PROGRAM) {}
    template <typename PROGRAM>
    __device__ static void finalize(PROGRAM) {}

    template <typename PROGRAM>
    __device__ static bool make_work(PROGRAM prog) {
        const LazyState& s = prog.device;
        util::iter::Iter<unsigned int> it = s.starts->leap(LEAP);
        unsigned int i;
        while (it.step(i)) {
            prog.template async<Walk>(i, 0u, 0u, LazyLoad<unsigned int>(*(unsigned int*)&s.table[table_index(i, 0u)]),
                                      LazyLoad<Pair>(*(Pair*)&s.pairs[pair_index(i, 0u)]));
        }
        return !s.starts->done();
    }
};

using ProgType = PROGRAM_TYPE<LazySpec>;

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s COUNT STEPS OUT_FILE\n", argv[0]);
        return 2;
    }
    const unsigned int count = (unsigned int)std::strtoul(argv[1], nullptr, 0);
    const unsigned int steps = (unsigned int)std::strtoul(argv[2], nullptr, 0);
    const bool is_async = std::is_same<ProgType, AsyncProgram<LazySpec>>::value;

    std::vector<unsigned int> table(TABLE_N);
    std::vector<Pair> pairs(PAIRS_N);
    unsigned int x = 12345u;
    for (auto& t : table) t = (x = x * 1664525u + 1013904223u);
    for (auto& p : pairs) {
        p.a = (x = x * 1664525u + 1013904223u);
        p.b = (x = x * 1664525u + 1013904223u);
    }
    util::host::DevBuf<unsigned int> d_table(TABLE_N);
    util::host::DevBuf<Pair> d_pairs(PAIRS_N);
    util::host::DevBuf<unsigned int> d_out((size_t)count);
    d_table << table;
    d_pairs << pairs;
    util::host::DevBuf<util::iter::AtomicIter<unsigned int>> starts;
    starts << util::iter::AtomicIter<unsigned int>(0u, count);
    LazyState state{d_table.data(), d_pairs.data(), d_out.data(), steps, starts.data()};

    ProgType::Instance instance(is_async ? (size_t)1 << 16 : (size_t)1 << 20, state);
    const size_t groups = 4096;
    init<ProgType>(instance, groups);
    unsigned int execs = 0;
    do {
        exec<ProgType>(instance, groups, is_async ? (size_t)1 << 20 : (size_t)1);
        util::host::check_error();
        execs++;
    } while (!instance.complete() && execs < 100000u);
    if (!instance.complete()) {
        std::fprintf(stderr, "no completion after %u execs\n", execs);
        return 1;
    }
    std::vector<unsigned int> host;
    d_out >> host;
    // The same walks on the host.
    unsigned int bad = 0;
    for (unsigned int i = 0; i < count; i++) {
        unsigned int acc = 0;
        for (unsigned int k = 0; k < steps; k++) acc = mix(acc, k, table[table_index(i, k)], pairs[pair_index(i, k)]);
        if (host[i] != acc && bad++ < 5) std::fprintf(stderr, "walk %u: %u, expected %u\n", i, host[i], acc);
    }
    FILE* f = std::fopen(argv[3], "wb");
    if (f == nullptr || std::fwrite(host.data(), sizeof(unsigned int), host.size(), f) != host.size()) return 1;
    std::fclose(f);
    std::printf("execs %u mismatches %u\n", execs, bad);
    return bad == 0 ? 0 : 3;
}
