// A user's spec written against the Harmonize spec API and run through its C++ host API
// (Instance, init<P>, exec<P>, complete) with no other code of this library: Collatz
// stopping times with one async function per parity. The program type is one line
// (PROGRAM_TYPE, AsyncProgram or EventProgram, given on the compiler's command line).
//
//     collatz_two_fn START COUNT OUT_FILE     writes COUNT uint32 stopping times
#include "harmonize.h"

#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <vector>

struct Even;
struct Odd;

struct ChainState {
    unsigned int start;
    unsigned int* steps;                            // steps[n - start] = stopping time of n
    util::iter::AtomicIter<unsigned int>* starts;  // start values not yet launched
};

// Sends value v (reached after `steps` steps from n) to the function for its parity, or
// records the stopping time once v is 1.
template <typename PROGRAM>
__device__ void advance(PROGRAM prog, unsigned long long v, unsigned int steps, unsigned int n) {
    if (v == 1ull) {
        prog.device.steps[n - prog.device.start] = steps;
    } else if (v & 1ull) {
        prog.template async<Odd>(v, steps, n);
    } else {
        prog.template async<Even>(v, steps, n);
    }
}

struct Even {
    using Type = void (*)(unsigned long long, unsigned int, unsigned int);
    template <typename PROGRAM>
    __device__ static void eval(PROGRAM prog, unsigned long long v, unsigned int steps, unsigned int n) {
        advance(prog, v >> 1, steps + 1u, n);
    }
};

struct Odd {
    using Type = void (*)(unsigned long long, unsigned int, unsigned int);
    template <typename PROGRAM>
    __device__ static void eval(PROGRAM prog, unsigned long long v, unsigned int steps, unsigned int n) {
        advance(prog, 3ull * v + 1ull, steps + 1u, n);
    }
};

struct ChainSpec {
    typedef OpUnion<Even, Odd> OpSet;
    typedef ChainState DeviceState;

    static const size_t STASH_SIZE = 8;
    static const size_t FRAME_SIZE = 8191;
    static const size_t POOL_SIZE = 8191;

    template <typename PROGRAM>
    __device__ static void initialize(PROGRAM) {}
    template <typename PROGRAM>
    __device__ static void finalize(PROGRAM) {}

    template <typename PROGRAM>
    __device__ static bool make_work(PROGRAM prog) {
        util::iter::Iter<unsigned int> it = prog.device.starts->leap(1u);
        unsigned int n;
        while (it.step(n)) advance(prog, (unsigned long long)n, 0u, n);
        return !prog.device.starts->done();
    }
};

using ProgType = PROGRAM_TYPE<ChainSpec>;

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s START COUNT OUT_FILE\n", argv[0]);
        return 2;
    }
    const unsigned int start = (unsigned int)std::strtoul(argv[1], nullptr, 0);
    const unsigned int count = (unsigned int)std::strtoul(argv[2], nullptr, 0);
    const bool is_async = std::is_same<ProgType, AsyncProgram<ChainSpec>>::value;

    util::host::DevBuf<unsigned int> steps((size_t)count);
    util::host::DevBuf<util::iter::AtomicIter<unsigned int>> starts;
    starts << util::iter::AtomicIter<unsigned int>(start, start + count);
    ChainState state{start, steps.data(), starts.data()};

    // AsyncProgram: arena links and a cycle budget per exec; EventProgram: promises per
    // function buffer and a chunk size per exec.
    ProgType::Instance instance(is_async ? (size_t)1 << 16 : (size_t)1 << 20, state);
    const size_t groups = 4096;
    init<ProgType>(instance, groups);
    unsigned int execs = 0;
    do {
        exec<ProgType>(instance, groups, is_async ? (size_t)1 << 12 : (size_t)1);
        util::host::check_error();
        execs++;
    } while (!instance.complete() && execs < 100000u);
    if (!instance.complete()) {
        std::fprintf(stderr, "no completion after %u execs\n", execs);
        return 1;
    }

    std::vector<unsigned int> host;
    steps >> host;
    FILE* f = std::fopen(argv[3], "wb");
    if (f == nullptr || std::fwrite(host.data(), sizeof(unsigned int), host.size(), f) != host.size()) {
        std::fprintf(stderr, "cannot write %s\n", argv[3]);
        return 1;
    }
    std::fclose(f);
    std::printf("execs %u\n", execs);
    return 0;
}
