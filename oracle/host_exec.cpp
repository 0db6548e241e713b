// host_exec.cpp — serial and OpenMP host executors of the built-in spec sources
// (TEST INFRASTRUCTURE ONLY; also the CPU baseline that bench.py reports).
//
// Harmonize has no CPU executor. These run the very same spec headers as the GPU runtime
// (harmonize_b200/csrc/specs/*.h) with a host program object: prog.async<F>(args) appends
// to a per-function queue, the executor evaluates promises until every queue is empty and
// make_work returns false (the completion rule of harmonize/cpp/program/async.h:2323-2393).
// With T threads each thread owns its queues and claims work through the spec's shared
// AtomicIter; because the specs' outputs are schedule-independent, any T gives the same
// outputs and the same per-function call counts.
#include "host_api.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include <omp.h>

#include "../harmonize_b200/csrc/specs/collatz.h"
#include "../harmonize_b200/csrc/specs/photon.h"
#include "../harmonize_b200/csrc/specs/bfs.h"

namespace {

template <typename T>
struct FnArgs;
template <typename R, typename... A>
struct FnArgs<R (*)(A...)> {
    using tuple = std::tuple<A...>;
};
template <typename F>
using ArgsOf = typename FnArgs<typename F::Type>::tuple;

template <typename F, typename U>
struct IndexOf;
template <typename F, typename... R>
struct IndexOf<F, OpUnion<F, R...>> {
    static const size_t value = 0;
};
template <typename F, typename H, typename... R>
struct IndexOf<F, OpUnion<H, R...>> {
    static const size_t value = 1 + IndexOf<F, OpUnion<R...>>::value;
};

template <typename U>
struct QueueTuple;
template <typename... Fs>
struct QueueTuple<OpUnion<Fs...>> {
    using type = std::tuple<std::deque<ArgsOf<Fs>>...>;
    static const size_t count = sizeof...(Fs);
};

template <typename Spec>
struct Exec;

// The program object handed to evals: a cheap handle, like the GPU program types.
template <typename Spec>
struct HostProg {
    using DeviceState = typename Spec::DeviceState;
    Exec<Spec>* ex;
    DeviceState& device;
    template <typename F, typename... A>
    void async(A... a) const {
        ex->template push<F>(a...);
    }
    template <typename F, typename... A>
    void sync(A... a) const {
        ex->template call<F>(ArgsOf<F>(a...));
    }
    template <typename F>
    float load_fraction() const {
        return NAN;
    }
    void halt_early() const {}
};

template <typename Spec>
struct Exec {
    using OpSet = typename Spec::OpSet;
    using DeviceState = typename Spec::DeviceState;
    static const size_t FN = QueueTuple<OpSet>::count;
    typename QueueTuple<OpSet>::type queues;
    unsigned long long calls[FN] = {};
    DeviceState& device;

    explicit Exec(DeviceState& d) : device(d) {}

    HostProg<Spec> prog() { return HostProg<Spec>{this, device}; }

    template <typename F, typename... A>
    void push(A... a) {
        std::get<IndexOf<F, OpSet>::value>(queues).emplace_back(ArgsOf<F>(a...));
    }

    template <typename F>
    void call(const ArgsOf<F>& args) {
        HostProg<Spec> p = prog();
        std::apply([&](auto... x) { F::template eval<HostProg<Spec>>(p, x...); }, args);
    }

    // Evaluates the oldest pending promise of the lowest-numbered non-empty function
    // (first-in first-out per function). Returns false when every queue is empty.
    template <size_t I, typename F, typename... R>
    bool step_impl(OpUnion<F, R...>*) {
        auto& q = std::get<I>(queues);
        if (!q.empty()) {
            ArgsOf<F> args = q.front();
            q.pop_front();
            calls[I]++;
            call<F>(args);
            return true;
        }
        return step_impl<I + 1>((OpUnion<R...>*)nullptr);
    }
    template <size_t I>
    bool step_impl(OpUnion<>*) {
        return false;
    }

    void run() {
        HostProg<Spec> p = prog();
        bool can_make_work = true;
        while (true) {
            if (step_impl<0>((OpSet*)nullptr)) continue;
            if (!can_make_work) break;
            can_make_work = Spec::template make_work<HostProg<Spec>>(p);
        }
    }
};

template <typename Spec>
void run_parallel(typename Spec::DeviceState& st, int threads, unsigned long long* calls_out) {
    const size_t FN = Exec<Spec>::FN;
    std::vector<unsigned long long> total(FN, 0);
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
    {
        Exec<Spec> ex(st);
        ex.run();
#pragma omp critical
        for (size_t i = 0; i < FN; i++) total[i] += ex.calls[i];
    }
    if (calls_out) {
        for (size_t i = 0; i < FN; i++) calls_out[i] = total[i];
    }
}

}  // namespace

extern "C" {

int oracle_max_threads(void) { return omp_get_max_threads(); }

// Collatz (collatz.h) over [start, start+count): out[i] = steps of start+i; calls_out[2].
void oracle_exec_collatz(unsigned int start, unsigned int count, unsigned int* out, int threads,
                         unsigned long long* calls_out) {
    util::iter::AtomicIter<unsigned int> it(start, start + count);
    hrm_specs::CollatzState st;
    st.start = start;
    st.limit = start + count;
    st.output = out;
    st.iterator = &it;
    st.leap = 64;
    run_parallel<hrm_specs::CollatzSpec<>>(st, threads, calls_out);
}

// Photon walk (photon.h) of photons [first, first+count); tally has n^3 + 3*1024 slots
// (zeroed by the caller); calls_out[3] = move, collide, tally calls.
void oracle_exec_photon(const float* mu_s, const float* absorb, const unsigned char* split, unsigned int n,
                        unsigned int seed_lo, unsigned int seed_hi, unsigned int first, unsigned int count,
                        unsigned long long* tally, int threads, unsigned long long* calls_out) {
    util::iter::AtomicIter<unsigned int> it(first, first + count);
    hrm_specs::PhotonState st;
    st.mu_s = mu_s;
    st.absorb = absorb;
    st.split = split;
    st.tally = tally;
    st.source = &it;
    st.n = n;
    st.seed_lo = seed_lo;
    st.seed_hi = seed_hi;
    st.leap = 16;
    st.load_limit = 2.0f;
    run_parallel<hrm_specs::PhotonSpec<>>(st, threads, calls_out);
}

// Label-correcting BFS (bfs.h) from `root`; levels[nv] must be pre-filled with 0xFFFFFFFF;
// calls_out[2] = relax, expand calls.
void oracle_exec_bfs(const unsigned int* rowptr, const unsigned int* col, unsigned int nv, unsigned int root,
                     unsigned int* levels, int threads, unsigned long long* calls_out) {
    util::iter::AtomicIter<unsigned int> it(0, 1);
    hrm_specs::BfsState st;
    st.rowptr = rowptr;
    st.col = col;
    st.levels = levels;
    st.roots = &it;
    st.root = root;
    st.nv = nv;
    run_parallel<hrm_specs::BfsSpec<>>(st, threads, calls_out);
}

}  // extern "C"
