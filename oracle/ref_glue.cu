// ref_glue.cu — runs the built-in spec sources on the ORIGINAL Harmonize runtime
// (TEST / BENCH INFRASTRUCTURE ONLY).
//
// Built by oracle/ref_build.py with the reference's own recipe:
//     nvcc -std=c++17 --restrict -x cu -arch=sm_100a -include <reference>/harmonize/cpp/harmonize.h
// (examples/cpp/collaz/Makefile:28), into oracle/_ref/libhrm_ref.so. The host drive loop is
// the one of the reference examples: Instance(arena_or_io, state); init<P>; do { exec<P>;
// sync } while (!complete()) (examples/cpp/collaz/collaz_hrm.cpp:212-225,
// examples/cpp/example_neutron/program.cpp:274-312), bounded here by max_execs so that a
// run that never completes returns an error instead of looping forever. Timing uses CUDA
// events around init + the exec loop, like util::Stopwatch (util/mod.h:88-134).
#include <chrono>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../harmonize_b200/csrc/specs/bfs.h"
#include "../harmonize_b200/csrc/specs/collatz.h"
#include "../harmonize_b200/csrc/specs/photon.h"

namespace {

thread_local std::string g_ref_error;

template <typename T>
struct DevArr {
    T* p = nullptr;
    explicit DevArr(size_t n) {
        if (n && cudaMalloc((void**)&p, n * sizeof(T)) != cudaSuccess) throw std::runtime_error("cudaMalloc");
    }
    ~DevArr() {
        if (p) cudaFree(p);
    }
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Drives one instance to completion; returns 0, 4 (incomplete within max_execs) or throws.
template <typename P>
int drive(typename P::Instance& inst, uint32_t wg_count, uint32_t n, uint32_t max_execs, float* ms, uint32_t* execs) {
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    ck(cudaDeviceSynchronize(), "sync");
    ck(cudaEventRecord(e0, 0), "event");
    init<P>(inst, wg_count);
    ck(cudaDeviceSynchronize(), "init");
    uint32_t k = 0;
    bool done = false;
    while (k < max_execs) {
        exec<P>(inst, wg_count, n);
        ck(cudaDeviceSynchronize(), "exec");
        k++;
        if (inst.complete()) {
            done = true;
            break;
        }
    }
    ck(cudaEventRecord(e1, 0), "event");
    ck(cudaEventSynchronize(e1), "event");
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = t;
    if (execs) *execs = k;
    return done ? 0 : 4;
}

template <template <size_t, size_t> class SPEC, typename STATE>
int drive_spec(int program_type, size_t arena, const STATE& st, uint32_t wg, uint32_t n, uint32_t max_execs,
               float* ms, uint32_t* execs) {
    if (program_type == 0) {
        using P = AsyncProgram<SPEC<2, 4>>;
        typename P::Instance inst((typename P::AdrType)arena, st);
        return drive<P>(inst, wg, n, max_execs, ms, execs);
    } else {
        using P = EventProgram<SPEC<2, 4>>;
        typename P::Instance inst(arena, st);
        return drive<P>(inst, wg, n, max_execs, ms, execs);
    }
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_ref_error.c_str(); }

// Collatz stopping times of [start, start+count) into out (host).
int ref_collatz_run(int program_type, uint32_t start, uint32_t count, uint32_t* out, uint32_t wg_count, uint32_t n,
                    uint32_t arena, uint32_t max_execs, float* ms, uint32_t* execs) {
    try {
        DevArr<uint32_t> d_out(count ? count : 1);
        DevArr<util::iter::AtomicIter<unsigned int>> it(1);
        util::iter::AtomicIter<unsigned int> h_it(start, start + count);
        ck(cudaMemcpy(it.p, &h_it, sizeof(h_it), cudaMemcpyHostToDevice), "iter");
        hrm_specs::CollatzState st;
        st.start = start;
        st.limit = start + count;
        st.output = d_out.p;
        st.iterator = it.p;
        st.leap = 1;
        int rc = drive_spec<hrm_specs::CollatzSpec>(program_type, arena, st, wg_count, n, max_execs, ms, execs);
        ck(cudaMemcpy(out, d_out.p, (size_t)count * 4u, cudaMemcpyDeviceToHost), "out");
        return rc;
    } catch (std::exception& e) {
        g_ref_error = e.what();
        return 2;
    }
}

// Photon walk: medium already on the device (device-resident timing); tally left in d_tally.
int ref_photon_run_device(int program_type, const float* d_mu, const float* d_ab, const uint8_t* d_sp, uint32_t n,
                          uint64_t seed, uint32_t first, uint32_t count, uint64_t* d_tally, uint32_t wg_count,
                          uint32_t nn, uint32_t arena, uint32_t max_execs, float load_limit, float* ms,
                          uint32_t* execs) {
    try {
        const size_t slots = (size_t)n * n * n + 3u * hrm_specs::PHOTON_SPREAD;
        ck(cudaMemset(d_tally, 0, slots * 8u), "tally");
        DevArr<util::iter::AtomicIter<unsigned int>> it(1);
        util::iter::AtomicIter<unsigned int> h_it(first, first + count);
        ck(cudaMemcpy(it.p, &h_it, sizeof(h_it), cudaMemcpyHostToDevice), "iter");
        hrm_specs::PhotonState st;
        st.mu_s = d_mu;
        st.absorb = d_ab;
        st.split = d_sp;
        st.tally = (unsigned long long*)d_tally;
        st.source = it.p;
        st.n = n;
        st.seed_lo = (uint32_t)seed;
        st.seed_hi = (uint32_t)(seed >> 32);
        st.leap = 1;
        // EventProgram: make_work stops launching photons while the move buffer is fuller than
        // this fraction (0 selects 1/64).
        st.load_limit = load_limit > 0.0f ? load_limit : 0.015625f;
        return drive_spec<hrm_specs::PhotonSpec>(program_type, arena, st, wg_count, nn, max_execs, ms, execs);
    } catch (std::exception& e) {
        g_ref_error = e.what();
        return 2;
    }
}

// BFS levels from root over a device CSR graph; levels (device) initialised here.
int ref_bfs_run_device(int program_type, const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t nv, uint32_t root,
                       uint32_t* d_levels, uint32_t wg_count, uint32_t nn, uint32_t arena, uint32_t max_execs,
                       float* ms, uint32_t* execs) {
    try {
        ck(cudaMemset(d_levels, 0xFF, (size_t)nv * 4u), "levels");
        DevArr<util::iter::AtomicIter<unsigned int>> it(1);
        util::iter::AtomicIter<unsigned int> h_it(0, 1);
        ck(cudaMemcpy(it.p, &h_it, sizeof(h_it), cudaMemcpyHostToDevice), "iter");
        hrm_specs::BfsState st;
        st.rowptr = d_rowptr;
        st.col = d_col;
        st.levels = d_levels;
        st.roots = it.p;
        st.root = root;
        st.nv = nv;
        return drive_spec<hrm_specs::BfsSpec>(program_type, arena, st, wg_count, nn, max_execs, ms, execs);
    } catch (std::exception& e) {
        g_ref_error = e.what();
        return 2;
    }
}

}  // extern "C"
