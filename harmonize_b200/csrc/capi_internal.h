// capi_internal.h — helpers shared by the translation units of libhrm.so (not exported).
#ifndef HRM_CAPI_INTERNAL_H
#define HRM_CAPI_INTERNAL_H

#include <cuda_runtime.h>

#include "../../include/hrm_capi.h"

#include <cstddef>
#include <stdexcept>
#include <string>
#include <type_traits>

template <typename PROGRAM_SPEC>
class AsyncProgram;

namespace hrm_capi {
// Records `msg` as the calling thread's last error (read by hrm_last_error) and returns code.
int set_error(int code, const std::string& msg);

// Tuning adapter: spec BASE compiled for at least MIN_CTAS resident CTAs per SM
// (__launch_bounds__), which caps its registers.
template <class BASE, size_t MIN_CTAS>
struct MinCtas : BASE {
    static const size_t MIN_CTAS_PER_SM = MIN_CTAS;
};

// What one CTA of a persistent exec kernel holds on an SM: registers per thread, threads and
// shared memory (static + dynamic) per CTA.
struct CtaFootprint {
    unsigned int regs_per_thread = 0;
    unsigned int threads = 0;
    size_t smem = 0;
};

// A photon walk through the whole-run helper (hrm_photon_run_device) on the cached program
// instance of `lane`: walks on different lanes may run at once (on different streams).
int photon_walk_lane(unsigned int lane, const float* d_mu_s, const float* d_absorb, const uint8_t* d_split,
                     uint32_t n, uint64_t seed, uint32_t first, uint32_t count, uint64_t* d_tally,
                     const hrm_run_config* cfg, hrm_run_result* res);

// Teams of the single-spec photon-walk AsyncProgram of tuning variant `variant` that fit on
// the current device at once.
size_t photon_resident_teams(int variant);

// The CTA footprint of the single-spec photon-walk AsyncProgram exec kernel of tuning variant
// `variant` on the current device (HRM_VARIANT_R4_T4_M5 only).
CtaFootprint photon_cta_footprint(int variant);

// What one SM offers the CTAs resident on it (B200: 233,472 B of shared memory with 1,024 B
// reserved per CTA, 65,536 registers in four sub-partitions, 2,048 threads, 32 CTAs).
struct SmLimits {
    size_t smem = 0;          // shared memory per SM
    size_t reserved = 0;      // shared memory reserved by the system per CTA
    size_t regs = 0;          // registers per SM
    size_t threads = 0;       // resident threads per SM
    unsigned int blocks = 0;  // resident CTAs per SM
};

// CTAs per SM of kernel B (at most 64) that fit beside `a_ctas` CTAs per SM of kernel A on an
// SM with limits `sm`: shared memory (with the per-CTA reservation), threads, CTA slots, and
// registers per SM sub-partition (a quarter of the register file; a CTA's warps spread over
// the four sub-partitions, so a kernel of w warps per CTA at c CTAs takes ceil(c*w/4) warps'
// registers from each, a warp's registers allocated in units of 256).
constexpr unsigned int ctas_beside(const CtaFootprint& a, unsigned int a_ctas, const CtaFootprint& b,
                                   const SmLimits& sm) {
    const auto warp_regs = [](unsigned int regs) { return (size_t)((regs * 32u + 255u) / 256u) * 256u; };
    const auto warps = [](const CtaFootprint& f) { return (f.threads + 31u) / 32u; };
    const size_t part_regs = sm.regs / 4u;
    for (unsigned int c = 64; c > 0; c--) {
        const size_t smem = (size_t)a_ctas * (a.smem + sm.reserved) + (size_t)c * (b.smem + sm.reserved);
        const size_t threads = (size_t)a_ctas * a.threads + (size_t)c * b.threads;
        const size_t regs = (size_t)((a_ctas * warps(a) + 3u) / 4u) * warp_regs(a.regs_per_thread) +
                            (size_t)((c * warps(b) + 3u) / 4u) * warp_regs(b.regs_per_thread);
        if (smem <= sm.smem && threads <= sm.threads && a_ctas + c <= sm.blocks && regs <= part_regs) return c;
    }
    return 0;
}

// The same on the current device.
unsigned int ctas_beside(const CtaFootprint& a, unsigned int a_ctas, const CtaFootprint& b);

// Two timing events, destroyed on every path out of the scope that made them (a failed
// launch or a device error flag throws between record and read).
struct EventPair {
    cudaEvent_t start = nullptr, stop = nullptr;
    EventPair() {
        if (cudaEventCreate(&start) != cudaSuccess || cudaEventCreate(&stop) != cudaSuccess) {
            release();
            throw std::runtime_error("cudaEventCreate failed");
        }
    }
    ~EventPair() { release(); }
    EventPair(const EventPair&) = delete;
    EventPair& operator=(const EventPair&) = delete;
    // Milliseconds between the two records (waits for the second one).
    float elapsed_ms() {
        if (cudaEventSynchronize(stop) != cudaSuccess) throw std::runtime_error("cudaEventSynchronize failed");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, start, stop);
        return ms;
    }

   private:
    void release() {
        if (start) cudaEventDestroy(start);
        if (stop) cudaEventDestroy(stop);
        start = stop = nullptr;
    }
};

// Runs `fn` on every path out of the scope that holds the returned object.
template <typename F>
struct ScopeExit {
    F fn;
    ~ScopeExit() { fn(); }
};
template <typename F>
ScopeExit<F> on_scope_exit(F fn) {
    return ScopeExit<F>{fn};
}

template <typename P>
struct is_async_program : std::false_type {};
template <typename S>
struct is_async_program<AsyncProgram<S>> : std::true_type {};
}  // namespace hrm_capi

#endif
