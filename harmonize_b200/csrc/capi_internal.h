// capi_internal.h — helpers shared by the translation units of libhrm.so (not exported).
#ifndef HRM_CAPI_INTERNAL_H
#define HRM_CAPI_INTERNAL_H

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <type_traits>

template <typename PROGRAM_SPEC>
class AsyncProgram;

namespace hrm_capi {
// Records `msg` as the calling thread's last error (read by hrm_last_error) and returns code.
int set_error(int code, const std::string& msg);

// Teams (32-lane work groups) of the single-spec photon-walk AsyncProgram of tuning variant
// `variant` that can be resident on one SM of the current device at once.
unsigned int photon_teams_per_sm(int variant);

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
