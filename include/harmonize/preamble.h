// preamble.h — platform aliases, debug macros and SFINAE detectors of the Harmonize
// source-level API, for CUDA on sm_100a only.
//
// Names kept from the original API (harmonize/cpp/preamble/mod.h:19-126 and
// harmonize/cpp/preamble/adapt.h:17-81) so that existing specifications and host
// programs compile unchanged: adapt::GPUrt*, adapt::WARP_SIZE, q_printf/rc_printf/
// db_printf, beg_time/end_time, is_detected, type_switch.
#ifndef HARMONIZE_B200_PREAMBLE_H
#define HARMONIZE_B200_PREAMBLE_H

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "spec_support.h"

#define HARMONIZE
#define HARMONIZE_B200

// Debug print hooks. All are compiled out; the names exist because specs use them.
#define NOOP(x) ;
#define q_printf(fmt, ...) ;
#define rc_printf(fmt, ...) ;
#define db_printf(fmt, ...) ;
#define beg_time(idx) ;
#define end_time(idx) ;

namespace adapt {

// Lanes per warp on every NVIDIA architecture, and the size of one coalesced batch of
// promises in this runtime.
static const size_t WARP_SIZE = 32;

using GPUrtError_t  = cudaError_t;
using GPUrtEvent_t  = cudaEvent_t;
using GPUrtStream_t = cudaStream_t;

static const auto GPUrtSuccess              = cudaSuccess;
static const auto GPUrtMemcpyDeviceToDevice = cudaMemcpyDeviceToDevice;
static const auto GPUrtMemcpyDeviceToHost   = cudaMemcpyDeviceToHost;
static const auto GPUrtMemcpyHostToDevice   = cudaMemcpyHostToDevice;
static const auto GPUrtMemcpyDefault        = cudaMemcpyDefault;

// Thin forwarding wrappers: same argument lists as the CUDA runtime calls they name.
#define HRM_FORWARD(name)                                                   \
    template <typename... ARGS>                                             \
    auto GPUrt##name(ARGS... args)->decltype(cuda##name(args...)) {         \
        return cuda##name(args...);                                         \
    }
HRM_FORWARD(Malloc)
HRM_FORWARD(MallocManaged)
HRM_FORWARD(DeviceSynchronize)
HRM_FORWARD(GetErrorString)
HRM_FORWARD(EventCreate)
HRM_FORWARD(EventRecord)
HRM_FORWARD(EventSynchronize)
HRM_FORWARD(EventElapsedTime)
HRM_FORWARD(GetLastError)
HRM_FORWARD(Memcpy)
HRM_FORWARD(Memset)
HRM_FORWARD(SetDevice)
HRM_FORWARD(Free)
#undef HRM_FORWARD

}  // namespace adapt

// Detection idiom (C++17 spelling of std::experimental::is_detected).
namespace detector {

template <class... TYPES>
using void_t = void;

template <template <class...> class LOOKUP, class GUARD, class... ARGS>
struct is_detected : std::false_type {};

template <template <class...> class LOOKUP, class... ARGS>
struct is_detected<LOOKUP, void_t<LOOKUP<ARGS...>>, ARGS...> : std::true_type {};

template <bool COND, class TRUE_TYPE = void, class FALSE_TYPE = void>
struct type_switch {
    using type = typename std::conditional<COND, TRUE_TYPE, FALSE_TYPE>::type;
};

}  // namespace detector

template <template <class...> class LOOKUP, class... ARGS>
using is_detected = typename detector::is_detected<LOOKUP, void, ARGS...>;

template <class DEFAULT, template <class> class LOOKUP, class TYPE>
using type_switch =
    typename detector::type_switch<is_detected<LOOKUP, TYPE>::value, TYPE, DEFAULT>::type;

#endif
