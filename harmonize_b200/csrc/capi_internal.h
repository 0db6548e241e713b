// capi_internal.h — helpers shared by the translation units of libhrm.so (not exported).
#ifndef HRM_CAPI_INTERNAL_H
#define HRM_CAPI_INTERNAL_H

#include <string>
#include <type_traits>

template <typename PROGRAM_SPEC>
class AsyncProgram;

namespace hrm_capi {
// Records `msg` as the calling thread's last error (read by hrm_last_error) and returns code.
int set_error(int code, const std::string& msg);

template <typename P>
struct is_async_program : std::false_type {};
template <typename S>
struct is_async_program<AsyncProgram<S>> : std::true_type {};
}  // namespace hrm_capi

#endif
