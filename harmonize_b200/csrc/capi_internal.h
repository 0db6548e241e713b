// capi_internal.h — helpers shared by the translation units of libhrm.so (not exported).
#ifndef HRM_CAPI_INTERNAL_H
#define HRM_CAPI_INTERNAL_H

#include <string>

namespace hrm_capi {
// Records `msg` as the calling thread's last error (read by hrm_last_error) and returns code.
int set_error(int code, const std::string& msg);
}  // namespace hrm_capi

#endif
