// errors.hpp -- the per-thread error record behind sov_last_error(), for host code in any file.
#pragma once

#include <string>

namespace sov {

// Record `msg` as the calling thread's sov_last_error() and return `code` (capi.cu).
int record_error(int code, const std::string& msg);
// SOV_OK when an sm_100 device is current, else the recorded SOV_E_NO_DEVICE (capi.cu).
int require_device();

}  // namespace sov
