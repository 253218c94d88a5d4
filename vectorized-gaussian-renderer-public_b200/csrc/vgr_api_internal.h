// Helpers shared by the C ABI translation units.
#pragma once

#include <stdint.h>

namespace vgr {

// Records a thread-local error message and returns code.
int fail(int code, const char* fmt, ...);
// Converts a pending CUDA launch error into VGR_ERR_CUDA.
int check_launch(const char* what, int launches = 1);
// Streaming-multiprocessor count of the current device (cached).
int device_sms(int* sms);

}  // namespace vgr
