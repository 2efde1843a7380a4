// errors.h -- per-thread error message of the C ABI (shared by the CUDA and
// the host translation units).
#pragma once

#include "../../include/mlbm.h"

namespace mlbm {
// Record `msg` as the calling thread's last error and return `st`.
mlbm_status set_error(mlbm_status st, const char* msg);
}  // namespace mlbm
