// errors.h -- per-thread error message of the C ABI (shared by the CUDA and
// the host translation units).
#pragma once

#include <cuda_runtime.h>

#include "../../include/mlbm.h"

namespace mlbm {
// Restores the calling thread's current device when it goes out of scope,
// so an entry point that switches to a lattice's device leaves the caller's
// device current on every return path.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      prev = -1;
      cudaGetLastError();
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Record `msg` as the calling thread's last error and return `st`.
mlbm_status set_error(mlbm_status st, const char* msg);
}  // namespace mlbm
