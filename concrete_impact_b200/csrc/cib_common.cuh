// Shared host-side helpers for the cib200 launchers: launch-error capture, grid sizing
// in whole waves over the SM count, and alignment checks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cib200.h"

namespace cib {

// Last CUDA error seen by a launcher in this host thread.
int& last_cuda_error_slot();

inline int check_launch() {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    last_cuda_error_slot() = (int)e;
    return CIB_ECUDA;
  }
  return CIB_OK;
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Number of SMs of the current device (cached per device).
int sm_count();

// Raise a kernel's dynamic shared-memory limit to `bytes` on the current device.  The
// attribute is per device, so the call is made (and remembered) once per kernel and device;
// returns CIB_OK or CIB_ECUDA (with the CUDA error recorded).
int allow_dynamic_smem(const void* kernel, int bytes);

// Grid for a grid-stride kernel: whole waves of resident blocks (SMs x blocks per SM),
// capped by the work available.
inline int persistent_grid(const void* kernel, int threads, int64_t work_items, size_t smem = 0) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int64_t full = (int64_t)sm_count() * per_sm;
  const int64_t needed = (work_items + threads - 1) / threads;
  return (int)(needed < full ? (needed > 0 ? needed : 1) : full);
}

}  // namespace cib
