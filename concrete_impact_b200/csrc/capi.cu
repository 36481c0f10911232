// Library-wide C entry points: names, reasons, version and error reporting.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "cib_common.cuh"

namespace cib {

int& last_cuda_error_slot() {
  static thread_local int slot = 0;
  return slot;
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cached[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

int allow_dynamic_smem(const void* kernel, int bytes) {
  struct Entry {
    const void* kernel;
    int dev;
    int bytes;
  };
  static std::mutex mutex;
  static std::vector<Entry> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    last_cuda_error_slot() = (int)e;
    return CIB_ECUDA;
  }
  std::lock_guard<std::mutex> lock(mutex);
  for (const Entry& x : done)
    if (x.kernel == kernel && x.dev == dev && x.bytes >= bytes) return CIB_OK;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) {
    last_cuda_error_slot() = (int)e;
    return CIB_ECUDA;
  }
  done.push_back({kernel, dev, bytes});
  return CIB_OK;
}

}  // namespace cib

namespace {
// Order of the rows written by cib_j2vp_update; the names are the reference's diagnostic
// keys (src/fem/materials/plasticity.py:565-708).
const char* const kDiagNames[CIB_J2_NDIAG] = {
    "yield_value",
    "plastic_work",
    "local_iterations",
    "active_surface",
    "plastic_multiplier",
    "viscoplastic_multiplier",
    "equivalent_stress",
    "trial_yield_value",
    "yield_scale",
    "yield_activation_threshold",
    "yield_activation_margin",
    "viscoplastic_active",
    "time_step",
    "equivalent_plastic_strain",
    "viscoplastic_hv",
    "plastic_power",
    "hardening_storage_rate",
    "local_residual",
    "root_lower_bound",
    "root_upper_bound",
    "incremental_work_density",
    "equivalent_stress_increment",
};

const char* const kReasons[] = {
    "ok",
    "non_finite_j2_invariant",
    "negative_j2_invariant",
    "invalid_yield_activation_tolerance",
    "non_finite_closed_form",
    "closed_form_solution_out_of_bounds",
    "invalid_iteration_limit",
    "non_finite_problem_scale",
    "invalid_corrected_overstress",
    "non_finite_iteration_value",
    "non_positive_derivative",
    "converged_solution_out_of_bounds",
    "non_finite_newton_candidate",
    "newton_candidate_out_of_bounds",
    "maximum_iterations_exceeded",
    "non_positive_tangent_overstress",
};
}  // namespace

extern "C" const char* cib_j2_diagnostic_name(int row) {
  return (row >= 0 && row < CIB_J2_NDIAG) ? kDiagNames[row] : nullptr;
}

extern "C" const char* cib_j2_reason(int code) {
  const int n = (int)(sizeof(kReasons) / sizeof(kReasons[0]));
  return (code >= 0 && code < n) ? kReasons[code] : "unknown";
}

extern "C" int cib_last_cuda_error(void) { return cib::last_cuda_error_slot(); }

extern "C" int cib_copy_rows_async(void* dst, int64_t dst_pitch, const void* src, int64_t src_pitch,
                                   int64_t row_bytes, int64_t rows, int kind, void* stream) {
  if (!dst || !src || row_bytes < 0 || rows < 0 || dst_pitch < row_bytes || src_pitch < row_bytes) return CIB_EINVAL;
  if (row_bytes == 0 || rows == 0) return CIB_OK;
  cudaMemcpyKind k;
  switch (kind) {
    case 1: k = cudaMemcpyHostToDevice; break;
    case 2: k = cudaMemcpyDeviceToHost; break;
    case 3: k = cudaMemcpyDeviceToDevice; break;
    default: return CIB_EINVAL;
  }
  const cudaError_t e = cudaMemcpy2DAsync(dst, (size_t)dst_pitch, src, (size_t)src_pitch, (size_t)row_bytes,
                                          (size_t)rows, k, reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    cib::last_cuda_error_slot() = (int)e;
    return CIB_ECUDA;
  }
  return CIB_OK;
}

extern "C" const char* cib_version(void) { return "cib200 0.1.0 sm_100a"; }
