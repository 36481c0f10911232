// Explicit macro time stepping for FE^2 (sm_100a): velocity-Verlet predictor and corrector
// with a lumped mass and homogeneous Dirichlet DOFs, restating the step of the reference's
// solve_material_explicit (src/fem/dynamics/material.py:164-219):
//   u' = u + dt v + dt^2/2 a                       (fixed DOFs set to 0)
//   a' = (load_scale * f_unit - f_int) / m         (fixed DOFs set to 0)
//   v' = v + dt/2 (a + a')                         (fixed DOFs set to 0)
#include <cuda_runtime.h>
#include <stdint.h>

#include "cib_common.cuh"

namespace cib {
namespace {

__global__ void verlet_predict_kernel(int64_t n, const double* __restrict__ u, const double* __restrict__ v,
                                      const double* __restrict__ a, const uint8_t* __restrict__ fixed, double dt,
                                      double* __restrict__ u_next) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u_next[i] = fixed[i] ? 0.0 : u[i] + dt * v[i] + 0.5 * dt * dt * a[i];
}

__global__ void verlet_correct_kernel(int64_t n, const double* __restrict__ f_unit, double load_scale,
                                      const double* __restrict__ f_int, const double* __restrict__ mass,
                                      const uint8_t* __restrict__ fixed, double dt, const double* __restrict__ a,
                                      const double* __restrict__ v, double* __restrict__ a_next,
                                      double* __restrict__ v_next) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (fixed[i]) {
    a_next[i] = 0.0;
    v_next[i] = 0.0;
    return;
  }
  const double an = (load_scale * f_unit[i] - f_int[i]) / mass[i];
  a_next[i] = an;
  v_next[i] = v[i] + 0.5 * dt * (a[i] + an);
}

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" int cib_verlet_predict(int64_t n, const double* u, const double* v, const double* a, const uint8_t* fixed,
                                  double dt, double* u_next, void* stream) {
  if (n < 0 || !u || !v || !a || !fixed || !u_next) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  verlet_predict_kernel<<<(unsigned)((n + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      n, u, v, a, fixed, dt, u_next);
  return check_launch();
}

extern "C" int cib_verlet_correct(int64_t n, const double* f_unit, double load_scale, const double* f_int,
                                  const double* mass, const uint8_t* fixed, double dt, const double* a, const double* v,
                                  double* a_next, double* v_next, void* stream) {
  if (n < 0 || !f_unit || !f_int || !mass || !fixed || !a || !v || !a_next || !v_next) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  verlet_correct_kernel<<<(unsigned)((n + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      n, f_unit, load_scale, f_int, mass, fixed, dt, a, v, a_next, v_next);
  return check_launch();
}
