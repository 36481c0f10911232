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

// Input stage of the surrogate's error gate for n macro points: the normalised fp32 inputs
// of the fused window kernel, the latent step coefficient, and the points (not yet
// flagged) whose strain or rate leaves the per-component training envelope `lim` (strain
// 0..5, rate 6..11, in normalised units) or is not finite.  `count` gains their number.
__global__ void rno_gate_prepare_kernel(int64_t n, const double* __restrict__ strain, const double* __restrict__ rate,
                                        double inv_se, double inv_sr, const double* __restrict__ lim, float coef,
                                        const uint8_t* __restrict__ flagged, float* __restrict__ sn,
                                        float* __restrict__ rn, float* __restrict__ cf, uint8_t* __restrict__ fresh,
                                        unsigned int* __restrict__ count) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool f = false;
  if (i < n) {
    bool over = false;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double e = strain[6 * i + k] * inv_se, r = rate[6 * i + k] * inv_sr;
      sn[6 * i + k] = (float)e;
      rn[6 * i + k] = (float)r;
      over |= !(fabs(e) <= lim[k]) || !(fabs(r) <= lim[6 + k]);  // also true for NaN
    }
    cf[i] = coef;
    f = over && !flagged[i];
    fresh[i] = f ? 1 : 0;
  }
  const unsigned m = __ballot_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(count, (unsigned)__popc(m));
}

// Output stage: physical stress = normalised stress * scale; a point whose surrogate answer
// is not finite is flagged as well (counted once).
__global__ void rno_gate_finish_kernel(int64_t n, const float* __restrict__ stress_n, double scale,
                                       const uint8_t* __restrict__ flagged, uint8_t* __restrict__ fresh,
                                       unsigned int* __restrict__ count, double* __restrict__ stress) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool f = false;
  if (i < n) {
    bool bad = false;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const float v = stress_n[6 * i + k];
      bad |= !isfinite(v);
      stress[6 * i + k] = (double)v * scale;
    }
    f = bad && !flagged[i] && !fresh[i];
    if (f) fresh[i] = 1;
  }
  const unsigned m = __ballot_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(count, (unsigned)__popc(m));
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

extern "C" int cib_rno_gate_prepare(int64_t n, const double* strain, const double* rate, double strain_scale,
                                    double rate_scale, const double* limits, double coef, const uint8_t* flagged,
                                    float* strain_n, float* rate_n, float* coef_out, uint8_t* fresh,
                                    unsigned int* count, void* stream) {
  if (n < 0 || !strain || !rate || !limits || !flagged || !strain_n || !rate_n || !coef_out || !fresh || !count ||
      !(strain_scale > 0.0) || !(rate_scale > 0.0))
    return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  rno_gate_prepare_kernel<<<(unsigned)((n + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      n, strain, rate, 1.0 / strain_scale, 1.0 / rate_scale, limits, (float)coef, flagged, strain_n, rate_n, coef_out,
      fresh, count);
  return check_launch();
}

extern "C" int cib_rno_gate_finish(int64_t n, const float* stress_n, double stress_scale, const uint8_t* flagged,
                                   uint8_t* fresh, unsigned int* count, double* stress, void* stream) {
  if (n < 0 || !stress_n || !flagged || !fresh || !count || !stress) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  rno_gate_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      n, stress_n, stress_scale, flagged, fresh, count, stress);
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
