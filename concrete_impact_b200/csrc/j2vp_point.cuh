// Device routine for one Gauss point of the rate-dependent (Perzyna) J2 return map.
//
// Restates, for one point and in registers, the algorithm of the reference's
// _update_j2_viscoplastic_point (src/fem/materials/plasticity.py:526-681),
// _solve_j2_viscoplastic_multiplier (:711-854), _compute_j2_viscoplastic_hv (:907-926),
// _j2_viscoplastic_consistent_tangent (:929-963) and _compute_j2_equivalent_stress
// (:1441-1465).  The arithmetic type T is float or double; the equivalent plastic strain
// history is always carried in double.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/cib200.h"

namespace cib {

// Material constants derived once on the host (in double) and converted to T.
template <typename T>
struct J2Consts {
  T G;          // shear modulus
  T K;          // bulk modulus
  T lam;        // Lame lambda
  T C11, C12;   // elasticity matrix entries lam + 2G and lam (C44 = G)
  T sy;         // yield stress
  T H;          // isotropic hardening modulus
  T slope;      // 3G + H
  T tau_sref;   // time_scale * reference_stress
  T tau;        // time_scale
  T sref;       // reference_stress
  T m;          // rate exponent
  int m_is_one; // rate_exponent == 1.0 exactly (closed form)
  int max_iterations;
  T yield_rel_tol;
  T res_abs_tol;
  T res_rel_tol;
};

template <typename T>
__host__ inline J2Consts<T> make_j2_consts(const cib_j2vp_material& m, const cib_update_settings& s) {
  const double E = m.young_modulus, nu = m.poisson_ratio;
  const double G = E / (2.0 * (1.0 + nu));
  const double K = E / (3.0 * (1.0 - 2.0 * nu));
  const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  J2Consts<T> c;
  c.G = (T)G;
  c.K = (T)K;
  c.lam = (T)lam;
  c.C11 = (T)(lam + 2.0 * G);
  c.C12 = (T)lam;
  c.sy = (T)m.yield_stress;
  c.H = (T)m.hardening_modulus;
  c.slope = (T)(3.0 * G + m.hardening_modulus);
  c.tau_sref = (T)(m.time_scale * m.reference_stress);
  c.tau = (T)m.time_scale;
  c.sref = (T)m.reference_stress;
  c.m = (T)m.rate_exponent;
  c.m_is_one = (m.rate_exponent == 1.0);
  c.max_iterations = s.max_iterations;
  c.yield_rel_tol = (T)s.yield_relative_tolerance;
  c.res_abs_tol = (T)s.residual_absolute_tolerance;
  c.res_rel_tol = (T)s.residual_relative_tolerance;
  return c;
}

__device__ __forceinline__ bool finite_(double x) { return isfinite(x); }
__device__ __forceinline__ bool finite_(float x) { return isfinite(x); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double pow_(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float pow_(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double fabs_(double x) { return fabs(x); }
__device__ __forceinline__ float fabs_(float x) { return fabsf(x); }
// Python's max(a, b): a unless b > a (so a NaN in b keeps a).
template <typename T>
__device__ __forceinline__ T pymax_(T a, T b) { return (b > a) ? b : a; }

// sigma = C eps for the isotropic elasticity matrix (engineering shear strains).
template <typename T>
__device__ __forceinline__ void elastic_stress(const J2Consts<T>& c, const T e[6], T s[6]) {
  s[0] = c.C11 * e[0] + c.C12 * e[1] + c.C12 * e[2];
  s[1] = c.C12 * e[0] + c.C11 * e[1] + c.C12 * e[2];
  s[2] = c.C12 * e[0] + c.C12 * e[1] + c.C11 * e[2];
  s[3] = c.G * e[3];
  s[4] = c.G * e[4];
  s[5] = c.G * e[5];
}

// Deviatoric part and the J2 radicand 1.5 * sum(w_i s_i^2), w = (1,1,1,2,2,2).
template <typename T>
__device__ __forceinline__ T j2_radicand(const T sig[6], T dev[6]) {
  const T p = (sig[0] + sig[1] + sig[2]) / (T)3;
  dev[0] = sig[0] - p;
  dev[1] = sig[1] - p;
  dev[2] = sig[2] - p;
  dev[3] = sig[3];
  dev[4] = sig[4];
  dev[5] = sig[5];
  const T ss = dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2] +
               (T)2 * (dev[3] * dev[3] + dev[4] * dev[4] + dev[5] * dev[5]);
  return (T)1.5 * ss;
}

// Result of one point update.  The consistent tangent is
//   C_alg = vol * (1 on the 3x3 normal block)
//         + f * (delta_ij - 1/3 on the normal block, 1/2 on the shear diagonal)
//         + c * n_i n_j
// for viscoplastic points (plasticity.py:929-963) and the elasticity matrix for elastic
// points (flag `active` = 0).
template <typename T>
struct J2Out {
  T sigma[6];
  T n[6];       // flow direction 1.5 s_tr / q_tr (zero when elastic)
  T dgamma;     // plastic multiplier increment
  T q_tr;       // trial equivalent stress
  T f_tr;       // trial yield value
  T yield_scale;
  T threshold;  // yield activation threshold
  T hv;         // local modulus h_v (0 when elastic)
  T tan_f;      // deviatoric tangent factor
  T tan_c;      // radial tangent factor
  T local_residual;
  int iters;
  int active;
};

// Failure snapshot writer (only compiled in when RECORD is true).
template <typename T>
struct J2Recorder {
  cib_j2vp_failure* rec;
  __device__ void newton(int reason, int it, T dt, T G, T slope, T ftr, T upper, T tol, int maxit, T x,
                         T over, bool has_res, T res, bool has_der, T der, bool has_cand, T cand) const {
    if (!rec) return;
    rec->reason = reason;
    rec->algorithm = 0;
    rec->iteration = it;
    rec->max_iterations = maxit;
    rec->time_step = (double)dt;
    rec->shear_modulus = (double)G;
    rec->hardening_slope = (double)slope;
    rec->trial_yield = (double)ftr;
    rec->physical_upper_bound = (double)upper;
    rec->residual_tolerance = (double)tol;
    rec->plastic_multiplier = (double)x;
    rec->corrected_overstress = (double)over;
    rec->has_residual = has_res;
    rec->residual = (double)res;
    rec->has_derivative = has_der;
    rec->derivative = (double)der;
    rec->has_newton_candidate = has_cand;
    rec->newton_candidate = (double)cand;
  }
};

// Scalar Perzyna multiplier (plasticity.py:711-854).  Returns a CIB_J2_* status.
template <typename T, bool RECORD>
__device__ __forceinline__ int j2vp_multiplier(const J2Consts<T>& c, T ftr, T dt, T& x_out, int& it_out,
                                               T& res_out, const J2Recorder<T>& rc) {
  const T slope = c.slope;
  const T upper = ftr / slope;
  const T scale = upper;
  const T tol = pymax_(c.res_abs_tol, c.res_rel_tol * scale);
  if (c.m_is_one) {
    const T denom = c.tau_sref / dt + slope;
    const T x = ftr / denom;
    const T corr = ftr - slope * x;
    const T res = x - dt * corr / c.tau_sref;
    const T der = (T)1 + dt * slope / c.tau_sref;
    if (!(finite_(denom) && finite_(x) && finite_(corr) && finite_(res) && finite_(der))) {
      if (RECORD) rc.newton(CIB_J2_NON_FINITE_CLOSED_FORM, 0, dt, c.G, slope, ftr, upper, tol,
                            c.max_iterations, x, corr, true, res, true, der, true, x);
      return CIB_J2_NON_FINITE_CLOSED_FORM;
    }
    if (!((T)0 < x && x < upper) || corr <= (T)0) {
      if (RECORD) rc.newton(CIB_J2_CLOSED_FORM_SOLUTION_OUT_OF_BOUNDS, 0, dt, c.G, slope, ftr, upper, tol,
                            c.max_iterations, x, corr, true, res, true, der, true, x);
      return CIB_J2_CLOSED_FORM_SOLUTION_OUT_OF_BOUNDS;
    }
    x_out = x;
    it_out = 0;
    res_out = res;
    return CIB_J2_OK;
  }
  if (c.max_iterations <= 0) {
    if (RECORD) rc.newton(CIB_J2_INVALID_ITERATION_LIMIT, 0, dt, c.G, slope, ftr, upper, tol,
                          c.max_iterations, (T)0, (T)0, false, (T)0, false, (T)0, false, (T)0);
    return CIB_J2_INVALID_ITERATION_LIMIT;
  }
  if (!(finite_(upper) && finite_(tol))) {
    if (RECORD) rc.newton(CIB_J2_NON_FINITE_PROBLEM_SCALE, 0, dt, c.G, slope, ftr, upper, tol,
                          c.max_iterations, (T)0, (T)0, false, (T)0, false, (T)0, false, (T)0);
    return CIB_J2_NON_FINITE_PROBLEM_SCALE;
  }
  T x = (T)0.5 * upper;
  for (int it = 1; it <= c.max_iterations; ++it) {
    const T over = ftr - slope * x;
    const T nov = over / c.sref;
    if (!finite_(nov) || nov <= (T)0) {
      if (RECORD) rc.newton(CIB_J2_INVALID_CORRECTED_OVERSTRESS, it, dt, c.G, slope, ftr, upper, tol,
                            c.max_iterations, x, over, false, (T)0, false, (T)0, false, (T)0);
      return CIB_J2_INVALID_CORRECTED_OVERSTRESS;
    }
    const T rate = pow_(nov, c.m) / c.tau;
    const T res = x - dt * rate;
    const T der = (T)1 + dt * c.m * slope * pow_(nov, c.m - (T)1) / (c.tau * c.sref);
    if (!(finite_(rate) && finite_(res) && finite_(der))) {
      if (RECORD) rc.newton(CIB_J2_NON_FINITE_ITERATION_VALUE, it, dt, c.G, slope, ftr, upper, tol,
                            c.max_iterations, x, over, true, res, true, der, false, (T)0);
      return CIB_J2_NON_FINITE_ITERATION_VALUE;
    }
    if (der <= (T)0) {
      if (RECORD) rc.newton(CIB_J2_NON_POSITIVE_DERIVATIVE, it, dt, c.G, slope, ftr, upper, tol,
                            c.max_iterations, x, over, true, res, true, der, false, (T)0);
      return CIB_J2_NON_POSITIVE_DERIVATIVE;
    }
    if (fabs_(res) <= tol) {
      if (!((T)0 < x && x < upper) || over <= (T)0) {
        if (RECORD) rc.newton(CIB_J2_CONVERGED_SOLUTION_OUT_OF_BOUNDS, it, dt, c.G, slope, ftr, upper, tol,
                              c.max_iterations, x, over, true, res, true, der, false, (T)0);
        return CIB_J2_CONVERGED_SOLUTION_OUT_OF_BOUNDS;
      }
      x_out = x;
      it_out = it;
      res_out = res;
      return CIB_J2_OK;
    }
    const T cand = x - res / der;
    if (!finite_(cand)) {
      if (RECORD) rc.newton(CIB_J2_NON_FINITE_NEWTON_CANDIDATE, it, dt, c.G, slope, ftr, upper, tol,
                            c.max_iterations, x, over, true, res, true, der, true, cand);
      return CIB_J2_NON_FINITE_NEWTON_CANDIDATE;
    }
    if (!((T)0 < cand && cand < upper)) {
      if (RECORD) rc.newton(CIB_J2_NEWTON_CANDIDATE_OUT_OF_BOUNDS, it, dt, c.G, slope, ftr, upper, tol,
                            c.max_iterations, x, over, true, res, true, der, true, cand);
      return CIB_J2_NEWTON_CANDIDATE_OUT_OF_BOUNDS;
    }
    if (it == c.max_iterations) {
      if (RECORD) rc.newton(CIB_J2_MAXIMUM_ITERATIONS_EXCEEDED, it, dt, c.G, slope, ftr, upper, tol,
                            c.max_iterations, x, over, true, res, true, der, true, cand);
      return CIB_J2_MAXIMUM_ITERATIONS_EXCEEDED;
    }
    x = cand;
  }
  return CIB_J2_MAXIMUM_ITERATIONS_EXCEEDED;  // not reached: the loop returns at it == max
}

// One point: trial stress sig_tr and committed equivalent plastic strain -> J2Out.
// Returns a CIB_J2_* status; on failure `o` is unspecified.
template <typename T, bool RECORD>
__device__ __forceinline__ int j2vp_point(const J2Consts<T>& c, T dt, const T sig_tr[6], double eqps_n,
                                          J2Out<T>& o, cib_j2vp_failure* rec = nullptr) {
  T dev[6];
  const T rad = j2_radicand(sig_tr, dev);
  if (!finite_(rad) || rad < (T)0) {
    const int code = finite_(rad) ? CIB_J2_NEGATIVE_J2_INVARIANT : CIB_J2_NON_FINITE_J2_INVARIANT;
    if (RECORD && rec) {
      rec->reason = code;
      rec->algorithm = 1;
      rec->radicand = (double)rad;
      for (int i = 0; i < 6; ++i) {
        rec->deviatoric_stress[i] = (double)dev[i];
        rec->trial_stress[i] = (double)sig_tr[i];
      }
      rec->equivalent_plastic_strain = eqps_n;
    }
    return code;
  }
  const T q = sqrt_(rad);
  const T radius = c.sy + c.H * (T)eqps_n;
  const T ftr = q - radius;
  const T yscale = pymax_(pymax_(c.sy, c.sref), q);
  const T thr = c.yield_rel_tol * yscale;
  o.q_tr = q;
  o.f_tr = ftr;
  o.yield_scale = yscale;
  o.threshold = thr;
  if (!finite_(c.yield_rel_tol) || c.yield_rel_tol < (T)0 || !finite_(thr)) {
    if (RECORD && rec) {
      rec->reason = CIB_J2_INVALID_YIELD_ACTIVATION_TOLERANCE;
      rec->algorithm = 2;
      rec->yield_scale = (double)yscale;
      rec->yield_activation_threshold = (double)thr;
      rec->trial_yield = (double)ftr;
    }
    return CIB_J2_INVALID_YIELD_ACTIVATION_TOLERANCE;
  }
  if (ftr <= thr) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      o.sigma[i] = sig_tr[i];
      o.n[i] = (T)0;
    }
    o.dgamma = (T)0;
    o.hv = (T)0;
    o.tan_f = (T)2 * c.G;
    o.tan_c = (T)0;
    o.local_residual = (T)0;
    o.iters = 0;
    o.active = 0;
    return CIB_J2_OK;
  }
  const T inv_q = (T)1.5 / q;
#pragma unroll
  for (int i = 0; i < 6; ++i) o.n[i] = dev[i] * inv_q;
  J2Recorder<T> rc{rec};
  if (RECORD && rec) {
    rec->trial_equivalent_stress = (double)q;
    rec->yield_radius = (double)radius;
    rec->equivalent_plastic_strain = eqps_n;
    for (int i = 0; i < 6; ++i) rec->trial_stress[i] = (double)sig_tr[i];
  }
  T dg, res;
  int iters;
  const int st = j2vp_multiplier<T, RECORD>(c, ftr, dt, dg, iters, res, rc);
  if (st != CIB_J2_OK) return st;
  const T two_g_dg = (T)2 * c.G * dg;
#pragma unroll
  for (int i = 0; i < 6; ++i) o.sigma[i] = sig_tr[i] - two_g_dg * o.n[i];
  o.dgamma = dg;
  o.iters = iters;
  o.local_residual = res;
  o.active = 1;
  // Local modulus h_v.  For m != 1 it needs the corrected overstress of the final state.
  T hv;
  if (c.m_is_one) {
    hv = c.tau_sref / dt + c.slope;
  } else {
    T dev2[6];
    const T qf = sqrt_(j2_radicand(o.sigma, dev2));
    const T fyield = qf - (c.sy + c.H * (T)(eqps_n + (double)dg));
    if (fyield <= (T)0) {
      if (RECORD && rec) {
        rec->reason = CIB_J2_NON_POSITIVE_TANGENT_OVERSTRESS;
        rec->algorithm = 3;
        rec->corrected_overstress = (double)fyield;
      }
      return CIB_J2_NON_POSITIVE_TANGENT_OVERSTRESS;
    }
    const T flow_der = c.m * pow_(fyield / c.sref, c.m - (T)1) / (c.tau * c.sref);
    hv = (T)1 / (dt * flow_der) + c.slope;
  }
  o.hv = hv;
  const T G2 = c.G * c.G;
  o.tan_f = (T)2 * c.G - (T)6 * G2 * dg / q;
  o.tan_c = (T)4 * G2 * (dg / q - (T)1 / hv);
  return CIB_J2_OK;
}

// Consistent tangent entry (i, j) from a J2Out (6x6, row-major, engineering strains).
template <typename T>
__device__ __forceinline__ T j2_tangent_entry(const J2Consts<T>& c, const J2Out<T>& o, int i, int j) {
  if (!o.active) {
    if (i < 3 && j < 3) return i == j ? c.C11 : c.C12;
    return (i == j) ? c.G : (T)0;
  }
  T base;
  if (i < 3 && j < 3) {
    base = c.K + o.tan_f * ((i == j ? (T)1 : (T)0) - (T)(1.0 / 3.0));
  } else {
    base = (i == j) ? (T)0.5 * o.tan_f : (T)0;
  }
  return base + o.tan_c * (o.n[i] * o.n[j]);
}

// Record "point p failed" as the lowest failing index.
__device__ __forceinline__ void flag_failure(unsigned long long* first_failure, int64_t p) {
  if (first_failure) atomicMin(first_failure, (unsigned long long)p);
}

}  // namespace cib
