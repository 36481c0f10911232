/*
 * Plain-C oracle of the batched J2 Perzyna return map -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates, point by point, the reference's _update_j2_viscoplastic_point
 * (src/fem/materials/plasticity.py:526-681), _solve_j2_viscoplastic_multiplier (:711-854),
 * _compute_j2_viscoplastic_hv (:907-926) and _j2_viscoplastic_consistent_tangent
 * (:929-963) in the incremental, stress-carried form (trial stress = stress_n + C dstrain).
 * Structure-of-arrays layout [component * n + point], float64, OpenMP over points.
 * Used as the checker for large batches and as the strong multi-core CPU baseline.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  double young_modulus, poisson_ratio, yield_stress, hardening_modulus, time_scale, reference_stress, rate_exponent;
  int max_iterations;
  double yield_relative_tolerance, residual_absolute_tolerance, residual_relative_tolerance;
} oracle_j2_params;

static double pymax(double a, double b) { return (b > a) ? b : a; }

/* Returns 0 or the status code of include/cib200.h. */
static int point_update(const oracle_j2_params* p, double G, double K, double lam, double dt, const double de[6],
                        const double s0[6], const double ep0[6], double q0, double s1[6], double ep1[6], double* q1,
                        double tan[36]) {
  double st[6], dev[6], n[6];
  const double c11 = lam + 2.0 * G, c12 = lam;
  st[0] = s0[0] + c11 * de[0] + c12 * de[1] + c12 * de[2];
  st[1] = s0[1] + c12 * de[0] + c11 * de[1] + c12 * de[2];
  st[2] = s0[2] + c12 * de[0] + c12 * de[1] + c11 * de[2];
  st[3] = s0[3] + G * de[3];
  st[4] = s0[4] + G * de[4];
  st[5] = s0[5] + G * de[5];
  const double pr = (st[0] + st[1] + st[2]) / 3.0;
  for (int k = 0; k < 6; ++k) dev[k] = st[k] - (k < 3 ? pr : 0.0);
  const double rad =
      1.5 * (dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2] + 2.0 * (dev[3] * dev[3] + dev[4] * dev[4] + dev[5] * dev[5]));
  if (!isfinite(rad)) return 1;
  if (rad < 0.0) return 2;
  const double q = sqrt(rad);
  const double ftr = q - (p->yield_stress + p->hardening_modulus * q0);
  const double ys = pymax(pymax(p->yield_stress, p->reference_stress), q);
  const double thr = p->yield_relative_tolerance * ys;
  if (!isfinite(p->yield_relative_tolerance) || p->yield_relative_tolerance < 0.0 || !isfinite(thr)) return 3;
  const double slope = 3.0 * G + p->hardening_modulus;
  double dg = 0.0, hv = 0.0;
  int active = ftr > thr;
  if (active) {
    for (int k = 0; k < 6; ++k) n[k] = 1.5 * dev[k] / q;
    const double upper = ftr / slope;
    const double tol = pymax(p->residual_absolute_tolerance, p->residual_relative_tolerance * upper);
    const double tau_sref = p->time_scale * p->reference_stress;
    if (p->rate_exponent == 1.0) {
      const double denom = tau_sref / dt + slope;
      const double x = ftr / denom;
      const double corr = ftr - slope * x;
      const double res = x - dt * corr / tau_sref;
      const double der = 1.0 + dt * slope / tau_sref;
      if (!(isfinite(denom) && isfinite(x) && isfinite(corr) && isfinite(res) && isfinite(der))) return 4;
      if (!(0.0 < x && x < upper) || corr <= 0.0) return 5;
      dg = x;
      hv = tau_sref / dt + slope;
    } else {
      if (p->max_iterations <= 0) return 6;
      if (!(isfinite(upper) && isfinite(tol))) return 7;
      double x = 0.5 * upper;
      int done = 0;
      for (int it = 1; it <= p->max_iterations && !done; ++it) {
        const double over = ftr - slope * x;
        const double nov = over / p->reference_stress;
        if (!isfinite(nov) || nov <= 0.0) return 8;
        const double rate = pow(nov, p->rate_exponent) / p->time_scale;
        const double res = x - dt * rate;
        const double der = 1.0 + dt * p->rate_exponent * slope * pow(nov, p->rate_exponent - 1.0) / tau_sref;
        if (!(isfinite(rate) && isfinite(res) && isfinite(der))) return 9;
        if (der <= 0.0) return 10;
        if (fabs(res) <= tol) {
          if (!(0.0 < x && x < upper) || over <= 0.0) return 11;
          done = 1;
          break;
        }
        const double cand = x - res / der;
        if (!isfinite(cand)) return 12;
        if (!(0.0 < cand && cand < upper)) return 13;
        if (it == p->max_iterations) return 14;
        x = cand;
      }
      dg = x;
    }
  }
  for (int k = 0; k < 6; ++k) {
    s1[k] = st[k] - 2.0 * G * dg * (active ? n[k] : 0.0);
    ep1[k] = ep0[k] + (active ? (k < 3 ? dg : 2.0 * dg) * n[k] : 0.0);
  }
  *q1 = q0 + dg;
  if (active && p->rate_exponent != 1.0) {
    const double pf = (s1[0] + s1[1] + s1[2]) / 3.0;
    double d2[6];
    for (int k = 0; k < 6; ++k) d2[k] = s1[k] - (k < 3 ? pf : 0.0);
    const double qf =
        sqrt(1.5 * (d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2] + 2.0 * (d2[3] * d2[3] + d2[4] * d2[4] + d2[5] * d2[5])));
    const double fy = qf - (p->yield_stress + p->hardening_modulus * (*q1));
    if (fy <= 0.0) return 15;
    const double flow = p->rate_exponent * pow(fy / p->reference_stress, p->rate_exponent - 1.0) /
                        (p->time_scale * p->reference_stress);
    hv = 1.0 / (dt * flow) + slope;
  }
  if (tan) {
    if (!active) {
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j)
          tan[6 * i + j] = (i < 3 && j < 3) ? (i == j ? c11 : c12) : (i == j ? G : 0.0);
    } else {
      const double f = 2.0 * G - 6.0 * G * G * dg / q;
      const double c = 4.0 * G * G * (dg / q - 1.0 / hv);
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
          double base;
          if (i < 3 && j < 3) base = K + f * ((i == j ? 1.0 : 0.0) - 1.0 / 3.0);
          else base = (i == j) ? 0.5 * f : 0.0;
          tan[6 * i + j] = base + c * n[i] * n[j];
        }
    }
  }
  return 0;
}

/* Batched update; returns the number of failing points (status per point if given). */
int64_t oracle_j2vp_incremental(const oracle_j2_params* p, int64_t n, double dt, const double* de, const double* s0,
                                const double* ep0, const double* q0, double* s1, double* ep1, double* q1, double* tan,
                                int32_t* status, int nthreads) {
  const double G = p->young_modulus / (2.0 * (1.0 + p->poisson_ratio));
  const double K = p->young_modulus / (3.0 * (1.0 - 2.0 * p->poisson_ratio));
  const double lam = p->young_modulus * p->poisson_ratio / ((1.0 + p->poisson_ratio) * (1.0 - 2.0 * p->poisson_ratio));
  int64_t failures = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(static) reduction(+ : failures)
  for (int64_t i = 0; i < n; ++i) {
    double a[6], b[6], c[6], o1[6], o2[6], t[36], qq;
    for (int k = 0; k < 6; ++k) {
      a[k] = de[k * n + i];
      b[k] = s0[k * n + i];
      c[k] = ep0[k * n + i];
    }
    const int st = point_update(p, G, K, lam, dt, a, b, c, q0[i], o1, o2, &qq, tan ? t : 0);
    if (status) status[i] = st;
    failures += (st != 0);
    for (int k = 0; k < 6; ++k) {
      s1[k * n + i] = o1[k];
      ep1[k * n + i] = o2[k];
    }
    q1[i] = qq;
    if (tan)
      for (int k = 0; k < 36; ++k) tan[(int64_t)k * n + i] = t[k];
  }
  return failures;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
