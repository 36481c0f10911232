// Batched J2 Perzyna return-map kernels (sm_100a).
//
//  * j2vp_soa_kernel: the streaming form used for large batches.  Structure-of-arrays
//    state (stress, plastic strain, equivalent plastic strain) with 128-bit vector loads
//    and cache-streaming stores; one thread owns VEC consecutive points so that every
//    warp touches 512 contiguous bytes per component stream.  HBM-bandwidth bound.
//  * j2vp_aos_kernel: the reference form of J2ViscoplasticMaterial.update
//    (src/fem/materials/plasticity.py:343-431): total strains, plastic_strain /
//    equivalent_plastic_strain / viscoplastic_multiplier state, tangents, free energy,
//    dissipation and the 22 per-point diagnostics rows (plasticity.py:565-681, 684-708).
//  * j2vp_diagnose_kernel: re-runs one failed point and writes its failure snapshot.
//  * linear_elastic_kernel: evaluate_linear_elastic_points (linear_elastic.py:74-100)
//    plus the elastic-phase increment diagnostics of phased.py:172-191.
#include <cuda_runtime.h>

#include "cib_common.cuh"
#include "j2vp_point.cuh"

namespace cib {

template <typename T, int VEC>
struct VecT;
template <>
struct VecT<double, 1> {
  using type = double;
};
template <>
struct VecT<double, 2> {
  using type = double2;
};
template <>
struct VecT<float, 1> {
  using type = float;
};
template <>
struct VecT<float, 4> {
  using type = float4;
};

template <typename T, int VEC>
__device__ __forceinline__ void ldv(const T* __restrict__ p, T (&out)[VEC]) {
  using V = typename VecT<T, VEC>::type;
  const V v = __ldcs(reinterpret_cast<const V*>(p));
  const T* t = reinterpret_cast<const T*>(&v);
#pragma unroll
  for (int k = 0; k < VEC; ++k) out[k] = t[k];
}

template <typename T, int VEC>
__device__ __forceinline__ void stv(T* __restrict__ p, const T (&in)[VEC]) {
  using V = typename VecT<T, VEC>::type;
  V v;
  T* t = reinterpret_cast<T*>(&v);
#pragma unroll
  for (int k = 0; k < VEC; ++k) t[k] = in[k];
  __stcs(reinterpret_cast<V*>(p), v);
}

// Equivalent plastic strain is always double: load/store VEC doubles (VEC = 1, 2 or 4).
template <int VEC>
__device__ __forceinline__ void ldq(const double* __restrict__ p, double (&out)[VEC]) {
  if constexpr (VEC == 1) {
    out[0] = __ldcs(p);
  } else {
#pragma unroll
    for (int k = 0; k < VEC; k += 2) {
      const double2 v = __ldcs(reinterpret_cast<const double2*>(p + k));
      out[k] = v.x;
      out[k + 1] = v.y;
    }
  }
}

template <int VEC>
__device__ __forceinline__ void stq(double* __restrict__ p, const double (&in)[VEC]) {
  if constexpr (VEC == 1) {
    __stcs(p, in[0]);
  } else {
#pragma unroll
    for (int k = 0; k < VEC; k += 2) __stcs(reinterpret_cast<double2*>(p + k), make_double2(in[k], in[k + 1]));
  }
}

// ---------------------------------------------------------------------------------------
// Streaming SoA kernel.  Component c of point p lives at [c * stride + p].  Points
// [0, count) of the (already offset) pointers are processed, VEC per thread.
// TAN: 0 no tangent, 1 the full 6x6 consistent tangent (36 rows), 2 the compact tangent
// (8 rows: flow direction n (6), f, c with C = K 1(x)1 + f P + c n(x)n, P the deviatoric
// projector in engineering-shear Voigt form; an elastic point has n = 0, f = 2G, c = 0).
template <typename T, int VEC, int TAN>
__global__ void __launch_bounds__(256) j2vp_soa_kernel(
    const J2Consts<T> c, const T dt, const int64_t nvec, const int64_t stride, const T* __restrict__ de,
    const T* __restrict__ s0, const T* __restrict__ ep0, const double* __restrict__ q0, T* __restrict__ s1,
    T* __restrict__ ep1, double* __restrict__ q1, T* __restrict__ tan, unsigned long long* first_failure,
    const int64_t index_offset) {
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvec; v += step) {
    const int64_t p0 = v * VEC;
    // Strain increment and committed stress -> trial stress.
    T sig[6][VEC];
    T ep[6][VEC];
    double q[VEC];
    {
      T d[6][VEC];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        ldv<T, VEC>(de + k * stride + p0, d[k]);
        ldv<T, VEC>(s0 + k * stride + p0, sig[k]);
        ldv<T, VEC>(ep0 + k * stride + p0, ep[k]);
      }
      ldq<VEC>(q0 + p0, q);
#pragma unroll
      for (int j = 0; j < VEC; ++j) {
        T e[6], ds[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) e[k] = d[k][j];
        elastic_stress(c, e, ds);
#pragma unroll
        for (int k = 0; k < 6; ++k) sig[k][j] += ds[k];
      }
    }
    T nn[6][VEC];
    T tf[VEC], tc[VEC];
    int act[VEC];
#pragma unroll
    for (int j = 0; j < VEC; ++j) {
      T st[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) st[k] = sig[k][j];
      J2Out<T> o;
      const int status = j2vp_point<T, false>(c, dt, st, q[j], o);
      if (status != CIB_J2_OK) {
        flag_failure(first_failure, index_offset + p0 + j);
        o.active = 0;
        o.dgamma = (T)0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          o.sigma[k] = st[k];
          o.n[k] = (T)0;
        }
      }
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        sig[k][j] = o.sigma[k];
        nn[k][j] = o.n[k];
        ep[k][j] += (k < 3 ? o.dgamma : (T)2 * o.dgamma) * o.n[k];
      }
      q[j] += (double)o.dgamma;
      tf[j] = o.tan_f;
      tc[j] = o.tan_c;
      act[j] = o.active;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      stv<T, VEC>(s1 + k * stride + p0, sig[k]);
      stv<T, VEC>(ep1 + k * stride + p0, ep[k]);
    }
    stq<VEC>(q1 + p0, q);
    if (TAN == 2) {
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        T row[VEC];
#pragma unroll
        for (int j = 0; j < VEC; ++j) row[j] = act[j] ? nn[i][j] : (T)0;
        stv<T, VEC>(tan + (int64_t)i * stride + p0, row);
      }
      T rf[VEC], rc[VEC];
#pragma unroll
      for (int j = 0; j < VEC; ++j) {
        rf[j] = act[j] ? tf[j] : (T)2 * c.G;
        rc[j] = act[j] ? tc[j] : (T)0;
      }
      stv<T, VEC>(tan + (int64_t)6 * stride + p0, rf);
      stv<T, VEC>(tan + (int64_t)7 * stride + p0, rc);
    }
    if (TAN == 1) {
#pragma unroll
      for (int i = 0; i < 6; ++i) {
#pragma unroll
        for (int jj = 0; jj < 6; ++jj) {
          T row[VEC];
#pragma unroll
          for (int j = 0; j < VEC; ++j) {
            T base;
            if (!act[j]) {
              base = (i < 3 && jj < 3) ? (i == jj ? c.C11 : c.C12) : (i == jj ? c.G : (T)0);
            } else {
              base = (i < 3 && jj < 3) ? c.K + tf[j] * ((i == jj ? (T)1 : (T)0) - (T)(1.0 / 3.0))
                                       : (i == jj ? (T)0.5 * tf[j] : (T)0);
              base += tc[j] * (nn[i][j] * nn[jj][j]);
            }
            row[j] = base;
          }
          stv<T, VEC>(tan + (int64_t)(6 * i + jj) * stride + p0, row);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// Reference-form kernel, one thread per point, row-major (n,6) / (n,6,6) arrays.
struct AosArgs {
  int64_t n;
  double dt;
  const double* strain;
  const double* rate;
  const double* ep0;
  const double* q0;
  const double* vpm0;
  double* stress;
  double* ep1;
  double* q1;
  double* vpm1;
  double* tangent;
  double* psi;
  double* diss;
  double* diag;
  unsigned long long* active_count;
  unsigned long long* first_failure;
};

__global__ void __launch_bounds__(128) j2vp_aos_kernel(const J2Consts<double> c, const AosArgs a) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool is_active = false;
  if (p < a.n) {
    double eps[6], epn[6], eel[6], st[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      eps[k] = a.strain[6 * p + k];
      epn[k] = a.ep0[6 * p + k];
      eel[k] = eps[k] - epn[k];
    }
    elastic_stress(c, eel, st);
    const double qn = a.q0[p];
    J2Out<double> o;
    int status = j2vp_point<double, false>(c, a.dt, st, qn, o);
    double qf = o.q_tr, fy = o.f_tr, pw = 0.0;
    double ep1[6];
    const double dg = o.dgamma;
    const double q1 = qn + (status == CIB_J2_OK ? dg : 0.0);
    if (status == CIB_J2_OK) {
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double inc = (k < 3 ? dg : 2.0 * dg) * o.n[k];
        ep1[k] = epn[k] + inc;
        pw += o.sigma[k] * inc;
      }
      if (o.active) {
        double dev[6];
        qf = sqrt(j2_radicand(o.sigma, dev));
        fy = qf - (c.sy + c.H * q1);
      }
    }
    // Increment diagnostics (plasticity.py:684-708).
    double iwd = 0.0, esi = 0.0;
    if (status == CIB_J2_OK && a.rate) {
      double de[6], eprev[6], sprev[6], dev[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        de[k] = a.dt * a.rate[6 * p + k];
        eprev[k] = (eps[k] - de[k]) - epn[k];
      }
      elastic_stress(c, eprev, sprev);
      const double rp = j2_radicand(sprev, dev);
      const double rc = j2_radicand(o.sigma, dev);
      if (!isfinite(rp) || rp < 0.0 || !isfinite(rc) || rc < 0.0) {
        status = (!isfinite(rp) || !isfinite(rc)) ? CIB_J2_NON_FINITE_J2_INVARIANT : CIB_J2_NEGATIVE_J2_INVARIANT;
      } else {
        double w = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) w += (sprev[k] + o.sigma[k]) * de[k];
        iwd = 0.5 * w;
        esi = sqrt(rc) - sqrt(rp);
      }
    }
    if (status != CIB_J2_OK) {
      flag_failure(a.first_failure, p);
    } else {
      is_active = o.active != 0;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        a.stress[6 * p + k] = o.sigma[k];
        a.ep1[6 * p + k] = ep1[k];
      }
      a.q1[p] = q1;
      a.vpm1[p] = a.vpm0[p] + dg;
      if (a.tangent) {
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
          for (int j = 0; j < 6; ++j) a.tangent[36 * p + 6 * i + j] = j2_tangent_entry(c, o, i, j);
      }
      const double hard_rate = o.active ? c.H * q1 * dg / a.dt : 0.0;
      if (a.psi) {
        double ee[6], se[6], w = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) ee[k] = eps[k] - ep1[k];
        elastic_stress(c, ee, se);
#pragma unroll
        for (int k = 0; k < 6; ++k) w += se[k] * ee[k];
        a.psi[p] = 0.5 * w + 0.5 * c.H * q1 * q1;
      }
      if (a.diss) a.diss[p] = o.active ? pw / a.dt - hard_rate : 0.0;
      if (a.diag) {
        const int64_t n = a.n;
        double* d = a.diag;
        const bool v = o.active != 0;
        d[0 * n + p] = fy;
        d[1 * n + p] = v ? pw : 0.0;
        d[2 * n + p] = (double)o.iters;
        d[3 * n + p] = v ? 4.0 : 0.0;
        d[4 * n + p] = dg;
        d[5 * n + p] = dg;
        d[6 * n + p] = qf;
        d[7 * n + p] = o.f_tr;
        d[8 * n + p] = o.yield_scale;
        d[9 * n + p] = o.threshold;
        d[10 * n + p] = (o.f_tr - o.threshold) / o.yield_scale;
        d[11 * n + p] = v ? 1.0 : 0.0;
        d[12 * n + p] = a.dt;
        d[13 * n + p] = q1;
        d[14 * n + p] = v ? o.hv : 0.0;
        d[15 * n + p] = v ? pw / a.dt : 0.0;
        d[16 * n + p] = hard_rate;
        d[17 * n + p] = v ? o.local_residual : 0.0;
        d[18 * n + p] = 0.0;
        d[19 * n + p] = v ? o.f_tr / c.slope : 0.0;
        d[20 * n + p] = iwd;
        d[21 * n + p] = esi;
      }
    }
  }
  if (a.active_count) {
    const unsigned ballot = __ballot_sync(0xffffffffu, is_active);
    if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(a.active_count, (unsigned long long)__popc(ballot));
  }
}

__global__ void j2vp_diagnose_kernel(const J2Consts<double> c, const AosArgs a, const int64_t p,
                                     cib_j2vp_failure* rec) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  cib_j2vp_failure r = {};
  double eps[6], epn[6], eel[6], st[6];
  for (int k = 0; k < 6; ++k) {
    eps[k] = a.strain[6 * p + k];
    epn[k] = a.ep0[6 * p + k];
    eel[k] = eps[k] - epn[k];
  }
  elastic_stress(c, eel, st);
  r.time_step = a.dt;
  r.max_iterations = c.max_iterations;
  J2Out<double> o;
  int status = j2vp_point<double, true>(c, a.dt, st, a.q0[p], o, &r);
  if (status == CIB_J2_OK && a.rate) {
    double de[6], eprev[6], sprev[6], dev[6];
    for (int k = 0; k < 6; ++k) {
      de[k] = a.dt * a.rate[6 * p + k];
      eprev[k] = (eps[k] - de[k]) - epn[k];
    }
    elastic_stress(c, eprev, sprev);
    double rad = j2_radicand(sprev, dev);
    if (isfinite(rad) && rad >= 0.0) rad = j2_radicand(o.sigma, dev);
    if (!isfinite(rad) || rad < 0.0) {
      status = isfinite(rad) ? CIB_J2_NEGATIVE_J2_INVARIANT : CIB_J2_NON_FINITE_J2_INVARIANT;
      r.reason = status;
      r.algorithm = 1;
      r.radicand = rad;
      for (int k = 0; k < 6; ++k) r.deviatoric_stress[k] = dev[k];
    }
  }
  r.reason = status;
  *rec = r;
}

// ---------------------------------------------------------------------------------------
struct ElasticArgs {
  int64_t n;
  double dt;
  double C11, C12, G;
  const double* strain;
  const double* rate;
  double* stress;
  double* tangent;
  double* psi;
  double* diss;
  double* incdiag;
};

__device__ __forceinline__ double eq_stress(const double s[6]) {
  const double p = (s[0] + s[1] + s[2]) / 3.0;
  const double a = s[0] - p, b = s[1] - p, cc = s[2] - p;
  return sqrt(1.5 * (a * a + b * b + cc * cc + 2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5])));
}

__global__ void __launch_bounds__(128) linear_elastic_kernel(const ElasticArgs a) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n) return;
  double e[6], s[6];
  for (int k = 0; k < 6; ++k) e[k] = a.strain[6 * p + k];
  s[0] = a.C11 * e[0] + a.C12 * e[1] + a.C12 * e[2];
  s[1] = a.C12 * e[0] + a.C11 * e[1] + a.C12 * e[2];
  s[2] = a.C12 * e[0] + a.C12 * e[1] + a.C11 * e[2];
  s[3] = a.G * e[3];
  s[4] = a.G * e[4];
  s[5] = a.G * e[5];
  for (int k = 0; k < 6; ++k) a.stress[6 * p + k] = s[k];
  if (a.tangent) {
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) {
        double v = 0.0;
        if (i < 3 && j < 3) v = (i == j) ? a.C11 : a.C12;
        else if (i == j) v = a.G;
        a.tangent[36 * p + 6 * i + j] = v;
      }
  }
  if (a.psi) {
    double w = 0.0;
    for (int k = 0; k < 6; ++k) w += e[k] * s[k];
    a.psi[p] = 0.5 * w;
  }
  if (a.diss) a.diss[p] = 0.0;
  if (a.incdiag && a.rate) {
    double de[6], ds[6], sp[6];
    for (int k = 0; k < 6; ++k) de[k] = a.dt * a.rate[6 * p + k];
    ds[0] = a.C11 * de[0] + a.C12 * de[1] + a.C12 * de[2];
    ds[1] = a.C12 * de[0] + a.C11 * de[1] + a.C12 * de[2];
    ds[2] = a.C12 * de[0] + a.C12 * de[1] + a.C11 * de[2];
    ds[3] = a.G * de[3];
    ds[4] = a.G * de[4];
    ds[5] = a.G * de[5];
    double w = 0.0;
    for (int k = 0; k < 6; ++k) {
      sp[k] = s[k] - ds[k];
      w += (sp[k] + s[k]) * de[k];
    }
    a.incdiag[p] = 0.5 * w;
    a.incdiag[a.n + p] = eq_stress(s) - eq_stress(sp);
  }
}

// ---------------------------------------------------------------------------------------
// Host launchers.

template <typename T, int VEC, int TAN>
static int launch_soa(const J2Consts<T>& c, T dt, int64_t count, int64_t stride, const T* de, const T* s0,
                      const T* ep0, const double* q0, T* s1, T* ep1, double* q1, T* tan,
                      unsigned long long* ff, cudaStream_t st, int64_t index_offset = 0) {
  const int64_t nvec = count / VEC;
  if (nvec <= 0) return CIB_OK;
  const int threads = 256;
  const int grid = persistent_grid(reinterpret_cast<const void*>(&j2vp_soa_kernel<T, VEC, TAN>), threads, nvec);
  j2vp_soa_kernel<T, VEC, TAN><<<grid, threads, 0, st>>>(c, dt, nvec, stride, de, s0, ep0, q0, s1, ep1, q1, tan, ff,
                                                          index_offset);
  return check_launch();
}

template <typename T, int VEC>
static int run_soa(const cib_j2vp_material* m, const cib_update_settings* s, int64_t n, int64_t ld, double dt,
                   const T* de, const T* s0, const T* ep0, const double* q0, T* s1, T* ep1, double* q1, T* tan,
                   unsigned long long* ff, void* stream, bool compact = false) {
  if (!m || !s || n < 0 || ld < n || !de || !s0 || !ep0 || !q0 || !s1 || !ep1 || !q1) return CIB_EINVAL;
  if (compact && !tan) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  const J2Consts<T> c = make_j2_consts<T>(*m, *s);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int mode = tan ? (compact ? 2 : 1) : 0;
  const bool aligned = (ld % VEC == 0) && aligned16(de) && aligned16(s0) && aligned16(ep0) && aligned16(q0) &&
                       aligned16(s1) && aligned16(ep1) && aligned16(q1) && (tan == nullptr || aligned16(tan));
  int64_t done = 0;
  if (aligned) {
    const int64_t main = n - n % VEC;
    int rc;
    switch (mode) {
      case 2: rc = launch_soa<T, VEC, 2>(c, (T)dt, main, ld, de, s0, ep0, q0, s1, ep1, q1, tan, ff, st); break;
      case 1: rc = launch_soa<T, VEC, 1>(c, (T)dt, main, ld, de, s0, ep0, q0, s1, ep1, q1, tan, ff, st); break;
      default: rc = launch_soa<T, VEC, 0>(c, (T)dt, main, ld, de, s0, ep0, q0, s1, ep1, q1, tan, ff, st); break;
    }
    if (rc != CIB_OK) return rc;
    done = main;
  }
  if (done == n) return CIB_OK;
  // Scalar path for the remaining points (pointers shifted by o; failure indices are
  // reported unshifted through index_offset).
  const int64_t o = done;
  T* to = tan ? tan + o : nullptr;
  switch (mode) {
    case 2:
      return launch_soa<T, 1, 2>(c, (T)dt, n - o, ld, de + o, s0 + o, ep0 + o, q0 + o, s1 + o, ep1 + o, q1 + o, to, ff,
                                 st, o);
    case 1:
      return launch_soa<T, 1, 1>(c, (T)dt, n - o, ld, de + o, s0 + o, ep0 + o, q0 + o, s1 + o, ep1 + o, q1 + o, to, ff,
                                 st, o);
    default:
      return launch_soa<T, 1, 0>(c, (T)dt, n - o, ld, de + o, s0 + o, ep0 + o, q0 + o, s1 + o, ep1 + o, q1 + o, to, ff,
                                 st, o);
  }
}

}  // namespace cib

using namespace cib;

extern "C" int cib_j2vp_update_soa_f64(const cib_j2vp_material* material, const cib_update_settings* settings,
                                       int64_t n, int64_t ld, double time_step, const double* dstrain, const double* stress_n,
                                       const double* plastic_strain_n, const double* eqps_n, double* stress,
                                       double* plastic_strain, double* eqps, double* tangent,
                                       unsigned long long* first_failure, void* stream) {
  return run_soa<double, 2>(material, settings, n, ld, time_step, dstrain, stress_n, plastic_strain_n, eqps_n, stress,
                            plastic_strain, eqps, tangent, first_failure, stream);
}

extern "C" int cib_j2vp_update_soa_f32(const cib_j2vp_material* material, const cib_update_settings* settings,
                                       int64_t n, int64_t ld, double time_step, const float* dstrain, const float* stress_n,
                                       const float* plastic_strain_n, const double* eqps_n, float* stress,
                                       float* plastic_strain, double* eqps, float* tangent,
                                       unsigned long long* first_failure, void* stream) {
  return run_soa<float, 4>(material, settings, n, ld, time_step, dstrain, stress_n, plastic_strain_n, eqps_n, stress,
                           plastic_strain, eqps, tangent, first_failure, stream);
}

extern "C" int cib_j2vp_update_soa_compact_f64(const cib_j2vp_material* material, const cib_update_settings* settings,
                                               int64_t n, int64_t ld, double time_step, const double* dstrain,
                                               const double* stress_n, const double* plastic_strain_n,
                                               const double* eqps_n, double* stress, double* plastic_strain,
                                               double* eqps, double* tangent8, unsigned long long* first_failure,
                                               void* stream) {
  return run_soa<double, 2>(material, settings, n, ld, time_step, dstrain, stress_n, plastic_strain_n, eqps_n, stress,
                            plastic_strain, eqps, tangent8, first_failure, stream, true);
}

extern "C" int cib_j2vp_update_soa_compact_f32(const cib_j2vp_material* material, const cib_update_settings* settings,
                                               int64_t n, int64_t ld, double time_step, const float* dstrain,
                                               const float* stress_n, const float* plastic_strain_n,
                                               const double* eqps_n, float* stress, float* plastic_strain,
                                               double* eqps, float* tangent8, unsigned long long* first_failure,
                                               void* stream) {
  return run_soa<float, 4>(material, settings, n, ld, time_step, dstrain, stress_n, plastic_strain_n, eqps_n, stress,
                           plastic_strain, eqps, tangent8, first_failure, stream, true);
}

extern "C" int cib_j2vp_update(const cib_j2vp_material* material, const cib_update_settings* settings, int64_t n,
                               double time_step, const double* strain, const double* strain_rate,
                               const double* plastic_strain_n, const double* eqps_n, const double* vpm_n,
                               double* stress, double* plastic_strain, double* eqps, double* vpm, double* tangent,
                               double* free_energy, double* dissipation, double* diagnostics,
                               unsigned long long* active_count, unsigned long long* first_failure, void* stream) {
  if (!material || !settings || n < 0 || !strain || !plastic_strain_n || !eqps_n || !vpm_n || !stress ||
      !plastic_strain || !eqps || !vpm)
    return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  const J2Consts<double> c = make_j2_consts<double>(*material, *settings);
  AosArgs a{n,     time_step, strain,      strain_rate, plastic_strain_n, eqps_n,       vpm_n,       stress,       plastic_strain,
            eqps,  vpm,       tangent,     free_energy, dissipation,      diagnostics,  active_count, first_failure};
  const int threads = 128;
  const int64_t blocks = (n + threads - 1) / threads;
  if (blocks > 0x7fffffff) return CIB_ERANGE;
  j2vp_aos_kernel<<<(unsigned)blocks, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(c, a);
  return check_launch();
}

extern "C" int cib_j2vp_diagnose_point(const cib_j2vp_material* material, const cib_update_settings* settings,
                                       int64_t n, double time_step, const double* strain, const double* strain_rate,
                                       const double* plastic_strain_n, const double* eqps_n, int64_t point,
                                       cib_j2vp_failure* record, void* stream) {
  if (!material || !settings || !strain || !plastic_strain_n || !eqps_n || !record || point < 0 || point >= n)
    return CIB_EINVAL;
  const J2Consts<double> c = make_j2_consts<double>(*material, *settings);
  AosArgs a{};
  a.n = n;
  a.dt = time_step;
  a.strain = strain;
  a.rate = strain_rate;
  a.ep0 = plastic_strain_n;
  a.q0 = eqps_n;
  j2vp_diagnose_kernel<<<1, 32, 0, reinterpret_cast<cudaStream_t>(stream)>>>(c, a, point, record);
  return check_launch();
}

extern "C" int cib_linear_elastic_update(double young_modulus, double poisson_ratio, int64_t n, double time_step,
                                         const double* strain, const double* strain_rate, double* stress,
                                         double* tangent, double* free_energy, double* dissipation,
                                         double* increment_diagnostics, void* stream) {
  if (n < 0 || !strain || !stress) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  const double G = young_modulus / (2.0 * (1.0 + poisson_ratio));
  const double lam = young_modulus * poisson_ratio / ((1.0 + poisson_ratio) * (1.0 - 2.0 * poisson_ratio));
  ElasticArgs a{n,           time_step, lam + 2.0 * G, lam, G, strain, strain_rate, stress, tangent,
                free_energy, dissipation, increment_diagnostics};
  const int threads = 128;
  const int64_t blocks = (n + threads - 1) / threads;
  if (blocks > 0x7fffffff) return CIB_ERANGE;
  linear_elastic_kernel<<<(unsigned)blocks, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  return check_launch();
}
