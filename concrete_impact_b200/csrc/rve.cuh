// Device-side argument structs of the periodic RVE kernels (see rve.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cib200.h"
#include "j2vp_point.cuh"

namespace cib {

constexpr int RVE_THREADS = 256;
constexpr int RVE_MAX_PHASES = CIB_RVE_MAX_PHASES;
constexpr int PHASE_ELASTIC = 0;
constexpr int PHASE_J2VP = 1;

// Slots of the per-RVE reduction written by rve_response_kernel (RVE_NOUT doubles per RVE).
constexpr int RS_SIGMA = 0;         // 6: sum sigma w
constexpr int RS_PSI = 6;           // sum psi w
constexpr int RS_DISS = 7;          // sum D w
constexpr int RS_MICRO_WORK = 8;    // sum sigma . (eps - eps_prev) w
constexpr int RS_POS_WORK = 9;      // sum max(iwd, 0) w
constexpr int RS_NEG_WORK = 10;     // sum min(iwd, 0) w
constexpr int RS_UNLOAD = 11;       // volume with iwd < 0
constexpr int RS_ACTIVE = 12;       // volume of viscoplastic points
constexpr int RS_EQPS = 13;         // sum eqps w (J2 points)
constexpr int RS_VW = 14;           // 6: A^T f (virtual work)
constexpr int RS_FNORM2 = 20;       // ||f_int||^2 over physical nodes
constexpr int RS_FACE = 21;         // 18: face resultants (axis, minus/plus, xyz)
constexpr int RS_PERIODIC = 39;     // max periodic fluctuation mismatch
constexpr int RS_PHASE = 40;        // per phase: volume, sigma (6), psi, D, eqps -> 10
constexpr int RS_PHASE_STRIDE = 10;
constexpr int RVE_NSUM = RS_PHASE + RS_PHASE_STRIDE * RVE_MAX_PHASES;  // 120
constexpr int RVE_NOUT = RVE_NSUM + 2 + RVE_MAX_PHASES;                 // + margin min/max + phase eqps max
static_assert(RVE_NOUT == CIB_RVE_NOUT, "reduction slot count must match the public header");

struct RveDesc {
  int nx, ny, nz, pad;
  int64_t eoff;
  double hx, hy, hz;
};
static_assert(sizeof(RveDesc) == sizeof(cib_rve_desc), "descriptor layout");

template <typename T>
struct PhaseMat {
  int kind;
  J2Consts<T> j2;  // elasticity entries are used by both kinds
  T C11, C12, G, K;
};

template <typename T>
struct PhaseTable {
  PhaseMat<T> m[RVE_MAX_PHASES];
};

template <typename T>
struct RveResidualArgs {
  const RveDesc* desc;
  int nrve;
  int64_t nelem;  // elements of the batch (RVE r owns [desc[r].eoff, desc[r].eoff + E_r))
  const uint8_t* phase;
  PhaseTable<T> mats;
  const double* macro;
  const double* w;
  const double* dw;
  const double* alpha;
  const int32_t* active;
  int64_t ngp;
  const T* ep_n;
  const double* q_n;
  const double* vpm_n;
  T* ep;
  double* q;
  double* vpm;
  T* stress;
  T* tparam;
  uint8_t* tflag;
  double* fe;
  double* de;
  const double* dt;  // per RVE
  unsigned long long* fail;
};

struct RveGatherArgs {
  const RveDesc* desc;
  int nrve;
  int64_t nelem;
  const double* fe;
  const double* de;
  const double* w;
  const double* dw;
  const double* alpha;
  const int32_t* active;
  double* res;
  double* dinv;
  double* rnorm2;
  double* wnorm2;
  double* class_max;
  double* w_out;
};

template <typename T>
struct RvePcgArgs {
  const RveDesc* desc;
  const uint8_t* phase;
  PhaseTable<T> mats;
  int64_t ngp;
  const T* tparam;
  const uint8_t* tflag;
  const int32_t* sys_rve;
  const int64_t* sys_off;
  const int32_t* active;
  const double* b;
  const double* dinv;
  double* x;
  double* r;
  double* p;
  double* Ap;
  double rtol;
  const double* rtol_dev = nullptr;  // when set, the relative tolerance is read here (device-side control)
  int maxit;
  int32_t* status;
  int32_t* iterations;
  double* rel_residual;
  double* xnorm;
  // Length of the vectors r, p, Ap when they belong to the library (no-allocation entry):
  // a system whose entries would leave [0, vec_len) is skipped with status 3.  -1: the
  // caller owns the vectors and sizes them (not checked).
  int64_t vec_len = -1;
};

template <typename T>
struct RveTangentArgs {
  const RveDesc* desc;
  const uint8_t* phase;
  PhaseTable<T> mats;
  int64_t ngp;
  int64_t ne_total;
  const T* tparam;
  const uint8_t* tflag;
  const int32_t* active;
  double* fe6;
  double* rhs;
  double* kee;
};

struct RveTangentFinishArgs {
  const RveDesc* desc;
  const int32_t* active;
  const double* rhs;
  const double* sol;
  const double* kee;
  double* ceff;
};

template <typename T>
struct RveResponseArgs {
  const RveDesc* desc;
  const uint8_t* phase;
  PhaseTable<double> mats;
  PhaseTable<T> mats_t;
  const double* macro;
  const double* macro_n;
  const double* w;
  const double* w_n;
  const int32_t* active;
  int64_t ngp;
  const T* ep_n;
  const double* q_n;
  const T* ep;
  const double* q;
  const T* stress;
  const uint8_t* tflag;
  const double* fe;
  const double* dt;  // per RVE
  double* sums;
  double* point_out;
  double* diag;
};

// ---------------------------------------------------------------------------------------
// Host-side argument builders from the public batch struct (shared by the C entry points).

// Gauss points per SoA row: the whole batch's, also for a view of its first RVEs.
inline int64_t rve_point_stride(const cib_rve_batch& b) { return b.point_stride > 0 ? b.point_stride : 8 * b.nelem; }

template <typename T>
inline PhaseTable<T> rve_phase_table(const cib_rve_batch& b) {
  PhaseTable<T> t;
  for (int i = 0; i < RVE_MAX_PHASES; ++i) {
    const cib_phase_material& pm = b.mats[i < b.nphase ? i : 0];
    PhaseMat<T>& m = t.m[i];
    m.kind = pm.kind;
    cib_j2vp_material params = pm.params;
    if (pm.kind == PHASE_ELASTIC) {
      // elastic phases only use the elasticity entries; keep the J2 block well defined
      params.yield_stress = 1.0;
      params.time_scale = 1.0;
      params.reference_stress = 1.0;
      params.rate_exponent = 1.0;
    }
    m.j2 = make_j2_consts<T>(params, b.settings);
    m.C11 = m.j2.C11;
    m.C12 = m.j2.C12;
    m.G = m.j2.G;
    m.K = m.j2.K;
  }
  return t;
}

template <typename T>
inline RveResidualArgs<T> rve_residual_args(const cib_rve_batch& b, const double* dt, const double* macro,
                                            const double* w, const double* dw, const double* alpha,
                                            const int32_t* active, unsigned long long* fail) {
  RveResidualArgs<T> a;
  a.desc = reinterpret_cast<const RveDesc*>(b.desc);
  a.nrve = b.nrve;
  a.nelem = b.nelem;
  a.phase = b.phase;
  a.mats = rve_phase_table<T>(b);
  a.macro = macro;
  a.w = w;
  a.dw = dw;
  a.alpha = alpha;
  a.active = active;
  a.ngp = rve_point_stride(b);
  a.ep_n = static_cast<const T*>(b.plastic_strain_n);
  a.q_n = b.eqps_n;
  a.vpm_n = b.vpm_n;
  a.ep = static_cast<T*>(b.plastic_strain);
  a.q = b.eqps;
  a.vpm = b.vpm;
  a.stress = static_cast<T*>(b.stress);
  a.tparam = static_cast<T*>(b.tparam);
  a.tflag = b.tflag;
  a.fe = b.fe;
  a.de = b.de;
  a.dt = dt;
  a.fail = fail;
  return a;
}

inline RveGatherArgs rve_gather_args(const cib_rve_batch& b, const double* w, const double* dw, const double* alpha,
                                     const int32_t* active, double* residual, double* dinv, double* rnorm2,
                                     double* wnorm2, double* class_max, double* w_out) {
  RveGatherArgs a;
  a.desc = reinterpret_cast<const RveDesc*>(b.desc);
  a.nrve = b.nrve;
  a.nelem = b.nelem;
  a.fe = b.fe;
  a.de = b.de;
  a.w = w;
  a.dw = dw;
  a.alpha = alpha;
  a.active = active;
  a.res = residual;
  a.dinv = dinv;
  a.rnorm2 = rnorm2;
  a.wnorm2 = wnorm2;
  a.class_max = class_max;
  a.w_out = w_out;
  return a;
}

template <typename T>
inline RvePcgArgs<T> rve_pcg_args(const cib_rve_batch& b, const int32_t* sys_rve, const int64_t* sys_off,
                                  const int32_t* active, const double* rhs, const double* dinv, double* x, double* r,
                                  double* p, double* Ap, double rtol, int32_t maxit, int32_t* status,
                                  int32_t* iterations, double* rel, double* xnorm) {
  RvePcgArgs<T> a;
  a.desc = reinterpret_cast<const RveDesc*>(b.desc);
  a.phase = b.phase;
  a.mats = rve_phase_table<T>(b);
  a.ngp = rve_point_stride(b);
  a.tparam = static_cast<const T*>(b.tparam);
  a.tflag = b.tflag;
  a.sys_rve = sys_rve;
  a.sys_off = sys_off;
  a.active = active;
  a.b = rhs;
  a.dinv = dinv;
  a.x = x;
  a.r = r;
  a.p = p;
  a.Ap = Ap;
  a.rtol = rtol;
  a.maxit = maxit;
  a.status = status;
  a.iterations = iterations;
  a.rel_residual = rel;
  a.xnorm = xnorm;
  return a;
}

// RVE owning batch element (or periodic node) e: the last r with desc[r].eoff <= e (RVEs
// are stored in element order).  A binary search over the descriptors, which stay in L1.
__device__ __forceinline__ int rve_of_element(const RveDesc* __restrict__ desc, int nrve, int64_t e) {
  int lo = 0, hi = nrve - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&desc[mid].eoff) <= e)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <typename T>
int launch_rve_residual(const RveResidualArgs<T>& a, int nrve, cudaStream_t st);
int launch_rve_gather(const RveGatherArgs& a, int nrve, cudaStream_t st);
template <typename T>
int launch_rve_pcg(const RvePcgArgs<T>& a, int nsys, int max_nxy, cudaStream_t st);
template <typename T>
int launch_rve_pcg_cluster(const RvePcgArgs<T>& a, int nsys, int max_nxy, int cluster, cudaStream_t st);
template <typename T>
int launch_rve_tangent_rhs(const RveTangentArgs<T>& a, int nrve, cudaStream_t st);
int launch_rve_tangent_finish(const RveTangentFinishArgs& a, int nrve, cudaStream_t st);
template <typename T>
int launch_rve_response(const RveResponseArgs<T>& a, int nrve, cudaStream_t st);

}  // namespace cib
