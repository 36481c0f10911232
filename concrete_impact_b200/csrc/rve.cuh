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
