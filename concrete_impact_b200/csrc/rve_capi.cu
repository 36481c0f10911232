// extern "C" entry points of the periodic RVE kernels (declared in include/cib200.h).
#include <cuda_runtime.h>

#include "cib_common.cuh"
#include "rve.cuh"

namespace cib {
namespace {

// CTAs per system (1, 2, 4, 8) in bits 0-3, launch shape (0-3) in bits 4-7.
bool pcg_cluster_ok(int32_t cluster) {
  const int c = cluster & 15;
  return cluster >= 0 && (cluster >> 8) == 0 && ((cluster >> 4) & 15) <= 3 && (c == 1 || c == 2 || c == 4 || c == 8);
}

bool batch_ok(const cib_rve_batch* b) {
  return b && b->nrve >= 0 && b->nphase >= 1 && b->nphase <= RVE_MAX_PHASES && b->nelem >= 0 && b->desc &&
         b->phase && (b->precision == 32 || b->precision == 64);
}

template <typename T>
int residual_t(const cib_rve_batch& b, const double* dt, const double* macro, const double* w, const double* dw,
               const double* alpha, const int32_t* active, unsigned long long* fail, cudaStream_t st) {
  return launch_rve_residual<T>(rve_residual_args<T>(b, dt, macro, w, dw, alpha, active, fail), b.nrve, st);
}

template <typename T>
int pcg_t(const cib_rve_batch& b, int32_t nsys, const int32_t* sys_rve, const int64_t* sys_off, const int32_t* active,
          const double* rhs, const double* dinv, double* x, double* r, double* p, double* Ap, double rtol,
          int32_t maxit, int32_t* status, int32_t* iterations, double* rel, double* xnorm, cudaStream_t st,
          int32_t cluster = 1) {
  const RvePcgArgs<T> a = rve_pcg_args<T>(b, sys_rve, sys_off, active, rhs, dinv, x, r, p, Ap, rtol, maxit, status,
                                          iterations, rel, xnorm);
  return launch_rve_pcg_cluster<T>(a, nsys, b.max_nxy, cluster, st);
}

template <typename T>
int tangent_rhs_t(const cib_rve_batch& b, const int32_t* active, double* fe6, double* rhs, double* kee,
                  cudaStream_t st) {
  RveTangentArgs<T> a;
  a.desc = reinterpret_cast<const RveDesc*>(b.desc);
  a.phase = b.phase;
  a.mats = rve_phase_table<T>(b);
  a.ngp = rve_point_stride(b);
  a.ne_total = rve_point_stride(b) / 8;
  a.tparam = static_cast<const T*>(b.tparam);
  a.tflag = b.tflag;
  a.active = active;
  a.fe6 = fe6;
  a.rhs = rhs;
  a.kee = kee;
  return launch_rve_tangent_rhs<T>(a, b.nrve, st);
}

template <typename T>
int response_t(const cib_rve_batch& b, const double* dt, const double* macro, const double* macro_n, const double* w,
               const double* w_n, const int32_t* active, double* sums, double* point_out, double* diag,
               cudaStream_t st) {
  RveResponseArgs<T> a;
  a.desc = reinterpret_cast<const RveDesc*>(b.desc);
  a.phase = b.phase;
  a.mats = rve_phase_table<double>(b);
  a.mats_t = rve_phase_table<T>(b);
  a.macro = macro;
  a.macro_n = macro_n;
  a.w = w;
  a.w_n = w_n;
  a.active = active;
  a.ngp = rve_point_stride(b);
  a.ep_n = static_cast<const T*>(b.plastic_strain_n);
  a.q_n = b.eqps_n;
  a.ep = static_cast<const T*>(b.plastic_strain);
  a.q = b.eqps;
  a.stress = static_cast<const T*>(b.stress);
  a.tflag = b.tflag;
  a.fe = b.fe;
  a.dt = dt;
  a.sums = sums;
  a.point_out = point_out;
  a.diag = diag;
  return launch_rve_response<T>(a, b.nrve, st);
}

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" int cib_rve_residual(const cib_rve_batch* batch, const double* time_step, const double* macro, const double* w,
                                const double* dw, const double* alpha, const int32_t* active,
                                unsigned long long* fail, void* stream) {
  if (!batch_ok(batch) || !macro || !w || !batch->plastic_strain_n || !batch->eqps_n || !batch->vpm_n ||
      !batch->plastic_strain || !batch->eqps || !batch->vpm || !batch->stress || !batch->tparam || !batch->tflag ||
      !batch->fe || !batch->de || !time_step)
    return CIB_EINVAL;
  if (batch->nrve == 0) return CIB_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return batch->precision == 64 ? residual_t<double>(*batch, time_step, macro, w, dw, alpha, active, fail, st)
                                : residual_t<float>(*batch, time_step, macro, w, dw, alpha, active, fail, st);
}

extern "C" int cib_rve_gather(const cib_rve_batch* batch, const double* w, const double* dw, const double* alpha,
                              const int32_t* active, double* residual, double* dinv, double* rnorm2,
                              double* wnorm2, double* class_max, double* w_out, void* stream) {
  if (!batch_ok(batch) || !w || !residual || !dinv || !rnorm2 || !batch->fe || !batch->de) return CIB_EINVAL;
  if (batch->nrve == 0) return CIB_OK;
  const RveGatherArgs a = rve_gather_args(*batch, w, dw, alpha, active, residual, dinv, rnorm2, wnorm2, class_max,
                                          w_out);
  return launch_rve_gather(a, batch->nrve, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int cib_rve_pcg(const cib_rve_batch* batch, int32_t nsys, const int32_t* sys_rve, const int64_t* sys_off,
                           const int32_t* active, const double* b, const double* dinv, double* x, double* r, double* p,
                           double* Ap, double rtol, int32_t maxit, int32_t* status, int32_t* iterations,
                           double* rel_residual, double* xnorm, void* stream) {
  if (!batch_ok(batch) || nsys < 0 || !sys_rve || !sys_off || !b || !dinv || !x || !r || !p || !Ap || !status ||
      !iterations || !rel_residual || !xnorm || maxit < 0 || !batch->tparam || !batch->tflag || batch->max_nxy <= 0)
    return CIB_EINVAL;
  if (nsys == 0) return CIB_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return batch->precision == 64
             ? pcg_t<double>(*batch, nsys, sys_rve, sys_off, active, b, dinv, x, r, p, Ap, rtol, maxit, status,
                             iterations, rel_residual, xnorm, st)
             : pcg_t<float>(*batch, nsys, sys_rve, sys_off, active, b, dinv, x, r, p, Ap, rtol, maxit, status,
                            iterations, rel_residual, xnorm, st);
}

extern "C" int cib_rve_pcg_cluster(const cib_rve_batch* batch, int32_t nsys, const int32_t* sys_rve,
                                   const int64_t* sys_off, const int32_t* active, const double* b, const double* dinv,
                                   double* x, double* r, double* p, double* Ap, double rtol, int32_t maxit,
                                   int32_t cluster, int32_t* status, int32_t* iterations, double* rel_residual,
                                   double* xnorm, void* stream) {
  if (!batch_ok(batch) || nsys < 0 || !sys_rve || !sys_off || !b || !dinv || !x || !r || !p || !Ap || !status ||
      !iterations || !rel_residual || !xnorm || maxit < 0 || !batch->tparam || !batch->tflag || batch->max_nxy <= 0 ||
      !pcg_cluster_ok(cluster))
    return CIB_EINVAL;
  if (nsys == 0) return CIB_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return batch->precision == 64
             ? pcg_t<double>(*batch, nsys, sys_rve, sys_off, active, b, dinv, x, r, p, Ap, rtol, maxit, status,
                             iterations, rel_residual, xnorm, st, cluster)
             : pcg_t<float>(*batch, nsys, sys_rve, sys_off, active, b, dinv, x, r, p, Ap, rtol, maxit, status,
                            iterations, rel_residual, xnorm, st, cluster);
}

extern "C" int cib_rve_tangent_rhs(const cib_rve_batch* batch, const int32_t* active, double* fe6, double* rhs,
                                   double* kee, void* stream) {
  if (!batch_ok(batch) || !fe6 || !rhs || !kee || !batch->tparam || !batch->tflag) return CIB_EINVAL;
  if (batch->nrve == 0) return CIB_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return batch->precision == 64 ? tangent_rhs_t<double>(*batch, active, fe6, rhs, kee, st)
                                : tangent_rhs_t<float>(*batch, active, fe6, rhs, kee, st);
}

extern "C" int cib_rve_tangent_finish(const cib_rve_batch* batch, const int32_t* active, const double* rhs,
                                      const double* sol, const double* kee, double* ceff, void* stream) {
  if (!batch_ok(batch) || !rhs || !sol || !kee || !ceff) return CIB_EINVAL;
  if (batch->nrve == 0) return CIB_OK;
  RveTangentFinishArgs a;
  a.desc = reinterpret_cast<const RveDesc*>(batch->desc);
  a.active = active;
  a.rhs = rhs;
  a.sol = sol;
  a.kee = kee;
  a.ceff = ceff;
  return launch_rve_tangent_finish(a, batch->nrve, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int cib_rve_response(const cib_rve_batch* batch, const double* time_step, const double* macro,
                                const double* macro_n, const double* w, const double* w_n, const int32_t* active,
                                double* sums, double* point_out, double* diagnostics, void* stream) {
  if (!batch_ok(batch) || !macro || !macro_n || !w || !w_n || !sums || !batch->stress || !batch->fe || !time_step)
    return CIB_EINVAL;
  if (batch->nrve == 0) return CIB_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return batch->precision == 64
             ? response_t<double>(*batch, time_step, macro, macro_n, w, w_n, active, sums, point_out, diagnostics, st)
             : response_t<float>(*batch, time_step, macro, macro_n, w, w_n, active, sums, point_out, diagnostics, st);
}
