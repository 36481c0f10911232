// Device-controlled batched Newton solve of periodic RVEs, as one CUDA graph per step.
//
// Restates the Newton iteration of the reference's solve_rve_microequilibrium
// (src/fem/rve/solver.py:62-227, without the Armijo search) for a whole batch of RVEs with
// the decisions on the device.  Each iteration is the body of a conditional WHILE graph
// node:
//   residual pass (strains, return map, element forces)  -> rve_residual_kernel
//   periodic gather and norms                            -> rve_gather_nodes/norms_kernel
//   convergence check                                    -> newton_check_kernel
//   PCG on the live RVEs (tolerance read on the device)  -> rve_pcg(_cluster)_kernel
//   increment check and step                             -> newton_update_kernel
//   w <- w - dw on the live RVEs                         -> newton_axpy_kernel
// newton_update_kernel sets the loop condition, so the host enqueues one graph per step and
// reads nothing until the step is over.  The tests and their order are the host driver's
// (rve.py::solve_batch_step): a material failure among the unconverged RVEs stops the
// solve; an RVE converges when ||r|| <= tol and (first iteration or its last increment
// <= the increment tolerance), or when ||r|| <= tol and its new increment <= the increment
// tolerance; an unconverged RVE at the iteration limit stops the solve; a PCG breakdown or
// a non-finite increment stops it.  The Eisenstat-Walker forcing (gamma 0.9, alpha 2, with
// its safeguard, at most 0.1) takes the largest residual ratio over the live RVEs.
// The control kernels are single CTAs looping over the RVEs; their reductions (max, min,
// count) are order-independent, so every run takes the same decisions.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <new>

#include "cib_common.cuh"
#include "rve.cuh"

namespace cib {
namespace {

constexpr int NW_THREADS = 256;
constexpr int CTL = 16;  // leading control words of iwork and dwork
constexpr int IW_ITER = 0, IW_ERROR = 1, IW_ERR_RVE = 2, IW_ERR_INFO = 3, IW_LIVE = 4;
constexpr int DW_ETA = 0, DW_RTOL = 1;
constexpr int NEWTON_MATERIAL = 1, NEWTON_NONFINITE_INCREMENT = 2, NEWTON_MAX_ITERATIONS = 3;
constexpr unsigned long long NO_FAILURE = ~0ull;

struct NewtonArgs {
  int nrve;
  int64_t nelem;
  const RveDesc* desc;
  cib_rve_newton s;
  cudaGraphConditionalHandle cond;
};

// Per-RVE slices of the workspace (layout documented in include/cib200.h).
struct NewtonView {
  int32_t *its, *pcg, *done;
  double *rnorm, *tol, *inc, *inc_tol, *init, *last_inc, *prev;
};

__device__ __forceinline__ NewtonView newton_view(const NewtonArgs& a) {
  const int R = a.nrve;
  NewtonView v;
  v.its = a.s.iwork + CTL;
  v.pcg = v.its + R;
  v.done = v.pcg + R;
  v.rnorm = a.s.dwork + CTL;
  v.tol = v.rnorm + R;
  v.inc = v.tol + R;
  v.inc_tol = v.inc + R;
  v.init = v.inc_tol + R;
  v.last_inc = v.init + R;
  v.prev = v.last_inc + R;
  return v;
}

// CTA-wide min / max / sum (order-independent results).
__device__ int cta_min_int(int v, int* sh) {
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  int r = INT_MAX;
  for (int k = 0; k < nw; ++k) r = min(r, sh[k]);
  __syncthreads();
  return r;
}

__device__ int cta_sum_int(int v, int* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  int r = 0;
  for (int k = 0; k < nw; ++k) r += sh[k];
  __syncthreads();
  return r;
}

__device__ double cta_max_double(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = -INFINITY;
  for (int k = 0; k < nw; ++k) r = fmax(r, sh[k]);
  __syncthreads();
  return r;
}

// Before the loop: the live set, fresh per-RVE records, no recorded failure.
__global__ void __launch_bounds__(NW_THREADS) newton_init_kernel(const NewtonArgs a) {
  const NewtonView v = newton_view(a);
  for (int r = threadIdx.x; r < a.nrve; r += blockDim.x) {
    const int live = a.s.live_mask ? (a.s.live_mask[r] != 0) : 1;
    v.done[r] = !live;
    a.s.active[r] = live;
    v.its[r] = 0;
    v.pcg[r] = 0;
    v.rnorm[r] = v.tol[r] = v.inc[r] = v.inc_tol[r] = 0.0;
    v.init[r] = NAN;
    v.last_inc[r] = INFINITY;
    v.prev[r] = NAN;
    a.s.fail[r] = NO_FAILURE;
  }
  if (threadIdx.x < CTL) {
    a.s.iwork[threadIdx.x] = 0;
    a.s.dwork[threadIdx.x] = 0.0;
  }
  if (threadIdx.x == 0) {
    a.s.dwork[DW_ETA] = 0.1;
    a.s.dwork[DW_RTOL] = a.s.pcg_rtol;
  }
}

// After the residual pass and gather of iteration it.
__global__ void __launch_bounds__(NW_THREADS) newton_check_kernel(const NewtonArgs a) {
  __shared__ int ish[32];
  __shared__ double dsh[32];
  const NewtonView v = newton_view(a);
  const cib_rve_newton& s = a.s;
  const int it = s.iwork[IW_ITER];
  if (s.iwork[IW_ERROR] != 0) return;
  // material failures among the unconverged RVEs come first (the lowest RVE is reported)
  int fail_r = INT_MAX;
  unsigned long long fail_point = 0;
  for (int r = threadIdx.x; r < a.nrve; r += blockDim.x) {
    const unsigned long long f = s.fail[r];
    if (!v.done[r] && f != NO_FAILURE && r < fail_r) {
      fail_r = r;
      fail_point = f;
    }
    s.fail[r] = NO_FAILURE;  // for the next residual pass
  }
  const int first_fail = cta_min_int(fail_r, ish);
  if (first_fail != INT_MAX) {
    if (fail_r == first_fail) {
      s.iwork[IW_ERROR] = NEWTON_MATERIAL;
      s.iwork[IW_ERR_RVE] = first_fail;
      s.iwork[IW_ERR_INFO] = (int)fail_point;
    }
    for (int r = threadIdx.x; r < a.nrve; r += blockDim.x) s.active[r] = 0;
    return;
  }
  int maxit_r = INT_MAX, live = 0;
  double ratio = -INFINITY;
  for (int r = threadIdx.x; r < a.nrve; r += blockDim.x) {
    if (v.done[r]) {
      s.active[r] = 0;
      continue;
    }
    const double rn = sqrt(s.rnorm2[r]);
    if (isnan(v.init[r])) v.init[r] = rn;
    const double tol = fmax(s.residual_absolute_tolerance, s.residual_relative_tolerance * v.init[r]);
    const double inc_tol =
        fmax(s.increment_absolute_tolerance, s.increment_relative_tolerance * fmax(sqrt(s.wnorm2[r]), 1.0));
    v.rnorm[r] = rn;
    v.tol[r] = tol;
    v.inc_tol[r] = inc_tol;
    if (rn <= tol && (it == 0 || v.last_inc[r] <= inc_tol)) {
      v.done[r] = 1;
      v.its[r] = it;
      s.active[r] = 0;
      continue;
    }
    if (it == s.max_iterations) maxit_r = min(maxit_r, r);
    const double pr = v.prev[r];
    if (isfinite(pr) && pr > 0.0) ratio = fmax(ratio, rn / pr);
    v.prev[r] = rn;
    s.active[r] = 1;
    ++live;
  }
  const int first_maxit = cta_min_int(maxit_r, ish);
  const double ratio_max = cta_max_double(ratio, dsh);
  live = cta_sum_int(live, ish);
  if (first_maxit != INT_MAX) {
    if (threadIdx.x == 0) {
      s.iwork[IW_ERROR] = NEWTON_MAX_ITERATIONS;
      s.iwork[IW_ERR_RVE] = first_maxit;
    }
    for (int r = threadIdx.x; r < a.nrve; r += blockDim.x) s.active[r] = 0;
    return;
  }
  if (threadIdx.x == 0) {
    s.iwork[IW_LIVE] = live;
    double eta = s.dwork[DW_ETA];
    if (s.inexact && ratio_max > -INFINITY) {
      double next = 0.9 * ratio_max * ratio_max;
      if (0.9 * eta * eta > 0.1) next = fmax(next, 0.9 * eta * eta);
      eta = fmin(next, 0.1);
      s.dwork[DW_ETA] = eta;
    }
    s.dwork[DW_RTOL] = s.inexact ? fmax(s.pcg_rtol, eta) : s.pcg_rtol;
  }
}

// After the PCG: increment checks, the step size of every live RVE, the loop condition.
__global__ void __launch_bounds__(NW_THREADS) newton_update_kernel(const NewtonArgs a) {
  __shared__ int ish[32];
  const NewtonView v = newton_view(a);
  const cib_rve_newton& s = a.s;
  const int it = s.iwork[IW_ITER];
  int bad_r = INT_MAX, bad_status = 0;
  if (s.iwork[IW_ERROR] == 0) {
    for (int r = threadIdx.x; r < a.nrve; r += blockDim.x) {
      if (!s.active[r]) continue;
      const double xn = s.pcg_xnorm[r];
      v.pcg[r] += s.pcg_iterations[r];
      v.inc[r] = xn;
      if ((s.pcg_status[r] == 2 || !isfinite(xn)) && r < bad_r) {
        bad_r = r;
        bad_status = s.pcg_status[r];
      }
    }
  }
  const int first_bad = cta_min_int(bad_r, ish);
  int live = 0;
  if (first_bad != INT_MAX) {
    if (bad_r == first_bad) {
      s.iwork[IW_ERROR] = NEWTON_NONFINITE_INCREMENT;
      s.iwork[IW_ERR_RVE] = first_bad;
      s.iwork[IW_ERR_INFO] = bad_status;
    }
  }
  __syncthreads();
  const bool stop = s.iwork[IW_ERROR] != 0;
  for (int r = threadIdx.x; r < a.nrve; r += blockDim.x) {
    if (stop || !s.active[r]) {
      s.active[r] = 0;
      s.alpha[r] = 0.0;
      continue;
    }
    if (v.rnorm[r] <= v.tol[r] && v.inc[r] <= v.inc_tol[r]) {  // converged on the unapplied increment
      v.done[r] = 1;
      v.its[r] = it;
      s.active[r] = 0;
      s.alpha[r] = 0.0;
      continue;
    }
    s.alpha[r] = -1.0;  // w <- w - dw (the PCG solved K dw = r)
    v.last_inc[r] = 1.0 * v.inc[r];
    ++live;
  }
  live = cta_sum_int(live, ish);
  if (threadIdx.x == 0) {
    s.iwork[IW_ITER] = it + 1;
    cudaGraphSetConditional(a.cond, (!stop && live > 0) ? 1u : 0u);
  }
}

// w <- w + alpha x on the periodic nodes of the active RVEs (class 0 stays zero).
__global__ void __launch_bounds__(NW_THREADS) newton_axpy_kernel(const NewtonArgs a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; node < a.nelem; node += stride) {
    const int r = rve_of_element(a.desc, a.nrve, node);
    if (!a.s.active[r]) continue;
    const int64_t c = node - a.desc[r].eoff;
    const double al = a.s.alpha[r];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double v = a.s.w[3 * node + d];
      v += al * a.s.x[3 * node + d];
      a.s.w[3 * node + d] = (c == 0) ? 0.0 : v;
    }
  }
}

// After the loop: the live set is the active set again (the response and tangent passes).
__global__ void __launch_bounds__(NW_THREADS) newton_finish_kernel(const NewtonArgs a) {
  for (int r = threadIdx.x; r < a.nrve; r += blockDim.x) a.s.active[r] = a.s.live_mask ? (a.s.live_mask[r] != 0) : 1;
}

struct NewtonGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

#define CIB_TRY(expr)                      \
  do {                                     \
    const cudaError_t e_ = (expr);         \
    if (e_ != cudaSuccess) {               \
      last_cuda_error_slot() = (int)e_;    \
      return CIB_ECUDA;                    \
    }                                      \
  } while (0)

template <typename T>
int capture_body(const cib_rve_batch& b, const NewtonArgs& a, cudaStream_t st) {
  const cib_rve_newton& s = a.s;
  int rc = launch_rve_residual<T>(
      rve_residual_args<T>(b, s.time_step, s.macro, s.w, nullptr, nullptr, s.active, s.fail), b.nrve, st);
  if (rc != CIB_OK) return rc;
  rc = launch_rve_gather(
      rve_gather_args(b, s.w, nullptr, nullptr, s.active, s.residual, s.dinv, s.rnorm2, s.wnorm2, s.class_max, s.w_out),
      b.nrve, st);
  if (rc != CIB_OK) return rc;
  newton_check_kernel<<<1, NW_THREADS, 0, st>>>(a);
  if ((rc = check_launch()) != CIB_OK) return rc;
  RvePcgArgs<T> pa = rve_pcg_args<T>(b, s.sys_rve, s.sys_off, s.active, s.residual, s.dinv, s.x, s.r, s.p, s.Ap,
                                     s.pcg_rtol, s.pcg_maxit, s.pcg_status, s.pcg_iterations, s.pcg_rel_residual,
                                     s.pcg_xnorm);
  pa.rtol_dev = s.dwork + DW_RTOL;
  rc = launch_rve_pcg_cluster<T>(pa, b.nrve, b.max_nxy, s.cluster, st);
  if (rc != CIB_OK) return rc;
  newton_update_kernel<<<1, NW_THREADS, 0, st>>>(a);
  if ((rc = check_launch()) != CIB_OK) return rc;
  const int grid = persistent_grid(reinterpret_cast<const void*>(newton_axpy_kernel), NW_THREADS, b.nelem);
  newton_axpy_kernel<<<grid, NW_THREADS, 0, st>>>(a);
  return check_launch();
}

int add_kernel_node(cudaGraphNode_t* node, cudaGraph_t g, const cudaGraphNode_t* dep, size_t ndep, void* fn,
                    const NewtonArgs* args) {
  void* params[1] = {const_cast<NewtonArgs*>(args)};
  cudaKernelNodeParams kp = {};
  kp.func = fn;
  kp.gridDim = dim3(1, 1, 1);
  kp.blockDim = dim3(NW_THREADS, 1, 1);
  kp.sharedMemBytes = 0;
  kp.kernelParams = params;
  kp.extra = nullptr;
  CIB_TRY(cudaGraphAddKernelNode(node, g, dep, ndep, &kp));
  return CIB_OK;
}

int build_graph(const cib_rve_batch& b, const cib_rve_newton& s, NewtonGraph& out) {
  NewtonArgs a;
  a.nrve = b.nrve;
  a.nelem = b.nelem;
  a.desc = reinterpret_cast<const RveDesc*>(b.desc);
  a.s = s;
  cudaGraph_t g = nullptr;
  CIB_TRY(cudaGraphCreate(&g, 0));
  out.graph = g;
  CIB_TRY(cudaGraphConditionalHandleCreate(&a.cond, g, 1u, cudaGraphCondAssignDefault));
  // w = w_n for every RVE (the solve starts from the committed fluctuation), then the
  // per-RVE records
  cudaGraphNode_t copy = nullptr, init = nullptr, loop = nullptr, finish = nullptr;
  CIB_TRY(cudaGraphAddMemcpyNode1D(&copy, g, nullptr, 0, s.w, s.w_n, (size_t)(3 * b.nelem) * sizeof(double),
                                   cudaMemcpyDeviceToDevice));
  int rc = add_kernel_node(&init, g, &copy, 1, reinterpret_cast<void*>(newton_init_kernel), &a);
  if (rc != CIB_OK) return rc;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = a.cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  CIB_TRY(cudaGraphAddNode(&loop, g, &init, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaStream_t st = nullptr;
  CIB_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    rc = b.precision == 64 ? capture_body<double>(b, a, st) : capture_body<float>(b, a, st);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(st, &captured);
  }
  cudaStreamDestroy(st);
  if (rc != CIB_OK) return rc;
  CIB_TRY(e);
  rc = add_kernel_node(&finish, g, &loop, 1, reinterpret_cast<void*>(newton_finish_kernel), &a);
  if (rc != CIB_OK) return rc;
  CIB_TRY(cudaGraphInstantiate(&out.exec, g, 0));
  return CIB_OK;
}

void destroy_graph(NewtonGraph* h) {
  if (!h) return;
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  delete h;
}

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" void cib_rve_newton_workspace(int32_t nrve, int64_t* n_int, int64_t* n_double) {
  const int64_t R = nrve > 0 ? nrve : 0;
  if (n_int) *n_int = CTL + 3 * R;
  if (n_double) *n_double = CTL + 7 * R;
}

extern "C" int cib_rve_newton_graph_create(const cib_rve_batch* batch, const cib_rve_newton* s, void** graph) {
  if (!graph) return CIB_EINVAL;
  *graph = nullptr;
  if (!batch || batch->nrve < 1 || batch->nelem < 1 || batch->nphase < 1 || batch->nphase > RVE_MAX_PHASES ||
      !batch->desc || !batch->phase || (batch->precision != 32 && batch->precision != 64) || batch->max_nxy <= 0 ||
      !batch->plastic_strain_n || !batch->eqps_n || !batch->vpm_n || !batch->plastic_strain || !batch->eqps ||
      !batch->vpm || !batch->stress || !batch->tparam || !batch->tflag || !batch->fe || !batch->de)
    return CIB_EINVAL;
  if (!s || s->max_iterations < 0 || s->pcg_maxit < 0 ||
      s->cluster < 0 || (s->cluster >> 8) != 0 || ((s->cluster >> 4) & 15) > 3 ||
      ((s->cluster & 15) != 1 && (s->cluster & 15) != 2 && (s->cluster & 15) != 4 && (s->cluster & 15) != 8) ||
      !s->time_step || !s->macro ||
      !s->w_n || !s->w || !s->w_out || !s->x || !s->r || !s->p || !s->Ap || !s->residual || !s->dinv || !s->rnorm2 ||
      !s->wnorm2 || !s->class_max || !s->alpha || !s->active || !s->fail || !s->sys_rve || !s->sys_off ||
      !s->pcg_status || !s->pcg_iterations || !s->pcg_rel_residual || !s->pcg_xnorm || !s->iwork || !s->dwork)
    return CIB_EINVAL;
  NewtonGraph* h = new (std::nothrow) NewtonGraph();
  if (!h) return CIB_ECUDA;
  const int rc = build_graph(*batch, *s, *h);
  if (rc != CIB_OK) {
    destroy_graph(h);
    return rc;
  }
  *graph = h;
  return CIB_OK;
}

extern "C" int cib_rve_newton_graph_launch(void* graph, void* stream) {
  if (!graph) return CIB_EINVAL;
  const NewtonGraph* h = static_cast<NewtonGraph*>(graph);
  const cudaError_t e = cudaGraphLaunch(h->exec, reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    last_cuda_error_slot() = (int)e;
    return CIB_ECUDA;
  }
  return CIB_OK;
}

extern "C" int cib_rve_newton_graph_destroy(void* graph) {
  destroy_graph(static_cast<NewtonGraph*>(graph));
  return CIB_OK;
}
