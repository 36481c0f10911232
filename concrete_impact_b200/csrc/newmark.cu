// Implicit Newmark macro dynamics on the GPU, sm_100a.
//
// The device side of the reference's implicit Newmark step
//   solve_material_implicit_newmark / _solve_implicit_step / _evaluate_implicit_trial
//   (src/fem/dynamics/material.py:300-701)
// on the CSR pattern of the Hex8 tangent (the consistent mass shares it, see
// cib_hex8_mass_csr):
//   * Newmark kinematics   a = (u - u_pred) / (beta dt^2),  v = v_pred + (gamma dt) a
//   * residual             r = (M a + f_int) - f_ext on the free DOFs, 0 on the fixed ones
//   * effective tangent    K + M / (beta dt^2) and its Jacobi inverse diagonal
//   * a Jacobi-preconditioned conjugate gradient on the free DOFs in place of the
//     reference's sparse direct solve (src/fem/solvers/linear.py:15).
//
// CSR rows are handled one warp per row (a Hex8 row has at most 81 entries, so the lanes
// read contiguous values and column indices).  The CG runs as three kernels per iteration
// (matrix product + p.q partials; x, r, z update + r.z and r.r partials; new direction).
// Every dot product is reduced in a fixed order: one partial per block, then each block
// of the next kernel sums all partials in the same order, so every block holds the same
// scalar and results are bitwise repeatable.  The iteration count is bounded by `maxit`;
// the host reads the device status every `check_every` iterations, and kernels launched
// after convergence return at once.  Nothing waits on another block.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "cib_common.cuh"

namespace cib {
namespace {

constexpr int NM_THREADS = 256;
constexpr int NM_WARPS = NM_THREADS / 32;
constexpr unsigned NM_FULL = 0xffffffffu;

// Work buffer layout (doubles), CIB_CSR_PCG_WORK_DOUBLES in total.
constexpr int PCG_MAX_GRID = CIB_CSR_PCG_MAX_GRID;
constexpr int PART_PQ = 0;                      // [PCG_MAX_GRID]
constexpr int PART_RZ = PCG_MAX_GRID;           // [2 * PCG_MAX_GRID] (r.z, r.r) per block
constexpr int ST = 3 * PCG_MAX_GRID;            // scalars:
constexpr int ST_STATUS = ST + 0;               //   0 running, 1 converged, 2 breakdown
constexpr int ST_ITER = ST + 1;                 //   iterations done
constexpr int ST_REL = ST + 2;                  //   ||r|| / ||b||
constexpr int ST_BNORM = ST + 3;                //   ||b|| (free DOFs)
constexpr int ST_RZ = ST + 4;                   //   r.z of the current direction, two slots
static_assert(ST_RZ + 2 <= CIB_CSR_PCG_WORK_DOUBLES, "work layout");

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(NM_FULL, v, o);
  return v;
}

// Block sum with a fixed order: warps reduce, then thread 0 adds the warp sums in warp
// order.  The result is valid in thread 0 only.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();  // sh may still be read by a previous call
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < NM_WARPS; ++w) s += sh[w];
  return s;
}

// Ordered sum of partials part[k * stride] for k < count, broadcast to the whole block.
__device__ __forceinline__ double sum_partials(const double* part, int count, int stride, double* sh, double* bcast) {
  double v = 0.0;
  for (int k = threadIdx.x; k < count; k += NM_THREADS) v += part[(int64_t)k * stride];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) *bcast = v;
  __syncthreads();
  return *bcast;
}

// One read of the status per block (uniform early exit for the whole block).
__device__ __forceinline__ bool block_stopped(const double* work, int* flag) {
  if (threadIdx.x == 0) *flag = (*reinterpret_cast<const volatile double*>(work + ST_STATUS) != 0.0) ? 1 : 0;
  __syncthreads();
  return *flag != 0;
}

__global__ void __launch_bounds__(NM_THREADS) newmark_kinematics_kernel(int64_t n, const double* __restrict__ u,
                                                                       const double* __restrict__ u_pred,
                                                                       const double* __restrict__ v_pred,
                                                                       double beta_dt2, double gamma_dt,
                                                                       double* __restrict__ a, double* __restrict__ v) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double ai = (u[i] - u_pred[i]) / beta_dt2;
    a[i] = ai;
    v[i] = v_pred[i] + gamma_dt * ai;
  }
}

// r = (M a + f_int) - f_ext on free rows, 0 on fixed rows; one warp per row.
__global__ void __launch_bounds__(NM_THREADS) newmark_residual_kernel(
    int64_t n, const int64_t* __restrict__ indptr, const int64_t* __restrict__ indices, const double* __restrict__ mass,
    const double* __restrict__ a, const double* __restrict__ f_int, const double* __restrict__ f_ext,
    const uint8_t* __restrict__ free_mask, double* __restrict__ r) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * NM_WARPS;
  for (int64_t row = (int64_t)blockIdx.x * NM_WARPS + (threadIdx.x >> 5); row < n; row += nw) {
    double s = 0.0;
    for (int64_t k = indptr[row] + lane; k < indptr[row + 1]; k += 32) s += mass[k] * a[indices[k]];
    s = warp_sum(s);
    if (lane == 0) r[row] = free_mask[row] ? (s + f_int[row]) - f_ext[row] : 0.0;
  }
}

// out = k + m / beta_dt2 (k may be NULL: out = m / beta_dt2); dinv = 1 / diag on free rows
// (1 where the diagonal is not positive), 0 on fixed rows.
__global__ void __launch_bounds__(NM_THREADS) newmark_effective_kernel(
    int64_t n, const int64_t* __restrict__ indptr, const int64_t* __restrict__ indices, const double* __restrict__ k_values,
    const double* __restrict__ m_values, double beta_dt2, const uint8_t* __restrict__ free_mask,
    double* __restrict__ out, double* __restrict__ dinv) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * NM_WARPS;
  for (int64_t row = (int64_t)blockIdx.x * NM_WARPS + (threadIdx.x >> 5); row < n; row += nw) {
    double diag = 0.0;
    for (int64_t k = indptr[row] + lane; k < indptr[row + 1]; k += 32) {
      const double v = (k_values ? k_values[k] : 0.0) + m_values[k] / beta_dt2;
      out[k] = v;
      if (indices[k] == row) diag = v;
    }
    diag = warp_sum(diag);  // one lane holds the diagonal, the others add zeros
    if (lane == 0) dinv[row] = free_mask[row] ? (diag > 0.0 ? 1.0 / diag : 1.0) : 0.0;
  }
}

// y = A x (all rows); one warp per row.
__global__ void __launch_bounds__(NM_THREADS) csr_spmv_kernel(int64_t n, const int64_t* __restrict__ indptr,
                                                             const int64_t* __restrict__ indices,
                                                             const double* __restrict__ values,
                                                             const double* __restrict__ x, double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * NM_WARPS;
  for (int64_t row = (int64_t)blockIdx.x * NM_WARPS + (threadIdx.x >> 5); row < n; row += nw) {
    double s = 0.0;
    for (int64_t k = indptr[row] + lane; k < indptr[row + 1]; k += 32) s += values[k] * x[indices[k]];
    s = warp_sum(s);
    if (lane == 0) y[row] = s;
  }
}

// x = 0, r = b on free rows (0 on fixed), z = dinv r, p = z; partials of r.z and r.r.
__global__ void __launch_bounds__(NM_THREADS) pcg_init_kernel(int64_t n, const uint8_t* __restrict__ free_mask,
                                                             const double* __restrict__ dinv,
                                                             const double* __restrict__ b, double* __restrict__ x,
                                                             double* __restrict__ r, double* __restrict__ z,
                                                             double* __restrict__ p, double* __restrict__ work) {
  __shared__ double sh[NM_WARPS];
  double rz = 0.0, rr = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double ri = free_mask[i] ? b[i] : 0.0;
    const double zi = dinv[i] * ri;
    x[i] = 0.0;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  rz = block_sum(rz, sh);
  if (threadIdx.x == 0) work[PART_RZ + 2 * blockIdx.x] = rz;
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) work[PART_RZ + 2 * blockIdx.x + 1] = rr;
}

__global__ void __launch_bounds__(NM_THREADS) pcg_init_finish_kernel(double* __restrict__ work, int grid) {
  __shared__ double sh[NM_WARPS];
  __shared__ double bc;
  const double rz = sum_partials(work + PART_RZ, grid, 2, sh, &bc);
  const double rr = sum_partials(work + PART_RZ + 1, grid, 2, sh, &bc);
  if (threadIdx.x == 0) {
    work[ST_RZ] = rz;
    work[ST_RZ + 1] = rz;
    work[ST_BNORM] = sqrt(rr);
    work[ST_ITER] = 0.0;
    work[ST_REL] = rr > 0.0 ? 1.0 : 0.0;
    work[ST_STATUS] = !(isfinite(rz) && isfinite(rr)) ? 2.0 : (rr == 0.0 ? 1.0 : 0.0);
  }
}

// q = A p on free rows (0 on fixed); per-block partial of p.q.
__global__ void __launch_bounds__(NM_THREADS) pcg_spmv_kernel(int64_t n, const int64_t* __restrict__ indptr,
                                                             const int64_t* __restrict__ indices,
                                                             const double* __restrict__ values,
                                                             const uint8_t* __restrict__ free_mask,
                                                             const double* __restrict__ p, double* __restrict__ q,
                                                             double* __restrict__ work) {
  __shared__ double sh[NM_WARPS];
  __shared__ int stop;
  if (block_stopped(work, &stop)) return;
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * NM_WARPS;
  double acc = 0.0;
  for (int64_t row = (int64_t)blockIdx.x * NM_WARPS + (threadIdx.x >> 5); row < n; row += nw) {
    double s = 0.0;
    for (int64_t k = indptr[row] + lane; k < indptr[row + 1]; k += 32) s += values[k] * p[indices[k]];
    s = warp_sum(s);
    if (lane == 0) {
      const double qv = free_mask[row] ? s : 0.0;
      q[row] = qv;
      acc += p[row] * qv;
    }
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) work[PART_PQ + blockIdx.x] = acc;
}

// alpha = rz / pq; x += alpha p; r -= alpha q; z = dinv r; partials of r.z and r.r.
__global__ void __launch_bounds__(NM_THREADS) pcg_update_kernel(int64_t n, int it, int grid,
                                                               const double* __restrict__ dinv,
                                                               const double* __restrict__ p,
                                                               const double* __restrict__ q, double* __restrict__ x,
                                                               double* __restrict__ r, double* __restrict__ z,
                                                               double* __restrict__ work) {
  __shared__ double sh[NM_WARPS];
  __shared__ double bc;
  __shared__ int stop;
  if (block_stopped(work, &stop)) return;
  const double pq = sum_partials(work + PART_PQ, grid, 1, sh, &bc);
  if (!(pq > 0.0) || !isfinite(pq)) {  // every block sees the same pq
    if (blockIdx.x == 0 && threadIdx.x == 0) work[ST_STATUS] = 2.0;
    return;
  }
  const double alpha = work[ST_RZ + (it & 1)] / pq;
  double rz = 0.0, rr = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * q[i];
    const double zi = dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  rz = block_sum(rz, sh);
  if (threadIdx.x == 0) work[PART_RZ + 2 * blockIdx.x] = rz;
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) work[PART_RZ + 2 * blockIdx.x + 1] = rr;
}

// beta = rz_new / rz_old; p = z + beta p; block 0 records rz_new, the iteration count and
// the relative residual, and sets the status (converged when ||r|| <= rtol ||b||).
__global__ void __launch_bounds__(NM_THREADS) pcg_direction_kernel(int64_t n, int it, int grid, double rtol,
                                                                  const double* __restrict__ z, double* __restrict__ p,
                                                                  double* __restrict__ work) {
  __shared__ double sh[NM_WARPS];
  __shared__ double bc;
  __shared__ int stop;
  if (block_stopped(work, &stop)) return;
  const double rz = sum_partials(work + PART_RZ, grid, 2, sh, &bc);
  const double rr = sum_partials(work + PART_RZ + 1, grid, 2, sh, &bc);
  const double beta = rz / work[ST_RZ + (it & 1)];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = z[i] + beta * p[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    work[ST_RZ + ((it + 1) & 1)] = rz;
    work[ST_ITER] = (double)(it + 1);
    const double rel = sqrt(rr) / work[ST_BNORM];
    work[ST_REL] = rel;
    if (!(isfinite(rz) && isfinite(rr)))
      work[ST_STATUS] = 2.0;
    else if (rel <= rtol)
      work[ST_STATUS] = 1.0;
  }
}

inline int rows_grid(int64_t n) {
  const int64_t g = (n + NM_WARPS - 1) / NM_WARPS;
  const int64_t cap = 4 * (int64_t)sm_count();
  return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

inline int vec_grid(int64_t n) {
  const int64_t g = (n + NM_THREADS - 1) / NM_THREADS;
  const int64_t cap = 4 * (int64_t)sm_count();
  return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" int cib_newmark_kinematics(int64_t n, const double* u, const double* u_pred, const double* v_pred,
                                      double beta_dt2, double gamma_dt, double* a, double* v, void* stream) {
  if (n < 0 || !u || !u_pred || !v_pred || !a || !v || !(beta_dt2 > 0.0)) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  newmark_kinematics_kernel<<<vec_grid(n), NM_THREADS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      n, u, u_pred, v_pred, beta_dt2, gamma_dt, a, v);
  return check_launch();
}

extern "C" int cib_newmark_residual(int64_t n, const int64_t* indptr, const int64_t* indices, const double* mass,
                                    const double* a, const double* f_int, const double* f_ext,
                                    const uint8_t* free_mask, double* r, void* stream) {
  if (n < 0 || !indptr || !indices || !mass || !a || !f_int || !f_ext || !free_mask || !r) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  newmark_residual_kernel<<<rows_grid(n), NM_THREADS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      n, indptr, indices, mass, a, f_int, f_ext, free_mask, r);
  return check_launch();
}

extern "C" int cib_newmark_effective_tangent(int64_t n, const int64_t* indptr, const int64_t* indices,
                                             const double* k_values, const double* m_values, double beta_dt2,
                                             const uint8_t* free_mask, double* out, double* dinv, void* stream) {
  if (n < 0 || !indptr || !indices || !m_values || !free_mask || !out || !dinv || !(beta_dt2 > 0.0)) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  newmark_effective_kernel<<<rows_grid(n), NM_THREADS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      n, indptr, indices, k_values, m_values, beta_dt2, free_mask, out, dinv);
  return check_launch();
}

extern "C" int cib_csr_spmv(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values,
                            const double* x, double* y, void* stream) {
  if (n < 0 || !indptr || !indices || !values || !x || !y) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  csr_spmv_kernel<<<rows_grid(n), NM_THREADS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(n, indptr, indices, values,
                                                                                          x, y);
  return check_launch();
}

extern "C" int cib_csr_pcg(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values,
                           const uint8_t* free_mask, const double* dinv, const double* b, double* x, double* r,
                           double* z, double* p, double* q, double* work, double rtol, int32_t maxit,
                           int32_t check_every, int32_t* status, int32_t* iterations, double* relative_residual,
                           void* stream) {
  if (n <= 0 || !indptr || !indices || !values || !free_mask || !dinv || !b || !x || !r || !z || !p || !q || !work ||
      !status || !iterations || !relative_residual || maxit < 0 || check_every <= 0 || !(rtol >= 0.0))
    return CIB_EINVAL;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int g_rows = rows_grid(n), g_vec = vec_grid(n);
  if (g_rows > PCG_MAX_GRID || g_vec > PCG_MAX_GRID) return CIB_ERANGE;
  pcg_init_kernel<<<g_vec, NM_THREADS, 0, st>>>(n, free_mask, dinv, b, x, r, z, p, work);
  pcg_init_finish_kernel<<<1, NM_THREADS, 0, st>>>(work, g_vec);
  if (check_launch() != CIB_OK) return CIB_ECUDA;
  double host[3] = {0.0, 0.0, 0.0};  // status, iterations, relative residual
  int it = 0;
  for (;;) {
    if (cudaMemcpyAsync(host, work + ST_STATUS, sizeof(host), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      last_cuda_error_slot() = (int)cudaGetLastError();
      return CIB_ECUDA;
    }
    if (host[0] != 0.0 || it >= maxit) break;
    for (int c = 0; c < check_every && it < maxit; ++c, ++it) {
      pcg_spmv_kernel<<<g_rows, NM_THREADS, 0, st>>>(n, indptr, indices, values, free_mask, p, q, work);
      pcg_update_kernel<<<g_vec, NM_THREADS, 0, st>>>(n, it, g_rows, dinv, p, q, x, r, z, work);
      pcg_direction_kernel<<<g_vec, NM_THREADS, 0, st>>>(n, it, g_vec, rtol, z, p, work);
    }
    if (check_launch() != CIB_OK) return CIB_ECUDA;
  }
  *status = host[0] == 1.0 ? 0 : (host[0] == 2.0 ? 2 : 1);
  *iterations = (int32_t)host[1];
  *relative_residual = host[2];
  return CIB_OK;
}
