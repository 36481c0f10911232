// General Hex8 element kernels (arbitrary node coordinates and connectivity), sm_100a.
//
// Restates, for the GPU, the reference's
//   _build_hex8_quadrature_geometry   (src/fem/assembly/nonlinear_solid.py:391-425)
//   _compute_hex8_strain_fields       (:428-454)
//   _assemble_force_and_tangent       (:457-493)
//   assemble_consistent_mass_matrix   (src/fem/assembly/elasticity.py:50-70, 109-140)
// with the reference's conventions: lexicographic node signs (elements/lagrange.py:50-76),
// 2x2x2 Gauss points in itertools.product order (quadrature/rules.py:24-33), DOF 3 n + c,
// Voigt (xx, yy, zz, yz, xz, xy) with engineering shear (assembly/elasticity.py:160-183).
//
// Thread mapping: one thread per Gauss point; the 8 threads of an element share nodal
// values by warp shuffles and reduce-scatter their B^T sigma contributions.  Global
// assembly is deterministic: node forces and CSR values are gathered from precomputed
// contribution lists in a fixed order (no atomics).
#include <cuda_runtime.h>
#include <stdint.h>

#include "cib_common.cuh"

namespace cib {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int HEX_THREADS = 256;

__device__ __forceinline__ void ref_grad(int q, int a, double g[3]) {
  const double gp = 0.57735026918962576451;
  const double xi = (q & 4) ? gp : -gp, eta = (q & 2) ? gp : -gp, zeta = (q & 1) ? gp : -gp;
  const double sx = (a & 1) ? 1.0 : -1.0, sy = (a & 2) ? 1.0 : -1.0, sz = (a & 4) ? 1.0 : -1.0;
  const double fx = 1.0 + sx * xi, fy = 1.0 + sy * eta, fz = 1.0 + sz * zeta;
  g[0] = 0.125 * sx * fy * fz;
  g[1] = 0.125 * sy * fx * fz;
  g[2] = 0.125 * sz * fx * fy;
}

// Geometry: dN/dx for every (element, GP, node) and J*w; bad[0] counts det <= 0.
__global__ void __launch_bounds__(HEX_THREADS) hex8_geometry_kernel(int64_t ne, const double* __restrict__ nodes,
                                                                   const int64_t* __restrict__ elements,
                                                                   double* __restrict__ grads, double* __restrict__ jw,
                                                                   unsigned long long* bad) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 8 * ne) return;
  const int64_t e = t >> 3;
  const int q = (int)(t & 7);
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double gr[8][3];
  for (int a = 0; a < 8; ++a) {
    ref_grad(q, a, gr[a]);
    const int64_t n = elements[8 * e + a];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) J[i][j] += nodes[3 * n + i] * gr[a][j];  // X^T dN
  }
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  if (!(det > 0.0)) atomicAdd(bad, 1ull);
  double inv[3][3];
  const double id = 1.0 / det;
  inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  for (int a = 0; a < 8; ++a)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += gr[a][k] * inv[k][j];  // dN_ref @ inv(J)
      grads[((8 * e + q) * 8 + a) * 3 + j] = v;
    }
  jw[8 * e + q] = det;  // Gauss weights are 1 for the 2-point rule
}

__device__ __forceinline__ void load_grads(const double* __restrict__ grads, int64_t g, double G[8][3]) {
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int d = 0; d < 3; ++d) G[a][d] = grads[(g * 8 + a) * 3 + d];
}

__device__ __forceinline__ void strain_of(const double G[8][3], const double u[8][3], double e[6]) {
  double s[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    s[0] += G[a][0] * u[a][0];
    s[1] += G[a][1] * u[a][1];
    s[2] += G[a][2] * u[a][2];
    s[3] += G[a][2] * u[a][1] + G[a][1] * u[a][2];
    s[4] += G[a][2] * u[a][0] + G[a][0] * u[a][2];
    s[5] += G[a][1] * u[a][0] + G[a][0] * u[a][1];
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) e[c] = s[c];
}

__device__ __forceinline__ void gather8(const double mine[3], double u[8][3]) {
  const int base = (threadIdx.x & 31) & ~7;
#pragma unroll
  for (int b = 0; b < 8; ++b)
#pragma unroll
    for (int d = 0; d < 3; ++d) u[b][d] = __shfl_sync(FULL, mine[d], base + b);
}

__device__ __forceinline__ void reduce_scatter8(double v[8][3], int q, double out[3]) {
  double h[4][3], g[2][3];
#pragma unroll
  for (int t = 0; t < 4; ++t)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double send = (q & 4) ? v[t][d] : v[t + 4][d];
      h[t][d] = ((q & 4) ? v[t + 4][d] : v[t][d]) + __shfl_xor_sync(FULL, send, 4);
    }
#pragma unroll
  for (int t = 0; t < 2; ++t)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double send = (q & 2) ? h[t][d] : h[t + 2][d];
      g[t][d] = ((q & 2) ? h[t + 2][d] : h[t][d]) + __shfl_xor_sync(FULL, send, 2);
    }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double send = (q & 1) ? g[0][d] : g[1][d];
    out[d] = ((q & 1) ? g[1][d] : g[0][d]) + __shfl_xor_sync(FULL, send, 1);
  }
}

// strains (8E, 6) and strain rates B (u - u_prev) / dt (reference layout, row per point).
__global__ void __launch_bounds__(HEX_THREADS) hex8_strain_kernel(int64_t ne, const int64_t* __restrict__ elements,
                                                                 const double* __restrict__ grads,
                                                                 const double* __restrict__ u,
                                                                 const double* __restrict__ u_prev, double dt,
                                                                 double* __restrict__ strain,
                                                                 double* __restrict__ rate) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = t < 8 * ne;
  const int64_t e = live ? (t >> 3) : 0;
  const int q = (int)(t & 7);
  double mu[3] = {0, 0, 0}, md[3] = {0, 0, 0};
  if (live) {
    const int64_t n = elements[8 * e + q];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      mu[d] = u[3 * n + d];
      md[d] = mu[d] - u_prev[3 * n + d];
    }
  }
  double U[8][3], D[8][3];
  gather8(mu, U);
  gather8(md, D);
  if (!live) return;
  double G[8][3];
  load_grads(grads, 8 * e + q, G);
  double eps[6], de[6];
  strain_of(G, U, eps);
  strain_of(G, D, de);
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    strain[6 * t + c] = eps[c];
    if (rate) rate[6 * t + c] = de[c] / dt;
  }
}

// Element nodal forces fe[(8 e + a) * 3 + d] = sum_q w (B_q^T sigma_q).
__global__ void __launch_bounds__(HEX_THREADS) hex8_force_kernel(int64_t ne, const double* __restrict__ grads,
                                                                const double* __restrict__ jw,
                                                                const double* __restrict__ stress,
                                                                double* __restrict__ fe) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = t < 8 * ne;
  const int q = (int)(t & 7);
  double f[8][3];
  if (live) {
    double G[8][3], s[6];
    load_grads(grads, t, G);
#pragma unroll
    for (int c = 0; c < 6; ++c) s[c] = stress[6 * t + c];
    const double w = jw[t];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      f[a][0] = w * (G[a][0] * s[0] + G[a][2] * s[4] + G[a][1] * s[5]);
      f[a][1] = w * (G[a][1] * s[1] + G[a][2] * s[3] + G[a][0] * s[5]);
      f[a][2] = w * (G[a][2] * s[2] + G[a][1] * s[3] + G[a][0] * s[4]);
    }
  } else {
#pragma unroll
    for (int a = 0; a < 8; ++a) f[a][0] = f[a][1] = f[a][2] = 0.0;
  }
  double out[3];
  reduce_scatter8(f, q, out);
  if (live)
#pragma unroll
    for (int d = 0; d < 3; ++d) fe[t * 3 + d] = out[d];
}

// Node-centric deterministic gather: force[3 n + d] = sum over list[ptr[n] .. ptr[n+1]) of fe.
__global__ void __launch_bounds__(HEX_THREADS) hex8_node_gather_kernel(int64_t nnode, const int64_t* __restrict__ ptr,
                                                                      const int64_t* __restrict__ list,
                                                                      const double* __restrict__ fe,
                                                                      double* __restrict__ force) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  double f[3] = {0, 0, 0};
  for (int64_t k = ptr[n]; k < ptr[n + 1]; ++k) {
    const int64_t slot = list[k];
#pragma unroll
    for (int d = 0; d < 3; ++d) f[d] += fe[slot * 3 + d];
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) force[3 * n + d] = f[d];
}

// Element stiffness ke[e][i][j] = sum_q w B_q[:, i]^T C_q B_q[:, j]; one thread per (e, i).
__global__ void __launch_bounds__(HEX_THREADS) hex8_stiffness_kernel(int64_t ne, const double* __restrict__ grads,
                                                                    const double* __restrict__ jw,
                                                                    const double* __restrict__ tangent,
                                                                    double* __restrict__ ke) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 24 * ne) return;
  const int64_t e = t / 24;
  const int i = (int)(t % 24);
  const int ai = i / 3, di = i % 3;
  double row[24];
#pragma unroll
  for (int j = 0; j < 24; ++j) row[j] = 0.0;
  for (int q = 0; q < 8; ++q) {
    const int64_t g = 8 * e + q;
    double G[8][3];
    load_grads(grads, g, G);
    double bi[6] = {0, 0, 0, 0, 0, 0};  // B column i
    if (di == 0) {
      bi[0] = G[ai][0];
      bi[4] = G[ai][2];
      bi[5] = G[ai][1];
    } else if (di == 1) {
      bi[1] = G[ai][1];
      bi[3] = G[ai][2];
      bi[5] = G[ai][0];
    } else {
      bi[2] = G[ai][2];
      bi[3] = G[ai][1];
      bi[4] = G[ai][0];
    }
    double v[6];  // C^T b_i (row i of B^T C)
    const double* C = tangent + 36 * g;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) s += bi[k] * C[6 * k + c];
      v[c] = s;
    }
    const double w = jw[g];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      row[3 * a + 0] += w * (v[0] * G[a][0] + v[4] * G[a][2] + v[5] * G[a][1]);
      row[3 * a + 1] += w * (v[1] * G[a][1] + v[3] * G[a][2] + v[5] * G[a][0]);
      row[3 * a + 2] += w * (v[2] * G[a][2] + v[3] * G[a][1] + v[4] * G[a][0]);
    }
  }
#pragma unroll
  for (int j = 0; j < 24; ++j) ke[(e * 24 + i) * 24 + j] = row[j];
}

// Trilinear shape value N_a at Gauss point q (same node signs and point order as ref_grad).
__device__ __forceinline__ double shape_value(int q, int a) {
  const double gp = 0.57735026918962576451;
  const double xi = (q & 4) ? gp : -gp, eta = (q & 2) ? gp : -gp, zeta = (q & 1) ? gp : -gp;
  const double sx = (a & 1) ? 1.0 : -1.0, sy = (a & 2) ? 1.0 : -1.0, sz = (a & 4) ? 1.0 : -1.0;
  return 0.125 * (1.0 + sx * xi) * (1.0 + sy * eta) * (1.0 + sz * zeta);
}

// Element consistent mass me[e][i][j] = rho sum_q J w N_q(a_i) N_q(a_j) delta(d_i, d_j), in the
// 24 x 24 layout of the element stiffness (src/fem/assembly/elasticity.py:109-140); one
// thread per (e, i).
__global__ void __launch_bounds__(HEX_THREADS) hex8_mass_kernel(int64_t ne, const double* __restrict__ jw, double density,
                                                               double* __restrict__ me) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 24 * ne) return;
  const int64_t e = t / 24;
  const int i = (int)(t % 24);
  const int ai = i / 3, di = i % 3;
  double row[8];
#pragma unroll
  for (int b = 0; b < 8; ++b) row[b] = 0.0;
  for (int q = 0; q < 8; ++q) {
    const double w = density * shape_value(q, ai) * jw[8 * e + q];
#pragma unroll
    for (int b = 0; b < 8; ++b) row[b] += w * shape_value(q, b);
  }
  double* out = me + (e * 24 + i) * 24;
#pragma unroll
  for (int j = 0; j < 24; ++j) out[j] = (j % 3 == di) ? row[j / 3] : 0.0;
}

// CSR values: values[k] = sum over list[ptr[k] .. ptr[k+1]) of ke (fixed order).
__global__ void __launch_bounds__(HEX_THREADS) csr_gather_kernel(int64_t nnz, const int64_t* __restrict__ ptr,
                                                                const int64_t* __restrict__ list,
                                                                const double* __restrict__ ke,
                                                                double* __restrict__ values) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  double s = 0.0;
  for (int64_t m = ptr[k]; m < ptr[k + 1]; ++m) s += ke[list[m]];
  values[k] = s;
}

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + HEX_THREADS - 1) / HEX_THREADS); }

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" int cib_hex8_geometry(int64_t nelem, const double* nodes, const int64_t* elements, double* grads,
                                 double* jw, unsigned long long* bad_count, void* stream) {
  if (nelem < 0 || !nodes || !elements || !grads || !jw || !bad_count) return CIB_EINVAL;
  if (nelem == 0) return CIB_OK;
  hex8_geometry_kernel<<<blocks_for(8 * nelem), HEX_THREADS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      nelem, nodes, elements, grads, jw, bad_count);
  return check_launch();
}

extern "C" int cib_hex8_strains(int64_t nelem, const int64_t* elements, const double* grads, const double* u,
                                const double* u_prev, double time_step, double* strain, double* rate, void* stream) {
  if (nelem < 0 || !elements || !grads || !u || !u_prev || !strain || !(time_step > 0.0)) return CIB_EINVAL;
  if (nelem == 0) return CIB_OK;
  hex8_strain_kernel<<<blocks_for(8 * nelem), HEX_THREADS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      nelem, elements, grads, u, u_prev, time_step, strain, rate);
  return check_launch();
}

extern "C" int cib_hex8_internal_force(int64_t nelem, int64_t nnode, const double* grads, const double* jw,
                                       const double* stress, const int64_t* node_ptr, const int64_t* node_list,
                                       double* fe, double* force, void* stream) {
  if (nelem < 0 || nnode < 0 || !grads || !jw || !stress || !node_ptr || !node_list || !fe || !force)
    return CIB_EINVAL;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (nelem > 0) hex8_force_kernel<<<blocks_for(8 * nelem), HEX_THREADS, 0, st>>>(nelem, grads, jw, stress, fe);
  if (nnode > 0) hex8_node_gather_kernel<<<blocks_for(nnode), HEX_THREADS, 0, st>>>(nnode, node_ptr, node_list, fe, force);
  return check_launch();
}

extern "C" int cib_csr_gather(int64_t nnz, const int64_t* ptr, const int64_t* list, const double* src, double* dst,
                              void* stream) {
  if (nnz < 0 || !ptr || !list || !src || !dst) return CIB_EINVAL;
  if (nnz == 0) return CIB_OK;
  csr_gather_kernel<<<blocks_for(nnz), HEX_THREADS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(nnz, ptr, list, src,
                                                                                                 dst);
  return check_launch();
}

extern "C" int cib_hex8_mass_csr(int64_t nelem, const double* jw, double density, int64_t nnz, const int64_t* csr_ptr,
                                 const int64_t* csr_list, double* me, double* values, void* stream) {
  if (nelem < 0 || nnz < 0 || !jw || !csr_ptr || !csr_list || !me || !values || !(density > 0.0)) return CIB_EINVAL;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (nelem > 0) hex8_mass_kernel<<<blocks_for(24 * nelem), HEX_THREADS, 0, st>>>(nelem, jw, density, me);
  if (nnz > 0) csr_gather_kernel<<<blocks_for(nnz), HEX_THREADS, 0, st>>>(nnz, csr_ptr, csr_list, me, values);
  return check_launch();
}

extern "C" int cib_hex8_tangent_csr(int64_t nelem, const double* grads, const double* jw, const double* tangent,
                                    int64_t nnz, const int64_t* csr_ptr, const int64_t* csr_list, double* ke,
                                    double* values, void* stream) {
  if (nelem < 0 || nnz < 0 || !grads || !jw || !tangent || !csr_ptr || !csr_list || !ke || !values) return CIB_EINVAL;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (nelem > 0) hex8_stiffness_kernel<<<blocks_for(24 * nelem), HEX_THREADS, 0, st>>>(nelem, grads, jw, tangent, ke);
  if (nnz > 0) csr_gather_kernel<<<blocks_for(nnz), HEX_THREADS, 0, st>>>(nnz, csr_ptr, csr_list, ke, values);
  return check_launch();
}
