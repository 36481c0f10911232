// Periodic structured Hex8 RVE kernels (sm_100a): fused residual, deterministic periodic
// gather, matrix-free PCG, homogenisation.
//
// Restates, for structured periodic boxes, the reference's
//   _compute_hex8_strain_fields + material update + _assemble_force_and_tangent
//       (src/fem/assembly/nonlinear_solid.py:428-493) -- fused into rve_residual_kernel;
//   u = T w + A ebar and r = T^T f_int (src/fem/rve/solver.py:88-100, periodic.py:20-169);
//   the reduced solve K_red dw = -r (solver.py:143-144), done here by Jacobi-PCG with a
//       matrix-free tangent apply instead of SuperLU;
//   the homogenisation and diagnostics of _build_rve_response (solver.py:253-364);
//   the Schur-complement effective tangent (solver.py:438-461) via multi-RHS PCG.
//
// Layout.  Batch of R RVEs; RVE r has nx*ny*nz elements starting at element eoff; its
// periodic node (equivalence class) c = i + nx (j + ny k) is stored at batch node eoff + c,
// so classes and elements share offsets.  Class 0 is the eliminated reference class (its
// entries stay zero).  Gauss-point arrays are SoA over all 8 E points of the batch; GP q
// of element e is point 8 e + q, q = 4 a + 2 b + c for the Gauss coordinates
// (xi_a, eta_b, zeta_c) (itertools.product order, quadrature/rules.py:24-33).  Element
// node a has signs (a&1, a&2, a&4) -> lexicographic order of elements/lagrange.py:50-76.
//
// Parallel mapping.  One CTA per RVE (or per linear system): every reduction is CTA-local
// and in a fixed order, so results are bitwise reproducible.  Within a CTA, one thread per
// Gauss point; the 8 threads of an element exchange nodal values with warp shuffles and
// reduce-scatter their B^T sigma contributions so that thread q ends with element node q.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cooperative_groups.h>

#include "cib_common.cuh"
#include "j2vp_point.cuh"
#include "rve.cuh"

namespace cg = cooperative_groups;

namespace cib {

namespace {

constexpr unsigned FULL_MASK = 0xffffffffu;

template <typename T>
struct Grad8 {
  T x[8], y[8], z[8];
};

// Physical gradients of a box element (edges hx, hy, hz): dN/dx = dN/dxi * 2 / hx, in the
// element precision T.  The three reciprocals are formed once (a division per entry would
// be 24 divisions per Gauss point in every residual pass); the node factors 1 -/+ xi are
// selected at compile time per node.  Node a sits at (+/-1, +/-1, +/-1) by its bits 0, 1,
// 2 and point q at (+/-, +/-, +/-) 1/sqrt(3) by its bits 2, 1, 0; dN_a/dxi = s_a / 8 (1 + s_b
// eta)(1 + s_c zeta).
template <typename T>
__device__ __forceinline__ void physical_grads(int q, const RveDesc& d, Grad8<T>& G) {
  const T sx = (T)2 / (T)d.hx, sy = (T)2 / (T)d.hy, sz = (T)2 / (T)d.hz;
  const T gp = (T)0.57735026918962576451;  // 1/sqrt(3)
  const T xi = (q & 4) ? gp : -gp;
  const T eta = (q & 2) ? gp : -gp;
  const T zeta = (q & 1) ? gp : -gp;
  const T fx[2] = {(T)1 - xi, (T)1 + xi}, fy[2] = {(T)1 - eta, (T)1 + eta}, fz[2] = {(T)1 - zeta, (T)1 + zeta};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int ax = a & 1, ay = (a >> 1) & 1, az = (a >> 2) & 1;
    const T e8x = ax ? (T)0.125 : (T)-0.125, e8y = ay ? (T)0.125 : (T)-0.125, e8z = az ? (T)0.125 : (T)-0.125;
    G.x[a] = e8x * fy[ay] * fz[az] * sx;
    G.y[a] = e8y * fx[ax] * fz[az] * sy;
    G.z[a] = e8z * fx[ax] * fy[ay] * sz;
  }
}

// The gradients of all 8 Gauss points of a box element in shared memory, entry (a, d) of
// point q at tab[(3 a + d) * 8 + q]: the lanes of a warp that share q read the same word.
// The PCG kernels fill it once per solve (one RVE per system; a thread's Gauss point is
// fixed because the item stride is a multiple of 8) instead of forming the gradients for
// every element of every CG iteration.
template <typename T>
__device__ __forceinline__ void fill_grad_table(const RveDesc& d, T* tab) {
  if (threadIdx.x < 8) {
    Grad8<T> G;
    physical_grads((int)threadIdx.x, d, G);
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      tab[(3 * a + 0) * 8 + threadIdx.x] = G.x[a];
      tab[(3 * a + 1) * 8 + threadIdx.x] = G.y[a];
      tab[(3 * a + 2) * 8 + threadIdx.x] = G.z[a];
    }
  }
}

template <typename T>
__device__ __forceinline__ void load_grads(const T* tab, int q, Grad8<T>& G) {
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    G.x[a] = tab[(3 * a + 0) * 8 + q];
    G.y[a] = tab[(3 * a + 1) * 8 + q];
    G.z[a] = tab[(3 * a + 2) * 8 + q];
  }
}

// eps = B u for the 24 nodal values u[a][d] (Voigt xx,yy,zz,yz,xz,xy; engineering shear).
template <typename T>
__device__ __forceinline__ void strain_from(const Grad8<T>& G, const T u[8][3], T e[6]) {
  T exx = 0, eyy = 0, ezz = 0, gyz = 0, gxz = 0, gxy = 0;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    exx += G.x[a] * u[a][0];
    eyy += G.y[a] * u[a][1];
    ezz += G.z[a] * u[a][2];
    gyz += G.z[a] * u[a][1] + G.y[a] * u[a][2];
    gxz += G.z[a] * u[a][0] + G.x[a] * u[a][2];
    gxy += G.y[a] * u[a][0] + G.x[a] * u[a][1];
  }
  e[0] = exx;
  e[1] = eyy;
  e[2] = ezz;
  e[3] = gyz;
  e[4] = gxz;
  e[5] = gxy;
}

// f[a][d] = w * (B_a^T s)_d
template <typename T>
__device__ __forceinline__ void bt_stress(const Grad8<T>& G, const T s[6], T w, T f[8][3]) {
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    f[a][0] = w * (G.x[a] * s[0] + G.z[a] * s[4] + G.y[a] * s[5]);
    f[a][1] = w * (G.y[a] * s[1] + G.z[a] * s[3] + G.x[a] * s[5]);
    f[a][2] = w * (G.z[a] * s[2] + G.y[a] * s[3] + G.x[a] * s[4]);
  }
}

// Gauss point tangent: tau = C eps, for an elastic phase (params unused) or a J2 point with
// tangent parameters (n[6], f, c, active flag encoded by c/f).
template <typename T>
struct TangentParams {
  T n[6];
  T f;
  T c;
  int elastic;  // 1: use the elasticity matrix of the phase
};

// One formula for both kinds of point, so that a warp holding elastic and viscoplastic
// points runs it once: the isotropic elasticity is K 1(x)1 + 2G P, i.e. f = 2G, c = 0.
template <typename T>
__device__ __forceinline__ void tangent_apply(const PhaseMat<T>& m, const TangentParams<T>& tp, const T e[6],
                                              T s[6]) {
  const T f = tp.elastic ? (T)2 * m.G : tp.f;
  const T c = tp.elastic ? (T)0 : tp.c;
  const T tr = e[0] + e[1] + e[2];
  const T ne = tp.n[0] * e[0] + tp.n[1] * e[1] + tp.n[2] * e[2] + tp.n[3] * e[3] + tp.n[4] * e[4] + tp.n[5] * e[5];
  const T cne = c * ne;
  const T vol = m.K * tr - f * tr * (T)(1.0 / 3.0);
#pragma unroll
  for (int i = 0; i < 3; ++i) s[i] = vol + f * e[i] + cne * tp.n[i];
  const T hf = (T)0.5 * f;
#pragma unroll
  for (int i = 3; i < 6; ++i) s[i] = hf * e[i] + cne * tp.n[i];
}

// Butterfly reduce-scatter of 24 values over the 8 lanes of an element group: on return,
// out[0..2] of lane q holds the sum over the group of v[3q .. 3q+2].
template <typename T>
__device__ __forceinline__ void reduce_scatter8(const T (&v)[8][3], int q, T out[3]) {
  T h[4][3];  // after xor 4: nodes (q&4) .. (q&4)+3
#pragma unroll
  for (int t = 0; t < 4; ++t)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T send = (q & 4) ? v[t][d] : v[t + 4][d];
      const T keep = (q & 4) ? v[t + 4][d] : v[t][d];
      h[t][d] = keep + __shfl_xor_sync(FULL_MASK, send, 4);
    }
  T g[2][3];  // after xor 2: nodes (q&6), (q&6)+1
#pragma unroll
  for (int t = 0; t < 2; ++t)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T send = (q & 2) ? h[t][d] : h[t + 2][d];
      const T keep = (q & 2) ? h[t + 2][d] : h[t][d];
      g[t][d] = keep + __shfl_xor_sync(FULL_MASK, send, 2);
    }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const T send = (q & 1) ? g[0][d] : g[1][d];
    const T keep = (q & 1) ? g[1][d] : g[0][d];
    out[d] = keep + __shfl_xor_sync(FULL_MASK, send, 1);
  }
}

// Broadcast the 3 nodal values held by each lane of the 8-lane group to all of them.
template <typename T>
__device__ __forceinline__ void allgather8(const T mine[3], T u[8][3]) {
  const int base = (threadIdx.x & 31) & ~7;
#pragma unroll
  for (int b = 0; b < 8; ++b)
#pragma unroll
    for (int d = 0; d < 3; ++d) u[b][d] = __shfl_sync(FULL_MASK, mine[d], base + b);
}

// Index arithmetic avoids integer division by the runtime box sizes where it can (a
// division or remainder by a runtime divisor costs tens of instructions, and these run per
// Gauss point in every residual pass and every CG iteration): wraps are conditional
// subtractions, and local element indices are 32-bit (an RVE has far fewer than 2^31).
__device__ __forceinline__ int wrap_up(int i, int n) { return i >= n ? i - n : i; }      // i in [0, 2n)
__device__ __forceinline__ int wrap_down(int i, int n) { return i < 0 ? i + n : i; }     // i in [-n, n)

// Periodic batch node of physical node (i, j, k), 0 <= i <= nx etc.
__device__ __forceinline__ int64_t periodic_node(const RveDesc& d, int i, int j, int k) {
  i = wrap_up(i, d.nx);
  j = wrap_up(j, d.ny);
  k = wrap_up(k, d.nz);
  return d.eoff + i + (int64_t)d.nx * (j + (int64_t)d.ny * k);
}

// Node a of local element (i, j, k): periodic batch node.
__device__ __forceinline__ int64_t element_node(const RveDesc& d, int i, int j, int k, int a) {
  return periodic_node(d, i + (a & 1), j + ((a >> 1) & 1), k + ((a >> 2) & 1));
}

__device__ __forceinline__ void local_ijk(const RveDesc& d, int64_t le, int& i, int& j, int& k) {
  const int l = (int)le;
  const int row = l / d.nx;  // j + ny k
  i = l - row * d.nx;
  k = row / d.ny;
  j = row - k * d.ny;
}

// CTA-wide sum of NV doubles (fixed order: warp tree, then warp 0 over warps).
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch /* >= 32 * NV */) {
#pragma unroll
  for (int k = 0; k < NV; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(FULL_MASK, v[k], o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) scratch[warp * NV + k] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = lane < nw ? scratch[lane * NV + k] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL_MASK, x, o);
      v[k] = x;
    }
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < NV; ++k) scratch[k] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = scratch[k];
  __syncthreads();
}

__device__ __forceinline__ double block_max(double v, double* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL_MASK, v, o));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double x = lane < nw ? scratch[lane] : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(FULL_MASK, x, o));
    if (lane == 0) scratch[0] = x;
  }
  __syncthreads();
  v = scratch[0];
  __syncthreads();
  return v;
}

__device__ __forceinline__ double block_min(double v, double* scratch) { return -block_max(-v, scratch); }

// Current fluctuation at a batch node: w_base + alpha * dw (dw may be null).
__device__ __forceinline__ void load_w(const double* w, const double* dw, double alpha, int64_t node, double out[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double v = w[3 * node + d];
    if (dw) v += alpha * dw[3 * node + d];
    out[d] = v;
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Fused residual: strains, return map, trial state, tangent parameters, element nodal
// forces and Jacobi diagonal contributions.  The grid covers all Gauss points of the batch
// (one thread each, grid-stride in whole waves), whatever RVE they belong to, so an uneven
// batch keeps every SM busy until the last element; each 8-lane group looks up its RVE.
// FP32: capped at 80 registers for three CTAs (24 warps) per SM, 32 B of spills; FP64 keeps
// its 170 registers.
template <typename T>
__global__ void __launch_bounds__(RVE_THREADS, sizeof(T) == 4 ? 3 : 1) rve_residual_kernel(const RveResidualArgs<T> a) {
  const int64_t G_all = 8 * a.nelem;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t rounds = (G_all + stride - 1) / stride;  // the same for every thread (shuffles)
  for (int64_t it = 0; it < rounds; ++it) {
    const int64_t gl = it * stride + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t e = gl < G_all ? (gl >> 3) : 0;  // whole 8-lane groups are in range or not
    const int q = (int)(gl & 7);
    const int r = rve_of_element(a.desc, a.nrve, e);
    const RveDesc d = a.desc[r];
    const int64_t E = (int64_t)d.nx * d.ny * d.nz;
    const int64_t le = e - d.eoff;
    const bool live = gl < G_all && le >= 0 && le < E && (!a.active || a.active[r]);
    const double alpha = a.alpha ? a.alpha[r] : 1.0;
    T ebar[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) ebar[k] = (T)a.macro[6 * r + k];
    const T jw = (T)(d.hx * d.hy * d.hz / 8.0);
    int i, j, k;
    local_ijk(d, live ? le : 0, i, j, k);
    const int64_t g = 8 * e + q;
    double wq[3] = {0.0, 0.0, 0.0};
    if (live) load_w(a.w, a.dw, alpha, element_node(d, i, j, k, q), wq);
    T mine[3] = {(T)wq[0], (T)wq[1], (T)wq[2]};
    T u[8][3];
    allgather8(mine, u);
    Grad8<T> Gr;
    physical_grads(q, d, Gr);
    T eps[6];
    strain_from(Gr, u, eps);
#pragma unroll
    for (int c = 0; c < 6; ++c) eps[c] += ebar[c];
    const int ph = live ? (int)a.phase[e] : 0;
    const PhaseMat<T>& m = a.mats.m[ph];
    T sig[6];
    TangentParams<T> tp;
    tp.elastic = 1;
    tp.f = (T)0;
    tp.c = (T)0;
#pragma unroll
    for (int c = 0; c < 6; ++c) tp.n[c] = (T)0;
    if (live) {
      if (m.kind == PHASE_J2VP) {
        T ep[6], eel[6], st[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          ep[c] = a.ep_n[c * a.ngp + g];
          eel[c] = eps[c] - ep[c];
        }
        elastic_stress(m.j2, eel, st);
        const double qn = a.q_n[g];
        J2Out<T> o;
        const int status = j2vp_point<T, false>(m.j2, (T)a.dt[r], st, qn, o);
        if (status != CIB_J2_OK) {
          if (a.fail) atomicMin(&a.fail[r], (unsigned long long)(8 * le + q));
#pragma unroll
          for (int c = 0; c < 6; ++c) o.sigma[c] = st[c];
          o.active = 0;
          o.dgamma = (T)0;
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          sig[c] = o.sigma[c];
          a.ep[c * a.ngp + g] = ep[c] + (c < 3 ? o.dgamma : (T)2 * o.dgamma) * (o.active ? o.n[c] : (T)0);
        }
        a.q[g] = qn + (double)o.dgamma;
        a.vpm[g] = a.vpm_n[g] + (double)o.dgamma;
        if (o.active) {
          tp.elastic = 0;
          tp.f = o.tan_f;
          tp.c = o.tan_c;
#pragma unroll
          for (int c = 0; c < 6; ++c) tp.n[c] = o.n[c];
        }
      } else {
        elastic_stress(m.j2, eps, sig);
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        a.stress[c * a.ngp + g] = sig[c];
        a.tparam[c * a.ngp + g] = tp.n[c];
      }
      a.tparam[6 * a.ngp + g] = tp.f;
      a.tparam[7 * a.ngp + g] = tp.elastic ? (T)0 : tp.c;
      a.tflag[g] = (uint8_t)(tp.elastic ? 0 : 1);
    } else {
#pragma unroll
      for (int c = 0; c < 6; ++c) sig[c] = (T)0;
    }
    // Element nodal forces w_q B_q^T sigma_q and Jacobi diagonal contributions
    // w e^T C e for the B column e of every (node, direction): e has the node's gradient
    // component g on the direction's normal strain and the other two components s1, s2 on
    // its two engineering shears, so with C = K 1(x)1 + f P + c n(x)n
    //   e^T C e = K g^2 + f (2/3 g^2 + 1/2 (s1^2 + s2^2)) + c (n . e)^2
    // (elastic: C11 g^2 + G (s1^2 + s2^2)).
    // Per point the diagonal is  A g^2 + B (s1^2 + s2^2) + c (n . e)^2  with (A, B) =
    // (K + 2/3 f, f / 2), or (C11, G) for an elastic point (n = 0, c = 0 there); the
    // integration weight is folded into the three coefficients.
    T f[8][3];
    bt_stress(Gr, sig, jw, f);
    const T jwl = live ? jw : (T)0;
    const T ca = jwl * (tp.elastic ? m.C11 : m.K + (T)(2.0 / 3.0) * tp.f);
    const T cb = jwl * (tp.elastic ? m.G : (T)0.5 * tp.f);
    const T cc = jwl * tp.c;
    T diag[8][3];
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const T gx = Gr.x[b], gy = Gr.y[b], gz = Gr.z[b];
      const T gx2 = gx * gx, gy2 = gy * gy, gz2 = gz * gz;
      // n . e for the B columns of directions x, y, z (Voigt xx yy zz yz xz xy)
      const T nx = tp.n[0] * gx + tp.n[4] * gz + tp.n[5] * gy;
      const T ny = tp.n[1] * gy + tp.n[3] * gz + tp.n[5] * gx;
      const T nz = tp.n[2] * gz + tp.n[3] * gy + tp.n[4] * gx;
      diag[b][0] = ca * gx2 + cb * (gy2 + gz2) + cc * nx * nx;
      diag[b][1] = ca * gy2 + cb * (gx2 + gz2) + cc * ny * ny;
      diag[b][2] = ca * gz2 + cb * (gx2 + gy2) + cc * nz * nz;
    }
    T fo[3], dgo[3];
    reduce_scatter8(f, q, fo);
    reduce_scatter8(diag, q, dgo);
    if (live) {
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) {
        a.fe[(8 * e + q) * 3 + dd] = (double)fo[dd];
        a.de[(8 * e + q) * 3 + dd] = (double)dgo[dd];
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// Periodic gather: reduced residual r = T^T f (class 0 removed), Jacobi inverse diagonal,
// squared norm, class-reaction maximum (class 0 included) and, optionally, the
// materialised trial fluctuation w_out = w + alpha dw.  Two kernels: the node pass does the
// gathers (8 element contributions of f and of the diagonal per periodic node) over a grid
// that covers every node of the batch, so an uneven batch keeps every SM busy; the norm
// pass then forms the per-RVE reductions from the gathered residual, one CTA per RVE, in a
// fixed order (bitwise reproducible).
__device__ __forceinline__ void gather_node_force(const RveDesc& d, const double* __restrict__ fe,
                                                  const double* __restrict__ de, int64_t c, double f[3],
                                                  double dg[3]) {
  int i, j, k;
  local_ijk(d, c, i, j, k);
#pragma unroll
  for (int dd = 0; dd < 3; ++dd) f[dd] = dg[dd] = 0.0;
  for (int n = 0; n < 8; ++n) {
    const int di = n & 1, dj = (n >> 1) & 1, dk = (n >> 2) & 1;
    const int ie = wrap_down(i - di, d.nx), je = wrap_down(j - dj, d.ny), ke = wrap_down(k - dk, d.nz);
    const int64_t e = d.eoff + ie + (int64_t)d.nx * (je + (int64_t)d.ny * ke);
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      f[dd] += fe[(8 * e + n) * 3 + dd];
      if (de) dg[dd] += de[(8 * e + n) * 3 + dd];
    }
  }
}

__global__ void __launch_bounds__(RVE_THREADS) rve_gather_nodes_kernel(const RveGatherArgs a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; node < a.nelem; node += stride) {
    const int r = rve_of_element(a.desc, a.nrve, node);
    if (a.active && !a.active[r]) continue;
    const RveDesc d = a.desc[r];
    const int64_t E = (int64_t)d.nx * d.ny * d.nz;
    const int64_t c = node - d.eoff;
    if (c < 0 || c >= E) continue;
    double f[3], dg[3];
    gather_node_force(d, a.fe, a.de, c, f, dg);
    const bool fixed = (c == 0);
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      a.res[3 * node + dd] = fixed ? 0.0 : f[dd];
      a.dinv[3 * node + dd] = fixed ? 0.0 : 1.0 / dg[dd];
    }
    if (a.w_out) {
      double w[3];
      load_w(a.w, a.dw, a.alpha ? a.alpha[r] : 1.0, node, w);
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) a.w_out[3 * node + dd] = fixed ? 0.0 : w[dd];
    }
  }
}

__global__ void __launch_bounds__(RVE_THREADS) rve_gather_norms_kernel(const RveGatherArgs a) {
  __shared__ double scratch[32 * 2];
  const int r = blockIdx.x;
  if (a.active && !a.active[r]) return;
  const RveDesc d = a.desc[r];
  const int64_t E = (int64_t)d.nx * d.ny * d.nz;
  const double alpha = a.alpha ? a.alpha[r] : 1.0;
  double acc[2] = {0.0, 0.0};  // ||r||^2, ||w + alpha dw||^2
  double cmax = 0.0;
  for (int64_t c = threadIdx.x; c < E; c += blockDim.x) {
    const int64_t node = d.eoff + c;
    double f[3];
    if (c == 0) {  // the eliminated class: its force is not in the reduced residual
      double dg[3];
      gather_node_force(d, a.fe, nullptr, 0, f, dg);
    } else {
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) f[dd] = a.res[3 * node + dd];
    }
    cmax = fmax(cmax, sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]));
    if (c != 0)
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) acc[0] += f[dd] * f[dd];
    double w[3];
    if (a.w_out) {
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) w[dd] = a.w_out[3 * node + dd];
    } else {
      load_w(a.w, a.dw, alpha, node, w);
    }
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      const double wv = (c == 0) ? 0.0 : w[dd];
      acc[1] += wv * wv;
    }
  }
  block_sum<2>(acc, scratch);
  cmax = block_max(cmax, scratch);
  if (threadIdx.x == 0) {
    a.rnorm2[r] = acc[0];
    if (a.wnorm2) a.wnorm2[r] = acc[1];
    if (a.class_max) a.class_max[r] = cmax;
  }
}

// ---------------------------------------------------------------------------------------
// One element-Gauss-point item of the matrix-free apply and its loads.  The apply loops
// fetch the next round's item (the vector values at its node, its phase and tangent flag,
// then its tangent parameters) while the current round computes, so that the L2 latency of
// those loads overlaps the arithmetic instead of stalling every round.
template <typename T>
struct ApplyItem {
  bool live;
  int el, q, ph, flag;
  int64_t g;
  T mine[3];
  T tp[8];
};

template <typename T>
__device__ __forceinline__ void fetch_item(const RvePcgArgs<T>& a, const RveDesc& d, const double* __restrict__ p,
                                           int items, int nxy, int k, int it, ApplyItem<T>& x) {
  const int gl = it * blockDim.x + threadIdx.x;
  x.live = gl < items;
  x.el = x.live ? (gl >> 3) : 0;
  x.q = gl & 7;
  const int j = x.el / d.nx, i = x.el - j * d.nx;
  const int64_t e = d.eoff + x.el + (int64_t)nxy * k;
  x.g = 8 * e + x.q;
  x.ph = 0;
  x.flag = 0;
#pragma unroll
  for (int dd = 0; dd < 3; ++dd) x.mine[dd] = (T)0;
  if (x.live) {
    const int64_t node = element_node(d, i, j, k, x.q);
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) x.mine[dd] = (T)__ldcg(p + 3 * node + dd);  // other ranks may have written p
    x.ph = (int)a.phase[e];
    x.flag = (int)a.tflag[x.g];
  }
}

template <typename T>
__device__ __forceinline__ void fetch_tangent(const RvePcgArgs<T>& a, ApplyItem<T>& x) {
  if (x.live && x.flag) {
#pragma unroll
    for (int c = 0; c < 8; ++c) x.tp[c] = a.tparam[c * a.ngp + x.g];
  }
}

// Element-node contributions w B^T C B u of one item (valid on every lane; zero when the
// item is not live), reduce-scattered so that lane q holds node q's three values.
template <typename T>
__device__ __forceinline__ void apply_item(const RvePcgArgs<T>& a, const ApplyItem<T>& x, const T* gtab, T jw,
                                           T out[3]) {
  T u[8][3];
  allgather8(x.mine, u);
  Grad8<T> Gr;
  load_grads(gtab, x.q, Gr);
  T eps[6], sig[6];
  strain_from(Gr, u, eps);
  TangentParams<T> tp;
  tp.elastic = 1;
  tp.f = (T)0;
  tp.c = (T)0;
#pragma unroll
  for (int c = 0; c < 6; ++c) tp.n[c] = (T)0;
  if (x.live && x.flag) {
    tp.elastic = 0;
#pragma unroll
    for (int c = 0; c < 6; ++c) tp.n[c] = x.tp[c];
    tp.f = x.tp[6];
    tp.c = x.tp[7];
  }
  tangent_apply(a.mats.m[x.ph], tp, eps, sig);
  T f[8][3];
  bt_stress(Gr, sig, x.live ? jw : (T)0, f);
  reduce_scatter8(f, x.q, out);
}

// ---------------------------------------------------------------------------------------
// Matrix-free apply of the reduced tangent to one periodic vector, streaming the RVE in
// z-layers: element results of a layer go to shared memory, then every node of the layer
// gathers its 4 bottom and 4 top contributions in a fixed order.  Returns p . Ap (CTA-wide).
template <typename T>
__device__ double apply_tangent(const RvePcgArgs<T>& a, const RveDesc& d, const double* __restrict__ p,
                                double* __restrict__ Ap, double* smem, double* scratch, const T* gtab) {
  const int nxy = d.nx * d.ny;
  double* ye = smem;                  // nxy * 24
  double* acc_cur = ye + 24 * nxy;    // nxy * 3
  double* acc_next = acc_cur + 3 * nxy;
  double* acc_first = acc_next + 3 * nxy;
  const T jw = (T)(d.hx * d.hy * d.hz / 8.0);
  double pap[1] = {0.0};
  const int items = 8 * nxy;
  const int rounds = (items + blockDim.x - 1) / blockDim.x;
  for (int k = 0; k < d.nz; ++k) {
    ApplyItem<T> cur, nxt;
    fetch_item(a, d, p, items, nxy, k, 0, cur);
    fetch_tangent(a, cur);
    for (int it = 0; it < rounds; ++it) {
      if (it + 1 < rounds) fetch_item(a, d, p, items, nxy, k, it + 1, nxt);
      T out[3];
      apply_item(a, cur, gtab, jw, out);
      if (cur.live)
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) ye[(8 * cur.el + cur.q) * 3 + dd] = (double)out[dd];
      if (it + 1 < rounds) {
        fetch_tangent(a, nxt);
        cur = nxt;
      }
    }
    __syncthreads();
    for (int n = threadIdx.x; n < nxy; n += blockDim.x) {
      const int j = n / d.nx, i = n - j * d.nx;
      double bot[3] = {0, 0, 0}, top[3] = {0, 0, 0};
      for (int s = 0; s < 4; ++s) {
        const int di = s & 1, dj = s >> 1;
        const int el = wrap_down(i - di, d.nx) + d.nx * wrap_down(j - dj, d.ny);
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) {
          bot[dd] += ye[(8 * el + s) * 3 + dd];
          top[dd] += ye[(8 * el + s + 4) * 3 + dd];
        }
      }
      if (k == 0) {
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) acc_first[3 * n + dd] = bot[dd];
      } else {
        const int64_t node = d.eoff + n + (int64_t)nxy * k;
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) {
          const double v = acc_cur[3 * n + dd] + bot[dd];
          Ap[3 * node + dd] = v;
          pap[0] += p[3 * node + dd] * v;
        }
      }
      if (k == d.nz - 1) {
        const int64_t node = d.eoff + n;
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) {
          const double v = (n == 0) ? 0.0 : acc_first[3 * n + dd] + top[dd];
          Ap[3 * node + dd] = v;
          pap[0] += p[3 * node + dd] * v;
        }
      } else {
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) acc_next[3 * n + dd] = top[dd];
      }
    }
    __syncthreads();
    double* t = acc_cur;
    acc_cur = acc_next;
    acc_next = t;
  }
  block_sum<1>(pap, scratch);
  return pap[0];
}

// Jacobi-PCG on one reduced periodic system per CTA: K x = b, x0 = 0.  Bounded iterations;
// status 0 converged (||r|| <= rtol ||b|| or ||b|| == 0), 1 iteration limit, 2 breakdown
// (p.Ap <= 0 or non-finite).  Two CTAs per SM in both precisions: the FP64 build then fits
// 128 registers with ~140 B of spills, and the second CTA hides more of the latency of the
// per-layer barriers and reductions (2,048 8^3 systems: 23 % less time than at 252
// registers and one CTA per SM, bitwise the same results).
template <typename T>
__global__ void __launch_bounds__(RVE_THREADS, 2) rve_pcg_kernel(const RvePcgArgs<T> a) {
  extern __shared__ double smem[];
  __shared__ double scratch[64];
  const int s = blockIdx.x;
  const int r = a.sys_rve[s];
  if (a.active && !a.active[r]) return;
  const RveDesc d = a.desc[r];
  const int64_t E = (int64_t)d.nx * d.ny * d.nz;
  const int64_t off = a.sys_off[s];  // vector offset of this system (3 * node base)
  if (a.vec_len >= 0 && (off < 0 || E < 0 || off + 3 * E > a.vec_len)) {  // uniform over the CTA
    if (threadIdx.x == 0) {
      a.status[s] = 3;
      a.iterations[s] = 0;
      a.rel_residual[s] = 0.0;
      a.xnorm[s] = 0.0;
    }
    return;
  }
  const double* b = a.b + off;
  double* x = a.x + off;
  double* rr = a.r + off;
  double* p = a.p + off;
  double* Ap = a.Ap + off;
  const double* dinv = a.dinv + 3 * d.eoff;
  __shared__ T gtab[24 * 8];
  fill_grad_table(d, gtab);  // visible after the block sum below
  // Shift the vector pointers so that batch node indices address them directly.
  const int64_t shift = 3 * d.eoff;
  double* x_ = x - shift;
  double* r_ = rr - shift;
  double* p_ = p - shift;
  double* Ap_ = Ap - shift;
  double v[2] = {0.0, 0.0};  // rz, bb
  for (int64_t n = threadIdx.x; n < 3 * E; n += blockDim.x) {
    const double bi = b[n];
    x[n] = 0.0;
    rr[n] = bi;
    const double z = dinv[n] * bi;
    p[n] = z;
    v[0] += bi * z;
    v[1] += bi * bi;
  }
  block_sum<2>(v, scratch);
  double rz = v[0];
  const double bnorm = sqrt(v[1]);
  const double tol = (a.rtol_dev ? *a.rtol_dev : a.rtol) * bnorm;
  int status = 1, iters = 0;
  double rnorm = bnorm;
  if (bnorm == 0.0 || !(bnorm == bnorm)) {
    status = (bnorm == 0.0) ? 0 : 2;
  } else {
    for (iters = 0; iters < a.maxit;) {
      const double pap = apply_tangent<T>(a, d, p_, Ap_, smem, scratch, gtab);
      if (!(pap > 0.0) || !isfinite(pap)) {
        status = 2;
        break;
      }
      const double alpha = rz / pap;
      double w2[2] = {0.0, 0.0};  // r.r, r.z
      for (int64_t n = threadIdx.x; n < 3 * E; n += blockDim.x) {
        x[n] += alpha * p[n];
        const double rn = rr[n] - alpha * Ap[n];
        rr[n] = rn;
        w2[0] += rn * rn;
        w2[1] += rn * dinv[n] * rn;
      }
      block_sum<2>(w2, scratch);
      ++iters;
      rnorm = sqrt(w2[0]);
      if (!isfinite(rnorm)) {
        status = 2;
        break;
      }
      if (rnorm <= tol) {
        status = 0;
        break;
      }
      const double beta = w2[1] / rz;
      rz = w2[1];
      for (int64_t n = threadIdx.x; n < 3 * E; n += blockDim.x) p[n] = dinv[n] * rr[n] + beta * p[n];
      __syncthreads();
    }
  }
  double xn[1] = {0.0};
  for (int64_t n = threadIdx.x; n < 3 * E; n += blockDim.x) xn[0] += x[n] * x[n];
  block_sum<1>(xn, scratch);
  if (threadIdx.x == 0) {
    a.status[s] = status;
    a.iterations[s] = iters;
    a.rel_residual[s] = bnorm > 0.0 ? rnorm / bnorm : 0.0;
    a.xnorm[s] = sqrt(xn[0]);
  }
  (void)x_;
  (void)r_;
}

// ---------------------------------------------------------------------------------------
// Cluster variant of the PCG: C CTAs of one thread-block cluster share one system.  Rank q
// owns the node layers [k0, k1) = [q nz / C, (q + 1) nz / C) of its RVE: it streams its
// element layers like apply_tangent, keeps the bottom contributions of its first node layer
// (acc_first) and exports the top contributions of its last element layer, which belong to
// the next rank's first node layer (the last rank's wrap to node layer 0 is the periodic
// closure); after a cluster barrier every rank adds its predecessor's export through
// distributed shared memory.  Dot products are CTA sums combined over the ranks in rank
// order (every rank forms the same totals, so all ranks take the same branches).  Four
// cluster barriers per iteration: export, p.Ap, r.r / r.z, and p visibility.  The layer's
// element contributions are kept in the element type T (exact: they are computed in T),
// the node sums in double as in rve_pcg_kernel; in FP32 mode that is 192 bytes per node of
// a layer, and with at most 128 registers two CTAs fit on an SM.
template <typename T>
__device__ double apply_tangent_slab(const RvePcgArgs<T>& a, const RveDesc& d, const double* __restrict__ p,
                                     double* __restrict__ Ap, unsigned char* smem, int k0, int k1,
                                     cg::cluster_group& cl, unsigned prev_rank,
                                     const T* gtab) {
  const int nxy = d.nx * d.ny;
  T* ye = reinterpret_cast<T*>(smem);  // nxy * 24 element-node contributions of one layer (exact in T)
  double* acc_cur = reinterpret_cast<double*>(smem + (size_t)24 * nxy * sizeof(T));  // nxy * 3 node sums
  double* acc_next = acc_cur + 3 * nxy;
  double* acc_first = acc_next + 3 * nxy;
  double* exported = acc_first + 3 * nxy;
  const T jw = (T)(d.hx * d.hy * d.hz / 8.0);
  double pap = 0.0;
  const int items = 8 * nxy;
  const int rounds = (items + blockDim.x - 1) / blockDim.x;
  for (int k = k0; k < k1; ++k) {
    ApplyItem<T> cur, nxt;
    fetch_item(a, d, p, items, nxy, k, 0, cur);
    fetch_tangent(a, cur);
    for (int it = 0; it < rounds; ++it) {
      if (it + 1 < rounds) fetch_item(a, d, p, items, nxy, k, it + 1, nxt);
      T out[3];
      apply_item(a, cur, gtab, jw, out);
      if (cur.live)
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) ye[(8 * cur.el + cur.q) * 3 + dd] = out[dd];
      if (it + 1 < rounds) {
        fetch_tangent(a, nxt);
        cur = nxt;
      }
    }
    __syncthreads();
    for (int n = threadIdx.x; n < nxy; n += blockDim.x) {
      const int j = n / d.nx, i = n - j * d.nx;
      double bot[3] = {0, 0, 0}, top[3] = {0, 0, 0};
      for (int s = 0; s < 4; ++s) {
        const int di = s & 1, dj = s >> 1;
        const int el = wrap_down(i - di, d.nx) + d.nx * wrap_down(j - dj, d.ny);
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) {
          bot[dd] += (double)ye[(8 * el + s) * 3 + dd];
          top[dd] += (double)ye[(8 * el + s + 4) * 3 + dd];
        }
      }
      if (k == k0) {
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) acc_first[3 * n + dd] = bot[dd];
      } else {
        const int64_t node = d.eoff + n + (int64_t)nxy * k;
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) {
          const double v = acc_cur[3 * n + dd] + bot[dd];
          Ap[3 * node + dd] = v;
          pap += p[3 * node + dd] * v;
        }
      }
      if (k == k1 - 1) {
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) exported[3 * n + dd] = top[dd];
      } else {
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) acc_next[3 * n + dd] = top[dd];
      }
    }
    __syncthreads();
    double* t = acc_cur;
    acc_cur = acc_next;
    acc_next = t;
  }
  cl.sync();  // every rank's export is complete
  const double* prev = cl.map_shared_rank(exported, prev_rank);
  for (int n = threadIdx.x; n < nxy; n += blockDim.x) {
    const int64_t node = d.eoff + n + (int64_t)nxy * k0;
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      const double v = (k0 == 0 && n == 0) ? 0.0 : acc_first[3 * n + dd] + prev[3 * n + dd];
      Ap[3 * node + dd] = v;
      pap += p[3 * node + dd] * v;
    }
  }
  return pap;
}

// Sum of NV doubles over the CTAs of the cluster, the same on every thread of every rank.
// `slots` (NV doubles of this CTA's shared memory) must not be rewritten before the next
// cluster barrier that follows every rank's read.
template <int NV>
__device__ __forceinline__ void cluster_sum(double (&v)[NV], double* scratch, double* slots, cg::cluster_group& cl) {
  block_sum<NV>(v, scratch);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) slots[k] = v[k];
  cl.sync();
  double t[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) t[k] = 0.0;
  const unsigned nr = cl.num_blocks();
  for (unsigned q = 0; q < nr; ++q) {
    const double* rem = cl.map_shared_rank(slots, q);
#pragma unroll
    for (int k = 0; k < NV; ++k) t[k] += rem[k];
  }
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = t[k];
}

// Launch shapes of the cluster PCG (threads per CTA, resident CTAs per SM -> register cap),
// chosen per batch by the tuner: 0 is the default, 1-3 trade threads for registers.
template <typename T, int SHAPE>
struct PcgShape;
template <typename T>
struct PcgShape<T, 0> {
  static constexpr int threads = 256, min_blocks = sizeof(T) == 4 ? 2 : 1;
};
template <typename T>
struct PcgShape<T, 1> {
  static constexpr int threads = 128, min_blocks = sizeof(T) == 4 ? 4 : 2;
};
template <typename T>
struct PcgShape<T, 2> {
  static constexpr int threads = 512, min_blocks = 1;
};
template <typename T>
struct PcgShape<T, 3> {
  static constexpr int threads = 256, min_blocks = sizeof(T) == 4 ? 1 : 2;
};

template <typename T, int SHAPE>
__global__ void __launch_bounds__(PcgShape<T, SHAPE>::threads, PcgShape<T, SHAPE>::min_blocks)
    rve_pcg_cluster_kernel(const RvePcgArgs<T> a) {
  extern __shared__ double smem_dyn[];  // the layer buffers of apply_tangent_slab
  unsigned char* smem = reinterpret_cast<unsigned char*>(smem_dyn);
  __shared__ double scratch[64];
  __shared__ double slot_init[2], slot_pap[1], slot_rr[2], slot_xn[1];
  cg::cluster_group cl = cg::this_cluster();
  const unsigned C = cl.num_blocks();
  const unsigned rank = cl.block_rank();
  const int s = blockIdx.x / C;
  const int r = a.sys_rve[s];
  if (a.active && !a.active[r]) return;  // the whole cluster leaves together
  const RveDesc d = a.desc[r];
  if (d.nz < (int)C) {  // every rank must own a layer
    if (rank == 0 && threadIdx.x == 0) {
      a.status[s] = 3;
      a.iterations[s] = 0;
      a.rel_residual[s] = 0.0;
      a.xnorm[s] = 0.0;
    }
    return;
  }
  const int nxy = d.nx * d.ny;
  __shared__ T gtab[24 * 8];
  fill_grad_table(d, gtab);  // visible after the first cluster sum
  const int k0 = (int)((rank * (unsigned)d.nz) / C), k1 = (int)(((rank + 1) * (unsigned)d.nz) / C);
  const unsigned prev_rank = (rank + C - 1) % C;
  const int64_t off = a.sys_off[s];
  const int64_t shift = 3 * d.eoff;
  const int64_t lo = 3 * (int64_t)nxy * k0, hi = 3 * (int64_t)nxy * k1;  // this rank's vector entries
  const double* b = a.b + off;
  double* x = a.x + off;
  double* rr = a.r + off;
  double* p = a.p + off;
  double* Ap = a.Ap + off;
  const double* dinv = a.dinv + 3 * d.eoff;
  double v[2] = {0.0, 0.0};  // r.z, b.b
  for (int64_t n = lo + threadIdx.x; n < hi; n += blockDim.x) {
    const double bi = b[n];
    x[n] = 0.0;
    rr[n] = bi;
    const double z = dinv[n] * bi;
    p[n] = z;
    v[0] += bi * z;
    v[1] += bi * bi;
  }
  cluster_sum<2>(v, scratch, slot_init, cl);  // its barrier also publishes p
  double rz = v[0];
  const double bnorm = sqrt(v[1]);
  const double tol = (a.rtol_dev ? *a.rtol_dev : a.rtol) * bnorm;
  int status = 1, iters = 0;
  double rnorm = bnorm;
  if (bnorm == 0.0 || !(bnorm == bnorm)) {
    status = (bnorm == 0.0) ? 0 : 2;
  } else {
    for (iters = 0; iters < a.maxit;) {
      double pap[1] = {apply_tangent_slab<T>(a, d, p - shift, Ap - shift, smem, k0, k1, cl, prev_rank, gtab)};
      cluster_sum<1>(pap, scratch, slot_pap, cl);
      if (!(pap[0] > 0.0) || !isfinite(pap[0])) {
        status = 2;
        break;
      }
      const double alpha = rz / pap[0];
      double w2[2] = {0.0, 0.0};  // r.r, r.z
      for (int64_t n = lo + threadIdx.x; n < hi; n += blockDim.x) {
        x[n] += alpha * p[n];
        const double rn = rr[n] - alpha * Ap[n];
        rr[n] = rn;
        w2[0] += rn * rn;
        w2[1] += rn * dinv[n] * rn;
      }
      cluster_sum<2>(w2, scratch, slot_rr, cl);
      ++iters;
      rnorm = sqrt(w2[0]);
      if (!isfinite(rnorm)) {
        status = 2;
        break;
      }
      if (rnorm <= tol) {
        status = 0;
        break;
      }
      const double beta = w2[1] / rz;
      rz = w2[1];
      for (int64_t n = lo + threadIdx.x; n < hi; n += blockDim.x) p[n] = dinv[n] * rr[n] + beta * p[n];
      cl.sync();  // p of every rank visible before the next apply
    }
  }
  double xn[1] = {0.0};
  for (int64_t n = lo + threadIdx.x; n < hi; n += blockDim.x) xn[0] += x[n] * x[n];
  cluster_sum<1>(xn, scratch, slot_xn, cl);
  if (rank == 0 && threadIdx.x == 0) {
    a.status[s] = status;
    a.iterations[s] = iters;
    a.rel_residual[s] = bnorm > 0.0 ? rnorm / bnorm : 0.0;
    a.xnorm[s] = sqrt(xn[0]);
  }
  cl.sync();  // no rank leaves while another may still read its shared memory
}

// ---------------------------------------------------------------------------------------
// Right-hand sides of the effective-tangent solves and K_ee.  For macro strain unit j,
// element forces f_e^(j) = sum_q w B_q^T C_q e_j; gathered periodically they give column j
// of K_we = T^T K A; K_ee = A^T K A = sum_q w C_q (since B_q A e_j = e_j on a box).
// One CTA per RVE; rhs is (6, 3E) per RVE at offset 18 * eoff; kee is (R, 36).
template <typename T>
__global__ void __launch_bounds__(RVE_THREADS) rve_tangent_rhs_kernel(const RveTangentArgs<T> a) {
  __shared__ double scratch[32 * 36];
  const int r = blockIdx.x;
  if (a.active && !a.active[r]) return;
  const RveDesc d = a.desc[r];
  const int64_t E = (int64_t)d.nx * d.ny * d.nz;
  const int64_t G = 8 * E;
  const T jw = (T)(d.hx * d.hy * d.hz / 8.0);
  double kee[36];
#pragma unroll
  for (int t = 0; t < 36; ++t) kee[t] = 0.0;
  const int64_t rounds = (G + blockDim.x - 1) / blockDim.x;
  for (int64_t it = 0; it < rounds; ++it) {
    const int64_t gl = it * blockDim.x + threadIdx.x;
    const bool live = gl < G;
    const int64_t le = live ? (gl >> 3) : 0;
    const int q = (int)(gl & 7);
    const int64_t e = d.eoff + le;
    const int64_t g = 8 * e + q;
    Grad8<T> Gr;
    physical_grads(q, d, Gr);
    const int ph = live ? (int)a.phase[e] : 0;
    TangentParams<T> tp;
    tp.elastic = 1;
    tp.f = (T)0;
    tp.c = (T)0;
#pragma unroll
    for (int c = 0; c < 6; ++c) tp.n[c] = (T)0;
    if (live && a.tflag[g]) {
      tp.elastic = 0;
#pragma unroll
      for (int c = 0; c < 6; ++c) tp.n[c] = a.tparam[c * a.ngp + g];
      tp.f = a.tparam[6 * a.ngp + g];
      tp.c = a.tparam[7 * a.ngp + g];
    }
#pragma unroll 1
    for (int jcol = 0; jcol < 6; ++jcol) {
      T ej[6] = {0, 0, 0, 0, 0, 0};
      ej[jcol] = (T)1;
      T sc[6];
      tangent_apply(a.mats.m[ph], tp, ej, sc);
      if (live)
#pragma unroll
        for (int i = 0; i < 6; ++i) kee[6 * i + jcol] += (double)jw * (double)sc[i];
      T f[8][3];
      bt_stress(Gr, sc, live ? jw : (T)0, f);
      T out[3];
      reduce_scatter8(f, q, out);
      if (live)
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) a.fe6[((int64_t)jcol * a.ne_total * 8 + 8 * e + q) * 3 + dd] = (double)out[dd];
    }
  }
  block_sum<36>(kee, scratch);
  if (threadIdx.x == 0)
    for (int t = 0; t < 36; ++t) a.kee[36 * r + t] = kee[t];
  __syncthreads();
  // Periodic gather of the 6 columns into rhs (class 0 removed).
  for (int64_t c = threadIdx.x; c < E; c += blockDim.x) {
    int i, j, k;
    local_ijk(d, c, i, j, k);
    for (int jcol = 0; jcol < 6; ++jcol) {
      double f[3] = {0.0, 0.0, 0.0};
      for (int n = 0; n < 8; ++n) {
        const int di = n & 1, dj = (n >> 1) & 1, dk = (n >> 2) & 1;
        const int ie = wrap_down(i - di, d.nx), je = wrap_down(j - dj, d.ny), ke = wrap_down(k - dk, d.nz);
        const int64_t e = d.eoff + ie + (int64_t)d.nx * (je + (int64_t)d.ny * ke);
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) f[dd] += a.fe6[((int64_t)jcol * a.ne_total * 8 + 8 * e + n) * 3 + dd];
      }
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) a.rhs[18 * d.eoff + (int64_t)jcol * 3 * E + 3 * c + dd] = (c == 0) ? 0.0 : f[dd];
    }
  }
}

// C_eff = (K_ee - K_we^T S) / V, with S the 6 PCG solutions (same layout as rhs).
__global__ void __launch_bounds__(RVE_THREADS) rve_tangent_finish_kernel(const RveTangentFinishArgs a) {
  __shared__ double scratch[32 * 36];
  const int r = blockIdx.x;
  if (a.active && !a.active[r]) return;
  const RveDesc d = a.desc[r];
  const int64_t E = (int64_t)d.nx * d.ny * d.nz;
  double acc[36];
#pragma unroll
  for (int t = 0; t < 36; ++t) acc[t] = 0.0;
  const double* rhs = a.rhs + 18 * d.eoff;
  const double* sol = a.sol + 18 * d.eoff;
  for (int64_t n = threadIdx.x; n < 3 * E; n += blockDim.x) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const double ki = rhs[i * 3 * E + n];
#pragma unroll
      for (int j = 0; j < 6; ++j) acc[6 * i + j] += ki * sol[j * 3 * E + n];
    }
  }
  block_sum<36>(acc, scratch);
  if (threadIdx.x == 0) {
    const double vol = d.hx * d.hy * d.hz * (double)E;
    for (int t = 0; t < 36; ++t) a.ceff[36 * r + t] = (a.kee[36 * r + t] - acc[t]) / vol;
  }
}

// ---------------------------------------------------------------------------------------
// Response pass: homogenised stress, energies, work/activity statistics, phase averages,
// virtual-work, periodicity and reaction diagnostics (solver.py:253-364, 464-494), and
// optionally the per-point strains, strain rates, free energy, dissipation and the J2
// diagnostics rows.  One CTA per RVE.
template <typename T>
__global__ void __launch_bounds__(RVE_THREADS) rve_response_kernel(const RveResponseArgs<T> a) {
  __shared__ double scratch[32 * RVE_NSUM];
  const int r = blockIdx.x;
  if (a.active && !a.active[r]) return;
  const RveDesc d = a.desc[r];
  const int64_t E = (int64_t)d.nx * d.ny * d.nz;
  const int64_t G = 8 * E;
  const double jw = d.hx * d.hy * d.hz / 8.0;
  const double dt = a.dt[r];
  double S[RVE_NSUM];
#pragma unroll
  for (int t = 0; t < RVE_NSUM; ++t) S[t] = 0.0;
  double mmin = INFINITY, mmax = -INFINITY, qmax[RVE_MAX_PHASES];
#pragma unroll
  for (int t = 0; t < RVE_MAX_PHASES; ++t) qmax[t] = -INFINITY;
  const int64_t rounds = (G + blockDim.x - 1) / blockDim.x;
  for (int64_t it = 0; it < rounds; ++it) {
    const int64_t gl = it * blockDim.x + threadIdx.x;
    const bool live = gl < G;
    const int64_t le = live ? (gl >> 3) : 0;
    const int q = (int)(gl & 7);
    int i, j, k;
    local_ijk(d, le, i, j, k);
    const int64_t e = d.eoff + le;
    const int64_t g = 8 * e + q;
    double w1[3] = {0, 0, 0}, w0[3] = {0, 0, 0};
    if (live) {
      const int64_t node = element_node(d, i, j, k, q);
      load_w(a.w, nullptr, 0.0, node, w1);
      load_w(a.w_n, nullptr, 0.0, node, w0);
    }
    double u1[8][3], u0[8][3];
    allgather8(w1, u1);
    allgather8(w0, u0);
    Grad8<double> Gr;
    physical_grads(q, d, Gr);
    double eps[6], eps0[6];
    strain_from(Gr, u1, eps);
    strain_from(Gr, u0, eps0);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      eps[c] += a.macro[6 * r + c];
      eps0[c] += a.macro_n[6 * r + c];
    }
    if (!live) continue;
    const int ph = (int)a.phase[e];
    const PhaseMat<double>& m = a.mats.m[ph];
    double sig[6], de[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      sig[c] = (double)a.stress[c * a.ngp + g];
      de[c] = eps[c] - eps0[c];
    }
    // Per-point energy, dissipation and increment diagnostics.
    double psi, diss = 0.0, iwd, esi, margin = NAN, active = 0.0;
    double sprev[6];
    if (m.kind == PHASE_J2VP) {
      // Re-run the return map of this update in the kernel precision (same inputs and
      // operation order as the residual pass) for the local-solver diagnostics.
      const PhaseMat<T>& mt = a.mats_t.m[ph];
      T wt[3] = {(T)w1[0], (T)w1[1], (T)w1[2]};
      T ut[8][3];
      // all lanes of this group are live here; the group never straddles the G boundary
      {
        const int base = (threadIdx.x & 31) & ~7;
        const unsigned gmask = 0xffu << base;
#pragma unroll
        for (int b = 0; b < 8; ++b)
#pragma unroll
          for (int dd = 0; dd < 3; ++dd) ut[b][dd] = __shfl_sync(gmask, wt[dd], base + b);
      }
      Grad8<T> Gt;
      physical_grads(q, d, Gt);
      T et[6], ep0t[6], eelt[6], stt[6];
      strain_from(Gt, ut, et);
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        et[c] += (T)a.macro[6 * r + c];
        ep0t[c] = a.ep_n[c * a.ngp + g];
        eelt[c] = et[c] - ep0t[c];
      }
      elastic_stress(mt.j2, eelt, stt);
      const double q0 = a.q_n[g];
      J2Out<T> o;
      const int st_code = j2vp_point<T, false>(mt.j2, (T)dt, stt, q0, o);
      const bool act = (st_code == CIB_J2_OK) && o.active;
      double ep1[6], ep0[6], ee[6], se[6], e_prev[6];
      const double q1 = a.q[g];
      const double dg = q1 - q0;
      double pw = 0.0, wsum = 0.0;
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        ep1[c] = (double)a.ep[c * a.ngp + g];
        ep0[c] = (double)a.ep_n[c * a.ngp + g];
        ee[c] = eps[c] - ep1[c];
        pw += sig[c] * (ep1[c] - ep0[c]);
        e_prev[c] = (eps[c] - de[c]) - ep0[c];
      }
      elastic_stress(m.j2, ee, se);
#pragma unroll
      for (int c = 0; c < 6; ++c) wsum += se[c] * ee[c];
      psi = 0.5 * wsum + 0.5 * m.j2.H * q1 * q1;
      active = act ? 1.0 : 0.0;
      if (act) diss = pw / dt - m.j2.H * q1 * dg / dt;
      elastic_stress(m.j2, e_prev, sprev);
      const double ftr = (double)o.f_tr, ys = (double)o.yield_scale, thr = (double)o.threshold;
      margin = (ftr - thr) / ys;
      if (a.diag) {
        const int64_t Gt_ = a.ngp;
        double* dgr = a.diag;
        double dv2[6];
        const double qf = act ? sqrt(fmax(j2_radicand(sig, dv2), 0.0)) : (double)o.q_tr;
        const double fy = act ? qf - (m.j2.sy + m.j2.H * q1) : ftr;
        dgr[0 * Gt_ + g] = fy;
        dgr[1 * Gt_ + g] = act ? pw : 0.0;
        dgr[2 * Gt_ + g] = (double)o.iters;
        dgr[3 * Gt_ + g] = act ? 4.0 : 0.0;
        dgr[4 * Gt_ + g] = dg;
        dgr[5 * Gt_ + g] = dg;
        dgr[6 * Gt_ + g] = qf;
        dgr[7 * Gt_ + g] = ftr;
        dgr[8 * Gt_ + g] = ys;
        dgr[9 * Gt_ + g] = thr;
        dgr[10 * Gt_ + g] = margin;
        dgr[11 * Gt_ + g] = active;
        dgr[12 * Gt_ + g] = dt;
        dgr[13 * Gt_ + g] = q1;
        dgr[14 * Gt_ + g] = act ? (double)o.hv : 0.0;
        dgr[15 * Gt_ + g] = act ? pw / dt : 0.0;
        dgr[16 * Gt_ + g] = act ? m.j2.H * q1 * dg / dt : 0.0;
        dgr[17 * Gt_ + g] = act ? (double)o.local_residual : 0.0;
        dgr[18 * Gt_ + g] = 0.0;
        dgr[19 * Gt_ + g] = act ? ftr / m.j2.slope : 0.0;
      }
    } else {
      double w_ = 0.0;
#pragma unroll
      for (int c = 0; c < 6; ++c) w_ += eps[c] * sig[c];
      psi = 0.5 * w_;
      double ds[6];
      elastic_stress(m.j2, de, ds);
#pragma unroll
      for (int c = 0; c < 6; ++c) sprev[c] = sig[c] - ds[c];
    }
    {
      double w_ = 0.0, dv[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) w_ += (sprev[c] + sig[c]) * de[c];
      iwd = 0.5 * w_;
      esi = sqrt(fmax(j2_radicand(sig, dv), 0.0)) - sqrt(fmax(j2_radicand(sprev, dv), 0.0));
    }
    if (a.diag) {
      a.diag[20 * a.ngp + g] = iwd;
      a.diag[21 * a.ngp + g] = esi;
      if (m.kind != PHASE_J2VP) {
        // elastic phase: only the phased-model rows exist (others are NaN in the reference)
        for (int row = 0; row < 20; ++row) a.diag[row * a.ngp + g] = NAN;
        a.diag[11 * a.ngp + g] = 0.0;
      }
    }
    if (a.point_out) {
      // strains, strain rates, free energy, dissipation
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        a.point_out[c * a.ngp + g] = eps[c];
        a.point_out[(6 + c) * a.ngp + g] = de[c] / dt;
      }
      a.point_out[12 * a.ngp + g] = psi;
      a.point_out[13 * a.ngp + g] = diss;
    }
    double mw = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      S[RS_SIGMA + c] += sig[c] * jw;
      mw += sig[c] * de[c];
    }
    S[RS_PSI] += psi * jw;
    S[RS_DISS] += diss * jw;
    S[RS_MICRO_WORK] += mw * jw;
    S[RS_POS_WORK] += fmax(iwd, 0.0) * jw;
    S[RS_NEG_WORK] += fmin(iwd, 0.0) * jw;
    if (iwd < 0.0) S[RS_UNLOAD] += jw;
    if (active > 0.5) S[RS_ACTIVE] += jw;
    if (m.kind == PHASE_J2VP) {
      S[RS_EQPS] += a.q[g] * jw;
      if (isfinite(margin)) {
        mmin = fmin(mmin, margin);
        mmax = fmax(mmax, margin);
      }
    }
    if (ph < RVE_MAX_PHASES) {
      double* P = S + RS_PHASE + ph * RS_PHASE_STRIDE;
      P[0] += jw;
#pragma unroll
      for (int c = 0; c < 6; ++c) P[1 + c] += sig[c] * jw;
      P[7] += psi * jw;
      P[8] += diss * jw;
      if (m.kind == PHASE_J2VP) {
        P[9] += a.q[g] * jw;
        qmax[ph] = fmax(qmax[ph], a.q[g]);
      }
    }
  }
  // Virtual-work stress A^T f / V, full nodal force norm and face resultants from the
  // element nodal forces of the last residual pass (physical, non-periodic nodes).
  const int64_t NX = d.nx + 1, NY = d.ny + 1, NZ = d.nz + 1;
  const int64_t NN = NX * NY * NZ;
  for (int64_t n = threadIdx.x; n < NN; n += blockDim.x) {
    const int I = (int)(n % NX), J = (int)((n / NX) % NY), K = (int)(n / (NX * NY));
    double f[3] = {0, 0, 0};
    for (int s = 0; s < 8; ++s) {
      const int di = s & 1, dj = (s >> 1) & 1, dk = (s >> 2) & 1;
      const int ie = I - di, je = J - dj, ke = K - dk;
      if (ie < 0 || je < 0 || ke < 0 || ie >= d.nx || je >= d.ny || ke >= d.nz) continue;
      const int64_t e = d.eoff + ie + (int64_t)d.nx * (je + (int64_t)d.ny * ke);
#pragma unroll
      for (int dd = 0; dd < 3; ++dd) f[dd] += a.fe[(8 * e + s) * 3 + dd];
    }
    const double x = I * d.hx, y = J * d.hy, z = K * d.hz;
    S[RS_VW + 0] += x * f[0];
    S[RS_VW + 1] += y * f[1];
    S[RS_VW + 2] += z * f[2];
    S[RS_VW + 3] += 0.5 * (z * f[1] + y * f[2]);
    S[RS_VW + 4] += 0.5 * (z * f[0] + x * f[2]);
    S[RS_VW + 5] += 0.5 * (y * f[0] + x * f[1]);
    S[RS_FNORM2] += f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
    const int idx[3] = {I, J, K};
    const int64_t mx[3] = {d.nx, d.ny, d.nz};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      if (idx[ax] == 0)
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) S[RS_FACE + 6 * ax + dd] += f[dd];
      if (idx[ax] == mx[ax])
#pragma unroll
        for (int dd = 0; dd < 3; ++dd) S[RS_FACE + 6 * ax + 3 + dd] += f[dd];
    }
    // periodic fluctuation mismatch of u = T w + A ebar against the class representative
    double w[3];
    load_w(a.w, nullptr, 0.0, periodic_node(d, I, J, K), w);
    const double* eb = a.macro + 6 * r;
    const double ua[3] = {x * eb[0] + 0.5 * z * eb[4] + 0.5 * y * eb[5], y * eb[1] + 0.5 * z * eb[3] + 0.5 * x * eb[5],
                          z * eb[2] + 0.5 * y * eb[3] + 0.5 * x * eb[4]};
    const double xr = wrap_up(I, d.nx) * d.hx, yr = wrap_up(J, d.ny) * d.hy, zr = wrap_up(K, d.nz) * d.hz;
    const double ur[3] = {xr * eb[0] + 0.5 * zr * eb[4] + 0.5 * yr * eb[5],
                          yr * eb[1] + 0.5 * zr * eb[3] + 0.5 * xr * eb[5],
                          zr * eb[2] + 0.5 * yr * eb[3] + 0.5 * xr * eb[4]};
    double mis = 0.0;
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      const double fl = (w[dd] + ua[dd]) - ua[dd];
      const double flr = (w[dd] + ur[dd]) - ur[dd];
      mis += (fl - flr) * (fl - flr);
    }
    S[RS_PERIODIC] = fmax(S[RS_PERIODIC], sqrt(mis));
  }
  const double pmax = block_max(S[RS_PERIODIC], scratch);
  S[RS_PERIODIC] = 0.0;
  mmin = block_min(mmin, scratch);
  mmax = block_max(mmax, scratch);
  for (int t = 0; t < RVE_MAX_PHASES; ++t) qmax[t] = block_max(qmax[t], scratch);
  block_sum<RVE_NSUM>(S, scratch);
  if (threadIdx.x == 0) {
    double* o = a.sums + (int64_t)r * RVE_NOUT;
    for (int t = 0; t < RVE_NSUM; ++t) o[t] = S[t];
    o[RS_PERIODIC] = pmax;
    o[RVE_NSUM + 0] = mmin;
    o[RVE_NSUM + 1] = mmax;
    for (int t = 0; t < RVE_MAX_PHASES; ++t) o[RVE_NSUM + 2 + t] = qmax[t];
  }
}

// ---------------------------------------------------------------------------------------
// Host launchers.

template <typename T>
int launch_rve_residual(const RveResidualArgs<T>& a, int nrve, cudaStream_t st) {
  (void)nrve;
  if (a.nelem <= 0) return CIB_OK;
  const int grid = persistent_grid(reinterpret_cast<const void*>(rve_residual_kernel<T>), RVE_THREADS, 8 * a.nelem);
  rve_residual_kernel<T><<<grid, RVE_THREADS, 0, st>>>(a);
  return check_launch();
}

int launch_rve_gather(const RveGatherArgs& a, int nrve, cudaStream_t st) {
  if (a.nelem > 0) {
    const int grid = persistent_grid(reinterpret_cast<const void*>(rve_gather_nodes_kernel), RVE_THREADS, a.nelem);
    rve_gather_nodes_kernel<<<grid, RVE_THREADS, 0, st>>>(a);
    const int rc = check_launch();
    if (rc != CIB_OK) return rc;
  }
  rve_gather_norms_kernel<<<nrve, RVE_THREADS, 0, st>>>(a);
  return check_launch();
}

template <typename T>
int launch_rve_pcg(const RvePcgArgs<T>& a, int nsys, int max_nxy, cudaStream_t st) {
  const size_t smem = (size_t)max_nxy * (24 + 9) * sizeof(double);
  if (smem > 200 * 1024) return CIB_ERANGE;
  const int rc = allow_dynamic_smem(reinterpret_cast<const void*>(rve_pcg_kernel<T>), 200 * 1024);
  if (rc != CIB_OK) return rc;
  rve_pcg_kernel<T><<<nsys, RVE_THREADS, smem, st>>>(a);
  return check_launch();
}

template <typename T, int SHAPE>
int launch_rve_pcg_cluster_shape(const RvePcgArgs<T>& a, int nsys, int cluster, size_t smem, cudaStream_t st) {
  const void* fn = reinterpret_cast<const void*>(rve_pcg_cluster_kernel<T, SHAPE>);
  const int rc = allow_dynamic_smem(fn, 200 * 1024);
  if (rc != CIB_OK) return rc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)nsys * (unsigned)cluster, 1, 1);
  cfg.blockDim = dim3(PcgShape<T, SHAPE>::threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, rve_pcg_cluster_kernel<T, SHAPE>, a);
  return check_launch();
}

// cluster: the CTAs per system (1, 2, 4 or 8) in bits 0-3 and the launch shape (0-3, see
// PcgShape) in bits 4-7; cluster size 1 is the one-CTA kernel, whatever the shape.
template <typename T>
int launch_rve_pcg_cluster(const RvePcgArgs<T>& a, int nsys, int max_nxy, int cluster, cudaStream_t st) {
  const int c = cluster & 15, shape = (cluster >> 4) & 15;
  if ((cluster >> 8) != 0 || shape > 3) return CIB_EINVAL;
  if (c == 1) return launch_rve_pcg<T>(a, nsys, max_nxy, st);
  if (c != 2 && c != 4 && c != 8) return CIB_EINVAL;
  const size_t smem = (size_t)max_nxy * (24 * sizeof(T) + 12 * sizeof(double));
  if (smem > 200 * 1024) return CIB_ERANGE;
  switch (shape) {
    case 1: return launch_rve_pcg_cluster_shape<T, 1>(a, nsys, c, smem, st);
    case 2: return launch_rve_pcg_cluster_shape<T, 2>(a, nsys, c, smem, st);
    case 3: return launch_rve_pcg_cluster_shape<T, 3>(a, nsys, c, smem, st);
    default: return launch_rve_pcg_cluster_shape<T, 0>(a, nsys, c, smem, st);
  }
}

template <typename T>
int launch_rve_tangent_rhs(const RveTangentArgs<T>& a, int nrve, cudaStream_t st) {
  rve_tangent_rhs_kernel<T><<<nrve, RVE_THREADS, 0, st>>>(a);
  return check_launch();
}

int launch_rve_tangent_finish(const RveTangentFinishArgs& a, int nrve, cudaStream_t st) {
  rve_tangent_finish_kernel<<<nrve, RVE_THREADS, 0, st>>>(a);
  return check_launch();
}

template <typename T>
int launch_rve_response(const RveResponseArgs<T>& a, int nrve, cudaStream_t st) {
  rve_response_kernel<T><<<nrve, RVE_THREADS, 0, st>>>(a);
  return check_launch();
}

template int launch_rve_residual<float>(const RveResidualArgs<float>&, int, cudaStream_t);
template int launch_rve_residual<double>(const RveResidualArgs<double>&, int, cudaStream_t);
template int launch_rve_pcg<float>(const RvePcgArgs<float>&, int, int, cudaStream_t);
template int launch_rve_pcg<double>(const RvePcgArgs<double>&, int, int, cudaStream_t);
template int launch_rve_pcg_cluster<float>(const RvePcgArgs<float>&, int, int, int, cudaStream_t);
template int launch_rve_pcg_cluster<double>(const RvePcgArgs<double>&, int, int, int, cudaStream_t);
template int launch_rve_tangent_rhs<float>(const RveTangentArgs<float>&, int, cudaStream_t);
template int launch_rve_tangent_rhs<double>(const RveTangentArgs<double>&, int, cudaStream_t);
template int launch_rve_response<float>(const RveResponseArgs<float>&, int, cudaStream_t);
template int launch_rve_response<double>(const RveResponseArgs<double>&, int, cudaStream_t);

}  // namespace cib
