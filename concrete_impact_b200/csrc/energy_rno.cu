// Energy-based RVE-RNO update on the GPU (FP32), sm_100a.
//
// Restates the reference's EnergyDissipationRVERNO._constitutive_tensors
// (src/concrete_impact/nn/models/rve_rno.py:334-418; direct_rate evolution, both
// integrators), ScalarMLP.value_and_input_gradient (:110-129), the SiLU MultilayerPerceptron
// (:63-93) and prepare_energy_anchors (:227-247).  Per point and step: the equilibrium
// potential and its strain gradient, the non-equilibrium potential and its gradient at the
// previous state, the state-evolution network there, the forward-Euler latent candidate,
// and the non-equilibrium potential and gradient at the candidate -- four network passes and
// three hand-written input-gradient passes of 6/12 -> hidden^layers -> 1 (or 6) networks.
//
// One CTA of 128 threads per tile of 32 points.  Forward layers: thread j owns hidden unit j
// and keeps the 32 points' accumulators in registers; the layer's input sits in shared
// memory feature-major (the 32 points of a feature read as eight float4 broadcasts) and the
// transposed weights are read along j (coalesced).  Input-gradient layers: thread k owns
// input k and reads the weights along k (coalesced).  Pre-activations of every layer stay in
// shared memory for the backward pass.
// Everything is FP32 like the reference model (its dtype float32); no waits besides
// __syncthreads.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "cib_common.cuh"

namespace cib {
namespace {

constexpr int ER_TILE = 32;
constexpr int ER_THREADS = 128;
constexpr int ER_XLD = 16;  // input rows: 6 + latent <= 14, padded

// Parameter layout of one network (floats), for each hidden layer l: W [hidden][in_l],
// Wt [in_l][hidden], b [hidden]; then Wo [out][hidden], bo [out].
__host__ __device__ inline int64_t net_size(int in, int out, int hidden, int layers) {
  int64_t s = 0;
  for (int l = 0; l < layers; ++l) {
    const int in_l = l == 0 ? in : hidden;
    s += 2LL * hidden * in_l + hidden;
  }
  return s + (int64_t)out * hidden + out;
}

struct NetView {
  const float* base;
  int in, out;
};

__device__ __forceinline__ void layer_ptrs(const NetView& n, int hidden, int l, const float** W, const float** Wt,
                                           const float** b) {
  const float* p = n.base;
  for (int i = 0; i < l; ++i) {
    const int in_i = i == 0 ? n.in : hidden;
    p += 2LL * hidden * in_i + hidden;
  }
  const int in_l = l == 0 ? n.in : hidden;
  *W = p;
  *Wt = p + (int64_t)hidden * in_l;
  *b = p + 2LL * hidden * in_l;
}

__device__ __forceinline__ const float* output_ptr(const NetView& n, int hidden, int layers) {
  const float* p = n.base;
  for (int i = 0; i < layers; ++i) {
    const int in_i = i == 0 ? n.in : hidden;
    p += 2LL * hidden * in_i + hidden;
  }
  return p;  // Wo [out][hidden], then bo [out]
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }

__device__ __forceinline__ float silu_prime(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Shared buffers are feature-major, one row of ER_TILE floats per feature (input, hidden
// unit), so a layer reads the 32 points of one feature as eight float4 broadcasts.  The
// float4 groups of row r are XOR-swizzled by r & 7: a thread writing its own row and a
// thread reading one point across rows both hit 32 distinct banks.
__device__ __forceinline__ int sw(int row, int p) { return row * ER_TILE + ((((p >> 2) ^ (row & 7)) << 2) | (p & 3)); }

__device__ __forceinline__ float4* grp(float* buf, int row, int g) {
  return reinterpret_cast<float4*>(buf + row * ER_TILE + ((g ^ (row & 7)) << 2));
}

__device__ __forceinline__ const float4* grp(const float* buf, int row, int g) {
  return reinterpret_cast<const float4*>(buf + row * ER_TILE + ((g ^ (row & 7)) << 2));
}

struct Smem {
  float* x;    // [XLD rows][TILE] network input
  float* gin;  // [XLD rows][TILE] input gradient
  float* h0;   // [hidden rows][TILE]
  float* h1;   // [hidden rows][TILE]
  float* z;    // [layers][hidden rows][TILE] pre-activations
};

// Forward pass of the hidden layers; returns the buffer holding the last activation.
__device__ float* forward_hidden(const NetView& n, int hidden, int layers, const Smem& s) {
  const int j = threadIdx.x;
  const float* hin = s.x;
  float* hout = s.h0;
  for (int l = 0; l < layers; ++l) {
    const float *W, *Wt, *b;
    layer_ptrs(n, hidden, l, &W, &Wt, &b);
    const int in_l = l == 0 ? n.in : hidden;
    float* zl = s.z + (int64_t)l * hidden * ER_TILE;
    if (j < hidden) {
      float acc[ER_TILE];
      const float bj = b[j];
#pragma unroll
      for (int p = 0; p < ER_TILE; ++p) acc[p] = bj;
      int k = 0;
      for (; k + 4 <= in_l; k += 4) {  // four weights in flight per thread
        const float w0 = Wt[(int64_t)k * hidden + j], w1 = Wt[(int64_t)(k + 1) * hidden + j];
        const float w2 = Wt[(int64_t)(k + 2) * hidden + j], w3 = Wt[(int64_t)(k + 3) * hidden + j];
#pragma unroll
        for (int g = 0; g < ER_TILE / 4; ++g) {
          const float4 v0 = *grp(hin, k, g), v1 = *grp(hin, k + 1, g), v2 = *grp(hin, k + 2, g),
                       v3 = *grp(hin, k + 3, g);
          acc[4 * g] = fmaf(w3, v3.x, fmaf(w2, v2.x, fmaf(w1, v1.x, fmaf(w0, v0.x, acc[4 * g]))));
          acc[4 * g + 1] = fmaf(w3, v3.y, fmaf(w2, v2.y, fmaf(w1, v1.y, fmaf(w0, v0.y, acc[4 * g + 1]))));
          acc[4 * g + 2] = fmaf(w3, v3.z, fmaf(w2, v2.z, fmaf(w1, v1.z, fmaf(w0, v0.z, acc[4 * g + 2]))));
          acc[4 * g + 3] = fmaf(w3, v3.w, fmaf(w2, v2.w, fmaf(w1, v1.w, fmaf(w0, v0.w, acc[4 * g + 3]))));
        }
      }
      for (; k < in_l; ++k) {
        const float w = Wt[(int64_t)k * hidden + j];
#pragma unroll
        for (int g = 0; g < ER_TILE / 4; ++g) {
          const float4 v = *grp(hin, k, g);
          acc[4 * g] = fmaf(w, v.x, acc[4 * g]);
          acc[4 * g + 1] = fmaf(w, v.y, acc[4 * g + 1]);
          acc[4 * g + 2] = fmaf(w, v.z, acc[4 * g + 2]);
          acc[4 * g + 3] = fmaf(w, v.w, acc[4 * g + 3]);
        }
      }
#pragma unroll
      for (int g = 0; g < ER_TILE / 4; ++g) {
        *grp(zl, j, g) = make_float4(acc[4 * g], acc[4 * g + 1], acc[4 * g + 2], acc[4 * g + 3]);
        *grp(hout, j, g) = make_float4(silu(acc[4 * g]), silu(acc[4 * g + 1]), silu(acc[4 * g + 2]),
                                       silu(acc[4 * g + 3]));
      }
    }
    __syncthreads();
    hin = hout;
    hout = (hout == s.h0) ? s.h1 : s.h0;
  }
  return const_cast<float*>(hin);
}

// Scalar potential value per point (threads p < TILE) into value[p].
__device__ void scalar_output(const NetView& n, int hidden, int layers, const float* h, float* value) {
  const float* wo = output_ptr(n, hidden, layers);
  const int p = threadIdx.x;
  if (p < ER_TILE) {
    float v = 0.0f;
    for (int j = 0; j < hidden; ++j) v = fmaf(wo[j], h[sw(j, p)], v);
    value[p] = v;
  }
  __syncthreads();
}

// Input gradient of a scalar network into rows 0..in of s.gin (pre-activations in s.z).
__device__ void input_gradient(const NetView& n, int hidden, int layers, const Smem& s) {
  const float* wo = output_ptr(n, hidden, layers);
  const int t = threadIdx.x;
  float* g = s.h0;  // gradient wrt the activation of layer l
  float* d = s.h1;  // gradient wrt the pre-activation of layer l
  for (int l = layers - 1; l >= 0; --l) {
    const float* zl = s.z + (int64_t)l * hidden * ER_TILE;
    if (t < hidden) {
      const float wt = wo[t];
#pragma unroll
      for (int q = 0; q < ER_TILE / 4; ++q) {
        const float4 zz = *grp(zl, t, q);
        const float4 gv = (l == layers - 1) ? make_float4(wt, wt, wt, wt) : *grp(g, t, q);
        *grp(d, t, q) = make_float4(gv.x * silu_prime(zz.x), gv.y * silu_prime(zz.y), gv.z * silu_prime(zz.z),
                                    gv.w * silu_prime(zz.w));
      }
    }
    __syncthreads();
    const float *W, *Wt, *b;
    layer_ptrs(n, hidden, l, &W, &Wt, &b);
    const int in_l = l == 0 ? n.in : hidden;
    float* dst = l == 0 ? s.gin : g;
    if (t < in_l) {
      float acc[ER_TILE];
#pragma unroll
      for (int p = 0; p < ER_TILE; ++p) acc[p] = 0.0f;
      int jj = 0;
      for (; jj + 4 <= hidden; jj += 4) {
        const float w0 = W[(int64_t)jj * in_l + t], w1 = W[(int64_t)(jj + 1) * in_l + t];
        const float w2 = W[(int64_t)(jj + 2) * in_l + t], w3 = W[(int64_t)(jj + 3) * in_l + t];
#pragma unroll
        for (int q = 0; q < ER_TILE / 4; ++q) {
          const float4 v0 = *grp(d, jj, q), v1 = *grp(d, jj + 1, q), v2 = *grp(d, jj + 2, q), v3 = *grp(d, jj + 3, q);
          acc[4 * q] = fmaf(v3.x, w3, fmaf(v2.x, w2, fmaf(v1.x, w1, fmaf(v0.x, w0, acc[4 * q]))));
          acc[4 * q + 1] = fmaf(v3.y, w3, fmaf(v2.y, w2, fmaf(v1.y, w1, fmaf(v0.y, w0, acc[4 * q + 1]))));
          acc[4 * q + 2] = fmaf(v3.z, w3, fmaf(v2.z, w2, fmaf(v1.z, w1, fmaf(v0.z, w0, acc[4 * q + 2]))));
          acc[4 * q + 3] = fmaf(v3.w, w3, fmaf(v2.w, w2, fmaf(v1.w, w1, fmaf(v0.w, w0, acc[4 * q + 3]))));
        }
      }
      for (; jj < hidden; ++jj) {
        const float w = W[(int64_t)jj * in_l + t];
#pragma unroll
        for (int q = 0; q < ER_TILE / 4; ++q) {
          const float4 v = *grp(d, jj, q);
          acc[4 * q] = fmaf(v.x, w, acc[4 * q]);
          acc[4 * q + 1] = fmaf(v.y, w, acc[4 * q + 1]);
          acc[4 * q + 2] = fmaf(v.z, w, acc[4 * q + 2]);
          acc[4 * q + 3] = fmaf(v.w, w, acc[4 * q + 3]);
        }
      }
#pragma unroll
      for (int q = 0; q < ER_TILE / 4; ++q)
        *grp(dst, t, q) = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
    }
    __syncthreads();
  }
}

struct EnergyArgs {
  int hidden, layers, latent, integrator;
  float tau;
  const float* params;
  const float* scale;  // 6
  int64_t n;
  const float* strain;      // n x 6
  const float* latent_in;   // n x L
  const float* time_step;   // n
  const float* anchors;     // 14: eq value, eq grad (6), neq value, neq strain grad (6); NULL = zeros
  float* stress;            // n x 6
  float* latent_out;        // n x L
  float* rate;              // n x L
  float* rate_dimless;      // n x L
  float* scalars;           // 4 x n: dissipation, free energy, violation, energy increment
  float* anchors_out;       // anchor mode: 14 outputs (point 0 of a zero input)
  float* tangent;           // tangent kernel: n x 6 x 6
};

__global__ void __launch_bounds__(ER_THREADS) energy_rno_kernel(const EnergyArgs a) {
  extern __shared__ float sm[];
  const int hidden = a.hidden, layers = a.layers, L = a.latent;
  Smem s;
  s.x = sm;
  s.gin = s.x + ER_TILE * ER_XLD;
  s.h0 = s.gin + ER_TILE * ER_XLD;
  s.h1 = s.h0 + ER_TILE * hidden;
  s.z = s.h1 + ER_TILE * hidden;
  float* eps = s.z + (int64_t)layers * ER_TILE * hidden;  // [TILE][6] network strain
  float* zin = eps + ER_TILE * 6;                      // [TILE][8] previous latent
  float* zdl = zin + ER_TILE * 8;                      // [TILE][8] dimensionless rate
  float* zc = zdl + ER_TILE * 8;                       // [TILE][8] candidate latent
  float* geq = zc + ER_TILE * 8;                       // [TILE][6]
  float* gpr = geq + ER_TILE * 6;                      // [TILE][16]
  float* gca = gpr + ER_TILE * 16;                     // [TILE][16]
  float* val = gca + ER_TILE * 16;                     // [3][TILE]: eq, previous, candidate values
  const int t = threadIdx.x;
  const int64_t p0 = (int64_t)blockIdx.x * ER_TILE;
  const bool anchor_mode = a.anchors_out != nullptr;
  const NetView eq{a.params, 6, 1};
  const NetView neq{a.params + net_size(6, 1, hidden, layers), 6 + L, 1};
  const NetView evo{neq.base + net_size(6 + L, 1, hidden, layers), 6 + L, L};
  // per-point inputs (zeros beyond n and in anchor mode)
  for (int i = t; i < ER_TILE * 8; i += ER_THREADS) {
    const int p = i >> 3, c = i & 7;
    const bool live = !anchor_mode && p0 + p < a.n;
    if (c < 6) eps[p * 6 + c] = live ? a.strain[(p0 + p) * 6 + c] / a.scale[c] : 0.0f;
    zin[i] = (live && c < L) ? a.latent_in[(p0 + p) * L + c] : 0.0f;
  }
  __syncthreads();
  // 1. equilibrium potential and gradient at the network strain
  for (int i = t; i < ER_TILE * ER_XLD; i += ER_THREADS) {
    const int p = i / ER_XLD, c = i % ER_XLD;
    s.x[sw(c, p)] = c < 6 ? eps[p * 6 + c] : 0.0f;
  }
  __syncthreads();
  scalar_output(eq, hidden, layers, forward_hidden(eq, hidden, layers, s), val);
  input_gradient(eq, hidden, layers, s);
  for (int i = t; i < ER_TILE * 6; i += ER_THREADS) geq[i] = s.gin[sw(i % 6, i / 6)];
  // 2. previous state [eps, z_n]: non-equilibrium potential and gradient, then the evolution net
  for (int i = t; i < ER_TILE * ER_XLD; i += ER_THREADS) {
    const int p = i / ER_XLD, c = i % ER_XLD;
    s.x[sw(c, p)] = c < 6 ? eps[p * 6 + c] : (c < 6 + L ? zin[p * 8 + c - 6] : 0.0f);
  }
  __syncthreads();
  scalar_output(neq, hidden, layers, forward_hidden(neq, hidden, layers, s), val + ER_TILE);
  input_gradient(neq, hidden, layers, s);
  for (int i = t; i < ER_TILE * 16; i += ER_THREADS) gpr[i] = s.gin[sw(i % 16, i / 16)];
  __syncthreads();
  {
    const float* h = forward_hidden(evo, hidden, layers, s);  // s.x still holds the previous state
    const float* wo = output_ptr(evo, hidden, layers);
    const float* bo = wo + (int64_t)L * hidden;
    for (int i = t; i < ER_TILE * L; i += ER_THREADS) {
      const int p = i / L, o = i % L;
      float v = bo[o];
      for (int j = 0; j < hidden; ++j) v = fmaf(wo[(int64_t)o * hidden + j], h[sw(j, p)], v);
      zdl[p * 8 + o] = v;
    }
    __syncthreads();
  }
  // 3. forward-Euler candidate and the non-equilibrium potential there
  for (int i = t; i < ER_TILE * 8; i += ER_THREADS) {
    const int p = i >> 3, c = i & 7;
    const bool live = !anchor_mode && p0 + p < a.n;
    const float dt = live ? a.time_step[p0 + p] : 0.0f;
    zc[i] = c < L ? zin[i] + (dt / a.tau) * zdl[i] : 0.0f;
  }
  __syncthreads();
  for (int i = t; i < ER_TILE * ER_XLD; i += ER_THREADS) {
    const int p = i / ER_XLD, c = i % ER_XLD;
    s.x[sw(c, p)] = c < 6 ? eps[p * 6 + c] : (c < 6 + L ? zc[p * 8 + c - 6] : 0.0f);
  }
  __syncthreads();
  scalar_output(neq, hidden, layers, forward_hidden(neq, hidden, layers, s), val + 2 * ER_TILE);
  input_gradient(neq, hidden, layers, s);
  for (int i = t; i < ER_TILE * 16; i += ER_THREADS) gca[i] = s.gin[sw(i % 16, i / 16)];
  __syncthreads();
  if (anchor_mode) {
    if (t == 0) {
      a.anchors_out[0] = val[0];
      for (int c = 0; c < 6; ++c) a.anchors_out[1 + c] = geq[c];
      a.anchors_out[7] = val[ER_TILE];
      for (int c = 0; c < 6; ++c) a.anchors_out[8 + c] = gpr[c];
    }
    return;
  }
  // 4. anchored energies, stress, rates, dissipation (thread p owns point p)
  if (t < ER_TILE && p0 + t < a.n) {
    const int p = t;
    const int64_t q = p0 + p;
    float av_eq = 0.0f, av_neq = 0.0f, ag_eq[6], ag_neq[6];
    for (int c = 0; c < 6; ++c) {
      ag_eq[c] = a.anchors ? a.anchors[1 + c] : 0.0f;
      ag_neq[c] = a.anchors ? a.anchors[8 + c] : 0.0f;
    }
    if (a.anchors) {
      av_eq = a.anchors[0];
      av_neq = a.anchors[7];
    }
    float xe = 0.0f, xn = 0.0f;
    for (int c = 0; c < 6; ++c) {
      xe += eps[p * 6 + c] * ag_eq[c];
      xn += eps[p * 6 + c] * ag_neq[c];
    }
    const float equilibrium = val[p] - av_eq - xe;
    const float prev_neq = val[ER_TILE + p] - av_neq - xn;
    const float cand_neq = val[2 * ER_TILE + p] - av_neq - xn;
    float diss = 0.0f;
    for (int o = 0; o < L; ++o) {
      const float r = zdl[p * 8 + o] / a.tau;
      a.rate[q * L + o] = r;
      a.rate_dimless[q * L + o] = zdl[p * 8 + o];
      a.latent_out[q * L + o] = zc[p * 8 + o];
      diss += gpr[p * 16 + 6 + o] * r;
    }
    diss = -diss;
    const float* gresp = a.integrator == 1 ? gca + p * 16 : gpr + p * 16;
    for (int c = 0; c < 6; ++c)
      a.stress[q * 6 + c] = (geq[p * 6 + c] - ag_eq[c]) / a.scale[c] + (gresp[c] - ag_neq[c]) / a.scale[c];
    a.scalars[q] = diss;
    a.scalars[a.n + q] = equilibrium + (a.integrator == 1 ? cand_neq : prev_neq);
    a.scalars[2 * a.n + q] = fmaxf(-diss, 0.0f);
    a.scalars[3 * a.n + q] = cand_neq - prev_neq;
  }
}

// ---------------------------------------------------------------------------------------
// Algorithmic tangent d stress / d strain (the reference differentiates the stress with
// autograd, rve_rno.py:283-297).  With network strain e^ = strain / scale,
//   stress_i = (dW_eq/de^_i (e^) + dW_neq/de^_i (e^, z*)) / s_i  (+ constants)
// where z* is the candidate latent z + (dt / tau) f(e^, z) of the current-state integrator
// (the previous latent for the other integrator, which does not depend on the strain), so
//   C_ij = (H_eq(e^)_ij + [H_neq(e^, z*) v_j]_i) / (s_i s_j),  v_j = (e_j, (dt / tau) J_f e_j)
// with J_f the strain Jacobian of the evolution network.  Every Hessian-vector product is
// a forward-over-reverse pass of a SiLU MLP y = w_o . h_{L-1}, h_l = silu(a_l),
// a_l = W_l h_{l-1} + b_l:
//   primal:   a_l (kept), g_{L-1} = w_o, g_{l-1} = W_l^T (g_l * silu'(a_l)) (kept)
//   forward:  adot_0 = W_0 v, adot_l = W_l (silu'(a_{l-1}) * adot_{l-1}) (kept)
//   backward: ddot_{L-1} = w_o * silu''(a_{L-1}) adot_{L-1},
//             ddot_l = (W_{l+1}^T ddot_{l+1}) * silu'(a_l) + g_l * silu''(a_l) adot_l,
//             H v = W_0^T ddot_0.
// One CTA of 128 threads per tile of 32 points, the same feature-major shared layout as
// the update kernel; the tangent directions are looped (6 per network).

__device__ __forceinline__ float silu_second(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f - s) * (2.0f + z * (1.0f - 2.0f * s));
}

struct TanSmem {
  float* x;    // [XLD][TILE] primal input, then the tangent direction
  float* gin;  // [XLD][TILE] input gradient / Hessian-vector product
  float* h0;   // [hidden][TILE] work
  float* h1;   // [hidden][TILE] work
  float* z;    // [layers][hidden][TILE] pre-activations a_l
  float* ad;   // [layers][hidden][TILE] tangent pre-activations adot_l
  float* g;    // [layers - 1][hidden][TILE] activation gradients g_l, l < L - 1
};

// out[j][p] = sum_k W_l[j][k] in[k][p] (+ b_j), thread j < hidden (weights read transposed).
__device__ void tan_mat_forward(const float* Wt, const float* b, int in_l, int hidden, const float* in, float* out) {
  const int j = threadIdx.x;
  if (j < hidden) {
    float acc[ER_TILE];
    const float bj = b ? b[j] : 0.0f;
#pragma unroll
    for (int p = 0; p < ER_TILE; ++p) acc[p] = bj;
    for (int k = 0; k < in_l; ++k) {
      const float w = Wt[(int64_t)k * hidden + j];
#pragma unroll
      for (int q = 0; q < ER_TILE / 4; ++q) {
        const float4 v = *grp(in, k, q);
        acc[4 * q] = fmaf(w, v.x, acc[4 * q]);
        acc[4 * q + 1] = fmaf(w, v.y, acc[4 * q + 1]);
        acc[4 * q + 2] = fmaf(w, v.z, acc[4 * q + 2]);
        acc[4 * q + 3] = fmaf(w, v.w, acc[4 * q + 3]);
      }
    }
#pragma unroll
    for (int q = 0; q < ER_TILE / 4; ++q)
      *grp(out, j, q) = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
  }
  __syncthreads();
}

// out[t][p] = sum_j W_l[j][t] d[j][p], thread t < in_l.
__device__ void tan_mat_backward(const float* W, int in_l, int hidden, const float* d, float* out) {
  const int t = threadIdx.x;
  if (t < in_l) {
    float acc[ER_TILE];
#pragma unroll
    for (int p = 0; p < ER_TILE; ++p) acc[p] = 0.0f;
    for (int j = 0; j < hidden; ++j) {
      const float w = W[(int64_t)j * in_l + t];
#pragma unroll
      for (int q = 0; q < ER_TILE / 4; ++q) {
        const float4 v = *grp(d, j, q);
        acc[4 * q] = fmaf(v.x, w, acc[4 * q]);
        acc[4 * q + 1] = fmaf(v.y, w, acc[4 * q + 1]);
        acc[4 * q + 2] = fmaf(v.z, w, acc[4 * q + 2]);
        acc[4 * q + 3] = fmaf(v.w, w, acc[4 * q + 3]);
      }
    }
#pragma unroll
    for (int q = 0; q < ER_TILE / 4; ++q)
      *grp(out, t, q) = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
  }
  __syncthreads();
}

// Elementwise over a [hidden][TILE] buffer (thread j owns row j).
template <typename F>
__device__ __forceinline__ void tan_rows(int hidden, F f) {
  const int j = threadIdx.x;
  if (j < hidden)
#pragma unroll
    for (int p = 0; p < ER_TILE; ++p) f(j, p);
  __syncthreads();
}

// Primal forward (a_l kept) and backward (g_l kept) of a network at the input in s.x;
// returns the buffer of the last activation h_{L-1} (for the output layer).
__device__ const float* tan_primal(const NetView& n, int hidden, int layers, const TanSmem& s, bool backward) {
  const float* hin = s.x;
  float* hout = s.h0;
  for (int l = 0; l < layers; ++l) {
    const float *W, *Wt, *b;
    layer_ptrs(n, hidden, l, &W, &Wt, &b);
    float* zl = s.z + (int64_t)l * hidden * ER_TILE;
    tan_mat_forward(Wt, b, l == 0 ? n.in : hidden, hidden, hin, zl);
    tan_rows(hidden, [&](int j, int p) { hout[sw(j, p)] = silu(zl[sw(j, p)]); });
    hin = hout;
    hout = (hout == s.h0) ? s.h1 : s.h0;
  }
  const float* last = hin;
  if (!backward) return last;
  const float* wo = output_ptr(n, hidden, layers);
  // g_{L-1} = w_o; d = g * silu'(a); g_{l-1} = W_l^T d
  float* d = (last == s.h0) ? s.h1 : s.h0;  // keep h_{L-1} intact
  for (int l = layers - 1; l >= 1; --l) {
    const float* zl = s.z + (int64_t)l * hidden * ER_TILE;
    const float* gl = l == layers - 1 ? nullptr : s.g + (int64_t)l * hidden * ER_TILE;
    tan_rows(hidden, [&](int j, int p) {
      const float gv = gl ? gl[sw(j, p)] : wo[j];
      d[sw(j, p)] = gv * silu_prime(zl[sw(j, p)]);
    });
    const float *W, *Wt, *b;
    layer_ptrs(n, hidden, l, &W, &Wt, &b);
    tan_mat_backward(W, hidden, hidden, d, s.g + (int64_t)(l - 1) * hidden * ER_TILE);
  }
  return last;
}

// Forward tangent from the direction in s.x: adot_l kept in s.ad; returns the buffer of
// hdot_{L-1} = silu'(a_{L-1}) adot_{L-1}.
__device__ const float* tan_forward(const NetView& n, int hidden, int layers, const TanSmem& s) {
  const float* in = s.x;
  float* hd = s.h0;
  for (int l = 0; l < layers; ++l) {
    const float *W, *Wt, *b;
    layer_ptrs(n, hidden, l, &W, &Wt, &b);
    float* adl = s.ad + (int64_t)l * hidden * ER_TILE;
    tan_mat_forward(Wt, nullptr, l == 0 ? n.in : hidden, hidden, in, adl);
    const float* zl = s.z + (int64_t)l * hidden * ER_TILE;
    tan_rows(hidden, [&](int j, int p) { hd[sw(j, p)] = silu_prime(zl[sw(j, p)]) * adl[sw(j, p)]; });
    in = hd;
    hd = (hd == s.h0) ? s.h1 : s.h0;
  }
  return in;
}

// Backward tangent after tan_forward: H v into rows 0..in of s.gin.
__device__ void tan_backward(const NetView& n, int hidden, int layers, const TanSmem& s) {
  const float* wo = output_ptr(n, hidden, layers);
  float* gd = s.h0;  // W_{l+1}^T ddot_{l+1}
  float* dd = s.h1;  // ddot_l
  for (int l = layers - 1; l >= 0; --l) {
    const float* zl = s.z + (int64_t)l * hidden * ER_TILE;
    const float* adl = s.ad + (int64_t)l * hidden * ER_TILE;
    const float* gl = l == layers - 1 ? nullptr : s.g + (int64_t)l * hidden * ER_TILE;
    tan_rows(hidden, [&](int j, int p) {
      const float z = zl[sw(j, p)];
      const float second = (gl ? gl[sw(j, p)] : wo[j]) * silu_second(z) * adl[sw(j, p)];
      dd[sw(j, p)] = (gl ? gd[sw(j, p)] * silu_prime(z) : 0.0f) + second;
    });
    const float *W, *Wt, *b;
    layer_ptrs(n, hidden, l, &W, &Wt, &b);
    tan_mat_backward(W, l == 0 ? n.in : hidden, hidden, dd, l == 0 ? s.gin : gd);
  }
}

__global__ void __launch_bounds__(ER_THREADS) energy_rno_tangent_kernel(const EnergyArgs a) {
  extern __shared__ float sm[];
  const int hidden = a.hidden, layers = a.layers, L = a.latent;
  TanSmem s;
  s.x = sm;
  s.gin = s.x + ER_TILE * ER_XLD;
  s.h0 = s.gin + ER_TILE * ER_XLD;
  s.h1 = s.h0 + ER_TILE * hidden;
  s.z = s.h1 + ER_TILE * hidden;
  s.ad = s.z + (int64_t)layers * ER_TILE * hidden;
  s.g = s.ad + (int64_t)layers * ER_TILE * hidden;
  float* eps = s.g + (int64_t)(layers - 1) * ER_TILE * hidden;  // [TILE][6] network strain
  float* zin = eps + ER_TILE * 6;                                // [TILE][8] previous latent
  float* zc = zin + ER_TILE * 8;                                 // [TILE][8] candidate latent
  float* jf = zc + ER_TILE * 8;                                  // [TILE][8][6] (dt / tau) J_f
  float* cdt = jf + ER_TILE * 48;                                // [TILE] dt / tau
  const int t = threadIdx.x;
  const int64_t p0 = (int64_t)blockIdx.x * ER_TILE;
  const NetView eq{a.params, 6, 1};
  const NetView neq{a.params + net_size(6, 1, hidden, layers), 6 + L, 1};
  const NetView evo{neq.base + net_size(6 + L, 1, hidden, layers), 6 + L, L};
  for (int i = t; i < ER_TILE * 8; i += ER_THREADS) {
    const int p = i >> 3, c = i & 7;
    const bool live = p0 + p < a.n;
    if (c < 6) eps[p * 6 + c] = live ? a.strain[(p0 + p) * 6 + c] / a.scale[c] : 0.0f;
    zin[i] = (live && c < L) ? a.latent_in[(p0 + p) * L + c] : 0.0f;
    if (c == 0) cdt[p] = live ? a.time_step[p0 + p] / a.tau : 0.0f;
  }
  __syncthreads();
  auto set_input = [&](const float* latent) {  // s.x = [e^, latent]
    for (int i = t; i < ER_TILE * ER_XLD; i += ER_THREADS) {
      const int p = i / ER_XLD, c = i % ER_XLD;
      s.x[sw(c, p)] = c < 6 ? eps[p * 6 + c] : (latent && c < 6 + L ? latent[p * 8 + c - 6] : 0.0f);
    }
    __syncthreads();
  };
  // s.x = (e_j, latent part per point (or 0))
  auto set_direction = [&](int j, const float* latent_dir) {
    for (int i = t; i < ER_TILE * ER_XLD; i += ER_THREADS) {
      const int p = i / ER_XLD, c = i % ER_XLD;
      s.x[sw(c, p)] = c < 6 ? (c == j ? 1.0f : 0.0f) : (latent_dir && c < 6 + L ? latent_dir[p * 48 + (c - 6) * 6 + j] : 0.0f);
    }
    __syncthreads();
  };
  // accumulate rows 0..5 of s.gin as column j of the tangent (thread p < TILE owns point p)
  auto store_column = [&](int j, bool add) {
    if (t < ER_TILE && p0 + t < a.n) {
      float* out = a.tangent + (p0 + t) * 36;
      for (int i = 0; i < 6; ++i) {
        const float v = s.gin[sw(i, t)] / (a.scale[i] * a.scale[j]);
        out[6 * i + j] = add ? out[6 * i + j] + v : v;
      }
    }
    __syncthreads();
  };
  // 1. equilibrium potential: its Hessian in the strain block
  set_input(nullptr);
  tan_primal(eq, hidden, layers, s, true);
  for (int j = 0; j < 6; ++j) {
    set_direction(j, nullptr);
    tan_forward(eq, hidden, layers, s);
    tan_backward(eq, hidden, layers, s);
    store_column(j, false);
  }
  // 2. non-equilibrium potential at the stress state, in the total strain direction
  const float* latent_dir = nullptr;
  const float* state = zin;
  if (a.integrator == 1) {
    set_input(zin);
    const float* h = tan_primal(evo, hidden, layers, s, false);
    const float* wo = output_ptr(evo, hidden, layers);
    const float* bo = wo + (int64_t)L * hidden;
    for (int i = t; i < ER_TILE * 8; i += ER_THREADS) {
      const int p = i >> 3, o = i & 7;
      float v = 0.0f;
      if (o < L) {
        v = bo[o];
        for (int j = 0; j < hidden; ++j) v = fmaf(wo[(int64_t)o * hidden + j], h[sw(j, p)], v);
      }
      zc[i] = o < L ? zin[i] + cdt[p] * v : 0.0f;
    }
    __syncthreads();
    for (int j = 0; j < 6; ++j) {
      set_direction(j, nullptr);
      const float* hd = tan_forward(evo, hidden, layers, s);
      for (int i = t; i < ER_TILE * 8; i += ER_THREADS) {
        const int p = i >> 3, o = i & 7;
        float v = 0.0f;
        if (o < L)
          for (int k = 0; k < hidden; ++k) v = fmaf(wo[(int64_t)o * hidden + k], hd[sw(k, p)], v);
        jf[p * 48 + o * 6 + j] = cdt[p] * v;
      }
      __syncthreads();
    }
    latent_dir = jf;
    state = zc;
  }
  set_input(state);
  tan_primal(neq, hidden, layers, s, true);
  for (int j = 0; j < 6; ++j) {
    set_direction(j, latent_dir);
    tan_forward(neq, hidden, layers, s);
    tan_backward(neq, hidden, layers, s);
    store_column(j, true);
  }
}

inline size_t tangent_smem(int hidden, int layers) {
  const size_t floats = (size_t)ER_TILE * ER_XLD * 2 + (size_t)ER_TILE * hidden * (2 + 3 * layers - 1) +
                        (size_t)ER_TILE * (6 + 8 + 8 + 48 + 1);
  return floats * sizeof(float);
}

inline size_t energy_smem(int hidden, int layers) {
  const size_t floats = (size_t)ER_TILE * ER_XLD * 2 + (size_t)ER_TILE * hidden * (2 + layers) +
                        (size_t)ER_TILE * (6 + 8 + 8 + 8 + 6 + 16 + 16) + 3 * ER_TILE;
  return floats * sizeof(float);
}

int launch_energy(const cib_energy_rno* m, const EnergyArgs& a, int64_t blocks, cudaStream_t st) {
  const size_t smem = energy_smem(m->hidden, m->layers);
  if (smem > 200 * 1024) return CIB_ERANGE;
  const int rc = allow_dynamic_smem(reinterpret_cast<const void*>(energy_rno_kernel), 200 * 1024);
  if (rc != CIB_OK) return rc;
  energy_rno_kernel<<<(unsigned)blocks, ER_THREADS, smem, st>>>(a);
  return check_launch();
}

bool valid_model(const cib_energy_rno* m) {
  return m && m->params && m->strain_scale && m->hidden >= 1 && m->hidden <= ER_THREADS && m->layers >= 1 &&
         m->layers <= 8 && m->latent >= 1 && m->latent <= 8 && (m->integrator == 0 || m->integrator == 1) &&
         m->reference_time_scale > 0.0;
}

EnergyArgs base_args(const cib_energy_rno* m) {
  EnergyArgs a{};
  a.hidden = m->hidden;
  a.layers = m->layers;
  a.latent = m->latent;
  a.integrator = m->integrator;
  a.tau = (float)m->reference_time_scale;
  a.params = m->params;
  a.scale = m->strain_scale;
  return a;
}

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" int64_t cib_energy_rno_param_count(int32_t hidden, int32_t layers, int32_t latent) {
  if (hidden < 1 || layers < 1 || latent < 1) return -1;
  return net_size(6, 1, hidden, layers) + net_size(6 + latent, 1, hidden, layers) +
         net_size(6 + latent, latent, hidden, layers);
}

extern "C" int cib_energy_rno_anchors(const cib_energy_rno* model, float* anchors, void* stream) {
  if (!valid_model(model) || !anchors) return CIB_EINVAL;
  EnergyArgs a = base_args(model);
  a.n = 1;
  a.anchors_out = anchors;
  return launch_energy(model, a, 1, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int cib_energy_rno_update(const cib_energy_rno* model, int64_t n, const float* strain, const float* latent,
                                     const float* time_step, const float* anchors, float* stress, float* latent_out,
                                     float* state_rate, float* dimensionless_rate, float* scalars, void* stream) {
  if (!valid_model(model) || n < 0 || !strain || !latent || !time_step || !stress || !latent_out || !state_rate ||
      !dimensionless_rate || !scalars)
    return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  EnergyArgs a = base_args(model);
  a.n = n;
  a.strain = strain;
  a.latent_in = latent;
  a.time_step = time_step;
  a.anchors = anchors;
  a.stress = stress;
  a.latent_out = latent_out;
  a.rate = state_rate;
  a.rate_dimless = dimensionless_rate;
  a.scalars = scalars;
  return launch_energy(model, a, (n + ER_TILE - 1) / ER_TILE, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int cib_energy_rno_tangent(const cib_energy_rno* model, int64_t n, const float* strain, const float* latent,
                                      const float* time_step, float* tangent, void* stream) {
  if (!valid_model(model) || n < 0 || !strain || !latent || !time_step || !tangent) return CIB_EINVAL;
  if (model->layers < 2) return CIB_EINVAL;
  if (n == 0) return CIB_OK;
  const size_t smem = tangent_smem(model->hidden, model->layers);
  if (smem > 227 * 1024) return CIB_ERANGE;  // e.g. more than 4 hidden layers of 128
  const int rc = allow_dynamic_smem(reinterpret_cast<const void*>(energy_rno_tangent_kernel), 227 * 1024);
  if (rc != CIB_OK) return rc;
  EnergyArgs a = base_args(model);
  a.n = n;
  a.strain = strain;
  a.latent_in = latent;
  a.time_step = time_step;
  a.tangent = tangent;
  energy_rno_tangent_kernel<<<(unsigned)((n + ER_TILE - 1) / ER_TILE), ER_THREADS, smem,
                              reinterpret_cast<cudaStream_t>(stream)>>>(a);
  return check_launch();
}
