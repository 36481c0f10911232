// Fused recurrent window kernels of the material surrogate (sm_100a).
//
// The unfused path (mlp.cu GEMMs + rno.cu elementwise kernels) launches six kernels per
// time step, each of which re-stages its weights and runs on B / 128 CTAs.  Here one CTA
// owns 128 paths for the whole window: the four weight matrices stay in shared memory in
// the tcgen05 operand layout, the latent state stays in registers, and every time step
// runs its four layers as back-to-back tcgen05.mma (M = 128, accumulator in TMEM) with the
// bias/GELU epilogue writing the next layer's A operand straight into shared memory.  The
// epilogue is the step's critical path: 16 warps (four per TMEM lane quarter, each on a
// quarter of the columns) share it.
// The paths of a window are independent in time, so the recurrence needs no grid-wide
// synchronisation.  The forward kernel is persistent: one CTA per SM stages the weights
// once and runs its 128-path tiles one after another (a 131,072-point inference step is
// 1,024 tiles on 148 CTAs).
//
// Per step t and path p (normalised units; x = [strain, rate, z] padded to 32 bf16):
//   Z_l = H_{l-1} W_l^T + b_l, H_l = gelu(Z_l) (bf16), l = 1..3;  Y = H_3 W_4^T + b_4
//   s = Y[0:6] + K (strain - z)          (K: optional 6x6 elastic skip, else 0)
//   z' = z + coef * Y[6:12]
//   loss += scale * |s - target|^2,  gS = 2 scale (s - target)
// The backward kernel runs the same CTA tiling in reverse time with the transposed weights:
//   dY = [gS, coef dz', 0], dZ_3 = (dY W_4) * gelu'(Z_3), dZ_l = (dZ_{l+1} W_{l+1}) *
//   gelu'(Z_l), dX = dZ_1 W_1, dz = dz' + dX[12:18] - K^T gS
// and writes dY^T and dZ_l^T (bf16) for the split-K weight-gradient GEMMs of mlp.cu.
// The forward keeps Z_l (fp32) and X^T, H_l^T (bf16) for them.  Numerics follow the
// unfused kernels: bf16 activations and back-propagated signals, fp32 accumulation.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "cib200.h"
#include "cib_common.cuh"
#include "umma.cuh"

namespace cib {
namespace {

using namespace umma;

constexpr int RW_THREADS = 512;
constexpr int COL_GROUPS = RW_THREADS / 128;         // warps sharing one TMEM lane quarter
constexpr int GROUP_COLS = 128 / COL_GROUPS;         // epilogue columns of each of them
constexpr int GROUP_CHUNKS = GROUP_COLS / 16;        // 32x32b.x16 loads per layer and warp
constexpr int HID = 128;
constexpr int XIN = 32;
constexpr int YOUT = 16;
constexpr int TILE = 128;
constexpr uint32_t TMEM_COLS = 128;

struct __align__(1024) FwdSmem {
  uint8_t w1[HID * XIN * 2];
  uint8_t w2[HID * HID * 2];
  uint8_t w3[HID * HID * 2];
  uint8_t w4[YOUT * HID * 2];
  uint8_t x[TILE * XIN * 2];
  uint8_t h[TILE * HID * 2];
  float bias[3 * HID + YOUT];
  float skip[36];
  double red[RW_THREADS / 32];
  uint64_t bar;
  uint32_t tmem;
};

struct __align__(1024) BwdSmem {
  uint8_t w4t[HID * YOUT * 2];
  uint8_t w3t[HID * HID * 2];
  uint8_t w2t[HID * HID * 2];
  uint8_t w1t[XIN * HID * 2];
  uint8_t dy[TILE * YOUT * 2];
  uint8_t d[TILE * HID * 2];
  float skip[36];
  uint64_t bar;
  uint32_t tmem;
};

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// Store 8 consecutive bf16 (columns c..c+7 of tile row r) into an operand tile with k columns.
__device__ __forceinline__ void put8(uint8_t* tile, int r, int c, int k, const float* v) {
  uint4 q;
  q.x = pack_bf16(v[0], v[1]);
  q.y = pack_bf16(v[2], v[3]);
  q.z = pack_bf16(v[4], v[5]);
  q.w = pack_bf16(v[6], v[7]);
  *reinterpret_cast<uint4*>(tile + core_offset(r, c, k)) = q;
}

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// All threads: make shared-memory operands visible, issue one layer (thread 0), wait.
// Returns false on every thread when the wait timed out on any thread.
__device__ __forceinline__ bool run_layer(uint64_t* bar, uint32_t tmem, const uint8_t* a, const uint8_t* b, int k,
                                          int n, uint32_t& phase) {
  fence_smem_to_async();
  fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_after_sync();
    mma_bf16(tmem, smem_u32(a), smem_u32(b), k, n, false, bar);
  }
  const bool ok = mbar_wait(bar, phase);
  phase ^= 1u;
  fence_after_sync();
  return !__syncthreads_or(ok ? 0 : 1);
}

__global__ void __launch_bounds__(RW_THREADS, 1) rno_window_forward_kernel(const cib_rno_window w) {
  extern __shared__ uint8_t smem_raw[];
  FwdSmem& S = *reinterpret_cast<FwdSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, group = warp >> 2;
  const int row = quarter * 32 + lane;
  const int B = w.B, T = w.T;
  const int ntiles = (B + TILE - 1) / TILE;
  const size_t R = w.ldt > 0 ? (size_t)w.ldt : (size_t)B * T;

  stage_matrix(S.w1, static_cast<const __nv_bfloat16*>(w.W[0]), HID, XIN, XIN);
  stage_matrix(S.w2, static_cast<const __nv_bfloat16*>(w.W[1]), HID, HID, HID);
  stage_matrix(S.w3, static_cast<const __nv_bfloat16*>(w.W[2]), HID, HID, HID);
  stage_matrix(S.w4, static_cast<const __nv_bfloat16*>(w.W[3]), YOUT, HID, HID);
  for (int i = tid; i < 3 * HID + YOUT; i += RW_THREADS) S.bias[i] = w.bias[i / HID < 3 ? i / HID : 3][i % HID];
  for (int i = tid; i < 36; i += RW_THREADS) S.skip[i] = w.skip ? w.skip[i] : 0.0f;
  if (warp == 0) tmem_alloc(&S.tmem, TMEM_COLS);
  if (tid == 0) mbar_init(&S.bar, 1);
  fence_smem_to_async();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = S.tmem;
  const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16);
  const bool has_skip = w.skip != nullptr;
  uint32_t phase = 0;
  bool ok = true;

  // persistent over 128-path tiles: the weights are staged once per CTA
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int p = tile * TILE + row;
    const bool valid = p < B;
    float z[6] = {0, 0, 0, 0, 0, 0};
    if (group == 0 && valid)
#pragma unroll
      for (int k = 0; k < 6; ++k) z[k] = w.z[(size_t)p * 6 + k];
    double sq = 0.0;
    // inputs of the next step, loaded one step ahead so that their latency hides behind
    // the current step's layers
    float ne[6] = {0, 0, 0, 0, 0, 0}, nr[6] = {0, 0, 0, 0, 0, 0}, nt[6] = {0, 0, 0, 0, 0, 0}, nc = 0.0f;
    if (group == 0 && valid) {
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        ne[k] = w.strain[(size_t)p * 6 + k];
        nr[k] = w.rate[(size_t)p * 6 + k];
        if (w.target) nt[k] = w.target[(size_t)p * 6 + k];
      }
      nc = w.coef[p];
    }
    for (int t = 0; t < T && ok; ++t) {
      const size_t g = (size_t)t * B + p;  // (t, p) row of the window
      float e[6], tg[6];
      const float c = nc;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        e[k] = ne[k];
        tg[k] = nt[k];
      }
      if (group == 0) {
        float xin[XIN];
#pragma unroll
        for (int c2 = 0; c2 < XIN; ++c2) xin[c2] = 0.0f;
        if (valid) {
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            xin[k] = e[k];
            xin[6 + k] = nr[k];
            xin[12 + k] = z[k];
          }
        }
        if (valid && t + 1 < T) {
          const size_t gn = g + (size_t)B;
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            ne[k] = w.strain[gn * 6 + k];
            nr[k] = w.rate[gn * 6 + k];
            if (w.target) nt[k] = w.target[gn * 6 + k];
          }
          nc = w.coef[gn];
        }
#pragma unroll
        for (int c = 0; c < XIN; c += 8) put8(S.x, row, c, XIN, xin + c);
        if (w.Xt && valid) {
          __nv_bfloat16* xt = static_cast<__nv_bfloat16*>(w.Xt);
#pragma unroll
          for (int c = 0; c < XIN; ++c) xt[(size_t)c * R + g] = __float2bfloat16_rn(xin[c]);
        }
      }
      // hidden layers
      for (int l = 0; l < 3 && ok; ++l) {
        ok = run_layer(&S.bar, tmem, l == 0 ? S.x : S.h, l == 0 ? S.w1 : (l == 1 ? S.w2 : S.w3), l == 0 ? XIN : HID,
                       HID, phase);
        if (!ok) break;
        float* Zl = w.Z[l];
        __nv_bfloat16* Ht = static_cast<__nv_bfloat16*>(w.Ht[l]);
#pragma unroll 1
        for (int cb = 0; cb < GROUP_CHUNKS; ++cb) {
          const int c0 = GROUP_COLS * group + 16 * cb;
          float v[16];
          tmem_ld16(lane_addr + (uint32_t)c0, v);
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] += S.bias[l * HID + c0 + j];
          if (Zl && valid) {
            float4* dst = reinterpret_cast<float4*>(Zl + g * HID + c0);
#pragma unroll
            for (int j = 0; j < 4; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
          }
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = gelu(v[j]);
          put8(S.h, row, c0, HID, v);
          put8(S.h, row, c0 + 8, HID, v + 8);
          if (Ht && valid)
#pragma unroll
            for (int j = 0; j < 16; ++j) Ht[(size_t)(c0 + j) * R + g] = __float2bfloat16_rn(v[j]);
        }
      }
      if (!ok) break;
      // output layer and latent update
      ok = run_layer(&S.bar, tmem, S.h, S.w4, HID, YOUT, phase);
      if (!ok) break;
      if (group == 0) {
        float v[16];
        tmem_ld16(lane_addr, v);
        if (valid) {
          float s[6];
#pragma unroll
          for (int k = 0; k < 6; ++k) s[k] = v[k] + S.bias[3 * HID + k];
          if (has_skip) {
#pragma unroll
            for (int k = 0; k < 6; ++k) {
              float acc = 0.0f;
#pragma unroll
              for (int j = 0; j < 6; ++j) acc += S.skip[6 * k + j] * (e[j] - z[j]);
              s[k] += acc;
            }
          }
          if (w.stress)
#pragma unroll
            for (int k = 0; k < 6; ++k) w.stress[g * 6 + k] = s[k];
          if (w.target) {
#pragma unroll
            for (int k = 0; k < 6; ++k) {
              const float d = s[k] - tg[k];
              sq += (double)d * d;
              if (w.gS) w.gS[g * 6 + k] = w.loss_scale * 2.0f * d;
            }
          }
          float* zn = w.z + (size_t)(t + 1) * B * 6 + (size_t)p * 6;
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            z[k] = z[k] + c * (v[6 + k] + S.bias[3 * HID + 6 + k]);
            zn[k] = z[k];
          }
        }
      }
    }
    // window loss partial of this tile (first row of loss_part; the others zero)
    if (w.loss_part && ok) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
      if (lane == 0) S.red[warp] = sq;
      __syncthreads();
      if (tid == 0) {
        double tot = 0.0;
        for (int i = 0; i < RW_THREADS / 32; ++i) tot += S.red[i];
        w.loss_part[tile] = tot;
        for (int t = 1; t < T; ++t) w.loss_part[(size_t)t * ntiles + tile] = 0.0;
      }
    }
  }  // tile
  if (!ok && tid == 0 && w.err) atomicExch(w.err, 1u);
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

__global__ void __launch_bounds__(RW_THREADS, 1) rno_window_backward_kernel(const cib_rno_window w) {
  extern __shared__ uint8_t smem_raw[];
  BwdSmem& S = *reinterpret_cast<BwdSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, group = warp >> 2;
  const int row = quarter * 32 + lane;
  const int B = w.B, T = w.T;
  const int p = blockIdx.x * TILE + row;
  const bool valid = p < B;
  const size_t R = w.ldt > 0 ? (size_t)w.ldt : (size_t)B * T;

  stage_matrix(S.w4t, static_cast<const __nv_bfloat16*>(w.Wt[3]), HID, YOUT, YOUT);
  stage_matrix(S.w3t, static_cast<const __nv_bfloat16*>(w.Wt[2]), HID, HID, HID);
  stage_matrix(S.w2t, static_cast<const __nv_bfloat16*>(w.Wt[1]), HID, HID, HID);
  stage_matrix(S.w1t, static_cast<const __nv_bfloat16*>(w.Wt[0]), XIN, HID, HID);
  for (int i = tid; i < 36; i += RW_THREADS) S.skip[i] = w.skip ? w.skip[i] : 0.0f;
  if (warp == 0) tmem_alloc(&S.tmem, TMEM_COLS);
  if (tid == 0) mbar_init(&S.bar, 1);
  fence_smem_to_async();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = S.tmem;
  const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16);
  const bool has_skip = w.skip != nullptr;
  __nv_bfloat16* dYt = static_cast<__nv_bfloat16*>(w.dYt);

  float dz[6] = {0, 0, 0, 0, 0, 0};
  uint32_t phase = 0;
  bool ok = true;
  // loss gradient and coefficient of the next (earlier) step, loaded one step ahead
  float ng[6] = {0, 0, 0, 0, 0, 0}, ncf = 0.0f;
  if (group == 0 && valid) {
    const size_t gl = (size_t)(T - 1) * B + p;
#pragma unroll
    for (int k = 0; k < 6; ++k) ng[k] = w.gS[gl * 6 + k];
    ncf = w.coef[gl];
  }
  for (int t = T - 1; t >= 0 && ok; --t) {
    const size_t g = (size_t)t * B + p;
    float gs[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) gs[k] = ng[k];
    const float cf = ncf;
    if (group == 0) {
      float dy[YOUT];
#pragma unroll
      for (int c = 0; c < YOUT; ++c) dy[c] = 0.0f;
      if (valid) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          dy[k] = gs[k];
          dy[6 + k] = cf * dz[k];
        }
        if (t > 0) {
          const size_t gp = g - (size_t)B;
#pragma unroll
          for (int k = 0; k < 6; ++k) ng[k] = w.gS[gp * 6 + k];
          ncf = w.coef[gp];
        }
#pragma unroll
        for (int c2 = 0; c2 < YOUT; ++c2) dYt[(size_t)c2 * R + g] = __float2bfloat16_rn(dy[c2]);
      }
      put8(S.dy, row, 0, YOUT, dy);
      put8(S.dy, row, 8, YOUT, dy + 8);
    }
    // back through W_4, W_3, W_2 with the GELU derivative of Z_3, Z_2, Z_1
    for (int l = 2; l >= 0 && ok; --l) {
      const uint8_t* a = (l == 2) ? S.dy : S.d;
      const uint8_t* b = (l == 2) ? S.w4t : (l == 1 ? S.w3t : S.w2t);
      ok = run_layer(&S.bar, tmem, a, b, l == 2 ? YOUT : HID, HID, phase);
      if (!ok) break;
      const float* Zl = w.Z[l];
      __nv_bfloat16* dZt = static_cast<__nv_bfloat16*>(w.dZt[l]);
#pragma unroll 1
      for (int cb = 0; cb < GROUP_CHUNKS; ++cb) {
        const int c0 = GROUP_COLS * group + 16 * cb;
        float v[16];
        tmem_ld16(lane_addr + (uint32_t)c0, v);
        if (valid) {
          const float4* src = reinterpret_cast<const float4*>(Zl + g * HID + c0);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const float4 q = src[j];
            v[4 * j] = bf16r(v[4 * j] * gelu_grad(q.x));
            v[4 * j + 1] = bf16r(v[4 * j + 1] * gelu_grad(q.y));
            v[4 * j + 2] = bf16r(v[4 * j + 2] * gelu_grad(q.z));
            v[4 * j + 3] = bf16r(v[4 * j + 3] * gelu_grad(q.w));
          }
#pragma unroll
          for (int j = 0; j < 16; ++j) dZt[(size_t)(c0 + j) * R + g] = __float2bfloat16_rn(v[j]);
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = 0.0f;
        }
        put8(S.d, row, c0, HID, v);
        put8(S.d, row, c0 + 8, HID, v + 8);
      }
    }
    if (!ok) break;
    // dX = dZ_1 W_1: the latent columns 12..17 feed dz
    ok = run_layer(&S.bar, tmem, S.d, S.w1t, HID, XIN, phase);
    if (!ok) break;
    if (group == 0) {
      float v0[16], v1[16];
      tmem_ld16(lane_addr, v0);
      tmem_ld16(lane_addr + 16u, v1);
      if (valid) {
        const float dx[6] = {v0[12], v0[13], v0[14], v0[15], v1[0], v1[1]};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          float sk = 0.0f;
          if (has_skip)
#pragma unroll
            for (int j = 0; j < 6; ++j) sk += S.skip[6 * j + k] * gs[j];
          dz[k] = dz[k] + dx[k] - sk;
        }
      }
    }
  }
  if (!ok && tid == 0 && w.err) atomicExch(w.err, 1u);
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------------------
// Inference step (T = 1, nothing saved for a backward pass) over many tiles: the CTA's two
// halves of 8 warps each run their own 128-path tile with their own operand tiles, TMEM
// columns, mbarrier and named barrier, so that one half's bias/GELU epilogue overlaps the
// other half's tensor-core layer instead of every warp waiting on each MMA.  The weights are
// staged once per CTA and shared.  Same arithmetic per path as rno_window_forward_kernel
// (the same results bit for bit).
constexpr int INF_HALF = RW_THREADS / 2;       // threads of a half
constexpr int INF_GROUP_COLS = 64;             // epilogue columns per warp (2 groups per quarter)

struct __align__(1024) InfSmem {
  uint8_t w1[HID * XIN * 2];
  uint8_t w2[HID * HID * 2];
  uint8_t w3[HID * HID * 2];
  uint8_t w4[YOUT * HID * 2];
  uint8_t x[2][TILE * XIN * 2];
  uint8_t h[2][TILE * HID * 2];
  float bias[3 * HID + YOUT];
  float skip[36];
  uint64_t bar[2];
  uint32_t tmem;
};

// Named barrier of one half (ids 1 and 2; 0 is __syncthreads).
__device__ __forceinline__ void half_sync(int id) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(INF_HALF) : "memory");
}
// Same, returning whether any thread of the half passed a true flag.
__device__ __forceinline__ bool half_sync_or(int id, bool flag) {
  uint32_t out;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(out)
      : "r"((uint32_t)flag), "r"(id), "n"(INF_HALF)
      : "memory");
  return out != 0;
}

// run_layer for one half: its first thread issues, the half waits on its own mbarrier.
__device__ __forceinline__ bool run_layer_half(uint64_t* bar, uint32_t tmem, const uint8_t* a, const uint8_t* b, int k,
                                               int n, uint32_t& phase, int id, bool issuer) {
  fence_smem_to_async();
  fence_before_sync();
  half_sync(id);
  if (issuer) {
    fence_after_sync();
    mma_bf16(tmem, smem_u32(a), smem_u32(b), k, n, false, bar);
  }
  const bool ok = mbar_wait(bar, phase);
  phase ^= 1u;
  fence_after_sync();
  return !half_sync_or(id, !ok);
}

__global__ void __launch_bounds__(RW_THREADS, 1) rno_infer_kernel(const cib_rno_window w) {
  extern __shared__ uint8_t smem_raw[];
  InfSmem& S = *reinterpret_cast<InfSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int half = warp >> 3, quarter = warp & 3, group = (warp >> 2) & 1;
  const int row = quarter * 32 + lane;
  const int bar_id = 1 + half;
  const bool issuer = (tid & (INF_HALF - 1)) == 0;
  const int B = w.B;
  const int ntiles = (B + TILE - 1) / TILE;

  stage_matrix(S.w1, static_cast<const __nv_bfloat16*>(w.W[0]), HID, XIN, XIN);
  stage_matrix(S.w2, static_cast<const __nv_bfloat16*>(w.W[1]), HID, HID, HID);
  stage_matrix(S.w3, static_cast<const __nv_bfloat16*>(w.W[2]), HID, HID, HID);
  stage_matrix(S.w4, static_cast<const __nv_bfloat16*>(w.W[3]), YOUT, HID, HID);
  for (int i = tid; i < 3 * HID + YOUT; i += RW_THREADS) S.bias[i] = w.bias[i / HID < 3 ? i / HID : 3][i % HID];
  for (int i = tid; i < 36; i += RW_THREADS) S.skip[i] = w.skip ? w.skip[i] : 0.0f;
  if (warp == 0) tmem_alloc(&S.tmem, 2 * TMEM_COLS);
  if (tid == 0) {
    mbar_init(&S.bar[0], 1);
    mbar_init(&S.bar[1], 1);
  }
  fence_smem_to_async();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = S.tmem + (uint32_t)(half * TMEM_COLS);
  const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16);
  const bool has_skip = w.skip != nullptr;
  uint8_t* xs = S.x[half];
  uint8_t* hs = S.h[half];
  uint64_t* bar = &S.bar[half];
  uint32_t phase = 0;
  bool ok = true;

  for (int tile = 2 * blockIdx.x + half; tile < ntiles && ok; tile += 2 * gridDim.x) {
    const int p = tile * TILE + row;
    const bool valid = p < B;
    float z[6] = {0, 0, 0, 0, 0, 0}, e[6] = {0, 0, 0, 0, 0, 0};
    float c = 0.0f;
    if (group == 0) {
      float xin[XIN];
#pragma unroll
      for (int c2 = 0; c2 < XIN; ++c2) xin[c2] = 0.0f;
      if (valid) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          z[k] = w.z[(size_t)p * 6 + k];
          e[k] = w.strain[(size_t)p * 6 + k];
          xin[k] = e[k];
          xin[6 + k] = w.rate[(size_t)p * 6 + k];
          xin[12 + k] = z[k];
        }
        c = w.coef[p];
      }
#pragma unroll
      for (int c2 = 0; c2 < XIN; c2 += 8) put8(xs, row, c2, XIN, xin + c2);
    }
    for (int l = 0; l < 3 && ok; ++l) {
      ok = run_layer_half(bar, tmem, l == 0 ? xs : hs, l == 0 ? S.w1 : (l == 1 ? S.w2 : S.w3), l == 0 ? XIN : HID,
                          HID, phase, bar_id, issuer);
      if (!ok) break;
#pragma unroll 1
      for (int cb = 0; cb < INF_GROUP_COLS / 16; ++cb) {
        const int c0 = INF_GROUP_COLS * group + 16 * cb;
        float v[16];
        tmem_ld16(lane_addr + (uint32_t)c0, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = gelu(v[j] + S.bias[l * HID + c0 + j]);
        put8(hs, row, c0, HID, v);
        put8(hs, row, c0 + 8, HID, v + 8);
      }
    }
    if (!ok) break;
    ok = run_layer_half(bar, tmem, hs, S.w4, HID, YOUT, phase, bar_id, issuer);
    if (!ok) break;
    if (group == 0) {
      float v[16];
      tmem_ld16(lane_addr, v);
      if (valid) {
        float s[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) s[k] = v[k] + S.bias[3 * HID + k];
        if (has_skip) {
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            float acc = 0.0f;
#pragma unroll
            for (int j = 0; j < 6; ++j) acc += S.skip[6 * k + j] * (e[j] - z[j]);
            s[k] += acc;
          }
        }
        if (w.stress)
#pragma unroll
          for (int k = 0; k < 6; ++k) w.stress[(size_t)p * 6 + k] = s[k];
        float* zn = w.z + (size_t)B * 6 + (size_t)p * 6;
#pragma unroll
        for (int k = 0; k < 6; ++k) zn[k] = z[k] + c * (v[6 + k] + S.bias[3 * HID + 6 + k]);
      }
    }
  }
  if (!ok && issuer && w.err) atomicExch(w.err, 1u);
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(S.tmem, 2 * TMEM_COLS);
  }
}

// The dynamic shared-memory limit is raised once per device and kernel (so that launches
// recorded into a CUDA graph make no attribute call).
int validate_common(const cib_rno_window* w) {
  if (!w || w->B < 0 || w->T < 1 || w->hidden != HID || !w->strain || !w->rate || !w->coef || !w->z || !w->err)
    return CIB_EINVAL;
  if (w->ldt != 0 && w->ldt < (int64_t)w->B * w->T) return CIB_EINVAL;
  return CIB_OK;
}

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" int cib_rno_window_forward(const cib_rno_window* w, void* stream) {
  if (validate_common(w) != CIB_OK) return CIB_EINVAL;
  for (int l = 0; l < 4; ++l)
    if (!w->W[l] || !aligned16(w->W[l]) || !w->bias[l]) return CIB_EINVAL;
  for (int l = 0; l < 3; ++l)
    if (w->Z[l] && !aligned16(w->Z[l])) return CIB_EINVAL;
  if (w->gS && !w->target) return CIB_EINVAL;
  if (w->B == 0) return CIB_OK;
  const int64_t ntiles = (w->B + TILE - 1) / TILE;
  bool saves = w->target || w->gS || w->loss_part || w->Xt;
  for (int l = 0; l < 3; ++l) saves = saves || w->Z[l] || w->Ht[l];
  if (w->T == 1 && !saves && ntiles >= 2 * (int64_t)sm_count()) {
    // inference over at least two tiles per SM: two tiles in flight per CTA
    const size_t ibytes = sizeof(InfSmem);
    if (allow_dynamic_smem(reinterpret_cast<const void*>(rno_infer_kernel), (int)ibytes) != CIB_OK) return CIB_ECUDA;
    const unsigned igrid = (unsigned)std::min<int64_t>((ntiles + 1) / 2, sm_count());
    rno_infer_kernel<<<igrid, RW_THREADS, ibytes, reinterpret_cast<cudaStream_t>(stream)>>>(*w);
    return check_launch();
  }
  const size_t bytes = sizeof(FwdSmem);
  if (allow_dynamic_smem(reinterpret_cast<const void*>(rno_window_forward_kernel), (int)bytes) != CIB_OK)
    return CIB_ECUDA;
  // one CTA per SM (the staged weights fill most of its shared memory), each looping over tiles
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, sm_count());
  rno_window_forward_kernel<<<grid, RW_THREADS, bytes, reinterpret_cast<cudaStream_t>(stream)>>>(*w);
  return check_launch();
}

extern "C" int cib_rno_window_backward(const cib_rno_window* w, void* stream) {
  if (validate_common(w) != CIB_OK) return CIB_EINVAL;
  for (int l = 0; l < 4; ++l)
    if (!w->Wt[l] || !aligned16(w->Wt[l])) return CIB_EINVAL;
  for (int l = 0; l < 3; ++l)
    if (!w->Z[l] || !aligned16(w->Z[l]) || !w->dZt[l]) return CIB_EINVAL;
  if (!w->gS || !w->dYt) return CIB_EINVAL;
  if (w->B == 0) return CIB_OK;
  const size_t bytes = sizeof(BwdSmem);
  if (allow_dynamic_smem(reinterpret_cast<const void*>(rno_window_backward_kernel), (int)bytes) != CIB_OK)
    return CIB_ECUDA;
  const unsigned grid = (unsigned)((w->B + TILE - 1) / TILE);
  rno_window_backward_kernel<<<grid, RW_THREADS, bytes, reinterpret_cast<cudaStream_t>(stream)>>>(*w);
  return check_launch();
}
