// Elementwise kernels of the recurrent material surrogate (RNO) around the tensor-core
// GEMMs of mlp.cu: input assembly, latent update and stress loss, the backward recurrence
// through the latent state, bias-gradient row sums and the Adam update with bf16 refresh.
//
// Network (one time step, B paths): x = [strain (6), strain rate (6), latent z (6)] padded
// to 32 bf16 columns -> 128 -> 128 -> 128 (GELU) -> 16 (first 6 = normalised stress,
// next 6 = latent rate); z' = z + c * zdot with c = dt / tau_ref per path.  The latent
// update restates the forward-Euler latent step of the reference surrogate
// (src/concrete_impact/nn/models/rve_rno.py:383-387).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cib_common.cuh"

namespace cib {
namespace {

constexpr int RNO_IN = 32;
constexpr int RNO_OUT = 16;

__global__ void rno_input_kernel(int B, const float* __restrict__ strain, const float* __restrict__ rate,
                                 const float* __restrict__ z, __nv_bfloat16* __restrict__ X,
                                 __nv_bfloat16* __restrict__ Xt, int ldxt, int row_offset) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * RNO_IN) return;
  const int p = i / RNO_IN, c = i % RNO_IN;
  float v = 0.0f;
  if (c < 6) v = strain[6 * p + c];
  else if (c < 12) v = rate[6 * p + c - 6];
  else if (c < 18) v = z[6 * p + c - 12];
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  X[(size_t)p * RNO_IN + c] = h;
  if (Xt) Xt[(size_t)c * ldxt + row_offset + p] = h;
}

// z_next = z + coef * Y[:, 6:12]; gY = loss_scale * 2 (Y[:, 0:6] - target); per-block loss
// partial sums of (Y - target)^2 into loss_part[blockIdx.x].
__global__ void rno_forward_tail_kernel(int B, const float* __restrict__ Y, const float* __restrict__ target,
                                        const float* __restrict__ coef, const float* __restrict__ z,
                                        float* __restrict__ z_next, float* __restrict__ gY, float loss_scale,
                                        double* __restrict__ loss_part) {
  __shared__ double red[256];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  double se = 0.0;
  if (p < B) {
    const float c = coef[p];
#pragma unroll
    for (int k = 0; k < 6; ++k) z_next[6 * p + k] = z[6 * p + k] + c * Y[(size_t)p * RNO_OUT + 6 + k];
    if (target) {
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const float d = Y[(size_t)p * RNO_OUT + k] - target[6 * p + k];
        se += (double)d * d;
        if (gY) gY[6 * p + k] = loss_scale * 2.0f * d;
      }
    }
  }
  red[threadIdx.x] = se;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0 && loss_part) loss_part[blockIdx.x] = red[0];
}

// dY = [gY (6), coef * dz_next (6), 0 (4)] as bf16 rows, plus its transpose.
__global__ void rno_backward_head_kernel(int B, const float* __restrict__ gY, const float* __restrict__ coef,
                                         const float* __restrict__ dz_next, __nv_bfloat16* __restrict__ dY,
                                         __nv_bfloat16* __restrict__ dYt, int lddyt, int row_offset) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * RNO_OUT) return;
  const int p = i / RNO_OUT, c = i % RNO_OUT;
  float v = 0.0f;
  if (c < 6) v = gY[6 * p + c];
  else if (c < 12) v = coef[p] * dz_next[6 * p + c - 6];
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  dY[(size_t)p * RNO_OUT + c] = h;
  if (dYt) dYt[(size_t)c * lddyt + row_offset + p] = h;
}

// dz = dz_next + dX[:, 12:18]  (z enters the next step directly and the network input)
__global__ void rno_backward_tail_kernel(int B, const float* __restrict__ dz_next, const float* __restrict__ dX,
                                         float* __restrict__ dz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * 6) return;
  const int p = i / 6, k = i % 6;
  dz[i] = dz_next[i] + dX[(size_t)p * RNO_IN + 12 + k];
}

// out[n] = sum_r X[n * ld + r] for r < R (bf16 in, fp32/fp64 accumulation, fixed order)
__global__ void row_sum_bf16_kernel(int R, const __nv_bfloat16* __restrict__ X, int ld, float* __restrict__ out) {
  __shared__ double red[256];
  const int n = blockIdx.x;
  double s = 0.0;
  for (int r = threadIdx.x; r < R; r += blockDim.x) s += (double)__bfloat162float(X[(size_t)n * ld + r]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = (float)red[0];
}

// Adam (bias-corrected) on fp32 master weights w (rows x cols, row-major), then the bf16
// copy Wb (rows x ldb) and its transpose Wt (cols x ldt) when given.
__global__ void adam_kernel(int rows, int cols, float* __restrict__ w, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                            const int* __restrict__ step, __nv_bfloat16* __restrict__ Wb, int ldb,
                            __nv_bfloat16* __restrict__ Wt, int ldt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const float t = (float)(*step);
  const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  const int r = i / cols, c = i % cols;
  const __nv_bfloat16 h = __float2bfloat16_rn(wi);
  if (Wb) Wb[(size_t)r * ldb + c] = h;
  if (Wt) Wt[(size_t)c * ldt + r] = h;
}

__global__ void counter_increment_kernel(int* counter) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *counter += 1;
}

inline unsigned nblk(int n, int t) { return (unsigned)((n + t - 1) / t); }

// The elementwise kernels index with 32-bit ints: sizes whose element count (rows x
// components) would not fit are refused with CIB_ERANGE before anything is launched.
inline bool fits_int32(int64_t a, int64_t b) { return a * b <= (int64_t)INT32_MAX - 256; }

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" int cib_rno_input(int32_t B, const float* strain, const float* rate, const float* z, void* X, void* Xt,
                             int32_t ldxt, int32_t row_offset, void* stream) {
  if (B < 0 || !strain || !rate || !z || !X) return CIB_EINVAL;
  if (!fits_int32(B, RNO_IN)) return CIB_ERANGE;
  if (B == 0) return CIB_OK;
  rno_input_kernel<<<nblk(B * RNO_IN, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      B, strain, rate, z, static_cast<__nv_bfloat16*>(X), static_cast<__nv_bfloat16*>(Xt), ldxt, row_offset);
  return check_launch();
}

extern "C" int cib_rno_forward_tail(int32_t B, const float* Y, const float* target, const float* coef, const float* z,
                                    float* z_next, float* gY, float loss_scale, double* loss_part, void* stream) {
  if (B < 0 || !Y || !coef || !z || !z_next) return CIB_EINVAL;
  if (!fits_int32(B, RNO_OUT)) return CIB_ERANGE;
  if (B == 0) return CIB_OK;
  rno_forward_tail_kernel<<<nblk(B, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      B, Y, target, coef, z, z_next, gY, loss_scale, loss_part);
  return check_launch();
}

extern "C" int cib_rno_backward_head(int32_t B, const float* gY, const float* coef, const float* dz_next, void* dY,
                                     void* dYt, int32_t lddyt, int32_t row_offset, void* stream) {
  if (B < 0 || !gY || !coef || !dz_next || !dY) return CIB_EINVAL;
  if (!fits_int32(B, RNO_OUT)) return CIB_ERANGE;
  if (B == 0) return CIB_OK;
  rno_backward_head_kernel<<<nblk(B * RNO_OUT, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      B, gY, coef, dz_next, static_cast<__nv_bfloat16*>(dY), static_cast<__nv_bfloat16*>(dYt), lddyt, row_offset);
  return check_launch();
}

extern "C" int cib_rno_backward_tail(int32_t B, const float* dz_next, const float* dX, float* dz, void* stream) {
  if (B < 0 || !dz_next || !dX || !dz) return CIB_EINVAL;
  if (!fits_int32(B, RNO_IN)) return CIB_ERANGE;
  if (B == 0) return CIB_OK;
  rno_backward_tail_kernel<<<nblk(B * 6, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(B, dz_next, dX, dz);
  return check_launch();
}

extern "C" int cib_row_sum_bf16(int32_t rows, int32_t R, const void* X, int32_t ld, float* out, void* stream) {
  if (rows < 0 || R < 0 || !X || !out || ld < R) return CIB_EINVAL;
  if (rows == 0) return CIB_OK;
  row_sum_bf16_kernel<<<rows, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      R, static_cast<const __nv_bfloat16*>(X), ld, out);
  return check_launch();
}

extern "C" int cib_adam_step(int32_t rows, int32_t cols, float* w, const float* g, float* m, float* v, float lr,
                             float beta1, float beta2, float eps, const int32_t* step, void* Wb, int32_t ldb, void* Wt,
                             int32_t ldt, void* stream) {
  if (rows < 0 || cols < 0 || !w || !g || !m || !v || !step) return CIB_EINVAL;
  if (!fits_int32(rows, cols)) return CIB_ERANGE;
  if ((int64_t)rows * cols == 0) return CIB_OK;
  adam_kernel<<<nblk(rows * cols, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      rows, cols, w, g, m, v, lr, beta1, beta2, eps, step, static_cast<__nv_bfloat16*>(Wb), ldb,
      static_cast<__nv_bfloat16*>(Wt), ldt);
  return check_launch();
}

extern "C" int cib_counter_increment(int32_t* counter, void* stream) {
  if (!counter) return CIB_EINVAL;
  counter_increment_kernel<<<1, 32, 0, reinterpret_cast<cudaStream_t>(stream)>>>(counter);
  return check_launch();
}
