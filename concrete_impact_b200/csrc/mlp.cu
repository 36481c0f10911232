// Tensor-core (tcgen05) BF16 GEMM with fused MLP epilogues, and the elementwise kernels of
// the recurrent material surrogate (sm_100a).
//
// C[M x N] = A[M x K] . B[N x K]^T with A, B bf16 row-major (K contiguous), fp32 accumulation
// in tensor memory.  One CTA computes a 128-row tile over the full N (16..128, multiple of
// 16) and a K range (split-K over gridDim.y).  Operands are staged in shared memory in the
// K-major, no-swizzle canonical layout of tcgen05 (8-row x 16-byte core matrices) by
// cp.async through a three-slot pipeline, so that the copies of the next two K chunks
// overlap the MMA of the current one; one elected thread issues tcgen05.mma (M = 128, N,
// K = 16 per instruction) and commits each chunk to its slot's mbarrier; every wait is
// bounded in time and reports through an error word.  The epilogue
// reads the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows)
// and applies one of:
//   EPI_F32        C = acc                                   (fp32 out)
//   EPI_BIAS_F32   C = acc + bias                            (fp32 out; output layer)
//   EPI_BIAS_GELU  Z = acc + bias (fp32, optional), H = gelu(Z) (bf16), optional H^T (bf16)
//   EPI_GELU_BWD   dZ = acc * gelu'(Z) (bf16), optional dZ^T (bf16)
//   EPI_PARTIAL    fp32 partial of this K slice, reduced later in a fixed order
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cib_common.cuh"
#include "umma.cuh"

namespace cib {
namespace {

constexpr int GEMM_THREADS = 128;
constexpr int KC = 64;  // K elements staged per chunk
constexpr int GEMM_STAGES = 3;  // shared-memory slots of the copy/MMA pipeline

enum Epi { EPI_F32 = 0, EPI_BIAS_F32 = 1, EPI_BIAS_GELU = 2, EPI_GELU_BWD = 3, EPI_PARTIAL = 4 };

struct GemmArgs {
  int M, N, K;
  int lda, ldb;
  const __nv_bfloat16* A;
  const __nv_bfloat16* B;
  int k_per_split;     // K elements per gridDim.y slice (multiple of 16)
  // epilogue operands
  const float* bias;   // N
  float* C;            // fp32 out, ldc
  int ldc;
  float* Z;            // pre-activation fp32 (EPI_BIAS_GELU out / EPI_GELU_BWD in), ld = ldz
  int ldz;
  __nv_bfloat16* H;    // bf16 activation out, ld = ldh
  int ldh;
  __nv_bfloat16* Ht;   // optional transposed bf16 out: Ht[n * ldht + row_offset + m]
  int ldht;
  int row_offset;      // row index of this GEMM's row 0 inside the transposed buffer
  unsigned int* err;   // set to 1 when a wait times out
  int vec4;            // fp32 outputs: C 16-byte aligned and ldc a multiple of 4
};

using namespace umma;

// 16-byte asynchronous global->shared copy; src_bytes 0 fills the 16 bytes with zeros.
__device__ __forceinline__ void cp_async16(uint8_t* dst, const void* src, bool pred) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(pred ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

struct __align__(1024) GemmSmem {
  uint8_t a[GEMM_STAGES][128 * KC * 2];
  uint8_t b[GEMM_STAGES][128 * KC * 2];
  uint64_t bar[GEMM_STAGES];
  uint32_t tmem_base;
};

template <int EPI>
__global__ void __launch_bounds__(GEMM_THREADS) umma_gemm_kernel(const GemmArgs a) {
  extern __shared__ uint8_t smem_raw[];
  GemmSmem& S = *reinterpret_cast<GemmSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * 128;
  const int k_begin = blockIdx.y * a.k_per_split;
  const int k_end = min(a.K, k_begin + a.k_per_split);
  const int chunks = k_end > k_begin ? (k_end - k_begin + KC - 1) / KC : 0;
  const uint32_t ncols = a.N <= 32 ? 32u : (a.N <= 64 ? 64u : 128u);
  if (warp == 0) tmem_alloc(&S.tmem_base, ncols);
  if (tid == 0)
    for (int s = 0; s < GEMM_STAGES; ++s) mbar_init(&S.bar[s], 1);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = S.tmem_base;
  const uint32_t idesc = idesc_bf16(a.N);

  // stage chunk i (A: 128 x KC, B: N x KC) into slot st with cp.async, zero-filled outside
  // the matrices and the K range
  auto load_chunk = [&](int i, int st) {
    const int k0 = k_begin + i * KC;
    for (int v = tid; v < 128 * (KC / 8); v += GEMM_THREADS) {
      const int r = v / (KC / 8), c = (v % (KC / 8)) * 8;
      const bool in = m0 + r < a.M && k0 + c < k_end;
      cp_async16(S.a[st] + core_offset(r, c, KC), in ? a.A + (size_t)(m0 + r) * a.lda + k0 + c : a.A, in);
    }
    for (int v = tid; v < a.N * (KC / 8); v += GEMM_THREADS) {
      const int r = v / (KC / 8), c = (v % (KC / 8)) * 8;
      const bool in = k0 + c < k_end;
      cp_async16(S.b[st] + core_offset(r, c, KC), in ? a.B + (size_t)r * a.ldb + k0 + c : a.B, in);
    }
  };

  // Pipeline: GEMM_STAGES - 1 chunks in flight ahead of the MMA.  Chunk i lands in slot
  // i % GEMM_STAGES; the slot is refilled (with chunk i + GEMM_STAGES - 1) once the MMA of
  // chunk i - 1 that read it has completed, while the MMA of chunk i runs.
#pragma unroll
  for (int s = 0; s < GEMM_STAGES - 1; ++s) {
    if (s < chunks) load_chunk(s, s);
    cp_async_commit();
  }
  bool failed = false;
  for (int i = 0; i < chunks; ++i) {
    const int st = i % GEMM_STAGES;
    cp_async_wait<GEMM_STAGES - 2>();  // chunk i's group has landed (this thread's copies)
    fence_smem_to_async();
    __syncthreads();  // ... and every thread's
    if (tid == 0) {
      fence_after_sync();
      const int steps = min(KC, k_end - (k_begin + i * KC)) / 16;
      const uint32_t a0 = smem_u32(S.a[st]), b0 = smem_u32(S.b[st]);
      for (int s = 0; s < steps; ++s) {
        const uint64_t da = sdesc(a0 + 256 * s, 128, KC * 16);
        const uint64_t db = sdesc(b0 + 256 * s, 128, KC * 16);
        const uint32_t acc = (i > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&S.bar[st]))
                   : "memory");
    }
    const int j = i + GEMM_STAGES - 1;
    if (j < chunks) {
      if (i >= 1) {
        const int prev = i - 1;
        const bool ok = mbar_wait(&S.bar[prev % GEMM_STAGES], (uint32_t)((prev / GEMM_STAGES) & 1));
        if (__syncthreads_or(ok ? 0 : 1)) {
          failed = true;
          break;
        }
      }
      load_chunk(j, j % GEMM_STAGES);
    }
    cp_async_commit();
  }
  // the last commit covers every MMA issued before it
  if (!failed && chunks > 0) {
    const int last = chunks - 1;
    const bool ok = mbar_wait(&S.bar[last % GEMM_STAGES], (uint32_t)((last / GEMM_STAGES) & 1));
    failed = __syncthreads_or(ok ? 0 : 1) != 0;
  }
  cp_async_wait<0>();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (failed) {
    if (tid == 0 && a.err) atomicExch(a.err, 1u);
  } else {
    const int m = m0 + warp * 32 + lane;
    for (int cb = 0; cb < a.N / 16; ++cb) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16);
      if (chunks == 0) {
#pragma unroll
        for (int j = 0; j < 16; ++j) r[j] = 0u;
      } else {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
            "%15}, [%16];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      }
      const bool f32_out = EPI == EPI_F32 || EPI == EPI_BIAS_F32 || EPI == EPI_PARTIAL;
      if (f32_out && a.vec4 && m < a.M) {
        // fp32 rows as four 16-byte stores per 16 columns
        float* dst = a.C + ((EPI == EPI_PARTIAL ? (size_t)blockIdx.y * a.M : 0) + m) * a.ldc + cb * 16;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float4 v = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]), __uint_as_float(r[4 * q + 2]),
                                 __uint_as_float(r[4 * q + 3]));
          if (EPI == EPI_BIAS_F32) {
            const int n = cb * 16 + 4 * q;
            v.x += a.bias[n];
            v.y += a.bias[n + 1];
            v.z += a.bias[n + 2];
            v.w += a.bias[n + 3];
          }
          reinterpret_cast<float4*>(dst)[q] = v;
        }
      } else if (m < a.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = cb * 16 + j;
          const float acc = __uint_as_float(r[j]);
          if (EPI == EPI_F32) {
            a.C[(size_t)m * a.ldc + n] = acc;
          } else if (EPI == EPI_BIAS_F32) {
            a.C[(size_t)m * a.ldc + n] = acc + a.bias[n];
          } else if (EPI == EPI_BIAS_GELU) {
            const float z = acc + a.bias[n];
            if (a.Z) a.Z[(size_t)m * a.ldz + n] = z;
            const __nv_bfloat16 h = __float2bfloat16_rn(gelu(z));
            a.H[(size_t)m * a.ldh + n] = h;
            if (a.Ht) a.Ht[(size_t)n * a.ldht + a.row_offset + m] = h;
          } else if (EPI == EPI_GELU_BWD) {
            const float dz = acc * gelu_grad(a.Z[(size_t)m * a.ldz + n]);
            const __nv_bfloat16 h = __float2bfloat16_rn(dz);
            a.H[(size_t)m * a.ldh + n] = h;
            if (a.Ht) a.Ht[(size_t)n * a.ldht + a.row_offset + m] = h;
          } else {  // EPI_PARTIAL
            a.C[((size_t)blockIdx.y * a.M + m) * a.ldc + n] = acc;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

// out[m * ldo + n] = sum over s of partial[(s * M + m) * ldc + n]  (fixed order)
__global__ void splitk_reduce_kernel(int M, int N, int splits, const float* __restrict__ partial, int ldc,
                                     float* __restrict__ out, int ldo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M * N) return;
  const int m = i / N, n = i % N;
  float s = 0.0f;
  for (int k = 0; k < splits; ++k) s += partial[((size_t)k * M + m) * ldc + n];
  out[(size_t)m * ldo + n] = s;
}

}  // namespace
}  // namespace cib

using namespace cib;

extern "C" int cib_mlp_gemm(int32_t epilogue, int32_t M, int32_t N, int32_t K, const void* A, int32_t lda,
                            const void* B, int32_t ldb, int32_t splits, const float* bias, float* C, int32_t ldc,
                            float* Z, int32_t ldz, void* H, int32_t ldh, void* Ht, int32_t ldht, int32_t row_offset,
                            unsigned int* err, void* stream) {
  if (M < 0 || N < 16 || N > 128 || (N % 16) != 0 || K < 16 || (K % 16) != 0 || !A || !B || lda < K || ldb < K ||
      (lda % 8) != 0 || (ldb % 8) != 0 || !aligned16(A) || !aligned16(B) || splits < 1 || !err)
    return CIB_EINVAL;
  if (M == 0) return CIB_OK;
  GemmArgs a;
  a.M = M;
  a.N = N;
  a.K = K;
  a.lda = lda;
  a.ldb = ldb;
  a.A = static_cast<const __nv_bfloat16*>(A);
  a.B = static_cast<const __nv_bfloat16*>(B);
  int per = (K + splits - 1) / splits;
  per = ((per + KC - 1) / KC) * KC;
  a.k_per_split = per;
  const int ny = (K + per - 1) / per;
  a.bias = bias;
  a.C = C;
  a.ldc = ldc;
  a.Z = Z;
  a.ldz = ldz;
  a.H = static_cast<__nv_bfloat16*>(H);
  a.ldh = ldh;
  a.Ht = static_cast<__nv_bfloat16*>(Ht);
  a.ldht = ldht;
  a.row_offset = row_offset;
  a.err = err;
  a.vec4 = (C != nullptr && aligned16(C) && (ldc % 4) == 0) ? 1 : 0;
  switch (epilogue) {
    case EPI_F32:
    case EPI_BIAS_F32:
      if (!C || (epilogue == EPI_BIAS_F32 && !bias) || ny != 1) return CIB_EINVAL;
      break;
    case EPI_BIAS_GELU:
      if (!bias || !H || ny != 1) return CIB_EINVAL;
      break;
    case EPI_GELU_BWD:
      if (!Z || !H || ny != 1) return CIB_EINVAL;
      break;
    case EPI_PARTIAL:
      if (!C) return CIB_EINVAL;
      break;
    default:
      return CIB_EINVAL;
  }
  const dim3 grid((unsigned)((M + 127) / 128), (unsigned)ny);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int bytes = (int)sizeof(GemmSmem);
  const void* kernels[5] = {reinterpret_cast<const void*>(umma_gemm_kernel<EPI_F32>),
                            reinterpret_cast<const void*>(umma_gemm_kernel<EPI_BIAS_F32>),
                            reinterpret_cast<const void*>(umma_gemm_kernel<EPI_BIAS_GELU>),
                            reinterpret_cast<const void*>(umma_gemm_kernel<EPI_GELU_BWD>),
                            reinterpret_cast<const void*>(umma_gemm_kernel<EPI_PARTIAL>)};
  if (allow_dynamic_smem(kernels[epilogue], bytes) != CIB_OK) return CIB_ECUDA;
  switch (epilogue) {
    case EPI_F32: umma_gemm_kernel<EPI_F32><<<grid, GEMM_THREADS, bytes, st>>>(a); break;
    case EPI_BIAS_F32: umma_gemm_kernel<EPI_BIAS_F32><<<grid, GEMM_THREADS, bytes, st>>>(a); break;
    case EPI_BIAS_GELU: umma_gemm_kernel<EPI_BIAS_GELU><<<grid, GEMM_THREADS, bytes, st>>>(a); break;
    case EPI_GELU_BWD: umma_gemm_kernel<EPI_GELU_BWD><<<grid, GEMM_THREADS, bytes, st>>>(a); break;
    default: umma_gemm_kernel<EPI_PARTIAL><<<grid, GEMM_THREADS, bytes, st>>>(a); break;
  }
  return check_launch();
}

extern "C" int cib_splitk_reduce(int32_t M, int32_t N, int32_t splits, const float* partial, int32_t ldc, float* out,
                                 int32_t ldo, void* stream) {
  if (M < 0 || N < 0 || splits < 1 || !partial || !out) return CIB_EINVAL;
  if ((int64_t)M * N > (int64_t)INT32_MAX - 256) return CIB_ERANGE;  // 32-bit element index
  if ((int64_t)M * N == 0) return CIB_OK;
  const int threads = 256;
  splitk_reduce_kernel<<<(M * N + threads - 1) / threads, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      M, N, splits, partial, ldc, out, ldo);
  return check_launch();
}
