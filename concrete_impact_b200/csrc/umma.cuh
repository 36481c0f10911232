// tcgen05 (5th-generation tensor core) helpers shared by the GEMM and the fused recurrent
// surrogate kernels (sm_100a): shared-memory operand layout and descriptors, the BF16
// instruction descriptor, single-thread MMA issue with mbarrier commit, bounded mbarrier
// waits, TMEM allocation and 32x32b loads, and the GELU pair used by the MLP epilogues.
//
// Operand layout: K-major, no swizzle, 8-row x 16-byte core matrices.  Element (r, c) of a
// tile with K columns sits at byte ((r / 8) * (K / 8) + c / 8) * 128 + (r % 8) * 16 +
// (c % 8) * 2; the descriptor's leading byte offset is 128 (next core matrix along K) and
// its stride byte offset K * 16 (next 8-row group).  One MMA instruction consumes K = 16,
// i.e. two core matrices along K: step s starts 256 * s bytes into the tile.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace cib {
namespace umma {

constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;  // 2 s bound on every mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t core_offset(int r, int c, int k) {
  return (uint32_t)((((r >> 3) * (k >> 3)) + (c >> 3)) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// Shared-memory matrix descriptor: start address, leading byte offset, stride byte offset,
// descriptor version 1 (bit 46), no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D f32, A and B bf16, both K-major, M = 128, N.
__device__ __forceinline__ uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Waits for the phase with the given parity; false after WAIT_LIMIT_NS.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const uint64_t t0 = now_ns();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (now_ns() - t0 > WAIT_LIMIT_NS) return false;
  }
}

// Warp-wide: allocate ncols TMEM columns (power of two >= 32), address into *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One thread: D[tmem] (+)= A(smem, K = 16 * steps) . B(smem)^T, then commit to the mbarrier.
__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint32_t a_base, uint32_t b_base, int k, int n,
                                         bool accumulate, uint64_t* bar) {
  const uint32_t idesc = idesc_bf16(n);
  const int steps = k / 16;
  for (int s = 0; s < steps; ++s) {
    const uint64_t da = sdesc(a_base + 256 * s, 128, (uint32_t)k * 16);
    const uint64_t db = sdesc(b_base + 256 * s, 128, (uint32_t)k * 16);
    const uint32_t acc = (accumulate || s > 0) ? 1u : 0u;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
  }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane (warp w reads lanes 32 (w % 4) ..).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// Copy a row-major bf16 matrix (rows x k, leading dimension ld) into the canonical layout.
// Each thread issues four 16-byte loads before its stores, so that the copy waits on the
// memory latency once per four chunks instead of once per chunk.
__device__ __forceinline__ void stage_matrix(uint8_t* dst, const __nv_bfloat16* src, int rows, int k, int ld) {
  constexpr int U = 4;
  const int chunks = k / 8, total = rows * chunks;
  for (int base = threadIdx.x; base < total; base += U * blockDim.x) {
    uint4 q[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int v = base + u * (int)blockDim.x;
      if (v < total) q[u] = *reinterpret_cast<const uint4*>(src + (size_t)(v / chunks) * ld + (v % chunks) * 8);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int v = base + u * (int)blockDim.x;
      if (v < total) *reinterpret_cast<uint4*>(dst + core_offset(v / chunks, (v % chunks) * 8, k)) = q[u];
    }
  }
}

}  // namespace umma
}  // namespace cib
