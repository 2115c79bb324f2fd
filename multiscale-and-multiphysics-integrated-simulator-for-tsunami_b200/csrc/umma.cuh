// umma.cuh -- the fifth-generation tensor-core (tcgen05) building blocks of
// the learned warm start: shared-memory matrix descriptors, the instruction
// descriptor of a BF16 x BF16 -> FP32 MMA, TMEM allocation, the MMA, its
// commit to an mbarrier, TMEM loads, and mbarrier waits with an iteration
// limit.
//
// Operand layout: K-major without swizzle.  A tile of R rows (R a multiple
// of 8) and KC columns (KC a multiple of 16 BF16 values) is stored as core
// matrices of 8 rows x 16 bytes (8 BF16): element (r, k) sits at byte
//   ((k / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// so consecutive 8-row groups are 128 bytes apart (the stride byte offset,
// SBO) and the two 8-value halves of one MMA's K = 16 are R * 16 bytes
// apart (the leading byte offset, LBO).  One MMA (M = 128, K = 16) then
// reads the descriptor at start + kk * 2 * R * 16 for its K slice kk.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cadmas {
namespace umma {

// byte offset of element (r, k) in an R-row K-major tile
__host__ __device__ constexpr uint32_t kmajor_offset(uint32_t R, uint32_t r, uint32_t k) {
  return ((k >> 3) * (R >> 3) + (r >> 3)) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor (64 bits): start address >> 4 in bits
// [0,14), leading byte offset >> 4 in [16,30), stride byte offset >> 4 in
// [32,46), version 1 (this architecture) in [46,48), base offset 0 in
// [49,52), LBO mode 0 in bit 52, layout type 0 (no swizzle) in [61,64).
__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1u << 46);
}

// Instruction descriptor of kind::f16 (32 bits): dense, D format F32 (1) in
// bits [4,6), A and B format BF16 (1) in [7,10) and [10,13), no negation,
// both K-major (bits 15, 16 clear), N >> 3 in [17,23), M >> 4 in [24,29).
__host__ __device__ constexpr uint32_t idesc_bf16_f32(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// TMEM columns to allocate for N FP32 accumulator columns: a power of two
// of at least 32.
__host__ __device__ constexpr uint32_t tmem_cols(uint32_t N) {
  uint32_t c = 32;
  while (c < N) c <<= 1;
  return c;
}

#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// one warp: allocate ncols TMEM columns, address to *dst (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
// the same warp: free them
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A * B^T, M x N x 16, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// the mbarrier at bar gets one arrival when the MMAs issued so far by this
// thread have completed
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase with the given parity to complete; false after about
// two seconds (the caller records an error and stops using the tile).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > 4000000000LL) return false;
  }
  return true;
}

// 32 lanes x 32 bits x 8 columns from TMEM (lane quarter of this warp)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
#endif

}  // namespace umma
}  // namespace cadmas
