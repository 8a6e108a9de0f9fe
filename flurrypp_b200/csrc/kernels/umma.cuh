// 5th-generation tensor-core (tcgen05) helpers for sm_100a, as inline PTX:
// tensor-memory allocation, shared-memory matrix descriptors, the kind::tf32
// MMA issued by one thread, its completion on an mbarrier, and tensor-memory
// loads for the epilogue.  One CTA, no clusters, no multicast.
#pragma once
#include <stdint.h>

#include "tma.cuh"

namespace frk {

// Shared-memory matrix descriptor of a K-major operand in the no-swizzle
// canonical layout: 8-row x 16-byte core matrices, `lbo` bytes between the
// two 16-byte K chunks of one MMA step, `sbo` bytes between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  // base offset 0, absolute LBO mode, layout type 0 (no swizzle)
  return d;
}

// Instruction descriptor of tcgen05.mma kind::tf32: FP32 accumulate, A and B
// TF32, both K-major, shape M x N.
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4)                    // D format F32
         | (2u << 7)                  // A format TF32
         | (2u << 10)                 // B format TF32
         | ((uint32_t)(N >> 3) << 17) // N / 8
         | ((uint32_t)(M >> 4) << 24);// M / 16
}

// D[tmem] (+)= A[desc] * B[desc]^T, issued by the calling thread only.
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

// Arrive once on `bar` when all previously issued tcgen05 operations of this
// thread have completed.
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Tensor-memory allocation by one whole warp; the column base lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Eight consecutive 32-bit columns of this thread's lane (warp w reads lanes
// 32w .. 32w+31); taddr carries the warp's lane base in bits 16..31.  The
// wait is in the same statement, so the outputs are complete on return.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// Round to the nearest TF32 value (10-bit mantissa, ties away from zero) and
// clear the 13 low bits, so the tensor core sees the value exactly: the hi
// part of the 3xTF32 split; x - hi is exact in FP32 and is itself rounded to
// TF32 as the lo part.
__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r & 0xFFFFE000u);
}

}  // namespace frk
