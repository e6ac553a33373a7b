// tcgen05.cuh -- thin wrappers of the sm_100a tensor-core (tcgen05) PTX used
// by the integer-slice FF kernel: tensor-memory allocation, the kind::i8 MMA
// with shared-memory operand descriptors, commit to an mbarrier, and
// tensor-memory loads.  Descriptor bit layouts follow the PTX ISA (shared
// memory matrix descriptor, instruction descriptor for .kind::i8).
#pragma once

#include <stdint.h>

#include "bgw_internal.cuh"

namespace bgw {
namespace tc {

// Shared-memory matrix descriptor, K-major, no swizzle ("interleave"):
// core matrices of 8 rows x 16 bytes stored as 128 contiguous bytes; `lbo`
// is the byte distance between the two 16-byte halves of a K step (K
// direction), `sbo` between consecutive 8-row groups (M/N direction).
__device__ __forceinline__ uint64_t smem_desc(uint32_t smem_addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);          // bits  0-13 start address
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;          // bits 16-29 leading byte offset
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;          // bits 32-45 stride byte offset
  d |= (uint64_t)1 << 46;                               // bits 46-47 descriptor version 1
  // base offset 0 (bits 49-51), lbo mode 0 (bit 52), layout 0 = no swizzle (61-63)
  return d;
}

// Instruction descriptor of tcgen05.mma .kind::i8: signed A and B, S32
// accumulator, both operands K-major, dense.  M = 128 takes N % 16 == 0,
// 16 <= N <= 256.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
  return (2u << 4)                       // D format: S32
         | (1u << 7)                     // A: signed 8-bit
         | (1u << 10)                    // B: signed 8-bit
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate), "r"(0u), "r"(0u), "r"(0u),
        "r"(0u)
      : "memory");
}

// Arrives on `bar` once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Warp-wide: allocates `ncols` tensor-memory columns, address to *dst (smem).
__device__ __forceinline__ void alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Warp-wide: 32 lanes x 16 consecutive 32-bit columns starting at taddr
// (lane field = the warp's 32-lane quarter).
__device__ __forceinline__ void ld16(uint32_t taddr, int32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
// Warp-wide: 32 lanes x 4 consecutive 32-bit columns.
__device__ __forceinline__ void ld4(uint32_t taddr, int32_t (&v)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr));
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Orders this thread's earlier generic-proxy shared-memory writes before
// later async-proxy reads (operands written with st.shared, read by MMAs).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Plain mbarrier arrive (count 1) by this thread.
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

}  // namespace tc
}  // namespace bgw
