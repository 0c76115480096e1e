// tcgen05 (5th-generation tensor core) building blocks for sm_100a: TMEM allocation, the
// shared-memory matrix and instruction descriptors of a BF16 x BF16 -> FP32 MMA with K-major
// operands in the 128-byte-swizzled layout that a TMA tile load with
// CU_TENSOR_MAP_SWIZZLE_128B writes, the MMA issue and commit, and the TMEM -> register
// loads of the epilogue.  Used by the proposal network's GEMMs (cnn.cu); single-CTA
// (cta_group::1), no cluster multicast.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tma.cuh"

namespace aldic {

// ------------------------------------------------------------------ TMEM allocation
// One warp allocates ncols (a power of two, >= 32) TMEM columns; the base address is written
// to *slot (shared memory).  The same warp frees them.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ------------------------------------------------------------------ descriptors
// Shared-memory matrix descriptor of a K-major operand tile in the 128-byte swizzle layout:
// rows of 64 BF16 (128 bytes), 8-row core groups 1024 bytes apart (the stride byte offset),
// the tile 1024-byte aligned.  Bits: [0,14) address >> 4, [16,30) leading byte offset >> 4
// (unused by swizzled K-major layouts; 1), [32,46) stride byte offset >> 4, [46,48) version 1,
// [49,52) base offset 0, [61,64) layout 2 = 128-byte swizzle.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t smem_addr) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// The same for a K-major tile of 32 BF16 per row in the 64-byte swizzle layout: rows of 64
// bytes, 8-row core groups 512 bytes apart, chunk c (16 bytes) of row r stored at
// r * 64 + ((c ^ ((r >> 1) & 3)) << 4), the tile 512-byte aligned; layout 4 = 64-byte swizzle.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t smem_addr) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)((512u >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)4u << 61;
  return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 D, both K-major, M x N:
// [4,6) D format (1 = F32), [7,10) A format (1 = BF16), [10,13) B format (1 = BF16),
// [15] A major (0 = K), [16] B major (0 = K), [17,23) N >> 3, [24,29) M >> 4.
__host__ __device__ constexpr uint32_t bf16_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ------------------------------------------------------------------ MMA and commit
// D[tmem] (+)= A[adesc] x B[bdesc]^T, one instruction of K = 16, issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

// Arrive on bar once every MMA this thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// One arrival on bar (its expected count set at init).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tcgen05_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tcgen05_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

}  // namespace aldic
