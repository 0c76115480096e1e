// Tensor-memory-accelerator (TMA) 2-D tile staging for the IC-GN warp passes (sm_100a).
//
// Host side: a 2-D tiled tensor map over a column-major FP32 image (dim 0 = the M rows,
// contiguous; dim 1 = the N columns), built with the driver's cuTensorMapEncodeTiled through
// the runtime's driver entry point (no link against libcuda).  Device side: one mbarrier per
// staging buffer, a single-lane cp.async.bulk.tensor load with complete_tx accounting, and a
// bounded wait.  No load here uses .multicast::cluster, and every tensor map covers an image
// of the launching GPU.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace aldic {

// ---------------------------------------------------------------------------------- host
// Tensor map of a column-major M x N FP32 image with a box of box_r rows by box_c columns.
// Returns false when the layout cannot be described (row pitch M * 4 not a multiple of 16
// bytes, base not 16-byte aligned, box beyond the hardware limits) or the driver entry
// point is unavailable; callers then use the gather path.  Out-of-image box elements read 0.
bool make_tmap_2d_f32(CUtensorMap* map, const float* base, int M, int N, int box_r, int box_c);

// ---------------------------------------------------------------------------------- device
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make the initialised mbarrier and earlier generic-proxy shared-memory accesses of this thread
// visible to the async proxy (the TMA unit).
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// One 2-D tile: box at (row c0, column c1) of the tensor map into shared memory dst (128-byte
// aligned); completion is signalled on bar.  c0 * 4 must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

// Wait for phase `parity` of bar to complete, for at most max_cycles SM clock cycles (each
// try_wait returns within a hardware time limit); false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long max_cycles) {
  const uint32_t addr = smem_u32(bar);
  const long long start = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - start > max_cycles) return false;
  }
}

}  // namespace aldic
