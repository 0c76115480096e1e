// aldic_local_icgn_noalloc: the batched local IC-GN for callers that cannot allocate
// device memory.
//
// Some hosts of this library own every device allocation themselves: a MATLAB MEX that
// hands over gpuArray buffers, an application with a fixed memory budget or its own pool,
// code running inside a framework that forbids stray cudaMalloc calls.  They can pass
// inputs and outputs but cannot let the library call cudaMalloc for its work queue.  This
// entry point keeps that queue in a fixed file-scope device array instead, so it performs
// no allocation at all.
//
// Limits and sharing:
//   * at most ALDIC_NOALLOC_MAX_SUBSETS subsets per call (larger n is rejected with
//     ALDIC_ERR_ARG before any work is queued);
//   * the array (3 buckets x ALDIC_NOALLOC_MAX_SUBSETS x 3 ints, then the counters: the
//     three bucket counts and the two work counters of the solver passes; ~2.4 MB) is held
//     by every GPU that loads the library until the process exits;
//   * all calls share the one array: calls that overlap on the GPU (different streams, or
//     different host threads) race on it and must be serialised by the caller.  Each call
//     clears the counters before use; the queue entries are rewritten.
//   * every array must be device (or managed) memory of the current device; a pointer to
//     another GPU's memory is refused with ALDIC_ERR_ARG.
//   * a CUDA error already pending from the caller's earlier work is reported as
//     ALDIC_ERR_CUDA before anything is queued, and left pending for the caller.
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) once for that device; make that first call before any stream
//     capture.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/aldic_b200.h"
#include "kernels.h"

namespace {

constexpr long long kMaxSubsets = ALDIC_NOALLOC_MAX_SUBSETS;
constexpr int kMaxDevices = 64;

// queue (3 buckets x kMaxSubsets x 3 ints) followed by the counters: the counts of the three
// buckets and the two work counters (launch_icgn clears eight ints), padded to 64 ints
constexpr int kCounterInts = 64;
static_assert(kCounterInts >= 8, "launch_icgn clears eight counters after the queue");
constexpr long long kQueueInts = (long long)aldic::kIcgnQueueBuckets * kMaxSubsets * 3;
__device__ __align__(256) int g_noalloc_scratch[kQueueInts + kCounterInts];

std::mutex g_setup_mutex;
int* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
int scratch_address(int** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return ALDIC_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "aldic_local_icgn_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return ALDIC_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<int*>(p);
  }
  *out = g_scratch_addr[dev];
  return ALDIC_OK;
}

// Device or managed memory that belongs to device `dev` (the current device).
bool on_device(const void* p, int dev) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type == cudaMemoryTypeDevice) return at.device == dev;
  if (at.type == cudaMemoryTypeManaged) return true;  // reachable from every device
  return false;
}

}  // namespace

extern "C" int aldic_local_icgn_noalloc(int variant, const float* ref, const float* def, const uint8_t* mask,
                                        const float* dfdx, const float* dfdy, int M, int N, int64_t n,
                                        const double* coords, const double* U0, int winsize, double tol,
                                        double* U, double* F, double* H, int32_t* conv, uint8_t* markHole,
                                        void* stream) {
  if (variant != ALDIC_UNIFORM && variant != ALDIC_QUADTREE) return ALDIC_ERR_ARG;
  if (n < 0 || M < 8 || N < 8 || winsize < 2 || winsize > 200) return ALDIC_ERR_ARG;
  if (n > kMaxSubsets) {
    std::fprintf(stderr,
                 "aldic_local_icgn_noalloc: %lld subsets requested, the fixed work queue holds at most %lld; "
                 "split the batch or use aldic_local_icgn\n",
                 (long long)n, kMaxSubsets);
    return ALDIC_ERR_ARG;
  }
  if (n == 0) return ALDIC_OK;
  // an error left pending by the caller's earlier work: report it, queue nothing, and leave
  // it pending (cudaPeekAtLastError does not clear it)
  if (cudaPeekAtLastError() != cudaSuccess) return ALDIC_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ALDIC_ERR_CUDA;
  const void* need[] = {ref, def, dfdx, dfdy, coords, U0, U, F, conv};
  for (const void* p : need)
    if (!on_device(p, dev)) return ALDIC_ERR_ARG;  // every array must be memory of the current device
  if ((mask && !on_device(mask, dev)) || (H && !on_device(H, dev)) || (markHole && !on_device(markHole, dev)))
    return ALDIC_ERR_ARG;
  const double w = winsize;
  int wmax = variant == ALDIC_QUADTREE ? (int)(2 * std::ceil(std::sqrt(1.0 / 0.6) * w / 2)) + 2
                                       : (int)std::round(std::sqrt(2.0) * w);
  if (wmax < winsize) wmax = winsize;
  if (aldic::icgn_smem_bytes(wmax) > 200 * 1024) return ALDIC_ERR_ARG;
  int* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  aldic::IcgnArgs a;
  a.fr.ref = ref;
  a.fr.def = def;
  a.fr.mask = mask;
  a.fr.gx = dfdx;
  a.fr.gy = dfdy;
  a.fr.M = M;
  a.fr.N = N;
  a.variant = variant;
  a.n = n;
  a.coords = coords;
  a.U0 = U0;
  a.winsize = winsize;
  a.tol = tol;
  a.max_iter = 100;
  a.warp_cap = aldic::kDefaultWarpCap;
  a.crop = 3;
  a.U = U;
  a.F = F;
  a.H = H;
  a.conv = conv;
  a.mark = variant == ALDIC_QUADTREE ? markHole : nullptr;
  a.znssd = nullptr;
  a.queue = scratch;
  a.qcount = scratch + kQueueInts;  // cleared by launch_icgn before the classify kernel
  a.carry = nullptr;  // slow subsets restart from their initial guess (no state buffer here)
  a.band = aldic::icgn_smem_bytes_f64(wmax) <= 200 * 1024 ? aldic::kDefaultFp64Band : 0.0;
  a.noise = aldic::kDefaultFp64Noise;
  a.F0 = nullptr;
  a.staging = 0;
  a.slow_nw = 2;
  a.slow_fp64 = 0;
  a.fp64_threads = 128;
  a.zncc = nullptr;
  aldic::launch_icgn(a, wmax, static_cast<cudaStream_t>(stream));
  return cudaGetLastError() == cudaSuccess ? ALDIC_OK : ALDIC_ERR_CUDA;
}
