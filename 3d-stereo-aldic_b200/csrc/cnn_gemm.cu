// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a) for the
// proposal network: C[M x N] = A[M x K] * B[N x K]^T with both operands K-major (rows of K
// contiguous BF16), the product the network's convolutions (implicit GEMM over im2col rows),
// their data and weight gradients and its fully connected layers all reduce to.
//
// Persistent and warp-specialised: each CTA (192 threads) walks the output tiles
// (128 rows x BN columns x one K range of the split-K division) t = blockIdx.x,
// blockIdx.x + gridDim.x, ...; the N tiles of one row block are consecutive, so CTAs running
// side by side share A tiles in L2.
//   * warp 0 (one lane) issues the TMA loads (A: 64 K x 128 rows, B: 64 K x BN rows, 128-byte
//     swizzle, out-of-range rows and K read as zero) into a 4-stage ring, across tile
//     boundaries, each stage's refill gated by the tcgen05.commit of the MMAs that read it;
//   * warp 1 (one lane) issues the tcgen05.mma instructions (M 128, N BN, K 16 each) into one
//     of two FP32 TMEM accumulators of BN columns, alternating per tile, and commits each
//     finished accumulator;
//   * warps 2-5 read a finished accumulator back (tcgen05.ld 32x32b; warp w reads TMEM lanes
//     32 (w mod 4) ..) while the next tile's MMAs fill the other one, release it, and apply
//     the epilogue: store (+ bias), atomic add (split-K), or bias + ReLU to BF16 (16-byte
//     vector stores for whole 16-column runs at 16-byte aligned addresses).
// Every wait is bounded; a time-out sets *err and ends that role's loop (the others then
// time out too), the producer waits for its loads in flight and the MMA warp for its MMAs
// before the CTA frees TMEM and exits.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "cnn.h"
#include "umma.cuh"

namespace aldic {

namespace {

constexpr int kStages = 4;
constexpr int kBK = 64;             // K per stage: one 128-byte swizzle row of BF16
constexpr int kGemmThreads = 192;   // producer warp, MMA warp, 4 epilogue warps
constexpr long long kGemmWaitCycles = 4000000000LL;

template <int BN>
struct GemmSmem {
  static constexpr int a_bytes = 128 * kBK * 2;
  static constexpr int b_bytes = BN * kBK * 2;
  static constexpr int stage_bytes = a_bytes + b_bytes;
  static constexpr int bytes = kStages * stage_bytes + 1024;  // + 1024 for the alignment
  static constexpr uint32_t acc_cols = BN < 32 ? 32 : BN;     // TMEM columns of one accumulator
  static constexpr int per_sm = (227 * 1024) / bytes < 4 ? (227 * 1024) / bytes : 4;
};

struct TileGrid {
  int tiles_m, tiles_n, ntiles, kb_per_split, kb_total;
  // tile t -> first row, first column and K-block range [kb0, kb1)
  __device__ __forceinline__ void decode(int t, int& m0, int& n0, int& kb0, int& kb1) const {
    const int nt = t % tiles_n, r = t / tiles_n, mt = r % tiles_m, sp = r / tiles_m;
    m0 = mt * 128;
    n0 = nt;  // scaled by BN by the caller
    kb0 = sp * kb_per_split;
    kb1 = min(kb_total, kb0 + kb_per_split);
  }
};

template <int BN>
__device__ __forceinline__ void gemm_epilogue_tile(const GemmEpi& epi, uint32_t tacc, int row, int n0, int M, int N) {
#pragma unroll 1
  for (int c = 0; c < BN; c += 16) {
    float v[16];
    __syncwarp();  // tcgen05.ld is warp-collective: reconverge after the previous run's stores
    tmem_ld16(tacc + (uint32_t)c, v);
    const int col0 = n0 + c;
    if (row < M && col0 + 16 <= N && epi.mode != kEpiAtomic) {  // 16 whole columns: vector stores
      const size_t o = (size_t)row * epi.ldc + col0;
      if (epi.mode == kEpiBiasReluBf16 && ((reinterpret_cast<uintptr_t>(epi.c16 + o) & 15) == 0)) {
        __align__(16) __nv_bfloat16 h[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float x = v[j] + (epi.bias ? epi.bias[col0 + j] : 0.f);
          h[j] = __float2bfloat16_rn(x > 0.f ? x : 0.f);
        }
        uint4* dst = reinterpret_cast<uint4*>(epi.c16 + o);
        dst[0] = reinterpret_cast<const uint4*>(h)[0];
        dst[1] = reinterpret_cast<const uint4*>(h)[1];
        continue;
      }
      if (epi.mode == kEpiStore && ((reinterpret_cast<uintptr_t>(epi.c32 + o) & 15) == 0)) {
        float4* dst = reinterpret_cast<float4*>(epi.c32 + o);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          float4 q = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
          if (epi.bias) {
            q.x += epi.bias[col0 + 4 * j];
            q.y += epi.bias[col0 + 4 * j + 1];
            q.z += epi.bias[col0 + 4 * j + 2];
            q.w += epi.bias[col0 + 4 * j + 3];
          }
          dst[j] = q;
        }
        continue;
      }
    }
    if (row < M) {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int col = n0 + c + j;
        if (col >= N) continue;
        float x = v[j];
        const size_t o = (size_t)row * epi.ldc + col;
        switch (epi.mode) {
          case kEpiStore:
            if (epi.bias) x += epi.bias[col];
            epi.c32[o] = x;
            break;
          case kEpiAtomic:
            atomicAdd(epi.c32 + o, x);
            break;
          case kEpiBiasReluBf16:
            x += epi.bias ? epi.bias[col] : 0.f;
            epi.c16[o] = __float2bfloat16_rn(x > 0.f ? x : 0.f);
            break;
          default:
            break;
        }
      }
    }
  }
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmEpi epi,
                     int M, int N, TileGrid tg) {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N");
  constexpr uint32_t kCols = GemmSmem<BN>::acc_cols;
  constexpr uint32_t kAlloc = 2 * kCols;  // two accumulators (a power of two, <= 512)
  constexpr uint32_t kIdesc = bf16_idesc(128, BN);
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], acc_full[2], acc_empty[2], drain;
  __shared__ uint32_t s_tmem;
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);  // one arrival per epilogue warp
    }
    mbar_init(&drain, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(&s_tmem, kAlloc);
  tcgen05_before_sync();
  __syncthreads();
  tcgen05_after_sync();
  const uint32_t tmem = s_tmem;
  auto a_at = [&](int s) { return smem + s * GemmSmem<BN>::stage_bytes; };
  auto b_at = [&](int s) { return smem + s * GemmSmem<BN>::stage_bytes + GemmSmem<BN>::a_bytes; };
  if (warp == 0) {
    if (lane == 0) {
      int it = 0;  // stage fills issued (stage it % kStages, its use number it / kStages)
      bool ok = true;
      for (int t = blockIdx.x; t < tg.ntiles && ok; t += gridDim.x) {
        int m0, nt, kb0, kb1;
        tg.decode(t, m0, nt, kb0, kb1);
        for (int kb = kb0; kb < kb1; ++kb) {
          const int s = it % kStages;
          // the MMAs that read this stage's previous fill are done
          if (it >= kStages && !mbar_wait(&empty[s], (uint32_t)((it / kStages) - 1) & 1u, kGemmWaitCycles)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[s], (uint32_t)GemmSmem<BN>::stage_bytes);
          tma_load_2d(a_at(s), &ta, kb * kBK, m0, &full[s]);
          tma_load_2d(b_at(s), &tb, kb * kBK, nt * BN, &full[s]);
          ++it;
        }
      }
      if (!ok) atomicOr(epi.err, 1);
      // loads still in flight (after a time-out elsewhere) land before the CTA exits
      for (int s = 0; s < kStages && s < it; ++s) {
        const int last = it - 1 - ((it - 1 - s) % kStages);  // the last fill of stage s
        mbar_wait(&full[s], (uint32_t)(last / kStages) & 1u, kGemmWaitCycles);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int it = 0, tc = 0;
      bool ok = true, issued = false;
      for (int t = blockIdx.x; t < tg.ntiles && ok; t += gridDim.x, ++tc) {
        int m0, nt, kb0, kb1;
        tg.decode(t, m0, nt, kb0, kb1);
        const int b = tc & 1;
        // the epilogue has read this accumulator's previous tile (tile tc - 2)
        if (tc >= 2 && !mbar_wait(&acc_empty[b], (uint32_t)((tc >> 1) - 1) & 1u, kGemmWaitCycles)) {
          ok = false;
          break;
        }
        tcgen05_after_sync();
        const uint32_t d = tmem + (uint32_t)b * kCols;
        for (int kb = kb0; kb < kb1; ++kb) {
          const int s = it % kStages;
          if (!mbar_wait(&full[s], (uint32_t)(it / kStages) & 1u, kGemmWaitCycles)) {
            ok = false;
            break;
          }
          tcgen05_after_sync();
          const uint32_t a_addr = smem_u32(a_at(s)), b_addr = smem_u32(b_at(s));
#pragma unroll
          for (int k = 0; k < kBK / 16; ++k)  // 16 BF16 = 32 bytes along the swizzled row
            umma_bf16(d, sw128_desc(a_addr + 32 * k), sw128_desc(b_addr + 32 * k), kIdesc, kb > kb0 || k > 0);
          umma_commit(&empty[s]);
          issued = true;
          ++it;
        }
        if (!ok) break;
        umma_commit(&acc_full[b]);
      }
      if (!ok) atomicOr(epi.err, 1);
      if (issued) {  // every MMA issued above has completed before TMEM is freed
        umma_commit(&drain);
        if (!mbar_wait(&drain, 0u, kGemmWaitCycles)) atomicOr(epi.err, 1);
      }
    }
  } else {
    const int q = warp & 3;  // TMEM lanes 32 q .. 32 q + 31 = tile rows
    int tc = 0;
    for (int t = blockIdx.x; t < tg.ntiles; t += gridDim.x, ++tc) {
      int m0, nt, kb0, kb1;
      tg.decode(t, m0, nt, kb0, kb1);
      const int b = tc & 1;
      if (!mbar_wait(&acc_full[b], (uint32_t)(tc >> 1) & 1u, kGemmWaitCycles)) {
        if (lane == 0) atomicOr(epi.err, 2);
        break;
      }
      tcgen05_after_sync();
      gemm_epilogue_tile<BN>(epi, tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)b * kCols, m0 + q * 32 + lane,
                             nt * BN, M, N);
      tcgen05_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
    }
  }
  tcgen05_before_sync();
  __syncthreads();
  if (warp == 1) tmem_free(tmem, kAlloc);
}

// 2-D tensor map of a row-major BF16 matrix (rows x cols, cols contiguous with pitch ld
// elements) with a box of 64 columns (128 bytes, 128-byte swizzle) by box_rows rows.
bool make_tmap_bf16(CUtensorMap* map, const void* base, long long rows, long long cols, long long ld, int box_rows) {
  using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess && fn)
      encode = reinterpret_cast<EncodeFn>(fn);
    else
      cudaGetLastError();
  });
  if (!encode || !base || rows < 1 || cols < 1 || ld < cols) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (ld * 2) % 16 != 0) return false;
  if (box_rows < 1 || box_rows > 256) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int num_sms() {
  static int sms = 0;
  static std::once_flag once;
  std::call_once(once, [] {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sms = 148;
    cudaGetLastError();
  });
  return sms;
}

template <int BN>
int launch_bn(const GemmArgs& g, cudaStream_t st) {
  CUtensorMap ta, tb;
  std::memset(&ta, 0, sizeof(ta));
  std::memset(&tb, 0, sizeof(tb));
  if (!make_tmap_bf16(&ta, g.A, g.M, g.K, g.lda, 128) || !make_tmap_bf16(&tb, g.B, g.N, g.K, g.ldb, BN)) return -1;
  const int kb_total = (int)((g.K + kBK - 1) / kBK);
  int splits = g.splits < 1 ? 1 : g.splits;
  if (splits > kb_total) splits = kb_total;
  const int per = (kb_total + splits - 1) / splits;
  splits = (kb_total + per - 1) / per;  // every split holds at least one K block
  if (splits > 1 && g.epi.mode != kEpiAtomic) return -1;
  TileGrid tg;
  tg.tiles_m = (int)((g.M + 127) / 128);
  tg.tiles_n = (int)((g.N + BN - 1) / BN);
  tg.ntiles = tg.tiles_m * tg.tiles_n * splits;
  tg.kb_per_split = per;
  tg.kb_total = kb_total;
  // persistent: as many CTAs as fit on the GPU at once (shared memory bound), at most one
  // per tile
  const long long slots = (long long)num_sms() * GemmSmem<BN>::per_sm;
  const int grid = (int)(tg.ntiles < slots ? tg.ntiles : slots);
  auto k = umma_gemm_kernel<BN>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmSmem<BN>::bytes);
  cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  k<<<grid, kGemmThreads, GemmSmem<BN>::bytes, st>>>(ta, tb, g.epi, (int)g.M, (int)g.N, tg);
  return 1;
}

}  // namespace

// C = A * B^T (see GemmArgs); the BN tile is the smallest of 16, 32, 64, 128, 256 that holds
// N (larger N take several column tiles of 256).  Returns the launch count, -1 on a layout
// the tensor maps cannot describe.
int launch_umma_gemm(const GemmArgs& g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0) return 0;
  if (g.N <= 16) return launch_bn<16>(g, st);
  if (g.N <= 32) return launch_bn<32>(g, st);
  if (g.N <= 64) return launch_bn<64>(g, st);
  if (g.N <= 128) return launch_bn<128>(g, st);
  return launch_bn<256>(g, st);
}

}  // namespace aldic
