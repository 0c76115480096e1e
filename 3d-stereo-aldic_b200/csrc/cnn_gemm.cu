// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a) for the
// proposal network: C[M x N] = A[M x K] * B[N x K]^T with both operands K-major (rows of K
// contiguous BF16), the product the network's convolutions (implicit GEMM over im2col rows),
// their data and weight gradients and its fully connected layers all reduce to.
//
// One CTA of 128 threads per (128-row, BN-column) tile and K range (split-K over grid.z):
//   * one thread issues the TMA tile loads (A: 64 K x 128 rows, B: 64 K x BN rows, 128-byte
//     swizzle, out-of-range rows and K read as zero) into a 4-stage ring and the tcgen05.mma
//     instructions (M 128, N BN, K 16 each) into an FP32 accumulator of BN TMEM columns;
//     tcgen05.commit on a per-stage mbarrier frees a stage for the next load;
//   * the 4 warps then read their 32 accumulator rows back (tcgen05.ld 32x32b) and apply the
//     epilogue: store (+ bias), atomic add (split-K), or bias + ReLU to BF16 (16-byte vector
//     stores for whole 16-column runs at 16-byte aligned addresses).
// Every wait is bounded; a time-out sets *err, stops issuing, drains and frees TMEM.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "cnn.h"
#include "umma.cuh"

namespace aldic {

namespace {

constexpr int kStages = 4;
constexpr int kBK = 64;  // K per stage: one 128-byte swizzle row of BF16
constexpr long long kGemmWaitCycles = 4000000000LL;

template <int BN>
struct GemmSmem {
  static constexpr int a_bytes = 128 * kBK * 2;
  static constexpr int b_bytes = BN * kBK * 2;
  static constexpr int stage_bytes = a_bytes + b_bytes;
  static constexpr int bytes = kStages * stage_bytes + 1024;  // + 1024 for the alignment
};

template <int BN>
__global__ void __launch_bounds__(128, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmEpi epi,
                     int M, int N, int kb_per_split, int kb_total) {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N");
  constexpr uint32_t kCols = BN < 32 ? 32 : BN;  // TMEM columns (a power of two, >= 32)
  constexpr uint32_t kIdesc = bf16_idesc(128, BN);
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN;
  const int kb0 = blockIdx.z * kb_per_split;
  const int kb1 = min(kb_total, kb0 + kb_per_split);
  const int nkb = kb1 - kb0;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    fence_barrier_init();
    s_fail = 0;
  }
  if (warp == 0) tmem_alloc(&s_tmem, kCols);
  tcgen05_before_sync();
  __syncthreads();
  tcgen05_after_sync();
  const uint32_t tmem = s_tmem;
  if (tid == 0 && nkb > 0) {
    auto a_at = [&](int s) { return smem + s * GemmSmem<BN>::stage_bytes; };
    auto b_at = [&](int s) { return smem + s * GemmSmem<BN>::stage_bytes + GemmSmem<BN>::a_bytes; };
    auto load = [&](int kb, int s) {
      mbar_arrive_expect_tx(&full[s], (uint32_t)GemmSmem<BN>::stage_bytes);
      tma_load_2d(a_at(s), &ta, kb * kBK, m0, &full[s]);
      tma_load_2d(b_at(s), &tb, kb * kBK, n0, &full[s]);
    };
    const int pre = nkb < kStages ? nkb : kStages;
    for (int i = 0; i < pre; ++i) load(kb0 + i, i);
    bool ok = true;
    for (int i = 0; i < nkb && ok; ++i) {
      const int s = i % kStages;
      const uint32_t ph = (uint32_t)(i / kStages) & 1u;
      if (!mbar_wait(&full[s], ph, kGemmWaitCycles)) {
        ok = false;
        break;
      }
      tcgen05_after_sync();
      const uint32_t a_addr = smem_u32(a_at(s)), b_addr = smem_u32(b_at(s));
#pragma unroll
      for (int k = 0; k < kBK / 16; ++k)  // 16 BF16 = 32 bytes along the swizzled row
        umma_bf16(tmem, sw128_desc(a_addr + 32 * k), sw128_desc(b_addr + 32 * k), kIdesc, i > 0 || k > 0);
      umma_commit(&empty[s]);
      // refill the stage the previous MMAs read, once they are done (the MMAs just issued
      // keep the tensor pipe busy meanwhile)
      if (i >= 1) {
        const int ip = i - 1, sp = ip % kStages;
        if (ip + kStages < nkb) {
          if (!mbar_wait(&empty[sp], (uint32_t)(ip / kStages) & 1u, kGemmWaitCycles)) {
            ok = false;
            break;
          }
          load(kb0 + ip + kStages, sp);
        }
      }
    }
    umma_commit(&done);  // arrives once every MMA issued above has completed
    if (!ok) {
      s_fail = 1;
      atomicOr(epi.err, 1);
    }
  }
  __syncthreads();
  // accumulator ready (or nothing to do for an empty K range)
  bool ready = nkb > 0;
  if (ready) ready = mbar_wait(&done, 0, kGemmWaitCycles);
  if (ready && !s_fail) {
    tcgen05_after_sync();
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
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
  } else if (nkb > 0 && !ready) {
    atomicOr(epi.err, 2);
  }
  tcgen05_before_sync();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, kCols);
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
  splits = (kb_total + per - 1) / per;
  if (splits > 1 && g.epi.mode != kEpiAtomic) return -1;
  const dim3 grid((unsigned)((g.M + 127) / 128), (unsigned)((g.N + BN - 1) / BN), (unsigned)splits);
  auto k = umma_gemm_kernel<BN>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmSmem<BN>::bytes);
  k<<<grid, 128, GemmSmem<BN>::bytes, st>>>(ta, tb, g.epi, (int)g.M, (int)g.N, per, kb_total);
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
