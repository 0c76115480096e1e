// Proposal network of the learned initial guess: a small convolutional network that reads a
// 32 x 32 reference subset and the 64 x 64 deformed window around it and predicts the
// subset's displacement and displacement gradient, (u, v, du/dx, dv/dx, du/dy, dv/dy), the
// initial guess [F0 U0] of IC-GN in place of the FFT integer search.  No counterpart in the
// reference (its initial guess is the integer search, func/funIntegerSearch.m:132-180, which
// stays the fallback here).
//
// Architecture (NHWC BF16 activations, FP32 accumulation, ReLU after every convolution and the
// hidden fully connected layer; 3 x 3 convolutions with padding 1):
//   input 72 x 72 x 2 centred on the subset: channel 1 the frame's normalised deformed image,
//   channel 0 the normalised reference image in the centre 40 x 40 (zero elsewhere); zero
//   outside the image
//   the reference part R and the deformed window D through the same two convolutions:
//       conv1 1 -> 32 stride 2, conv2 32 -> 32 stride 2 (R: 10 x 10 x 32, D: 18 x 18 x 32), of
//       which the inner 8 x 8 (R, the 32 x 32 subset) and 16 x 16 (D, the 64 x 64 window) are
//       kept: the outer ring is the only part that sees the window's own zero padding, so the
//       kept features equal those of the two convolutions run over the whole image
//   correlation volume C[i, j, d] = sum_c fR[i, j, c] fD[i + 4 + di, j + 4 + dj, c] / 32 for
//       the 81 offsets d = (di + 4) 9 + (dj + 4), di, dj in -4..4 (+-16 px at stride 4)
//   conv3 81 -> 64 stride 2 (4 x 4), conv4 64 -> 64 stride 1 (4 x 4)
//   fully connected: 1024 -> 128 -> 6
// 227 152 parameters.  Training runs the network per subset window; prediction runs conv1 and
// conv2 once over each whole image and the correlation and the rest per subset, on feature
// crops at the subset's position (subset centres x = 1 mod 4 in both coordinates align the
// two).  Every convolution, data gradient, weight gradient and fully connected layer is one
// tcgen05 GEMM (cnn_gemm.cu) over im2col rows (conv4, on a 4 x 4 map, as one dense 1024 x 1024
// matrix on the flattened map instead); the correlation and the rest are the small
// kernels below (im2col, col2im, correlation and its gradient, transposes, ReLU gradient, loss,
// bias gradient, Adam, patch extraction).  Training: mean squared error on the scaled outputs
// (u / 8, v / 8, F x 20), Adam.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/aldic_b200.h"
#include "cnn.h"
#include "kernels.h"
#include "umma.cuh"

namespace aldic {
namespace {

typedef __nv_bfloat16 bf16;

// One convolution applied to one input: parameter layer, input Hin x Win x Cin, output
// Hout x Wout x Cout, K = 9 Cin im2col columns padded to Kp (a multiple of 8).
struct ConvI {
  int layer, Hin, Win, Cin, Hout, Wout, Cout, K, Kp, stride;
};
constexpr int kConvR1 = 0, kConvD1 = 1, kConvR2 = 2, kConvD2 = 3, kConv3 = 4, kConv4 = 5, kNumConv = 6;
constexpr ConvI kConv[kNumConv] = {{0, 40, 40, 1, 20, 20, 32, 9, 16, 2},      {0, 72, 72, 1, 36, 36, 32, 9, 16, 2},
                                   {1, 20, 20, 32, 10, 10, 32, 288, 288, 2},  {1, 36, 36, 32, 18, 18, 32, 288, 288, 2},
                                   {2, 8, 8, 81, 4, 4, 64, 729, 736, 2},      {3, 4, 4, 64, 4, 4, 64, 576, 576, 1}};
constexpr int kWin = 72, kRefWin = 40, kRefOff = 16;  // input window, reference part and its offset
constexpr int kDisp = 81, kFcIn = 1024, kFcHid = 128, kOut = 6, kOutP = 16;

// Where an input of a convolution sits: element (b, y, x, c) at base + off + b sb + y sy + x sx + c.
struct View {
  long long off, sb, sy, sx;
};
View nhwc(int H, int W, int C) { return View{0, (long long)H * W * C, (long long)W * C, C}; }
// the two image channels of the 72 x 72 x 2 input
constexpr View kViewRef{(kRefOff * kWin + kRefOff) * 2, kWin * kWin * 2, kWin * 2, 2};
constexpr View kViewDef{1, kWin * kWin * 2, kWin * 2, 2};

// Where the kept 8 x 8 (reference) and 16 x 16 (deformed) feature crops of sample b sit:
// element (i, j, c) at base + b sb + off + i row + j 32 + c.
struct Crop {
  long long sb, off, row;
};

// flat FP32 parameter layout: per layer W [rows x cols] then b [rows]: conv1 32 x 16 (9 used),
// conv2 32 x 288, conv3 64 x 736 (729 used), conv4 64 x 576, FC1 128 x 1024, FC2 16 x 128
// (rows 6..15 and bias entries 6..15 zero)
struct Layout {
  long long w[6], b[6], n;
  long long rows[6], cols[6];
  Layout() {
    const long long r[6] = {32, 32, 64, 64, kFcHid, kOutP}, c[6] = {16, 288, 736, 576, kFcIn, kFcHid};
    long long o = 0;
    for (int l = 0; l < 6; ++l) {
      rows[l] = r[l];
      cols[l] = c[l];
      w[l] = o;
      o += rows[l] * cols[l];
      b[l] = o;
      o += rows[l];
    }
    n = o;
  }
};
const Layout kL;

__device__ __forceinline__ long long ceil_div_ll(long long a, long long b) { return (a + b - 1) / b; }

// ------------------------------------------------------------------------- kernels
// im2col of a 3 x 3, pad-1 convolution: row p = (b, oy, ox), column k = (ky, kx, ci), zero
// outside the input and in the K padding.  Each thread writes 8 columns (one 16-byte store);
// with Cin a multiple of 8 (16-byte aligned channel runs) it also reads them in one load.
__global__ void im2col_kernel(const bf16* __restrict__ in, View v, bf16* __restrict__ A, long long P, ConvI L) {
  const int groups = L.Kp / 8;
  const long long total = P * groups;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long p = i / groups;
    const int k0 = (int)(i % groups) * 8;
    const int ox = (int)(p % L.Wout), oy = (int)((p / L.Wout) % L.Hout);
    const long long b = p / ((long long)L.Wout * L.Hout);
    const bf16* base = in + v.off + b * v.sb;
    if (L.Cin % 8 == 0) {  // the 8 columns are 8 channels of one tap: one 16-byte load
      uint4 val = make_uint4(0u, 0u, 0u, 0u);
      if (k0 < L.K) {
        const int tap = k0 / L.Cin, ci = k0 % L.Cin, ky = tap / 3, kx = tap % 3;
        const int iy = L.stride * oy - 1 + ky, ix = L.stride * ox - 1 + kx;
        if (iy >= 0 && iy < L.Hin && ix >= 0 && ix < L.Win)
          val = *reinterpret_cast<const uint4*>(base + iy * v.sy + ix * v.sx + ci);
      }
      *reinterpret_cast<uint4*>(A + p * L.Kp + k0) = val;
      continue;
    }
    __align__(16) bf16 vals[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = k0 + j;
      bf16 x = __float2bfloat16_rn(0.f);
      if (k < L.K) {
        const int tap = k / L.Cin, ci = k % L.Cin, ky = tap / 3, kx = tap % 3;
        const int iy = L.stride * oy - 1 + ky, ix = L.stride * ox - 1 + kx;
        if (iy >= 0 && iy < L.Hin && ix >= 0 && ix < L.Win) x = base[iy * v.sy + ix * v.sx + ci];
      }
      vals[j] = x;
    }
    *reinterpret_cast<uint4*>(A + p * L.Kp + k0) = *reinterpret_cast<const uint4*>(vals);
  }
}

// col2im (gather form, no atomics): the gradient of input pixel (b, iy, ix, ci) sums the
// im2col gradient entries that read it.
__global__ void col2im_kernel(const float* __restrict__ dA, float* __restrict__ dH, int batch, ConvI L) {
  const long long total = (long long)batch * L.Hin * L.Win * L.Cin;
  const int s = L.stride;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int ci = (int)(i % L.Cin);
    const int ix = (int)((i / L.Cin) % L.Win);
    const int iy = (int)((i / ((long long)L.Cin * L.Win)) % L.Hin);
    const long long b = i / ((long long)L.Cin * L.Win * L.Hin);
    float acc = 0.f;
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
      const int ty = iy + 1 - ky;
      if (ty < 0 || ty % s || ty / s >= L.Hout) continue;
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) {
        const int tx = ix + 1 - kx;
        if (tx < 0 || tx % s || tx / s >= L.Wout) continue;
        const long long p = (b * L.Hout + ty / s) * L.Wout + tx / s;
        acc += dA[p * L.Kp + (ky * 3 + kx) * L.Cin + ci];
      }
    }
    dH[i] = acc;
  }
}

// Gradients of the correlation with the ReLU of its inputs folded in, over the whole conv2
// output maps (zero on the ring outside the crops): dZR = dC fD / 32 where fR > 0 (B, 10, 10,
// 32), dZD = dC^T fR / 32 where fD > 0 (B, 18, 18, 32), BF16; dC (B, 8, 8, 81) FP32.
__global__ void corr_grad_ref_kernel(const float* __restrict__ dC, const bf16* __restrict__ fR,
                                     const bf16* __restrict__ fD, bf16* __restrict__ dZR, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % 32);
    const long long pix = i / 32;
    const int x = (int)(pix % 10) - 1, y = (int)((pix / 10) % 10) - 1;  // crop coordinates
    const long long b = pix / 100;
    float s = 0.f;
    if (x >= 0 && x < 8 && y >= 0 && y < 8 && __bfloat162float(fR[i]) > 0.f) {
      const long long pos = (b * 8 + y) * 8 + x;
      for (int d = 0; d < kDisp; ++d) {
        const int di = d / 9 - 4, dj = d % 9 - 4;
        s = fmaf(dC[pos * kDisp + d], __bfloat162float(fD[((b * 18 + y + 5 + di) * 18 + x + 5 + dj) * 32 + c]), s);
      }
    }
    dZR[i] = __float2bfloat16_rn(s * (1.f / 32.f));
  }
}

__global__ void corr_grad_def_kernel(const float* __restrict__ dC, const bf16* __restrict__ fR,
                                     const bf16* __restrict__ fD, bf16* __restrict__ dZD, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % 32);
    const long long pix = i / 32;
    const int q = (int)(pix % 18) - 1, p = (int)((pix / 18) % 18) - 1;  // crop coordinates
    const long long b = pix / 324;
    float s = 0.f;
    if (p >= 0 && p < 16 && q >= 0 && q < 16 && __bfloat162float(fD[i]) > 0.f) {
      for (int di = -4; di <= 4; ++di) {
        const int ii = p - 4 - di;
        if (ii < 0 || ii >= 8) continue;
        for (int dj = -4; dj <= 4; ++dj) {
          const int j = q - 4 - dj;
          if (j < 0 || j >= 8) continue;
          const long long rp = (b * 8 + ii) * 8 + j;
          s = fmaf(dC[rp * kDisp + (di + 4) * 9 + (dj + 4)], __bfloat162float(fR[((b * 10 + ii + 1) * 10 + j + 1) * 32 + c]), s);
        }
      }
    }
    dZD[i] = __float2bfloat16_rn(s * (1.f / 32.f));
  }
}

// conv1 (1 -> 32 channels, 3 x 3, stride 2, pad 1) + bias + ReLU computed directly (9 taps per
// output, FP32 sums in tap order): one thread per output pixel p = (b, oy, ox) of the input
// seen through v, 32 BF16 outputs (four 16-byte stores).  Weights W (32 x 16 BF16, 9 used).
__global__ void conv1_kernel(const bf16* __restrict__ in, View v, ConvI L, long long P, const bf16* __restrict__ W,
                             const float* __restrict__ bias, bf16* __restrict__ H) {
  __shared__ float w[32][9], bs[32];
  for (int i = threadIdx.x; i < 32 * 9; i += blockDim.x) w[i / 9][i % 9] = __bfloat162float(W[(i / 9) * 16 + i % 9]);
  for (int i = threadIdx.x; i < 32; i += blockDim.x) bs[i] = bias[i];
  __syncthreads();
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const int ox = (int)(p % L.Wout), oy = (int)((p / L.Wout) % L.Hout);
    const long long b = p / ((long long)L.Wout * L.Hout);
    const bf16* base = in + v.off + b * v.sb;
    float x[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int iy = 2 * oy - 1 + t / 3, ix = 2 * ox - 1 + t % 3;
      x[t] = (iy >= 0 && iy < L.Hin && ix >= 0 && ix < L.Win) ? __bfloat162float(base[iy * v.sy + ix * v.sx]) : 0.f;
    }
    uint4* out = reinterpret_cast<uint4*>(H + p * 32);
#pragma unroll 1
    for (int g = 0; g < 4; ++g) {
      __align__(16) bf16 o[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int c = g * 8 + k;
        float acc = 0.f;
#pragma unroll
        for (int t = 0; t < 9; ++t) acc = fmaf(w[c][t], x[t], acc);
        o[k] = __float2bfloat16_rn(fmaxf(acc + bs[c], 0.f));
      }
      out[g] = *reinterpret_cast<const uint4*>(o);
    }
  }
}

// Where the feature crops of sample t sit: per-window conv2 outputs (coords null; crops at
// offsets cr / cd of the (B, 10, 10, 32) and (B, 18, 18, 32) maps) or the whole-image maps
// FR, FD (Hf x Wf x 32) at the positions of subset t0 + t of coords (n x 2).
struct CorrSrc {
  const bf16 *R, *D;
  Crop cr, cd;
  const double* coords;
  long long n, t0;
  int Hf, Wf;
};

// crop bases and row pitches of sample t; false where a whole-image crop leaves the maps
__device__ __forceinline__ bool corr_crops(const CorrSrc& s, long long t, const bf16*& r, long long& rrow,
                                           const bf16*& d, long long& drow) {
  if (!s.coords) {
    r = s.R + t * s.cr.sb + s.cr.off;
    d = s.D + t * s.cd.sb + s.cd.off;
    rrow = s.cr.row;
    drow = s.cd.row;
    return true;
  }
  const long long x = 4 * llround((s.coords[s.t0 + t] - 1.0) / 4.0) + 1;
  const long long y = 4 * llround((s.coords[s.n + s.t0 + t] - 1.0) / 4.0) + 1;
  const long long rx = (x - 17) / 4, ry = (y - 17) / 4, dx = (x - 33) / 4, dy = (y - 33) / 4;
  if (x < 33 || y < 33 || rx + 7 >= s.Hf || ry + 7 >= s.Wf || dx + 15 >= s.Hf || dy + 15 >= s.Wf) return false;
  r = s.R + (rx * s.Wf + ry) * 32;
  d = s.D + (dx * s.Wf + dy) * 32;
  rrow = drow = (long long)s.Wf * 32;
  return true;
}

// The correlation volumes of samples 0 .. nb - 1 on the tensor cores and, from them, conv3's
// im2col rows; a persistent CTA takes samples blockIdx.x, + gridDim.x, ... and loads the next
// sample's crops into registers while it works on the current one.  Per sample: the 8 x 8
// reference feature crop (64 rows of 32 BF16 channels, written twice: A rows p and 64 + p) and
// the 16 x 16 deformed crop (256 rows) are staged in shared memory in the 64-byte-swizzled
// K-major layout (a row: the 32 channels, the two K = 16 steps).  In two passes (deformed rows 0..7, then 8..15) one thread issues
// two tcgen05.mma (M 128, N 128) into 128 TMEM columns: D[p, q] = fR[p] . fD[q] for the
// reference / deformed position pairs of the pass.  Each warp w reads TMEM lanes 32 w ..
// (reference positions p = 8 ii + j, rows 64.. repeating 0..63) and takes, with warp w + 2 or
// w - 2, the pass's deformed rows its lanes touch (tcgen05.ld, 16 columns each); for its own
// row ii it keeps the 9 offsets of each deformed row within ii .. ii + 8 (columns j .. j + 8,
// picked by a 3-stage rotation by j): the volume entries / 32, rounded to BF16, each written
// straight to the (at most 4) places conv3's im2col rows use it, in a shared-memory copy of
// the sample's 16 rows x 736 columns (zeroed once: the other places are the same for every
// sample).  All 128 threads then copy those rows out with 16-byte stores.  128 TMEM columns
// and 48 KB of shared memory let 4 CTAs share an SM.  ok[t] = 0 (whole-image crops leaving the maps) gives a zero volume.  The MMA waits are
// bounded (err bit 2 on time-out, the volumes then undefined).
constexpr int kCorrThreads = 128;
constexpr int kCorrA = 128 * 64, kCorrB = 256 * 64;  // operand tiles (bytes): 64-byte rows
constexpr int kCorrRows = 16 * 736 * 2;                // conv3's im2col rows of a sample
constexpr int kCorrSmem = 1024 + kCorrA + kCorrB + kCorrRows;  // + alignment slack
constexpr long long kCorrWaitCycles = 2000000000LL;

// chunk (16 bytes, 0..3) of a 64-byte-swizzled row (sw64_desc)
__device__ __forceinline__ void put_chunk64(unsigned char* tile, int row, int chunk, uint4 v) {
  *reinterpret_cast<uint4*>(tile + row * 64 + ((chunk ^ ((row >> 1) & 3)) << 4)) = v;
}

// this thread's 10 chunks of sample t's crops (A: chunks 0..255, B: 256..1279), zero outside
__device__ __forceinline__ bool corr_fetch(const CorrSrc& src, long long t, int tid, uint4 (&v)[10]) {
  const bf16 *r, *d;
  long long rrow, drow;
  const bool inside = corr_crops(src, t, r, rrow, d, drow);
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const int q = tid + i * kCorrThreads, row = i < 2 ? q / 4 : (q - 256) / 4, ch = q % 4;
    const bf16* src_row = i < 2 ? r + (row / 8) * rrow + (row % 8) * 32 : d + (row / 16) * drow + (row % 16) * 32;
    v[i] = inside ? *reinterpret_cast<const uint4*>(src_row + ch * 8) : zero;
  }
  return inside;
}

__global__ void __launch_bounds__(kCorrThreads) corr_im2col_kernel(CorrSrc src, int nb, bf16* __restrict__ A3,
                                                                   uint8_t* __restrict__ ok, int* __restrict__ err) {
  extern __shared__ unsigned char corr_raw[];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t s_tmem;
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(corr_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* tA = smem;
  unsigned char* tB = smem + kCorrA;
  bf16* rows = reinterpret_cast<bf16*>(smem + kCorrA + kCorrB);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    mbar_init(&done, 1);
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(&s_tmem, 128);
  tcgen05_before_sync();
  __syncthreads();
  tcgen05_after_sync();
  const uint32_t tmem = s_tmem;
  // warp w: reference positions p = 32 (w % 2) + lane (rows ii0 .. ii0 + 3), its half of the
  // deformed rows it needs in each pass
  const int p = (warp % 2) * 32 + lane, ii = p / 8, j = p % 8, ii0 = (warp % 2) * 4, half = warp / 2;
  // the im2col places of volume position (ii, j): output (oy, ox) with 2 oy - 1 + ky = ii and
  // 2 ox - 1 + kx = j, tap (ky, kx); at most 2 per axis
  int base[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int oy = ((ii + 1) >> 1) - (k >> 1), ox = ((j + 1) >> 1) - (k & 1);
    const int ky = ii + 1 - 2 * oy, kx = j + 1 - 2 * ox;
    base[k] = (oy >= 0 && oy < 4 && ox >= 0 && ox < 4 && ky >= 0 && ky <= 2 && kx >= 0 && kx <= 2)
                  ? (oy * 4 + ox) * 736 + (ky * 3 + kx) * kDisp
                  : -1;
  }
  // the im2col rows start at zero (padding taps and the 7 padding columns); every sample
  // rewrites the same (valid) places, so the zeros stay
  for (int q = tid; q < kCorrRows / 16; q += kCorrThreads)
    reinterpret_cast<uint4*>(rows)[q] = make_uint4(0u, 0u, 0u, 0u);
  bool ready = true;
  uint4 v[10];
  long long t = blockIdx.x;
  bool inside = t < nb ? corr_fetch(src, t, tid, v) : false;
#pragma unroll 1
  for (; t < nb; t += gridDim.x) {
    // this sample's crops into the tiles (free: the previous sample's MMAs are complete; its
    // im2col rows are free too: the previous copy-out finished before the loop's barrier)
#pragma unroll
    for (int i = 0; i < 10; ++i) {
      const int q = tid + i * kCorrThreads;
      if (i < 2) {  // A rows p and p + 64 (a copy: TMEM lanes 64..127 for warps 2 and 3)
        put_chunk64(tA, q / 4, q % 4, v[i]);
        put_chunk64(tA, 64 + q / 4, q % 4, v[i]);
      } else {
        put_chunk64(tB, (q - 256) / 4, q % 4, v[i]);
      }
    }
    if (ok && tid == 0) ok[t] = inside ? 1 : 0;
    const bool cur = inside;
    if (t + gridDim.x < nb) inside = corr_fetch(src, t + gridDim.x, tid, v);  // in flight meanwhile
    fence_proxy_async_shared();  // the generic-proxy tile writes, visible to the tensor cores
    tcgen05_before_sync();
    __syncthreads();
    tcgen05_after_sync();
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
      if (tid == 0) {
        constexpr uint32_t idesc = bf16_idesc(128, 128);
        const uint32_t a = smem_u32(tA), b = smem_u32(tB + pass * 128 * 64);
        umma_bf16(tmem, sw64_desc(a), sw64_desc(b), idesc, false);
        umma_bf16(tmem, sw64_desc(a + 32), sw64_desc(b + 32), idesc, true);
        umma_commit(&done);
      }
      __syncwarp();
      ready = mbar_wait(&done, (uint32_t)pass, kCorrWaitCycles) && ready;  // two phases per sample
      tcgen05_after_sync();
      // deformed rows of this pass that rows ii0 .. ii0 + 3 touch, split between the two warps
      const int lo = max(ii0, 8 * pass), hi = min(ii0 + 11, 8 * pass + 7);
      const int mid = lo + (hi - lo + 2) / 2;
#pragma unroll 1
      for (int dr = half ? mid : lo; dr <= (half ? hi : mid - 1); ++dr) {
        float w[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((dr - 8 * pass) * 16), w);
        const int di = dr - ii;  // deformed row dr = ii + di
        if (di < 0 || di > 8) continue;
        // rotate left by j (bits 4, 2, 1) so that w[0..8] = columns j .. j + 8
#pragma unroll
        for (int k = 0; k < 12; ++k) w[k] = (j & 4) ? w[k + 4] : w[k];
#pragma unroll
        for (int k = 0; k < 10; ++k) w[k] = (j & 2) ? w[k + 2] : w[k];
#pragma unroll
        for (int k = 0; k < 9; ++k) w[k] = (j & 1) ? w[k + 1] : w[k];
#pragma unroll
        for (int b = 0; b < 9; ++b) {
          const bf16 x = __float2bfloat16_rn(cur ? w[b] * (1.f / 32.f) : 0.f);
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (base[k] >= 0) rows[base[k] + di * 9 + b] = x;
        }
      }
      tcgen05_before_sync();
      __syncthreads();
      tcgen05_after_sync();
    }
    uint4* outA = reinterpret_cast<uint4*>(A3 + t * 16 * 736);
    for (int q = tid; q < kCorrRows / 16; q += kCorrThreads) outA[q] = reinterpret_cast<const uint4*>(rows)[q];
    __syncthreads();  // the rows are read before the next sample zeroes them
  }
  if (!ready && lane == 0) atomicOr(err, 4);
  tcgen05_before_sync();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, 128);
}

// conv1 and conv2 over whole frame images in a single pass (prediction): CTA (bx, i2, z)
// computes conv2's outputs (i2, 128 bx .. 128 bx + 127) of image z's (M2 x N2 x 32) map.  It loads
// the 7 x 515 image pixels they depend on (BF16-rounded, zero outside the image) into shared
// memory; for each output pixel the threads compute the 9 conv1 positions conv2's taps read
// (32 channels each, FP32 sums in tap order, + bias, ReLU, BF16: the arithmetic of
// conv1_kernel; zero outside conv1's map) straight into conv2's im2col row, written in the
// 128-byte-swizzled K-major layout as 5 K-blocks of 64 columns (288 used, as conv2's GEMM);
// conv2's weights are staged alike.  One thread issues the 20 tcgen05.mma (M 128, N 32,
// K 16) of the GEMM's K order into 32 TMEM columns; the 4 warps read their rows back and
// store bias + ReLU as BF16.  The results equal conv1_kernel + im2col + the tcgen05 GEMM
// bit for bit.  The MMA wait is bounded (err bit 3 on time-out).
constexpr int kFeatThreads = 128, kFeatCols = 4 * 128 + 3, kFeatKb = 5;
constexpr int kFeatA = 2 * 128 * 128, kFeatB = kFeatKb * 32 * 128;  // A: two K-block buffers
constexpr int kFeatSmem = 1024 + kFeatA + kFeatB + 7 * kFeatCols * 2;

__global__ void __launch_bounds__(kFeatThreads) image_features_kernel(const float* __restrict__ img0,
                                                                      const float* __restrict__ img1, int M, int N,
                                                                      const bf16* __restrict__ W1,
                                                                      const float* __restrict__ b1,
                                                                      const bf16* __restrict__ W2,
                                                                      const float* __restrict__ b2,
                                                                      bf16* __restrict__ out0,
                                                                      bf16* __restrict__ out1, int* __restrict__ err) {
  // grid.z selects the image: both images' CTAs in one launch (one tail, not two)
  const float* __restrict__ img = blockIdx.z ? img1 : img0;
  bf16* __restrict__ out = blockIdx.z ? out1 : out0;
  extern __shared__ unsigned char feat_raw[];
  __shared__ float w1[32][9], bs1[32], bs2[32];
  __shared__ __align__(8) uint64_t kbar[2];  // MMAs of the K-blocks in A buffer 0 / 1 done
  __shared__ uint32_t s_tmem;
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(feat_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* tA = smem;
  unsigned char* tB = smem + kFeatA;
  bf16* patch = reinterpret_cast<bf16*>(smem + kFeatA + kFeatB);  // [7][kFeatCols]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int M1 = (M + 1) / 2, N1 = (N + 1) / 2, N2 = (N1 + 1) / 2;
  const int i2 = blockIdx.y, j20 = blockIdx.x * 128;
  const int pi0 = 4 * i2 - 3, pj0 = 4 * j20 - 3;  // image pixel (0-based) of patch (0, 0)
  for (int q = tid; q < 32 * 9; q += kFeatThreads) w1[q / 9][q % 9] = __bfloat162float(W1[(q / 9) * 16 + q % 9]);
  if (tid < 32) {
    bs1[tid] = b1[tid];
    bs2[tid] = b2[tid];
  }
  // image patch: column-major image, 7 consecutive rows per column; every load of a thread is
  // issued before any store (one round of memory latency, not five)
  {
    constexpr int kIters = (kFeatCols + kFeatThreads - 1) / kFeatThreads;
    float v[kIters][7];
#pragma unroll
    for (int it = 0; it < kIters; ++it) {
      const int q = tid + it * kFeatThreads, j = pj0 + q;
#pragma unroll
      for (int a = 0; a < 7; ++a) {
        const int i = pi0 + a;
        v[it][a] = (q < kFeatCols && i >= 0 && i < M && j >= 0 && j < N) ? img[(size_t)i + (size_t)j * M] : 0.f;
      }
    }
#pragma unroll
    for (int it = 0; it < kIters; ++it) {
      const int q = tid + it * kFeatThreads;
      if (q < kFeatCols)
#pragma unroll
        for (int a = 0; a < 7; ++a) patch[a * kFeatCols + q] = __float2bfloat16_rn(v[it][a]);
    }
  }
  // conv2 weights: K-block kb, row n, chunk c = columns 64 kb + 8 c .. + 7 (zero from 288)
  {
    constexpr int kIters = kFeatKb * 32 * 8 / kFeatThreads;
    uint4 v[kIters];
#pragma unroll
    for (int it = 0; it < kIters; ++it) {
      const int q = tid + it * kFeatThreads, n = (q / 8) % 32, c = q % 8, col = (q / 256) * 64 + c * 8;
      v[it] = col < 288 ? *reinterpret_cast<const uint4*>(W2 + n * 288 + col) : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int it = 0; it < kIters; ++it) {
      const int q = tid + it * kFeatThreads, kb = q / 256, n = (q / 8) % 32, c = q % 8;
      *reinterpret_cast<uint4*>(tB + kb * 32 * 128 + n * 128 + ((c ^ (n & 7)) << 4)) = v[it];
    }
  }
  if (tid == 0) {
    mbar_init(&kbar[0], 1);
    mbar_init(&kbar[1], 1);
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(&s_tmem, 32);
  tcgen05_before_sync();
  __syncthreads();
  tcgen05_after_sync();
  // conv2's im2col row r (output pixel (i2, j20 + r)): tap t = (ky, kx) holds conv1 at
  // (2 i2 - 1 + ky, 2 j2 - 1 + kx), 32 channels = 4 chunks at K-block t / 2, chunks
  // 4 (t % 2) .. + 3; K-block 4's chunks 4..7 (columns 288..319) are zero.  K-blocks are built
  // into two alternating buffers while the previous one's MMAs run.  Thread: channel group cg
  // (8 channels, their weights in registers) of rows 4 rg .. 4 rg + 3.
  const int cg = tid & 3, rg = tid >> 2;
  float wr[8][9], br[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    br[k] = bs1[cg * 8 + k];
#pragma unroll
    for (int q = 0; q < 9; ++q) wr[k][q] = w1[cg * 8 + k][q];
  }
  const uint32_t tmem = s_tmem;
  bool ready = true;
#pragma unroll 1
  for (int kb = 0; kb < kFeatKb; ++kb) {
    const int buf = kb & 1;
    unsigned char* tAk = tA + buf * 128 * 128;
    if (kb >= 2) {  // the MMAs of K-block kb - 2 read this buffer
      ready = mbar_wait(&kbar[buf], (uint32_t)(((kb - 2) >> 1) & 1), kCorrWaitCycles) && ready;
      tcgen05_after_sync();
    }
#pragma unroll 1
    for (int rr = 0; rr < 4; ++rr) {
      const int r = rg * 4 + rr, j2 = j20 + r;
#pragma unroll 1
      for (int t = 2 * kb; t < 2 * kb + 2; ++t) {
        const int chunk0 = (t % 2) * 4;
        if (t >= 9) {  // K columns 288..319
          if (cg == 0)
#pragma unroll
            for (int chunk = 4; chunk < 8; ++chunk)
              *reinterpret_cast<uint4*>(tAk + r * 128 + ((chunk ^ (r & 7)) << 4)) = make_uint4(0u, 0u, 0u, 0u);
          continue;
        }
        const int ky = t / 3, kx = t % 3;
        const int i1 = 2 * i2 - 1 + ky, j1 = 2 * j2 - 1 + kx;
        const bool on_map = i1 >= 0 && i1 < M1 && j1 >= 0 && j1 < N1;
        float x[9];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b)
            x[a * 3 + b] = __bfloat162float(patch[(2 * ky + a) * kFeatCols + 4 * r + 2 * kx + b]);
        __align__(16) bf16 o[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          float acc = 0.f;
#pragma unroll
          for (int q = 0; q < 9; ++q) acc = fmaf(wr[k][q], x[q], acc);
          o[k] = __float2bfloat16_rn(on_map ? fmaxf(acc + br[k], 0.f) : 0.f);
        }
        const int chunk = chunk0 + cg;
        *reinterpret_cast<uint4*>(tAk + r * 128 + ((chunk ^ (r & 7)) << 4)) = *reinterpret_cast<const uint4*>(o);
      }
    }
    fence_proxy_async_shared();
    tcgen05_before_sync();
    __syncthreads();
    tcgen05_after_sync();
    if (tid == 0) {
      constexpr uint32_t idesc = bf16_idesc(128, 32);
      const uint32_t a = smem_u32(tAk), bb = smem_u32(tB + kb * 32 * 128);
#pragma unroll
      for (int k = 0; k < 4; ++k) umma_bf16(tmem, sw128_desc(a + 32 * k), sw128_desc(bb + 32 * k), idesc, kb > 0 || k > 0);
      umma_commit(&kbar[buf]);
    }
    __syncwarp();
  }
  // K-block 4's commit (buffer 0, its third phase) covers every MMA issued before it
  ready = mbar_wait(&kbar[0], 0u, kCorrWaitCycles) && ready;
  if (!ready && lane == 0) atomicOr(err, 8);
  tcgen05_after_sync();
  {
    const int r = warp * 32 + lane, j2 = j20 + r;
    float v[32];
    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16), *reinterpret_cast<float(*)[16]>(v));
    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + 16u, *reinterpret_cast<float(*)[16]>(v + 16));
    if (j2 < N2) {
      uint4* dst = reinterpret_cast<uint4*>(out + ((size_t)i2 * N2 + j2) * 32);
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        __align__(16) bf16 o[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float x = v[g * 8 + k] + bs2[g * 8 + k];
          o[k] = __float2bfloat16_rn(x > 0.f ? x : 0.f);
        }
        dst[g] = *reinterpret_cast<const uint4*>(o);
      }
    }
  }
  tcgen05_before_sync();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, 32);
}

// conv4 (3 x 3, stride 1, pad 1, 64 -> 64 channels on the 4 x 4 map) as one dense
// 1024 x 1024 matrix on the flattened map (index (y 4 + x) 64 + c): W4d[(oy, ox, co)][(iy, ix,
// ci)] = W4[co][(ky, kx, ci)] where (iy, ix) = (oy - 1 + ky, ox - 1 + kx), else 0; with its
// transpose and the bias per output entry.  One thread per entry.
__global__ void conv4_dense_kernel(const bf16* __restrict__ w4, const float* __restrict__ b4, bf16* __restrict__ W,
                                   bf16* __restrict__ WT, float* __restrict__ bd) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 1024 * 1024; e += gridDim.x * blockDim.x) {
    const int r = e / 1024, c = e % 1024;
    const int co = r % 64, oy = r / 256, ox = (r / 64) % 4;
    const int ci = c % 64, iy = c / 256, ix = (c / 64) % 4;
    const int ky = iy - oy + 1, kx = ix - ox + 1;
    const bf16 v = (ky >= 0 && ky <= 2 && kx >= 0 && kx <= 2) ? w4[co * 576 + (ky * 3 + kx) * 64 + ci]
                                                              : __float2bfloat16_rn(0.f);
    W[(size_t)r * 1024 + c] = v;
    WT[(size_t)c * 1024 + r] = v;
    if (c == 0) bd[r] = b4[co];
  }
}

// The conv4 weight gradient from the dense one: dW4[co][(ky, kx, ci)] sums dW4d over the
// output positions whose tap (ky, kx) stays on the map (fixed order).
__global__ void conv4_fold_kernel(const float* __restrict__ dWd, float* __restrict__ g) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 64 * 576; e += gridDim.x * blockDim.x) {
    const int co = e / 576, k = e % 576, tap = k / 64, ci = k % 64, ky = tap / 3, kx = tap % 3;
    float acc = 0.f;
    for (int oy = 0; oy < 4; ++oy) {
      const int iy = oy - 1 + ky;
      if (iy < 0 || iy >= 4) continue;
      for (int ox = 0; ox < 4; ++ox) {
        const int ix = ox - 1 + kx;
        if (ix < 0 || ix >= 4) continue;
        acc += dWd[(size_t)((oy * 4 + ox) * 64 + co) * 1024 + (iy * 4 + ix) * 64 + ci];
      }
    }
    g[e] += acc;
  }
}

// out[c, r] = in[r, c] (BF16, 32 x 32 tiles through shared memory)
__global__ void transpose_kernel(const bf16* __restrict__ in, bf16* __restrict__ out, long long R, long long Cn) {
  __shared__ bf16 t[32][33];
  const long long r0 = blockIdx.y * 32LL, c0 = blockIdx.x * 32LL;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const long long r = r0 + j, c = c0 + threadIdx.x;
    t[j][threadIdx.x] = (r < R && c < Cn) ? in[r * Cn + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const long long c = c0 + j, r = r0 + threadIdx.x;
    if (c < Cn && r < R) out[c * R + r] = t[threadIdx.x][j];
  }
}

// dZ = dH where the layer's output was positive (ReLU), as BF16
__global__ void relu_grad_kernel(const float* __restrict__ dH, const bf16* __restrict__ H, bf16* __restrict__ dZ,
                                 long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dZ[i] = __float2bfloat16_rn(__bfloat162float(H[i]) > 0.f ? dH[i] : 0.f);
}

// loss = mean over batch x 6 of (y - t)^2; dY = d loss / dy (BF16, the 6 outputs of 16 columns)
__global__ void mse_kernel(const float* __restrict__ Y, const float* __restrict__ T, int batch, bf16* __restrict__ dY,
                           float* __restrict__ loss) {
  __shared__ float red[256];
  float s = 0.f;
  const float scale = 2.f / (float)(batch * kOut);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch * kOutP; i += gridDim.x * blockDim.x) {
    const int b = i / kOutP, j = i % kOutP;
    float g = 0.f;
    if (j < kOut) {
      const float d = Y[(size_t)b * kOutP + j] - T[(size_t)b * kOut + j];
      s += d * d;
      g = scale * d;
    }
    dY[i] = __float2bfloat16_rn(g);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] / (float)(batch * kOut));
}

// db[c] += sum over rows of dZ[r, c] (each block sums a chunk of rows; one atomic per column)
__global__ void bias_grad_kernel(const bf16* __restrict__ dZ, long long R, int Cn, float* __restrict__ db) {
  const int c = threadIdx.x;
  if (c >= Cn) return;
  const long long per = ceil_div_ll(R, gridDim.x);
  const long long r0 = blockIdx.x * per, r1 = r0 + per < R ? r0 + per : R;
  float s = 0.f;
  for (long long r = r0; r < r1; ++r) s += __bfloat162float(dZ[r * Cn + c]);
  atomicAdd(db + c, s);
}

// Adam (Kingma & Ba 2015) on the flat FP32 parameters, refreshing their BF16 copies
__global__ void adam_kernel(float* __restrict__ w, bf16* __restrict__ wb, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, long long n, float lr, float b1, float b2,
                            float eps, float bc1, float bc2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ x, bf16* __restrict__ y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

// The network input of subset t (centre rounded to whole pixels): the frame's normalised
// deformed image over rows x0-36 .. x0+35 and columns y0-36 .. y0+35 (1-based) in channel 1,
// its normalised reference image over the centre 40 x 40 of that window (rows x0-20 .. x0+19)
// in channel 0, zero outside the image.  One block of 256 threads per subset.
__global__ void patch_kernel(FrameDev fr, const double* __restrict__ coords, long long n, bf16* __restrict__ X) {
  const long long t = blockIdx.x;
  if (t >= n) return;
  const int x0 = (int)llround(coords[t]), y0 = (int)llround(coords[n + t]);
  bf16* x = X + t * kWin * kWin * 2;
  for (int p = threadIdx.x; p < kWin * kWin; p += blockDim.x) {
    const int i = p / kWin, j = p % kWin;
    const int r1 = x0 - kWin / 2 + i, c1 = y0 - kWin / 2 + j;  // 1-based image pixel
    const bool in_img = r1 >= 1 && r1 <= fr.M && c1 >= 1 && c1 <= fr.N;
    const bool in_ref = i >= kRefOff && i < kRefOff + kRefWin && j >= kRefOff && j < kRefOff + kRefWin;
    const size_t o = (size_t)(r1 - 1) + (size_t)(c1 - 1) * fr.M;
    x[(size_t)p * 2] = __float2bfloat16_rn(in_img && in_ref ? fr.ref[o] : 0.f);
    x[(size_t)p * 2 + 1] = __float2bfloat16_rn(in_img ? fr.def[o] : 0.f);
  }
}

// Network outputs (scaled) -> IC-GN initial guess: U0 = (u, v), F0 = (du/dx, dv/dx, du/dy,
// dv/dy).  With coords, the prediction belongs to the aligned centre (x = 1 mod 4) nearest the
// subset's: U0 moves to the subset's own centre along F0; ok[t] = 0 gives NaN (no guess).
__global__ void unscale_kernel(const float* __restrict__ Y, long long n, double* __restrict__ U0,
                               double* __restrict__ F0, const double* __restrict__ coords, long long ncoords,
                               const uint8_t* __restrict__ ok) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const float* y = Y + t * kOutP;
    double f[4];
    for (int k = 0; k < 4; ++k) f[k] = y[2 + k] / 20.0;
    double u = 8.0 * y[0], v = 8.0 * y[1];
    if (coords) {
      const double x = coords[t], yy = coords[ncoords + t];
      const double ex = x - (4.0 * llround((x - 1.0) / 4.0) + 1.0), ey = yy - (4.0 * llround((yy - 1.0) / 4.0) + 1.0);
      u += f[0] * ex + f[2] * ey;
      v += f[1] * ex + f[3] * ey;
    }
    if (ok && !ok[t]) u = v = __longlong_as_double(0x7ff8000000000000LL);
    U0[2 * t] = u;
    U0[2 * t + 1] = v;
    for (int k = 0; k < 4; ++k) F0[4 * t + k] = f[k];
  }
}

inline unsigned blocks_for(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  return (unsigned)(b < 1 ? 1 : (b > 148 * 64 ? 148 * 64 : b));
}

}  // namespace

// ============================================================================ the network
struct ProposalNet {
  int device = 0, max_batch = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  std::string err;
  long long launches = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  bf16* wb = nullptr;
  bf16* wt[6] = {};  // transposed weights [cols x rows] for the data gradients
  int step_count = 0;
  // activations and their gradients (max_batch): per convolution its im2col rows A and their
  // transpose At, output H (NHWC) and output gradient dZ with its transpose dZt; the
  // FC1's input transposed (Ht5), output H6 (Ht6) and output gradient dZ6 (dZt6); the output
  // gradient dY (dYt).  conv3's im2col rows A[kConv3] come straight from the correlation.
  bf16 *A[kNumConv] = {}, *At[kNumConv] = {}, *H[kNumConv] = {}, *dZ[kNumConv] = {}, *dZt[kNumConv] = {};
  bf16 *Ht5 = nullptr, *H6 = nullptr, *Ht6 = nullptr, *dZ6 = nullptr, *dZt6 = nullptr;
  bf16 *W4d = nullptr, *W4dT = nullptr;  // conv4 as a dense 1024 x 1024 matrix and its transpose
  float* b4d = nullptr;                   // its bias per output entry
  bool w4d_valid = false;                 // W4d, W4dT, b4d match the current weights
  bf16 *dY = nullptr, *dYt = nullptr;
  float *dAf = nullptr, *dHf = nullptr, *Y = nullptr, *loss = nullptr;
  uint8_t* ok = nullptr;  // per predicted subset: its feature crops lie inside the maps
  // whole-image features for prediction (sized for the last frame size): the reference and
  // deformed conv2 maps
  int fM = 0, fN = 0;
  bf16 *FR = nullptr, *FD = nullptr;
  int* errflag = nullptr;
};

}  // namespace aldic

using aldic::ProposalNet;
struct aldic_net : ProposalNet {};

namespace aldic {
namespace {

#define NK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      net->err = std::string(#call) + ": " + cudaGetErrorString(e_);              \
      return ALDIC_ERR_CUDA;                                                      \
    }                                                                             \
  } while (0)

long long P_of(int i, int batch) { return (long long)batch * kConv[i].Hout * kConv[i].Hout; }

int gemm(ProposalNet* net, const void* A, long long lda, const void* B, long long ldb, long long M, long long N,
         long long K, int mode, float* c32, bf16* c16, const float* bias, long long ldc, int splits) {
  GemmArgs ga;
  ga.A = A;
  ga.lda = lda;
  ga.B = B;
  ga.ldb = ldb;
  ga.M = M;
  ga.N = N;
  ga.K = K;
  ga.splits = splits;
  ga.epi.mode = mode;
  ga.epi.c32 = c32;
  ga.epi.c16 = c16;
  ga.epi.bias = bias;
  ga.epi.ldc = ldc;
  ga.epi.err = net->errflag;
  const int r = launch_umma_gemm(ga, net->stream);
  if (r < 0) {
    net->err = "GEMM operand layout not describable by a tensor map";
    return ALDIC_ERR_ARG;
  }
  net->launches += r;
  return ALDIC_OK;
}

void transpose(ProposalNet* net, const bf16* in, bf16* out, long long R, long long Cn) {
  const dim3 grid((unsigned)((Cn + 31) / 32), (unsigned)((R + 31) / 32));
  transpose_kernel<<<grid, dim3(32, 8), 0, net->stream>>>(in, out, R, Cn);
  ++net->launches;
}

// split-K count for a weight gradient: enough blocks to fill the SMs
int wsplit(long long M, long long N, long long K) {
  const long long tiles = ((M + 127) / 128) * ((N + 255) / 256);
  long long s = (2 * 148) / (tiles < 1 ? 1 : tiles);
  const long long kb = (K + 63) / 64;
  if (s > kb) s = kb;
  return (int)(s < 1 ? 1 : s);
}

// im2col rows of convolution i's input (at `in` seen through v) into net->A[i]
void im2col(ProposalNet* net, int i, int batch, const bf16* in, View v) {
  const ConvI& L = kConv[i];
  const long long P = P_of(i, batch);
  im2col_kernel<<<blocks_for(P * (L.Kp / 8)), 256, 0, net->stream>>>(in, v, net->A[i], P, L);
  ++net->launches;
}

// im2col of convolution i's input and its GEMM with bias + ReLU
int conv_forward(ProposalNet* net, int i, int batch, const bf16* in, View v) {
  const ConvI& L = kConv[i];
  const long long P = P_of(i, batch);
  im2col(net, i, batch, in, v);
  return gemm(net, net->A[i], L.Kp, net->wb + kL.w[L.layer], L.Kp, P, L.Cout, L.Kp, kEpiBiasReluBf16, nullptr,
              net->H[i], net->w + kL.b[L.layer], L.Cout, 1);
}

// the layers after the correlation: conv3 (its im2col rows A[kConv3] written by the
// correlation kernel), conv4, FC1, FC2 (into net->Y)
int head(ProposalNet* net, int batch) {
  const ConvI& L3 = kConv[kConv3];
  int rc = gemm(net, net->A[kConv3], L3.Kp, net->wb + kL.w[L3.layer], L3.Kp, P_of(kConv3, batch), L3.Cout, L3.Kp,
                kEpiBiasReluBf16, nullptr, net->H[kConv3], net->w + kL.b[L3.layer], L3.Cout, 1);
  if (!rc) {  // conv4 as one dense GEMM on conv3's flattened output (no im2col)
    if (!net->w4d_valid) {  // rebuilt after every change of the weights
      conv4_dense_kernel<<<512, 256, 0, net->stream>>>(net->wb + kL.w[3], net->w + kL.b[3], net->W4d, net->W4dT,
                                                       net->b4d);
      ++net->launches;
      net->w4d_valid = true;
    }
    rc = gemm(net, net->H[kConv3], kFcIn, net->W4d, kFcIn, batch, kFcIn, kFcIn, kEpiBiasReluBf16, nullptr,
              net->H[kConv4], net->b4d, kFcIn, 1);
  }
  if (!rc)
    rc = gemm(net, net->H[kConv4], kFcIn, net->wb + kL.w[4], kFcIn, batch, kFcHid, kFcIn, kEpiBiasReluBf16, nullptr,
              net->H6, net->w + kL.b[4], kFcHid, 1);
  if (rc) return rc;
  return gemm(net, net->H6, kFcHid, net->wb + kL.w[5], kFcHid, batch, kOutP, kFcHid, kEpiStore, net->Y, nullptr,
              net->w + kL.b[5], kOutP, 1);
}

// crops of the kept features in the per-window conv2 outputs (B, 10, 10, 32) and (B, 18, 18, 32)
constexpr Crop kCropR{10 * 10 * 32, (10 + 1) * 32, 10 * 32};
constexpr Crop kCropD{18 * 18 * 32, (18 + 1) * 32, 18 * 32};

void conv1(ProposalNet* net, const bf16* in, View v, const ConvI& L, long long P, bf16* H) {
  conv1_kernel<<<blocks_for(P), 256, 0, net->stream>>>(in, v, L, P, net->wb + kL.w[0], net->w + kL.b[0], H);
  ++net->launches;
}

int corr_im2col(ProposalNet* net, const CorrSrc& src, int nb) {
  cudaFuncSetAttribute(corr_im2col_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kCorrSmem);
  cudaFuncSetAttribute(corr_im2col_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  int dev = 0, sms = 148, smem_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  // CTAs per SM by shared memory (1 KB reserved per CTA); TMEM (128 of 512 columns) allows 4
  const int per_sm = std::max(1, std::min(4, smem_sm / (kCorrSmem + 1024 + 64)));
  const int grid = std::max(1, std::min(nb, sms * per_sm));
  corr_im2col_kernel<<<(unsigned)grid, kCorrThreads, kCorrSmem, net->stream>>>(
      src, nb, net->A[kConv3], src.coords ? net->ok : nullptr, net->errflag);
  ++net->launches;
  return ALDIC_OK;
}

int forward(ProposalNet* net, int batch, const bf16* X) {
  conv1(net, X, kViewRef, kConv[kConvR1], P_of(kConvR1, batch), net->H[kConvR1]);
  conv1(net, X, kViewDef, kConv[kConvD1], P_of(kConvD1, batch), net->H[kConvD1]);
  int rc = conv_forward(net, kConvR2, batch, net->H[kConvR1], nhwc(20, 20, 32));
  if (!rc) rc = conv_forward(net, kConvD2, batch, net->H[kConvD1], nhwc(36, 36, 32));
  if (!rc) rc = corr_im2col(net, CorrSrc{net->H[kConvR2], net->H[kConvD2], kCropR, kCropD, nullptr, 0, 0, 0, 0}, batch);
  return rc ? rc : head(net, batch);
}

// weight and bias gradients of convolution i from its output gradient dZ[i] (added to net->g)
int conv_wgrad(ProposalNet* net, int i, int batch) {
  const ConvI& L = kConv[i];
  const long long P = P_of(i, batch);
  transpose(net, net->dZ[i], net->dZt[i], P, L.Cout);
  transpose(net, net->A[i], net->At[i], P, L.Kp);
  int rc = gemm(net, net->dZt[i], P, net->At[i], P, L.Cout, L.Kp, P, kEpiAtomic, net->g + kL.w[L.layer], nullptr,
                nullptr, L.Kp, wsplit(L.Cout, L.Kp, P));
  if (rc) return rc;
  bias_grad_kernel<<<148, L.Cout, 0, net->stream>>>(net->dZ[i], P, L.Cout, net->g + kL.b[L.layer]);
  ++net->launches;
  return ALDIC_OK;
}

// gradient of convolution i's input: dA = dZ W, then col2im into net->dHf (FP32, the input's
// NHWC layout)
int conv_dgrad(ProposalNet* net, int i, int batch) {
  const ConvI& L = kConv[i];
  const long long P = P_of(i, batch);
  int rc = gemm(net, net->dZ[i], L.Cout, net->wt[L.layer], L.Cout, P, L.Kp, L.Cout, kEpiStore, net->dAf, nullptr,
                nullptr, L.Kp, 1);
  if (rc) return rc;
  const long long nin = (long long)batch * L.Hin * L.Hin * L.Cin;
  col2im_kernel<<<blocks_for(nin), 256, 0, net->stream>>>(net->dAf, net->dHf, batch, L);
  ++net->launches;
  return ALDIC_OK;
}

void relu_grad(ProposalNet* net, const bf16* H, bf16* dZ, long long n) {
  relu_grad_kernel<<<blocks_for(n), 256, 0, net->stream>>>(net->dHf, H, dZ, n);
  ++net->launches;
}

// gradients of the mean squared error into net->g (zeroed here)
int backward(ProposalNet* net, int batch, const bf16* X, const float* T) {
  cudaStream_t st = net->stream;
  const long long B = batch;
  NK(cudaMemsetAsync(net->g, 0, sizeof(float) * kL.n, st));
  NK(cudaMemsetAsync(net->loss, 0, sizeof(float), st));
  mse_kernel<<<1, 256, 0, st>>>(net->Y, T, batch, net->dY, net->loss);
  ++net->launches;
  // transposed weights for the data gradients (conv1's input needs none)
  for (int l = 1; l < 6; ++l) transpose(net, net->wb + kL.w[l], net->wt[l], kL.rows[l], kL.cols[l]);
  // FC2: dW = dY^T H6, db = sum dY, dH6 = dY W
  transpose(net, net->dY, net->dYt, B, kOutP);
  transpose(net, net->H6, net->Ht6, B, kFcHid);
  int rc = gemm(net, net->dYt, B, net->Ht6, B, kOutP, kFcHid, B, kEpiAtomic, net->g + kL.w[5], nullptr, nullptr,
                kFcHid, wsplit(kOutP, kFcHid, B));
  if (rc) return rc;
  bias_grad_kernel<<<64, kOutP, 0, st>>>(net->dY, B, kOutP, net->g + kL.b[5]);
  ++net->launches;
  rc = gemm(net, net->dY, kOutP, net->wt[5], kOutP, B, kFcHid, kOutP, kEpiStore, net->dHf, nullptr, nullptr, kFcHid, 1);
  if (rc) return rc;
  relu_grad(net, net->H6, net->dZ6, B * kFcHid);
  // FC1: dW = dZ6^T F, db, dF = dZ6 W (F = conv4's output, flattened)
  transpose(net, net->dZ6, net->dZt6, B, kFcHid);
  transpose(net, net->H[kConv4], net->Ht5, B, kFcIn);
  rc = gemm(net, net->dZt6, B, net->Ht5, B, kFcHid, kFcIn, B, kEpiAtomic, net->g + kL.w[4], nullptr, nullptr, kFcIn,
            wsplit(kFcHid, kFcIn, B));
  if (rc) return rc;
  bias_grad_kernel<<<64, kFcHid, 0, st>>>(net->dZ6, B, kFcHid, net->g + kL.b[4]);
  ++net->launches;
  rc = gemm(net, net->dZ6, kFcHid, net->wt[4], kFcHid, B, kFcIn, kFcHid, kEpiStore, net->dHf, nullptr, nullptr, kFcIn,
            1);
  if (rc) return rc;
  relu_grad(net, net->H[kConv4], net->dZ[kConv4], B * kFcIn);
  // conv4, conv3
  // conv4 (dense): dW4d = dZ4^T H3 folded onto the 3 x 3 weights, db, dH3 = dZ4 W4d
  transpose(net, net->dZ[kConv4], net->dZt[kConv4], B, kFcIn);
  transpose(net, net->H[kConv3], net->At[kConv4], B, kFcIn);
  rc = gemm(net, net->dZt[kConv4], B, net->At[kConv4], B, kFcIn, kFcIn, B, kEpiStore, net->dAf, nullptr, nullptr,
            kFcIn, 1);
  if (rc) return rc;
  conv4_fold_kernel<<<144, 256, 0, st>>>(net->dAf, net->g + kL.w[3]);
  bias_grad_kernel<<<148, 64, 0, st>>>(net->dZ[kConv4], B * 16, 64, net->g + kL.b[3]);
  net->launches += 2;
  rc = gemm(net, net->dZ[kConv4], kFcIn, net->W4dT, kFcIn, B, kFcIn, kFcIn, kEpiStore, net->dHf, nullptr, nullptr,
            kFcIn, 1);
  if (rc) return rc;
  relu_grad(net, net->H[kConv3], net->dZ[kConv3], B * 16 * 64);
  if ((rc = conv_wgrad(net, kConv3, batch)) || (rc = conv_dgrad(net, kConv3, batch))) return rc;
  // correlation: dHf holds dC (B, 8, 8, 81); the ReLUs of conv2's outputs folded in
  corr_grad_ref_kernel<<<blocks_for(B * 100 * 32), 256, 0, st>>>(net->dHf, net->H[kConvR2], net->H[kConvD2],
                                                                  net->dZ[kConvR2], B * 100 * 32);
  corr_grad_def_kernel<<<blocks_for(B * 324 * 32), 256, 0, st>>>(net->dHf, net->H[kConvR2], net->H[kConvD2],
                                                                  net->dZ[kConvD2], B * 324 * 32);
  net->launches += 2;
  // conv2 and conv1 on the reference subset, then on the deformed window (shared weights)
  if ((rc = conv_wgrad(net, kConvR2, batch)) || (rc = conv_dgrad(net, kConvR2, batch))) return rc;
  relu_grad(net, net->H[kConvR1], net->dZ[kConvR1], B * 400 * 32);
  im2col(net, kConvR1, batch, X, kViewRef);  // conv1 ran directly: its im2col rows for dW
  if ((rc = conv_wgrad(net, kConvR1, batch))) return rc;
  if ((rc = conv_wgrad(net, kConvD2, batch)) || (rc = conv_dgrad(net, kConvD2, batch))) return rc;
  relu_grad(net, net->H[kConvD1], net->dZ[kConvD1], B * 1296 * 32);
  im2col(net, kConvD1, batch, X, kViewDef);
  return conv_wgrad(net, kConvD1, batch);
}

int check_errflag(ProposalNet* net) {
  int e = 0;
  NK(cudaMemcpyAsync(&e, net->errflag, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
  NK(cudaStreamSynchronize(net->stream));
  if (e) {
    net->err = "a tensor-core GEMM wait timed out";
    return ALDIC_ERR_TIMEOUT;
  }
  return ALDIC_OK;
}

}  // namespace

int launch_net_patches(const FrameDev& fr, const double* coords, long long n, void* X, cudaStream_t st) {
  patch_kernel<<<(unsigned)n, 256, 0, st>>>(fr, coords, n, reinterpret_cast<bf16*>(X));
  return 1;
}

}  // namespace aldic

using namespace aldic;

extern "C" {

int64_t aldic_net_param_count(void) { return kL.n; }

int aldic_net_create(aldic_net** out, int device, int max_batch) {
  if (!out || max_batch < 8 || max_batch % 8 != 0 || max_batch > 65536) return ALDIC_ERR_ARG;
  *out = nullptr;
  aldic_net* net = new aldic_net();
  net->device = device;
  net->max_batch = max_batch;
  auto fail = [&](cudaError_t e) {
    aldic_net_destroy(net);
    (void)e;
    return ALDIC_ERR_CUDA;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&net->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(e);
  net->stream = net->own;
  const long long B = max_batch, n = kL.n;
  e = cudaMalloc(&net->w, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->g, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->m, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->v, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->wb, n * 2);
  for (int l = 0; l < 6 && e == cudaSuccess; ++l) e = cudaMalloc(&net->wt[l], kL.rows[l] * kL.cols[l] * 2);
  long long maxA = (long long)kFcIn * kFcIn, maxH = B * kFcIn;  // dAf also holds conv4's dense gradient
  for (int i = 0; i < kNumConv && e == cudaSuccess; ++i) {
    const ConvI& L = kConv[i];
    const long long P = P_of(i, (int)B);
    maxA = std::max(maxA, P * L.Kp);
    maxH = std::max(maxH, B * L.Hin * L.Hin * L.Cin);
    e = cudaMalloc(&net->A[i], P * L.Kp * 2);
    if (e == cudaSuccess) e = cudaMalloc(&net->At[i], P * L.Kp * 2);
    if (e == cudaSuccess) e = cudaMalloc(&net->H[i], P * L.Cout * 2);
    if (e == cudaSuccess) e = cudaMalloc(&net->dZ[i], P * L.Cout * 2);
    if (e == cudaSuccess) e = cudaMalloc(&net->dZt[i], P * L.Cout * 2);
  }
  if (e == cudaSuccess) e = cudaMalloc(&net->Ht5, B * kFcIn * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->W4d, kFcIn * kFcIn * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->W4dT, kFcIn * kFcIn * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->b4d, kFcIn * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->H6, B * kFcHid * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->Ht6, B * kFcHid * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->dZ6, B * kFcHid * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->dZt6, B * kFcHid * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->dY, B * kOutP * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->dYt, B * kOutP * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->Y, B * kOutP * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->dAf, maxA * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->dHf, maxH * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->loss, 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->ok, B);
  if (e == cudaSuccess) e = cudaMalloc(&net->errflag, 4);
  if (e != cudaSuccess) return fail(e);
  cudaMemset(net->m, 0, n * 4);
  cudaMemset(net->v, 0, n * 4);
  cudaMemset(net->w, 0, n * 4);
  cudaMemset(net->wb, 0, n * 2);
  cudaMemset(net->errflag, 0, 4);
  *out = net;
  return ALDIC_OK;
}

void aldic_net_destroy(aldic_net* net) {
  if (!net) return;
  cudaSetDevice(net->device);
  if (net->stream) cudaStreamSynchronize(net->stream);
  void* bufs[] = {net->w,  net->g,   net->m,   net->v,   net->wb,  net->Ht5, net->H6,     net->Ht6,
                  net->dZ6, net->dZt6, net->dY, net->dYt, net->Y, net->dAf, net->dHf, net->loss, net->ok,  net->errflag,
                  net->FR, net->FD, net->W4d, net->W4dT, net->b4d};
  for (void* p : bufs)
    if (p) cudaFree(p);
  for (int l = 0; l < 6; ++l)
    if (net->wt[l]) cudaFree(net->wt[l]);
  for (int i = 0; i < kNumConv; ++i) {
    bf16* per[] = {net->A[i], net->At[i], net->H[i], net->dZ[i], net->dZt[i]};
    for (bf16* p : per)
      if (p) cudaFree(p);
  }
  if (net->own) cudaStreamDestroy(net->own);
  delete net;
}

const char* aldic_net_last_error(const aldic_net* net) { return net ? net->err.c_str() : "null network"; }

int aldic_net_set_stream(aldic_net* net, void* stream) {
  if (!net) return ALDIC_ERR_ARG;
  net->stream = stream ? static_cast<cudaStream_t>(stream) : net->own;
  return ALDIC_OK;
}

int64_t aldic_net_launch_count(const aldic_net* net) { return net ? net->launches : 0; }

int aldic_net_set_params(aldic_net* net, const float* params) {
  if (!net || !params) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  NK(cudaMemcpyAsync(net->w, params, sizeof(float) * kL.n, cudaMemcpyDefault, net->stream));
  to_bf16_kernel<<<blocks_for(kL.n), 256, 0, net->stream>>>(net->w, net->wb, kL.n);
  NK(cudaMemsetAsync(net->m, 0, sizeof(float) * kL.n, net->stream));
  NK(cudaMemsetAsync(net->v, 0, sizeof(float) * kL.n, net->stream));
  net->step_count = 0;
  net->w4d_valid = false;
  ++net->launches;
  NK(cudaStreamSynchronize(net->stream));
  return ALDIC_OK;
}

int aldic_net_get_params(aldic_net* net, float* params) {
  if (!net || !params) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  NK(cudaMemcpyAsync(params, net->w, sizeof(float) * kL.n, cudaMemcpyDefault, net->stream));
  NK(cudaStreamSynchronize(net->stream));
  return ALDIC_OK;
}

int aldic_net_forward(aldic_net* net, int batch, const void* x, float* y) {
  if (!net || !x || !y || batch < 8 || batch % 8 != 0 || batch > net->max_batch) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  int rc = forward(net, batch, reinterpret_cast<const bf16*>(x));
  if (rc) return rc;
  NK(cudaMemcpy2DAsync(y, kOut * 4, net->Y, kOutP * 4, kOut * 4, batch, cudaMemcpyDefault, net->stream));
  NK(cudaGetLastError());
  return ALDIC_OK;
}

int aldic_net_gradients(aldic_net* net, int batch, const void* x, const float* t, float* grads, float* loss) {
  if (!net || !x || !t || batch < 8 || batch % 8 != 0 || batch > net->max_batch) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  int rc = forward(net, batch, reinterpret_cast<const bf16*>(x));
  if (!rc) rc = backward(net, batch, reinterpret_cast<const bf16*>(x), t);
  if (rc) return rc;
  if (grads) NK(cudaMemcpyAsync(grads, net->g, sizeof(float) * kL.n, cudaMemcpyDefault, net->stream));
  if (loss) NK(cudaMemcpyAsync(loss, net->loss, sizeof(float), cudaMemcpyDefault, net->stream));
  NK(cudaGetLastError());
  return check_errflag(net);
}

int aldic_net_train_step(aldic_net* net, int batch, const void* x, const float* t, float lr, float* loss) {
  if (!net || !x || !t || batch < 8 || batch % 8 != 0 || batch > net->max_batch || !(lr > 0)) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  int rc = forward(net, batch, reinterpret_cast<const bf16*>(x));
  if (!rc) rc = backward(net, batch, reinterpret_cast<const bf16*>(x), t);
  if (rc) return rc;
  net->step_count += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.f - std::pow(b1, (float)net->step_count), bc2 = 1.f - std::pow(b2, (float)net->step_count);
  adam_kernel<<<blocks_for(kL.n), 256, 0, net->stream>>>(net->w, net->wb, net->g, net->m, net->v, kL.n, lr, b1, b2,
                                                          1e-8f, bc1, bc2);
  ++net->launches;
  net->w4d_valid = false;
  if (loss) {
    NK(cudaMemcpyAsync(loss, net->loss, sizeof(float), cudaMemcpyDefault, net->stream));
    NK(cudaStreamSynchronize(net->stream));
  }
  NK(cudaGetLastError());
  return ALDIC_OK;
}

int aldic_gemm_bf16(const void* A, int64_t lda, const void* B, int64_t ldb, int64_t M, int64_t N, int64_t K, float* C,
                    int64_t ldc, int splits, void* stream) {
  if (!A || !B || !C || M < 0 || N < 0 || K < 0 || lda < K || ldb < K || ldc < N || splits < 1) return ALDIC_ERR_ARG;
  if (M == 0 || N == 0 || K == 0) return ALDIC_OK;
  GemmArgs g;
  g.A = A;
  g.lda = lda;
  g.B = B;
  g.ldb = ldb;
  g.M = M;
  g.N = N;
  g.K = K;
  g.splits = splits;
  g.epi.mode = splits > 1 ? kEpiAtomic : kEpiStore;
  g.epi.c32 = C;
  g.epi.c16 = nullptr;
  g.epi.bias = nullptr;
  g.epi.ldc = ldc;
  static int* errflag = nullptr;  // the GEMM time-out flag of this entry (one per process)
  if (!errflag && cudaMalloc(&errflag, sizeof(int)) != cudaSuccess) return ALDIC_ERR_CUDA;
  g.epi.err = errflag;
  if (launch_umma_gemm(g, static_cast<cudaStream_t>(stream)) < 0) return ALDIC_ERR_ARG;
  return cudaGetLastError() == cudaSuccess ? ALDIC_OK : ALDIC_ERR_CUDA;
}

int aldic_net_status(aldic_net* net) {
  if (!net) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  return check_errflag(net);
}

}  // extern "C"

namespace aldic {
// conv1 and conv2 over the whole reference and deformed images of frame fr into net->FR and
// net->FD: (M + 3) / 4 x (N + 3) / 4 x 32 maps whose pixel (i, j) is centred on image pixel
// (4 i + 1, 4 j + 1) (1-based); one image_features_kernel launch for both images
int image_features(ProposalNet* net, const FrameDev& fr) {
  const int M = fr.M, N = fr.N, M2 = (M + 3) / 4, N2 = (N + 3) / 4;
  const size_t P2 = (size_t)M2 * N2;
  if (net->fM != M || net->fN != N) {
    NK(cudaStreamSynchronize(net->stream));
    bf16** bufs[] = {&net->FR, &net->FD};
    for (bf16** b : bufs) {
      if (*b) NK(cudaFree(*b));
      *b = nullptr;
    }
    net->fM = net->fN = 0;
    NK(cudaMalloc(&net->FR, P2 * 32 * 2));
    NK(cudaMalloc(&net->FD, P2 * 32 * 2));
    net->fM = M;
    net->fN = N;
  }
  NK(cudaFuncSetAttribute(image_features_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kFeatSmem));
  const dim3 grid((unsigned)((N2 + 127) / 128), (unsigned)M2, 2u);  // z: reference, deformed
  image_features_kernel<<<grid, kFeatThreads, kFeatSmem, net->stream>>>(
      fr.ref, fr.def, M, N, net->wb + kL.w[0], net->w + kL.b[0], net->wb + kL.w[1], net->w + kL.b[1], net->FR,
      net->FD, net->errflag);
  ++net->launches;
  NK(cudaGetLastError());
  return ALDIC_OK;
}

// Predict the initial guesses of n subsets (coords device n x 2) on the frame fr: the feature
// maps of both images once, then the correlation volumes and the rest in batches of the
// network's max_batch; U0 (2n) and F0 (4n) device arrays (U0 NaN where a subset's crops
// leave the maps: no guess).
int net_predict(aldic_net* net, const FrameDev& fr, const double* coords_dev, long long n, double* U0, double* F0) {
  NK(cudaSetDevice(net->device));
  int rc = image_features(net, fr);
  if (rc) return rc;
  const int Hf = (fr.M + 3) / 4, Wf = (fr.N + 3) / 4;
  const int B = net->max_batch;
  for (long long s = 0; s < n; s += B) {
    const int nb = (int)std::min<long long>(B, n - s);
    const int bpad = (nb + 7) / 8 * 8;
    corr_im2col(net, CorrSrc{net->FR, net->FD, Crop{}, Crop{}, coords_dev, n, s, Hf, Wf}, nb);
    if (bpad > nb)
      NK(cudaMemsetAsync(net->A[kConv3] + (size_t)nb * 16 * 736, 0, (size_t)(bpad - nb) * 16 * 736 * 2, net->stream));
    rc = head(net, bpad);
    if (rc) return rc;
    unscale_kernel<<<blocks_for(nb), 256, 0, net->stream>>>(net->Y, nb, U0 + 2 * s, F0 + 4 * s, coords_dev + s, n,
                                                           net->ok);
    ++net->launches;
  }
  NK(cudaGetLastError());
  return ALDIC_OK;
}
}  // namespace aldic
