// Image preparation kernels: ROI normalisation (funNormalizeImg), 7-tap gradients
// (funImgGradient), type conversion, and the point interpolation primitive
// (ba_interp2_spline).  All are HBM-bound streaming kernels.
#include "common.cuh"
#include "kernels.h"

namespace aldic {

template <typename T>
__device__ __forceinline__ double load_px(const T* p, size_t k) {
  return (double)p[k];
}

// Sum of (x - shift)^power (power 1 or 2) over the ROI rows [gx0, gx1) x cols [gy0, gy1)
// (0-based, half open), for floating-point images.  A block walks whole ROI columns
// (contiguous rows, no per-pixel index division).  Each block writes a partial; the last
// block to finish adds the partials in a fixed order (deterministic) and stores
//   POWER 1: stats[0] = sum, stats[2] = mean;
//   POWER 2: stats[1] = sum of squared deviations, stats[3] = std (N-1 normalised).
template <typename T, int POWER>
__global__ void roi_moment_kernel(const T* __restrict__ img, int M, int gx0, int gx1, int gy0, int gy1,
                                  const double* __restrict__ shift_ptr, double* __restrict__ partials,
                                  unsigned int* __restrict__ counter, double* __restrict__ stats, long long count) {
  __shared__ double red[32];
  __shared__ bool last;
  const double shift = shift_ptr ? shift_ptr[0] : 0.0;
  const int rows = gx1 - gx0, cols = gy1 - gy0;
  double s = 0;
  for (int b = blockIdx.x; b < cols; b += gridDim.x) {
    const T* col = img + (size_t)(gy0 + b) * M + gx0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
      const double v = load_px(col, (size_t)r) - shift;
      s += (POWER == 1) ? v : v * v;
    }
  }
  s = warp_sum(s);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    partials[blockIdx.x] = t;
    __threadfence();
    const unsigned int done = atomicAdd(counter, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (last) {
    // fixed-order sum of the partials by the whole block (a few L2 reads per thread, then
    // the warp and block sums in a fixed tree)
    double t = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) t += __ldcg(partials + i);
    t = warp_sum(t);
    if (lane == 0) red[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double u = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) u += red[w];
      stats[POWER - 1] = u;
      stats[POWER + 1] = (POWER == 1) ? u / (double)count : sqrt(u / (double)(count - 1));
      *counter = 0;  // re-arm for the next use
    }
  }
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// The same statistics for integer images (u8, u16) in one pass: exact integer sums S1 = sum x
// and S2 = sum x^2 over the ROI, then the sum of squared deviations (n S2 - S1^2) / n from
// exact 128-bit integers, which the reference's two FP64 passes (the mean, then the squared
// deviations from it; funNormalizeImg.m) approximate to within their rounding.  partials
// holds 2 entries per block.
constexpr int kMomentCols = 8;  // ROI columns per block step of roi_moment_int_kernel

template <typename T>
__global__ void roi_moment_int_kernel(const T* __restrict__ img, int M, int gx0, int gx1, int gy0, int gy1,
                                      unsigned long long* __restrict__ partials, unsigned int* __restrict__ counter,
                                      double* __restrict__ stats, long long count) {
  __shared__ unsigned long long red[2][32];
  __shared__ bool last;
  const int rows = gx1 - gx0, cols = gy1 - gy0;
  // a block step covers kMomentCols ROI columns: each thread's loads of those columns are
  // independent, so they are all in flight at once (a loop of one load per step would wait
  // out each load's latency before issuing the next)
  unsigned long long s1 = 0, s2 = 0;
  for (int b0 = blockIdx.x * kMomentCols; b0 < cols; b0 += gridDim.x * kMomentCols) {
    const T* col = img + (size_t)(gy0 + b0) * M + gx0;
    const int nc = min(kMomentCols, cols - b0);
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
      unsigned int v[kMomentCols];
#pragma unroll
      for (int k = 0; k < kMomentCols; ++k) v[k] = k < nc ? (unsigned int)col[(size_t)k * M + r] : 0u;
#pragma unroll
      for (int k = 0; k < kMomentCols; ++k) {
        s1 += v[k];
        s2 += (unsigned long long)v[k] * v[k];
      }
    }
  }
  s1 = warp_sum_u64(s1);
  s2 = warp_sum_u64(s2);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = s1;
    red[1][warp] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t1 = 0, t2 = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      t1 += red[0][w];
      t2 += red[1][w];
    }
    partials[2 * blockIdx.x] = t1;
    partials[2 * blockIdx.x + 1] = t2;
    __threadfence();
    const unsigned int done = atomicAdd(counter, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (last) {
    // the whole block sums the partials (L2 reads; integer sums, so any order is exact)
    unsigned long long t1 = 0, t2 = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
      t1 += __ldcg(partials + 2 * i);
      t2 += __ldcg(partials + 2 * i + 1);
    }
    t1 = warp_sum_u64(t1);
    t2 = warp_sum_u64(t2);
    if (lane == 0) {
      red[0][warp] = t1;
      red[1][warp] = t2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      t1 = 0;
      t2 = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        t1 += red[0][w];
        t2 += red[1][w];
      }
      const double n = (double)count;
      const unsigned __int128 d =
          (unsigned __int128)(unsigned long long)count * t2 - (unsigned __int128)t1 * t1;  // >= 0
      const double nd = (double)(unsigned long long)(d >> 64) * 18446744073709551616.0 + (double)(unsigned long long)d;
      const double ssd = nd / n;
      stats[0] = (double)t1;  // exact: t1 < 2^53
      stats[1] = ssd;
      stats[2] = (double)t1 / n;
      stats[3] = sqrt(ssd / (n - 1.0));
      *counter = 0;  // re-arm for the next use
    }
  }
}

template <typename T>
__global__ void normalize_map_kernel(const T* __restrict__ img, long long npx, const double* __restrict__ stats,
                                     const uint8_t* __restrict__ mask, float* __restrict__ out) {
  const double mean = stats[2], sd = stats[3];
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < npx; k += (long long)gridDim.x * blockDim.x) {
    double v = ((double)img[k] - mean) / sd;
    if (mask && !mask[k]) v = 0.0;
    out[k] = (float)v;
  }
}

// u8 images take at most 256 values: each block tabulates (x - mean) / sd (the same FP64
// division, so the same bits as normalize_map_kernel) and maps 4 pixels per thread step
// (4-byte loads, 16-byte stores); vec = 0 when a pointer is not aligned for that.
__global__ void normalize_u8_kernel(const uint8_t* __restrict__ img, long long npx, const double* __restrict__ stats,
                                    const uint8_t* __restrict__ mask, float* __restrict__ out, int vec) {
  __shared__ float lut[256];
  const double mean = stats[2], sd = stats[3];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = (float)(((double)i - mean) / sd);
  __syncthreads();
  const long long stride = (long long)gridDim.x * blockDim.x, first = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n4 = vec ? npx / 4 : 0;
  for (long long k = first; k < n4; k += stride) {
    const uchar4 v = reinterpret_cast<const uchar4*>(img)[k];
    float4 o = make_float4(lut[v.x], lut[v.y], lut[v.z], lut[v.w]);
    if (mask) {
      const uchar4 m = reinterpret_cast<const uchar4*>(mask)[k];
      if (!m.x) o.x = 0.f;
      if (!m.y) o.y = 0.f;
      if (!m.z) o.z = 0.f;
      if (!m.w) o.w = 0.f;
    }
    reinterpret_cast<float4*>(out)[k] = o;
  }
  for (long long k = 4 * n4 + first; k < npx; k += stride) out[k] = (mask && !mask[k]) ? 0.f : lut[img[k]];
}

__global__ void f64_to_f32_kernel(const double* __restrict__ in, long long n, float* __restrict__ out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    out[k] = (float)in[k];
}

__global__ void f32_to_f64_kernel(const float* __restrict__ in, long long n, double* __restrict__ out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    out[k] = (double)in[k];
}

__global__ void mask_binarize_kernel(const double* __restrict__ in, long long n, uint8_t* __restrict__ out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    out[k] = in ? (in[k] != 0.0) : 1;
}

// funImgGradient (func/funImgGradient.m:52-78): correlation with
// h = [-1 9 -45 0 45 -9 1]/60 along dim 1 (gx) and dim 2 (gy) at pixel (i+3, j+3),
// times the mask there.  A block computes a 64-row x 32-column output tile from a 70 x 38
// input tile staged in shared memory (each input pixel read from memory about 1.3 times
// instead of once per tap column); thread (r, g) computes rows r, columns 8 g .. 8 g + 7,
// consecutive threads consecutive rows (coalesced stores, conflict-free shared reads).
constexpr int kGradTR = 64, kGradTC = 32, kGradPR = kGradTR + 6, kGradPC = kGradTC + 6;
__global__ void __launch_bounds__(256) gradient_kernel(const float* __restrict__ img, const uint8_t* __restrict__ mask,
                                                       int M, int N, float* __restrict__ gx, float* __restrict__ gy) {
  __shared__ float t[kGradPC][kGradPR];
  const int gM = M - 6, gN = N - 6;
  const int i0 = blockIdx.x * kGradTR, j0 = blockIdx.y * kGradTC;  // output tile origin
  // input rows i0 .. i0 + 69, columns j0 .. j0 + 37 (output (ii, jj) centres on (ii + 3, jj + 3))
  for (int q = threadIdx.x; q < kGradPR * kGradPC; q += blockDim.x) {
    const int r = q % kGradPR, c = q / kGradPR, i = i0 + r, j = j0 + c;
    t[c][r] = (i < M && j < N) ? __ldg(img + (size_t)i + (size_t)j * M) : 0.f;
  }
  __syncthreads();
  const int r = threadIdx.x % kGradTR, g = threadIdx.x / kGradTR;
  const int ii = i0 + r;
  if (ii >= gM) return;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int c = g * 8 + k, jj = j0 + c;
    if (jj >= gN) break;
    const int R = r + 3, Cc = c + 3;
    const float dx = ((t[Cc][R + 3] - t[Cc][R - 3]) - 9.0f * (t[Cc][R + 2] - t[Cc][R - 2]) +
                      45.0f * (t[Cc][R + 1] - t[Cc][R - 1])) * (1.0f / 60.0f);
    const float dy = ((t[Cc + 3][R] - t[Cc - 3][R]) - 9.0f * (t[Cc + 2][R] - t[Cc - 2][R]) +
                      45.0f * (t[Cc + 1][R] - t[Cc - 1][R])) * (1.0f / 60.0f);
    const float mk = mask ? (float)mask[(size_t)(ii + 3) + (size_t)(jj + 3) * M] : 1.0f;
    const size_t o = (size_t)ii + (size_t)jj * gM;
    gx[o] = dx * mk;
    gy[o] = dy * mk;
  }
}

// ba_interp2_spline (ba_interp2_spline.cpp:235-331) at n points: X = dim-2 and
// Y = dim-1 coordinate, 1-based; taps clamped to the image.
__global__ void interp_points_kernel(const float* __restrict__ img, int M, int N, long long n,
                                     const double* __restrict__ X, const double* __restrict__ Y,
                                     double* __restrict__ Z) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double x = X[k], y = Y[k];
    const double fx = floor(x), fy = floor(y);
    if (!(fabs(fx) < 1e9 && fabs(fy) < 1e9)) {
      Z[k] = ALDIC_NAN;
      continue;
    }
    // taps at 1-based floor-1 .. floor+2, i.e. 0-based floor-2 .. floor+1
    const int r0 = (int)fy - 2, c0 = (int)fx - 2;
    Z[k] = (double)stencil16_clamped(img, M, N, r0, c0, (float)(y - fy), (float)(x - fx));
  }
}

}  // namespace aldic

// ----------------------------------------------------------------------------------
// host launchers
// ----------------------------------------------------------------------------------
namespace aldic {

static int grid_for(long long n, int threads, int cap) {
  long long g = (n + threads - 1) / threads;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

int launch_normalize(const void* img, int dtype, int M, int N, int gx0, int gx1, int gy0, int gy1,
                     const uint8_t* mask, float* out, double* stats, double* partials, int npartials,
                     unsigned int* counter, cudaStream_t st) {
  const long long cnt = (long long)(gx1 - gx0) * (gy1 - gy0);
  const int th = 256;
  const int cols = gy1 - gy0;
  const int g = cols < npartials ? cols : npartials;            // FP partials: 1 per block
  const int csteps = (cols + kMomentCols - 1) / kMomentCols;   // integer kernel: column groups
  const int gi = csteps < npartials / 2 ? csteps : npartials / 2;  // integer partials: 2 per block
  const long long npx = (long long)M * N;
  const int gm = grid_for(npx, th, 4 * 148 * 4);
  unsigned long long* ip = reinterpret_cast<unsigned long long*>(partials);
  switch (dtype) {
    case 0: {
      roi_moment_int_kernel<uint8_t><<<gi, th, 0, st>>>((const uint8_t*)img, M, gx0, gx1, gy0, gy1, ip, counter,
                                                        stats, cnt);
      const int vec = ((uintptr_t)img % 4 == 0) && ((uintptr_t)out % 16 == 0) && ((uintptr_t)mask % 4 == 0);
      normalize_u8_kernel<<<grid_for((npx + 3) / 4, th, 148 * 8), th, 0, st>>>((const uint8_t*)img, npx, stats,
                                                                            mask, out, vec);
      return 2;
    }
    case 1:
      roi_moment_int_kernel<uint16_t><<<gi, th, 0, st>>>((const uint16_t*)img, M, gx0, gx1, gy0, gy1, ip, counter,
                                                         stats, cnt);
      normalize_map_kernel<uint16_t><<<gm, th, 0, st>>>((const uint16_t*)img, npx, stats, mask, out);
      return 2;
#define ALDIC_NORM_CASE(T)                                                                                        \
  roi_moment_kernel<T, 1><<<g, th, 0, st>>>((const T*)img, M, gx0, gx1, gy0, gy1, nullptr, partials, counter,    \
                                            stats, cnt);                                                        \
  roi_moment_kernel<T, 2><<<g, th, 0, st>>>((const T*)img, M, gx0, gx1, gy0, gy1, stats + 2, partials, counter,  \
                                            stats, cnt);                                                        \
  normalize_map_kernel<T><<<gm, th, 0, st>>>((const T*)img, npx, stats, mask, out);
    case 2: { ALDIC_NORM_CASE(float) return 3; }
    case 3: { ALDIC_NORM_CASE(double) return 3; }
#undef ALDIC_NORM_CASE
    default: return -1;
  }
}

int launch_f64_to_f32(const double* in, long long n, float* out, cudaStream_t st) {
  f64_to_f32_kernel<<<grid_for(n, 256, 4096), 256, 0, st>>>(in, n, out);
  return 1;
}

int launch_f32_to_f64(const float* in, long long n, double* out, cudaStream_t st) {
  f32_to_f64_kernel<<<grid_for(n, 256, 4096), 256, 0, st>>>(in, n, out);
  return 1;
}

int launch_mask_binarize(const double* in, long long n, uint8_t* out, cudaStream_t st) {
  mask_binarize_kernel<<<grid_for(n, 256, 4096), 256, 0, st>>>(in, n, out);
  return 1;
}

int launch_gradient(const float* img, const uint8_t* mask, int M, int N, float* gx, float* gy, cudaStream_t st) {
  const dim3 grid((unsigned)((M - 6 + kGradTR - 1) / kGradTR), (unsigned)((N - 6 + kGradTC - 1) / kGradTC));
  gradient_kernel<<<grid, 256, 0, st>>>(img, mask, M, N, gx, gy);
  return 1;
}

int launch_interp_points(const float* img, int M, int N, long long n, const double* X, const double* Y, double* Z,
                         cudaStream_t st) {
  interp_points_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(img, M, N, n, X, Y, Z);
  return 1;
}

}  // namespace aldic
