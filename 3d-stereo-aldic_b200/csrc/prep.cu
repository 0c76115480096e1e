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
// (0-based, half open).  Each block writes a partial; the last block to finish adds
// the partials in a fixed order (deterministic) and stores
//   POWER 1: stats[0] = sum, stats[2] = mean;
//   POWER 2: stats[1] = sum of squared deviations, stats[3] = std (N-1 normalised).
template <typename T, int POWER>
__global__ void roi_moment_kernel(const T* __restrict__ img, int M, int gx0, int gx1, int gy0, int gy1,
                                  const double* __restrict__ shift_ptr, double* __restrict__ partials,
                                  unsigned int* __restrict__ counter, double* __restrict__ stats, long long count) {
  __shared__ double red[32];
  __shared__ bool last;
  const double shift = shift_ptr ? shift_ptr[0] : 0.0;
  const int rows = gx1 - gx0;
  const long long total = (long long)rows * (gy1 - gy0);
  double s = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(k % rows), b = (int)(k / rows);
    const double v = load_px(img, (size_t)(gx0 + a) + (size_t)(gy0 + b) * M) - shift;
    s += (POWER == 1) ? v : v * v;
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
    // fixed-order sum of the partials by one warp
    if (threadIdx.x < 32) {
      double t = 0;
      for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) t += ((volatile double*)partials)[i];
      t = warp_sum(t);
      if (threadIdx.x == 0) {
        stats[POWER - 1] = t;
        stats[POWER + 1] = (POWER == 1) ? t / (double)count : sqrt(t / (double)(count - 1));
        *counter = 0;  // re-arm for the next use
      }
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
// times the mask there.  One thread per output pixel; columns of the output are
// contiguous so a warp reads 32 consecutive rows (coalesced).
__global__ void gradient_kernel(const float* __restrict__ img, const uint8_t* __restrict__ mask, int M, int N,
                                float* __restrict__ gx, float* __restrict__ gy) {
  const int gM = M - 6, gN = N - 6;
  const long long total = (long long)gM * gN;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % gM) + 3, j = (int)(k / gM) + 3;
    const float* c = img + (size_t)i + (size_t)j * M;
    const float dx = ((__ldg(c + 3) - __ldg(c - 3)) - 9.0f * (__ldg(c + 2) - __ldg(c - 2)) +
                      45.0f * (__ldg(c + 1) - __ldg(c - 1))) * (1.0f / 60.0f);
    const float dy = ((__ldg(c + 3 * (size_t)M) - __ldg(c - 3 * (size_t)M)) -
                      9.0f * (__ldg(c + 2 * (size_t)M) - __ldg(c - 2 * (size_t)M)) +
                      45.0f * (__ldg(c + (size_t)M) - __ldg(c - (size_t)M))) * (1.0f / 60.0f);
    const float mk = mask ? (float)mask[(size_t)i + (size_t)j * M] : 1.0f;
    gx[k] = dx * mk;
    gy[k] = dy * mk;
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
  const int g = grid_for(cnt, th, npartials);
  const long long npx = (long long)M * N;
  const int gm = grid_for(npx, th, 4 * 148 * 4);
#define ALDIC_NORM_CASE(T)                                                                                        \
  roi_moment_kernel<T, 1><<<g, th, 0, st>>>((const T*)img, M, gx0, gx1, gy0, gy1, nullptr, partials, counter,    \
                                            stats, cnt);                                                        \
  roi_moment_kernel<T, 2><<<g, th, 0, st>>>((const T*)img, M, gx0, gx1, gy0, gy1, stats + 2, partials, counter,  \
                                            stats, cnt);                                                        \
  normalize_map_kernel<T><<<gm, th, 0, st>>>((const T*)img, npx, stats, mask, out);
  switch (dtype) {
    case 0: { ALDIC_NORM_CASE(uint8_t) break; }
    case 1: { ALDIC_NORM_CASE(uint16_t) break; }
    case 2: { ALDIC_NORM_CASE(float) break; }
    case 3: { ALDIC_NORM_CASE(double) break; }
    default: return -1;
  }
#undef ALDIC_NORM_CASE
  return 3;  // kernels launched
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
  const long long total = (long long)(M - 6) * (N - 6);
  gradient_kernel<<<grid_for(total, 256, 148 * 16), 256, 0, st>>>(img, mask, M, N, gx, gy);
  return 1;
}

int launch_interp_points(const float* img, int M, int N, long long n, const double* X, const double* Y, double* Z,
                         cudaStream_t st) {
  interp_points_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(img, M, N, n, X, Y, Z);
  return 1;
}

}  // namespace aldic
