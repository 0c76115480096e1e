// Shared device helpers for the ALDIC B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define ALDIC_NAN __longlong_as_double(0x7ff8000000000000LL)

namespace aldic {

// ---------------------------------------------------------------------------------
// Local 4x4 B-spline stencil of ba_interp2_spline.cpp:235-331 in separable form.
// The reference evaluates A = BC*Q*BC^T and sum a_ij tr^i tc^j; since the stencil is the
// outer product of one cubic basis per axis, the same value is
//   sum_r w_r(tr) * sum_c w_c(tc) * Q[r][c]
// with w(t) = [(-33t + 57t^2 - 24t^3), (56 - 3t - 117t^2 + 64t^3),
//              (45t + 75t^2 - 64t^3),  (-9t - 15t^2 + 24t^3)] / 56,
// the rows of BC = B*C (B the cubic B-spline basis, C the truncated prefilter inverse
// [71 -19 5 -1; ...]/56).  The weights sum to 1 and w(0) = [0 1 0 0].
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void bspline_weights(float t, float w[4]) {
  const float k = 1.0f / 56.0f;
  w[0] = k * (t * fmaf(t, fmaf(t, -24.0f, 57.0f), -33.0f));
  w[1] = k * fmaf(t, fmaf(t, fmaf(t, 64.0f, -117.0f), -3.0f), 56.0f);
  w[2] = k * (t * fmaf(t, fmaf(t, -64.0f, 75.0f), 45.0f));
  w[3] = k * (t * fmaf(t, fmaf(t, 24.0f, -15.0f), -9.0f));
}

// Interpolate the column-major M-row image `img` with tap 0 at 0-based (r0, c0), all 16
// taps in bounds, fractions tr (dim 1) and tc (dim 2).
__device__ __forceinline__ float stencil16(const float* __restrict__ img, int M, int r0, int c0, float tr, float tc) {
  float wr[4], wc[4];
  bspline_weights(tr, wr);
  bspline_weights(tc, wc);
  const float* p = img + (size_t)r0 + (size_t)c0 * M;
  float acc = 0.f;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float* q = p + (size_t)c * M;
    float col = wr[0] * __ldg(q);
    col = fmaf(wr[1], __ldg(q + 1), col);
    col = fmaf(wr[2], __ldg(q + 2), col);
    col = fmaf(wr[3], __ldg(q + 3), col);
    acc = fmaf(wc[c], col, acc);
  }
  return acc;
}

// The same stencil in FP64 arranged as the reference's double path computes it
// (ba_interp2_spline.cpp:235-331): per row i of the integer matrix K = 56 BC (up to sign and
// scale), T_ij = K_j . (K_i . Q), and the value sum_ij s_ij T_ij tr^i tc^j, where each
// scale s_ij is a float-literal constant of the reference rounded to float before it is
// promoted (3/56, 1/7, 9/3136, 3/392, 1/49; ba_interp2_spline.cpp:310-325).  It tracks the
// reference MEX to ~1e-13 and serves the FP64 re-solve of subsets whose FP32 convergence
// decision was too close to call.  All 16 taps in bounds.
__device__ __forceinline__ double stencil16_ref64(const float* __restrict__ img, int M, int r0, int c0, double tr,
                                                  double tc) {
  constexpr int K[4][4] = {{0, 1, 0, 0}, {11, 1, -15, 3}, {19, -39, 25, -5}, {-3, 8, -8, 3}};
  constexpr double sgn[4] = {1.0, -1.0, 1.0, 1.0};
  const double s356 = (double)(3.0f / 56.0f), s17 = (double)(1.0f / 7.0f);
  const double s9 = (double)((1.0f / 3136.0f) * 9.0f), s3392 = (double)(3.0f / 392.0f);
  const double s149 = (double)(1.0f / 49.0f);
  const double one[4] = {1.0, s356, s356, s17};
  const float* p = img + (size_t)r0 + (size_t)c0 * M;
  double rowc[4][4];  // rowc[i][c] = sum_r K_i[r] Q[r][c]
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double q0 = __ldg(p + (size_t)c * M), q1 = __ldg(p + (size_t)c * M + 1);
    const double q2 = __ldg(p + (size_t)c * M + 2), q3 = __ldg(p + (size_t)c * M + 3);
#pragma unroll
    for (int i = 0; i < 4; ++i) rowc[i][c] = ((K[i][0] * q0 + K[i][1] * q1) + K[i][2] * q2) + K[i][3] * q3;
  }
  const double pr[4] = {1.0, tr, tr * tr, tr * tr * tr};
  const double pc[4] = {1.0, tc, tc * tc, tc * tc * tc};
  double val = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const double t = ((K[j][0] * rowc[i][0] + K[j][1] * rowc[i][1]) + K[j][2] * rowc[i][2]) + K[j][3] * rowc[i][3];
      double s;
      if (i == 0 || j == 0) s = (i == 0) ? one[j] : one[i];
      else if (i == 3 && j == 3) s = s149;
      else if (i == 3 || j == 3) s = s3392;
      else s = s9;
      val += sgn[i] * sgn[j] * s * t * pr[i] * pc[j];
    }
  return val;
}

// Clamped version for arbitrary points (the MEX clamps taps to the image edge,
// ba_interp2_spline.cpp:60-66).
__device__ __forceinline__ float stencil16_clamped(const float* __restrict__ img, int M, int N, int r0, int c0, float tr,
                                                   float tc) {
  float wr[4], wc[4];
  bspline_weights(tr, wr);
  bspline_weights(tc, wc);
  float acc = 0.f;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int cc = min(max(c0 + c, 0), N - 1);
    float col = 0.f;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int rr = min(max(r0 + r, 0), M - 1);
      col = fmaf(wr[r], __ldg(img + (size_t)rr + (size_t)cc * M), col);
    }
    acc = fmaf(wc[c], col, acc);
  }
  return acc;
}

// ---------------------------------------------------------------------------------
// Packed FP32 pairs (sm_100 .f32x2 instructions): one instruction, two lanes of IEEE
// round-to-nearest results, each identical to the scalar operation.
// ---------------------------------------------------------------------------------
// The host forms (same IEEE results lane by lane) serve host-side checks of the
// functions built on them.
__host__ __device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
#ifndef __CUDA_ARCH__
  return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#else
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
#endif
}

__host__ __device__ __forceinline__ float2 fmul2(float2 a, float2 b) {
#ifndef __CUDA_ARCH__
  return make_float2(a.x * b.x, a.y * b.y);
#else
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
#endif
}

__host__ __device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
#ifndef __CUDA_ARCH__
  return make_float2(a.x + b.x, a.y + b.y);
#else
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
#endif
}

__host__ __device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
#ifndef __CUDA_ARCH__
  return make_float2(a.x - b.x, a.y - b.y);
#else
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
#endif
}

// Kahan-compensated accumulation (Kahan 1965), the compensation kept with the opposite sign:
// the running total is s + k.  The caller forms y = x + k, fused into the term's own
// operation (y = fma(a, b, k) for a product term), then
//   t = s + y;  k = (s - t) + y;  s = t
// (each operation rounded on its own: packed instructions or _rn intrinsics, never
// contracted or reassociated).  The error of the total is bounded by ~2 ulp of sum |x|,
// independent of the number of terms.
__host__ __device__ __forceinline__ void kahan2(float2& s, float2& k, float2 y) {
  const float2 t = fadd2(s, y);
  k = fadd2(fsub2(s, t), y);
  s = t;
}

__device__ __forceinline__ void kahan1(float& s, float& k, float y) {
  const float t = __fadd_rn(s, y);
  k = __fadd_rn(__fsub_rn(s, t), y);
  s = t;
}

// Two stencils at once with packed FP32 pairs (.x: point a, .y: point b); each lane's
// result is bit-identical to stencil16 at that point.
__device__ __forceinline__ void bspline_weights_x2(float2 t, float2 w[4]) {
  const float2 k = make_float2(1.0f / 56.0f, 1.0f / 56.0f);
  w[0] = fmul2(k, fmul2(t, ffma2(t, ffma2(t, make_float2(-24.0f, -24.0f), make_float2(57.0f, 57.0f)),
                                 make_float2(-33.0f, -33.0f))));
  w[1] = fmul2(k, ffma2(t, ffma2(t, ffma2(t, make_float2(64.0f, 64.0f), make_float2(-117.0f, -117.0f)),
                                 make_float2(-3.0f, -3.0f)),
                        make_float2(56.0f, 56.0f)));
  w[2] = fmul2(k, fmul2(t, ffma2(t, ffma2(t, make_float2(-64.0f, -64.0f), make_float2(75.0f, 75.0f)),
                                 make_float2(45.0f, 45.0f))));
  w[3] = fmul2(k, fmul2(t, ffma2(t, ffma2(t, make_float2(24.0f, 24.0f), make_float2(-15.0f, -15.0f)),
                                 make_float2(-9.0f, -9.0f))));
}

__device__ __forceinline__ float2 stencil16_x2(const float* __restrict__ img, int M, int ia, int ib, float2 tr,
                                               float2 tc) {
  // ia, ib: element index of tap 0 (r0 + c0 M) of the two points
  float2 wr[4], wc[4];
  bspline_weights_x2(tr, wr);
  bspline_weights_x2(tc, wc);
  const float* pa = img + ia;
  const float* pb = img + ib;
  float2 acc = make_float2(0.f, 0.f);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float* qa = pa + c * M;
    const float* qb = pb + c * M;
    float2 col = fmul2(wr[0], make_float2(__ldg(qa), __ldg(qb)));
    col = ffma2(wr[1], make_float2(__ldg(qa + 1), __ldg(qb + 1)), col);
    col = ffma2(wr[2], make_float2(__ldg(qa + 2), __ldg(qb + 2)), col);
    col = ffma2(wr[3], make_float2(__ldg(qa + 3), __ldg(qb + 3)), col);
    acc = ffma2(wc[c], col, acc);
  }
  return acc;
}

// The two stencils of stencil16_x2 read from a staged shared-memory tile (column-major,
// `pitch` rows); oa, ob are the tile offsets of tap 0.  Same operations in the same order,
// so each lane's value is bit-identical to stencil16_x2 on the image.
__device__ __forceinline__ float2 stencil16_x2_tile(const float* tile, int pitch, int oa, int ob, float2 tr,
                                                    float2 tc) {
  float2 wr[4], wc[4];
  bspline_weights_x2(tr, wr);
  bspline_weights_x2(tc, wc);
  const float* pa = tile + oa;
  const float* pb = tile + ob;
  float2 acc = make_float2(0.f, 0.f);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float* qa = pa + c * pitch;
    const float* qb = pb + c * pitch;
    float2 col = fmul2(wr[0], make_float2(qa[0], qb[0]));
    col = ffma2(wr[1], make_float2(qa[1], qb[1]), col);
    col = ffma2(wr[2], make_float2(qa[2], qb[2]), col);
    col = ffma2(wr[3], make_float2(qa[3], qb[3]), col);
    acc = ffma2(wc[c], col, acc);
  }
  return acc;
}

// stencil16 on a staged tile (see stencil16_x2_tile); bit-identical to stencil16.
__device__ __forceinline__ float stencil16_tile(const float* tile, int pitch, int o, float tr, float tc) {
  float wr[4], wc[4];
  bspline_weights(tr, wr);
  bspline_weights(tc, wc);
  const float* p = tile + o;
  float acc = 0.f;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float* q = p + c * pitch;
    float col = wr[0] * q[0];
    col = fmaf(wr[1], q[1], col);
    col = fmaf(wr[2], q[2], col);
    col = fmaf(wr[3], q[3], col);
    acc = fmaf(wc[c], col, acc);
  }
  return acc;
}

// ---------------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum of one double per thread over the block, returned to every thread (fixed order: warp
// shuffles, then the warp totals in warp order).  red holds blockDim.x / 32 doubles; the
// leading barrier lets the same red serve call after call.
__device__ __forceinline__ double block_sum_all(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
  return s;
}

// Block-wide sums of K doubles per thread; result in out[0..K) (shared), visible to all
// threads after return.  scratch must hold (NT/32)*K doubles.
template <int K, int NT>
__device__ __forceinline__ void block_sum(double (&v)[K], double* scratch, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double s = warp_sum(v[k]);
    if (lane == 0) scratch[warp * K + k] = s;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) s += scratch[w * K + threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// Block-wide FP64 sums of K per-thread FP32 partials, converting one value at a time so
// that only the FP32 partials stay live (low register pressure for wide one-off sums).
template <int K, int NT>
__device__ __forceinline__ void block_sum_f32(float (&v)[K], double* scratch, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double s = warp_sum((double)v[k]);
    if (lane == 0) scratch[warp * K + k] = s;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += NT) {
    double s = 0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) s += scratch[w * K + k];
    out[k] = s;
  }
  __syncthreads();
}

// Block-wide sums for a runtime number of warps (scratch holds nwarps*K doubles).
template <int K>
__device__ __forceinline__ void block_sum_dyn(double (&v)[K], double* scratch, double* out, int nwarps) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double s = warp_sum(v[k]);
    if (lane == 0) scratch[warp * K + k] = s;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0;
    for (int w = 0; w < nwarps; ++w) s += scratch[w * K + threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------
// bwselect: connected component of `on` pixels (rows x cols, column-major, u8) that
// contains the 0-based seed (sr, sc), 4- or 8-connected, into `lab` (u8).  Iterated
// in-place propagation until no pixel changes; bounded by rows*cols sweeps (every
// productive sweep adds at least one pixel).  All threads of the block must call it.
// ---------------------------------------------------------------------------------
__device__ inline void flood_select(const uint8_t* on, uint8_t* lab, int rows, int cols, int sr, int sc, int conn,
                             int* flag) {
  const int npx = rows * cols;
  for (int p = threadIdx.x; p < npx; p += blockDim.x) lab[p] = 0;
  __syncthreads();
  const bool seed_ok = sr >= 0 && sr < rows && sc >= 0 && sc < cols && on[sr + sc * rows];
  if (!seed_ok) {
    __syncthreads();
    return;
  }
  if (threadIdx.x == 0) lab[sr + sc * rows] = 1;
  __syncthreads();
  for (int sweep = 0; sweep < npx; ++sweep) {
    int changed = 0;
    for (int p = threadIdx.x; p < npx; p += blockDim.x) {
      if (lab[p] || !on[p]) continue;
      const int r = p % rows, c = p / rows;
      bool hit = false;
      if (r > 0 && lab[p - 1]) hit = true;
      if (r + 1 < rows && lab[p + 1]) hit = true;
      if (c > 0 && lab[p - rows]) hit = true;
      if (c + 1 < cols && lab[p + rows]) hit = true;
      if (!hit && conn == 8) {
        if (r > 0 && c > 0 && lab[p - 1 - rows]) hit = true;
        if (r + 1 < rows && c > 0 && lab[p + 1 - rows]) hit = true;
        if (r > 0 && c + 1 < cols && lab[p - 1 + rows]) hit = true;
        if (r + 1 < rows && c + 1 < cols && lab[p + 1 + rows]) hit = true;
      }
      if (hit) {
        lab[p] = 1;
        changed = 1;
      }
    }
    if (!__syncthreads_or(changed)) break;
  }
  (void)flag;
}

// MATLAB round(): half away from zero.
__device__ __forceinline__ double mround(double x) { return round(x); }

// Inverse-compositional update P <- P o dP^-1 (func/funICGN.m:289-307).  Returns false
// when det(dP) == 0.
__device__ __forceinline__ bool compose_inverse(double P[6], const double d[6]) {
  const double det = (1 + d[0]) * (1 + d[3]) - d[1] * d[2];
  if (!(det != 0)) return false;
  const double t1 = (-d[0] - d[0] * d[3] + d[1] * d[2]) / det;
  const double t2 = -d[1] / det;
  const double t3 = -d[2] / det;
  const double t4 = (-d[3] - d[0] * d[3] + d[1] * d[2]) / det;
  const double t5 = (-d[4] - d[3] * d[4] + d[2] * d[5]) / det;
  const double t6 = (-d[5] - d[0] * d[5] + d[1] * d[4]) / det;
  const double a00 = 1 + P[0], a01 = P[2], a02 = P[4];
  const double a10 = P[1], a11 = 1 + P[3], a12 = P[5];
  const double n00 = a00 * (1 + t1) + a01 * t2;
  const double n10 = a10 * (1 + t1) + a11 * t2;
  const double n01 = a00 * t3 + a01 * (1 + t4);
  const double n11 = a10 * t3 + a11 * (1 + t4);
  const double n02 = a00 * t5 + a01 * t6 + a02;
  const double n12 = a10 * t5 + a11 * t6 + a12;
  P[0] = n00 - 1;
  P[1] = n10;
  P[2] = n01;
  P[3] = n11 - 1;
  P[4] = n02;
  P[5] = n12;
  return true;
}

// x = A^-1 b for an n x n (n <= 6) column-major system, Gaussian elimination with
// partial pivoting in FP64 (mldivide's general path; a zero pivot yields Inf/NaN).
__device__ inline void solve_small(int n, const double* Ain, const double* bin, double* x) {
  double A[36], b[6];
  for (int i = 0; i < n * n; ++i) A[i] = Ain[i];
  for (int i = 0; i < n; ++i) b[i] = bin[i];
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = fabs(A[k + k * n]);
    for (int i = k + 1; i < n; ++i)
      if (fabs(A[i + k * n]) > best) {
        best = fabs(A[i + k * n]);
        piv = i;
      }
    if (piv != k) {
      for (int j = 0; j < n; ++j) {
        const double t = A[k + j * n];
        A[k + j * n] = A[piv + j * n];
        A[piv + j * n] = t;
      }
      const double t = b[k];
      b[k] = b[piv];
      b[piv] = t;
    }
    for (int i = k + 1; i < n; ++i) {
      const double l = A[i + k * n] / A[k + k * n];
      for (int j = k; j < n; ++j) A[i + j * n] -= l * A[k + j * n];
      b[i] -= l * b[k];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < n; ++j) s -= A[i + j * n] * x[j];
    x[i] = s / A[i + i * n];
  }
}

}  // namespace aldic
