// Per-point stereo triangulation (func_quadtree/stereoReconstruction_quadtree.m:30-52,
// which calls MATLAB's triangulate: linear DLT solved by SVD).  FP64 throughout: the
// 4x4 homogeneous system is ill-conditioned at small stereo angles.
#include "common.cuh"
#include "kernels.h"

namespace aldic {

// One-sided (Hestenes) Jacobi SVD of a 4x4 matrix A (row-major a[r][c]); returns the
// right singular vector of the smallest singular value in x.
__device__ void smallest_right_singular(double a[4][4], double x[4]) {
  double V[4][4];
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) V[r][c] = (r == c) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < 3; ++p)
      for (int q = p + 1; q < 4; ++q) {
        double alpha = 0, beta = 0, gamma = 0;
        for (int r = 0; r < 4; ++r) {
          alpha += a[r][p] * a[r][p];
          beta += a[r][q] * a[r][q];
          gamma += a[r][p] * a[r][q];
        }
        const double scale = sqrt(alpha * beta);
        if (!(scale > 0)) continue;
        const double rel = fabs(gamma) / scale;
        if (rel > off) off = rel;
        if (rel < 1e-17) continue;
        const double zeta = (beta - alpha) / (2.0 * gamma);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        for (int r = 0; r < 4; ++r) {
          const double ap = a[r][p], aq = a[r][q];
          a[r][p] = cs * ap - sn * aq;
          a[r][q] = sn * ap + cs * aq;
          const double vp = V[r][p], vq = V[r][q];
          V[r][p] = cs * vp - sn * vq;
          V[r][q] = sn * vp + cs * vq;
        }
      }
    if (off < 1e-15) break;
  }
  int kmin = 0;
  double smin = INFINITY;
  for (int c = 0; c < 4; ++c) {
    double s = 0;
    for (int r = 0; r < 4; ++r) s += a[r][c] * a[r][c];
    if (s < smin) {
      smin = s;
      kmin = c;
    }
  }
  for (int r = 0; r < 4; ++r) x[r] = V[r][kmin];
}

// pairs: n x 4 column-major [xL yL xR yR]; cams: PL then PR, 3x4 row-major, passed by
// value; xyz: n x 3 col-major.
__global__ void triangulate_kernel(long long n, const double* __restrict__ pairs, CamPair cams,
                                   double* __restrict__ xyz, double* __restrict__ err) {
  const double* PL = cams.P;
  const double* PR = cams.P + 12;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double x1 = pairs[k], y1 = pairs[n + k], x2 = pairs[2 * n + k], y2 = pairs[3 * n + k];
    if (!(isfinite(x1) && isfinite(y1) && isfinite(x2) && isfinite(y2))) {
      xyz[k] = xyz[n + k] = xyz[2 * n + k] = ALDIC_NAN;
      if (err) err[k] = ALDIC_NAN;
      continue;
    }
    double A[4][4];
    for (int c = 0; c < 4; ++c) {
      A[0][c] = x1 * PL[8 + c] - PL[c];
      A[1][c] = y1 * PL[8 + c] - PL[4 + c];
      A[2][c] = x2 * PR[8 + c] - PR[c];
      A[3][c] = y2 * PR[8 + c] - PR[4 + c];
    }
    double X[4];
    smallest_right_singular(A, X);
    const double X0 = X[0] / X[3], X1 = X[1] / X[3], X2 = X[2] / X[3];
    xyz[k] = X0;
    xyz[n + k] = X1;
    xyz[2 * n + k] = X2;
    if (err) {
      const double lz = PL[8] * X0 + PL[9] * X1 + PL[10] * X2 + PL[11];
      const double lx = (PL[0] * X0 + PL[1] * X1 + PL[2] * X2 + PL[3]) / lz;
      const double ly = (PL[4] * X0 + PL[5] * X1 + PL[6] * X2 + PL[7]) / lz;
      const double rz = PR[8] * X0 + PR[9] * X1 + PR[10] * X2 + PR[11];
      const double rx = (PR[0] * X0 + PR[1] * X1 + PR[2] * X2 + PR[3]) / rz;
      const double ry = (PR[4] * X0 + PR[5] * X1 + PR[6] * X2 + PR[7]) / rz;
      err[k] = 0.5 * (hypot(lx - x1, ly - y1) + hypot(rx - x2, ry - y2));
    }
  }
}

int launch_triangulate(long long n, const double* pairs, const CamPair& cams, double* xyz, double* err,
                       cudaStream_t st) {
  if (n <= 0) return 0;
  long long g = (n + 127) / 128;
  if (g > 148 * 16) g = 148 * 16;
  triangulate_kernel<<<(unsigned)g, 128, 0, st>>>(n, pairs, cams, xyz, err);
  return 1;
}

// funUndistortPoints (func/funUndistortPoints.m:8-39, MATLAB undistortPoints per camera):
// the inverse of the radial / tangential lens model of cameraParameters.  A pixel (u, v)
// (1-based, as K's principal point) maps to normalised coordinates (xd, yd) = K^-1 (u, v, 1);
// the undistorted (x, y) solves
//     xd = x (1 + k1 r^2 + k2 r^4 + k3 r^6) + 2 p1 x y + p2 (r^2 + 2 x^2)
//     yd = y (1 + k1 r^2 + k2 r^4 + k3 r^6) + p1 (r^2 + 2 y^2) + 2 p2 x y,   r^2 = x^2 + y^2,
// found by the fixed-point iteration x <- (xd - tangential(x)) / radial(x) from (xd, yd) until
// the update is below 1e-15 of the point's scale (at most 200 steps); the result goes back
// through K.  Non-finite input rows give NaN.  FP64 throughout.
struct Lens {
  double K[9];     // 3 x 3 row-major
  double Kinv[9];  // 3 x 3 row-major
  double k1, k2, k3, p1, p2;
};

__global__ void undistort_points_kernel(long long n, const double* __restrict__ pts, Lens L, double* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double u = pts[i], v = pts[n + i];
  if (!isfinite(u) || !isfinite(v)) {
    out[i] = NAN;
    out[n + i] = NAN;
    return;
  }
  const double* Ki = L.Kinv;
  const double w = Ki[6] * u + Ki[7] * v + Ki[8];
  const double xd = (Ki[0] * u + Ki[1] * v + Ki[2]) / w, yd = (Ki[3] * u + Ki[4] * v + Ki[5]) / w;
  double x = xd, y = yd;
  for (int it = 0; it < 200; ++it) {
    const double r2 = x * x + y * y;
    const double radial = 1.0 + r2 * (L.k1 + r2 * (L.k2 + r2 * L.k3));
    const double tx = 2.0 * L.p1 * x * y + L.p2 * (r2 + 2.0 * x * x);
    const double ty = L.p1 * (r2 + 2.0 * y * y) + 2.0 * L.p2 * x * y;
    const double xn = (xd - tx) / radial, yn = (yd - ty) / radial;
    const double step = fabs(xn - x) + fabs(yn - y);
    x = xn;
    y = yn;
    if (step <= 1e-15 * (1.0 + fabs(x) + fabs(y))) break;
  }
  const double* K = L.K;
  const double ww = K[6] * x + K[7] * y + K[8];
  out[i] = (K[0] * x + K[1] * y + K[2]) / ww;
  out[n + i] = (K[3] * x + K[4] * y + K[5]) / ww;
}

int launch_undistort_points(long long n, const double* pts, const double* Kcm, const double* dist, double* out,
                            cudaStream_t st) {
  if (n <= 0) return 0;
  Lens L;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) L.K[r * 3 + c] = Kcm[r + 3 * c];  // MATLAB column-major
  const double* a = L.K;
  const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                     a[2] * (a[3] * a[7] - a[4] * a[6]);
  L.Kinv[0] = (a[4] * a[8] - a[5] * a[7]) / det;
  L.Kinv[1] = (a[2] * a[7] - a[1] * a[8]) / det;
  L.Kinv[2] = (a[1] * a[5] - a[2] * a[4]) / det;
  L.Kinv[3] = (a[5] * a[6] - a[3] * a[8]) / det;
  L.Kinv[4] = (a[0] * a[8] - a[2] * a[6]) / det;
  L.Kinv[5] = (a[2] * a[3] - a[0] * a[5]) / det;
  L.Kinv[6] = (a[3] * a[7] - a[4] * a[6]) / det;
  L.Kinv[7] = (a[1] * a[6] - a[0] * a[7]) / det;
  L.Kinv[8] = (a[0] * a[4] - a[1] * a[3]) / det;
  L.k1 = dist[0];
  L.k2 = dist[1];
  L.k3 = dist[2];
  L.p1 = dist[3];
  L.p2 = dist[4];
  undistort_points_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, pts, L, out);
  return 1;
}

// FP32 FMA throughput probe: 8 independent FMA chains per thread, enough blocks to fill
// every SM; used only to state the measured FP32 roofline beside the kernels.
__global__ void fp32_probe_kernel(int iters, float seed, float* out) {
  float a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
        a7 = a0 + 7;
  const float m = 0.9999f, c = 1e-4f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fmaf(a0, m, c);
      a1 = fmaf(a1, m, c);
      a2 = fmaf(a2, m, c);
      a3 = fmaf(a3, m, c);
      a4 = fmaf(a4, m, c);
      a5 = fmaf(a5, m, c);
      a6 = fmaf(a6, m, c);
      a7 = fmaf(a7, m, c);
    }
  }
  const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 123.456f) out[0] = s;  // keep the chains live
}

// The same loop on packed pairs (fma.rn.f32x2): 8 independent float2 chains.
__global__ void fp32x2_probe_kernel(int iters, float seed, float* out) {
  float2 a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = make_float2(seed + threadIdx.x + 2 * i, seed + threadIdx.x + 2 * i + 1);
  const float2 m = make_float2(0.9999f, 0.9999f), c = make_float2(1e-4f, 1e-4f);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
#pragma unroll
      for (int j = 0; j < 8; ++j) a[j] = ffma2(a[j], m, c);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i].x + a[i].y;
  if (s == 123.456f) out[0] = s;  // keep the chains live
}

// FMAs per thread per iteration: 128 in both forms.
int launch_fp32_probe(int blocks, int threads, int iters, float* out, bool packed, cudaStream_t st) {
  if (packed)
    fp32x2_probe_kernel<<<blocks, threads, 0, st>>>(iters, 0.5f, out);
  else
    fp32_probe_kernel<<<blocks, threads, 0, st>>>(iters, 0.5f, out);
  return 1;
}

}  // namespace aldic
