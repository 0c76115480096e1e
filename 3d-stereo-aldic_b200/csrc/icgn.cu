// Batched local IC-GN (6-DOF, first-order shape function) and the ALDIC Subpb1
// augmented-Lagrangian local step on the B200.
//
// Structure of one batched call (all subsets of one frame):
//   1. classify kernel, one warp per subset: coordinate rounding, window bounds, the
//      zero-count rules of the reference (funICGN.m:57-68, funICGNQuadtree.m:61-79,
//      funICGN_Subpb1quadtree.m:68-89), final window size.  Subsets that end here
//      (solver error -> -1, too much masked -> 102) are written out; the others are
//      appended to one of two work queues: nominal window size, or enlarged window.
//   2. solve kernel per queue, persistent (grid = resident CTAs), one CTA of NT threads
//      per subset.  The subset's f, f_x, f_y live in shared memory for the whole solve;
//      each Gauss-Newton iteration interpolates g with the local 4x4 B-spline stencil
//      (FP32), accumulates the b-vector statistics in one pass (FP32 per thread, FP64
//      across threads), and thread 0 does the FP64 6x6 update and inverse composition.
//      Masked (quadtree) subsets additionally run the bwselect flood fills in shared
//      memory.
//
// The single-pass b-vector: with fn = (f - mean_f)/bf the reference's
//   b_k = bf * sum_p J_k(p) [fn(p) - (g(p) - mean_g)/bg]
// equals bf * (A_k - (C_k - mean_g * B_k) / bg) with A_k = sum J_k fn, B_k = sum J_k
// (constant per subset) and C_k = sum J_k g (per iteration); mean_g and bg come from
// sum g, sum g^2 over the same pass.
#include <cstring>
#include <mutex>
#include <type_traits>

#include "common.cuh"
#include "kernels.h"
#include "tma.cuh"

namespace aldic {

constexpr int kNT = 128;  // threads per solve CTA
constexpr int kSlowSubset = 2;   // queue-1 flag of a subset continued by the multi-warp pass
constexpr int kMovedSubset = 4;  // queue-1 flag of a subset moved to the FP64 re-solve queue
constexpr int kToFp64 = 5;       // hand-off code of the warp passes: re-solve in FP64

struct SolveCtl {
  double P[6];
  double Hinv[36];
  double H[21];
  double A[6], B[6];
  double meanf, bf, sabsf;
  double normNew, normAbs, normInit;
  double gsum_prev;
  double znssd;
  double d5, d6;  // P5 - round(P5), P6 - round(P6) (FP64 interpolation)
  float pf[4], f5, f6;
  int base_r, base_c;  // 0-based tap-0 row/col offsets: x0 + n5 - 2, y0 + n6 - 2
  int step, go, status, need_mask, fbw8_ready, done_error, to_fp64;
};

__device__ __forceinline__ bool is_intd(double v) { return floor(v) == v && fabs(v) < 1e9; }

// Window [x0 - wx/2, x0 + wx/2] x [y0 - wy/2, y0 + wy/2] (1-based) inside the image and,
// if need_grad, inside the gradient arrays shifted by crop.
__device__ __forceinline__ bool window_ok(const FrameDev& fr, double x0, double y0, double wx, double wy, bool need_grad,
                                          int crop) {
  const double r0 = x0 - wx / 2, r1 = x0 + wx / 2, c0 = y0 - wy / 2, c1 = y0 + wy / 2;
  if (!is_intd(r0) || !is_intd(r1) || !is_intd(c0) || !is_intd(c1)) return false;
  if (r0 < 1 || r1 > fr.M || c0 < 1 || c1 > fr.N) return false;
  if (need_grad) {
    if (r0 - crop < 1 || r1 - crop > fr.M - 6 || c0 - crop < 1 || c1 - crop > fr.N - 6) return false;
  }
  return true;
}

// Any corner of the warped window outside [3, M-2] x [3, N-2] (func/funICGN.m:121-124);
// the warp is affine so the extremes are at the corners.  Non-finite -> outside.
__device__ __forceinline__ bool warped_oob(const FrameDev& fr, const double P[6], double x0, double y0, double hx,
                                           double hy) {
  bool oob = false;
  for (int cx = -1; cx <= 1; cx += 2)
    for (int cy = -1; cy <= 1; cy += 2) {
      const double dx = cx * hx, dy = cy * hy;
      const double u = (1 + P[0]) * dx + P[2] * dy + (x0 + P[4]);
      const double v = P[1] * dx + (1 + P[3]) * dy + (y0 + P[5]);
      if (!(u >= 3 && u <= fr.M - 2 && v >= 3 && v <= fr.N - 2)) oob = true;
    }
  return oob;
}

// Per-iteration FP32 warp coefficients: u22 - (x0 + n5) = dx + P1 dx + P3 dy + f5 with
// n5 = round(P5), f5 = P5 - n5, so the coordinate keeps full FP32 precision relative to
// the subset centre.
__device__ __forceinline__ void prep_coeffs(SolveCtl& c, double x0, double y0) {
  const double n5 = mround(c.P[4]), n6 = mround(c.P[5]);
  c.pf[0] = (float)c.P[0];
  c.pf[1] = (float)c.P[1];
  c.pf[2] = (float)c.P[2];
  c.pf[3] = (float)c.P[3];
  c.d5 = c.P[4] - n5;
  c.d6 = c.P[5] - n6;
  c.f5 = (float)c.d5;
  c.f6 = (float)c.d6;
  c.base_r = (int)(x0 + n5) - 2;
  c.base_c = (int)(y0 + n6) - 2;
}

// Interpolate g at window pixel (dx, dy) with the current coefficients.
__device__ __forceinline__ float warp_g(const FrameDev& fr, const SolveCtl& c, float dx, float dy) {
  const float lx = dx + fmaf(c.pf[0], dx, fmaf(c.pf[2], dy, c.f5));
  const float ly = dy + fmaf(c.pf[3], dy, fmaf(c.pf[1], dx, c.f6));
  const float ix = floorf(lx), iy = floorf(ly);
  return stencil16(fr.def, fr.M, c.base_r + (int)ix, c.base_c + (int)iy, lx - ix, ly - iy);
}

// Gauss-Jordan inverse of a 6x6 (column-major) with partial pivoting, FP64.
__device__ void invert6(const double* Hin, double* Hinv) {
  double A[36], I[36];
  for (int k = 0; k < 36; ++k) {
    A[k] = Hin[k];
    I[k] = (k % 7 == 0) ? 1.0 : 0.0;
  }
  for (int k = 0; k < 6; ++k) {
    int piv = k;
    double best = fabs(A[k + 6 * k]);
    for (int i = k + 1; i < 6; ++i)
      if (fabs(A[i + 6 * k]) > best) {
        best = fabs(A[i + 6 * k]);
        piv = i;
      }
    if (piv != k)
      for (int j = 0; j < 6; ++j) {
        double t = A[k + 6 * j];
        A[k + 6 * j] = A[piv + 6 * j];
        A[piv + 6 * j] = t;
        t = I[k + 6 * j];
        I[k + 6 * j] = I[piv + 6 * j];
        I[piv + 6 * j] = t;
      }
    const double d = A[k + 6 * k];
    for (int j = 0; j < 6; ++j) {
      A[k + 6 * j] /= d;
      I[k + 6 * j] /= d;
    }
    for (int i = 0; i < 6; ++i) {
      if (i == k) continue;
      const double l = A[i + 6 * k];
      for (int j = 0; j < 6; ++j) {
        A[i + 6 * j] -= l * A[k + 6 * j];
        I[i + 6 * j] -= l * I[k + 6 * j];
      }
    }
  }
  for (int k = 0; k < 36; ++k) Hinv[k] = I[k];
}

// ================================================================================
// classify kernel (one warp per subset)
// ================================================================================
__global__ void icgn_classify_kernel(IcgnArgs a) {
  const long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= a.n) return;
  const FrameDev& fr = a.fr;
  double x0 = a.coords[t], y0 = a.coords[a.n + t];
  const bool quad = (a.variant == 1);
  if (quad) {
    x0 = mround(x0);
    y0 = mround(y0);
  }
  const double w = a.winsize;
  const double Nw = (w + 1) * (w + 1);
  int status = 0;  // 0 active, -1 error, 102 masked-out
  double wfin = w;
  uint8_t mark = 0;
  // zero counts over the nominal window
  const bool img_ok = window_ok(fr, x0, y0, w, w, false, a.crop);
  const bool grad_ok = img_ok && window_ok(fr, x0, y0, w, w, true, a.crop);
  long long cnt = 0;
  if (img_ok) {
    const int W1 = (int)w + 1;
    const int r0 = (int)(x0 - w / 2) - 1, c0 = (int)(y0 - w / 2) - 1;
    for (int p = lane; p < W1 * W1; p += 32) {
      const int aa = p % W1, bb = p / W1;
      const size_t k = (size_t)(r0 + aa) + (size_t)(c0 + bb) * fr.M;
      if (quad) {
        const float f = fr.ref[k];
        const bool mk = fr.mask ? (fr.mask[k] != 0) : true;
        cnt += (!mk || f == 0.f);
      } else if (grad_ok) {
        const size_t kg = (size_t)(r0 + aa - a.crop) + (size_t)(c0 + bb - a.crop) * (fr.M - 6);
        cnt += (fr.gx[kg] == 0.f);
      }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  if (quad) mark = (!img_ok || cnt > 0.6 * Nw) ? 1 : 0;
  if (!grad_ok) {
    status = -1;
  } else if (quad) {
    if (cnt < 0.4 * Nw) {
      if (cnt > 0) {
        wfin = 2 * ceil(sqrt(Nw / (Nw - (double)cnt)) * w / 2);
        if (!window_ok(fr, x0, y0, wfin, wfin, true, a.crop)) status = -1;
      }
    } else {
      status = 102;
    }
  } else {
    if (cnt < 0.5 * Nw) {
      if (cnt > 0.1 * Nw) {
        wfin = mround(1.4142135623730951 * w);
        if (!window_ok(fr, x0, y0, wfin, wfin, true, a.crop)) status = -1;
      }
    } else {
      status = 102;
    }
  }
  if (lane != 0) return;
  if (quad && a.mark) a.mark[t] = mark;
  if (status == 0) {
    const int bucket = (wfin == w) ? 0 : 1;
    const int pos = atomicAdd(&a.qcount[bucket], 1);
    int* q = a.queue + 3 * ((long long)bucket * a.n + pos);
    q[0] = (int)t;
    q[1] = (int)wfin;
    q[2] = (quad && cnt > 0) ? 1 : 0;
    return;
  }
  // finished here
  if (a.variant == 2) {
    a.znssd[t] = ALDIC_NAN;
    if (a.conv) a.conv[t] = status;
    return;
  }
  a.conv[t] = status;
  if (status == -1) {
    a.U[2 * t] = ALDIC_NAN;
    a.U[2 * t + 1] = ALDIC_NAN;
    for (int k = 0; k < 4; ++k) a.F[4 * t + k] = ALDIC_NAN;
  } else {  // 102: U = U0, F = 0
    a.U[2 * t] = a.U0[2 * t];
    a.U[2 * t + 1] = a.U0[2 * t + 1];
    for (int k = 0; k < 4; ++k) a.F[4 * t + k] = 0.0;
  }
  if (a.H)
    for (int k = 0; k < 21; ++k) a.H[t + a.n * k] = 0.0;
}

// ================================================================================
// 6-DOF solve kernel (general: masks, enlarged windows; FP32, or FP64 for re-solves)
// ================================================================================
// Shared-memory arrays of one subset: g (the interpolated deformed window, FP32 or FP64),
// f, f_x, f_y (FP32 image data), and the u8 masks of the flood fills.
template <bool F64>
struct SolveSmem {
  using G = typename std::conditional<F64, double, float>::type;
  G* g;
  float* f;
  float* gx;
  float* gy;
  uint8_t* on;    // f-mask pixel on (quadtree)
  uint8_t* lab;   // flood-fill output (bw4, then per-iteration g region)
  uint8_t* tmp;   // flood-fill input
  uint8_t* fbw8;  // 8-connected f-mask region (g-mask fallback)
};

template <bool F64>
__device__ __forceinline__ SolveSmem<F64> carve(unsigned char* base, int npx) {
  using G = typename SolveSmem<F64>::G;
  SolveSmem<F64> s;
  s.g = reinterpret_cast<G*>(base);  // first: 8-byte aligned for the FP64 form
  s.f = reinterpret_cast<float*>(s.g + npx);
  s.gx = s.f + npx;
  s.gy = s.gx + npx;
  uint8_t* u = reinterpret_cast<uint8_t*>(s.gy + npx);
  s.on = u;
  s.lab = u + npx;
  s.tmp = u + 2 * npx;
  s.fbw8 = u + 3 * npx;
  return s;
}

// Queue 2 receives a subset for the FP64 re-solve (from its initial guess): its entry keeps
// the window and the masked flag of the entry it came from.
__device__ __forceinline__ void push_fp64(const IcgnArgs& a, long long t, int w, int masked) {
  const int pos = atomicAdd(&a.qcount[4], 1);
  int* q2 = a.queue + 3 * (2 * a.n + pos);
  q2[0] = (int)t;
  q2[1] = w;
  q2[2] = masked;
}

// Whether a convergence test (funICGN.m:268-282: |b|/|b_1| < tol or |b| < tol) lies too close
// to tol for FP32 arithmetic to decide it as the FP64 reference does; such subsets are
// re-solved in FP64.  Two margins: a relative one, band * tol, and the FP32 noise of |b| at
// this iteration, sig = step * noise * 2^-24 * (bf / bg) * sqrt(tr(H) * sum(g^2) / n) (the
// rounding of the products J_k g and of the interpolated g, about sqrt(n) terms of size
// |J| |g|; it grows with the iterations behind it), which dominates when |b| itself is
// near tol.  The relative test |b| / |b_1| carries sig / |b_1|.
__device__ __forceinline__ bool too_close_to_call(double normRel, double normAbs, double normInit, double tol,
                                                  double band, double sig) {
  if (!(band > 0)) return false;
  if (!(fabs(normAbs - tol) > band * tol + sig)) return true;  // NaN also goes to FP64
  return normInit > tol && !(fabs(normRel - tol) > band * tol + sig / normInit);
}

__device__ __forceinline__ double fp32_noise(double factor, int step, double bf, double bg, double trH, double sum_g2,
                                             double n) {
  return step * factor * 5.9604644775390625e-08 * (bf / bg) * sqrt(fmax(trH * sum_g2 / n, 0.0));
}

// The FP32 form solves queue 1 (enlarged or masked subsets and those handed over by the warp
// passes) and moves subsets whose convergence test is too close to call to queue 2; the FP64
// form (interpolation in the reference's own double arithmetic, FP64 sums) re-solves queue 2
// from the initial guesses, so its decisions are the FP64 reference's.
template <bool F64, int NT>
__global__ void __launch_bounds__(NT) icgn_solve_kernel(IcgnArgs a, int bucket) {
  using G = typename SolveSmem<F64>::G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ SolveCtl c;
  __shared__ double red[(NT / 32) * 40];
  __shared__ double sums[40];
  const int tid = threadIdx.x;
  const FrameDev& fr = a.fr;
  const bool quad = (a.variant == 1);
  const bool epi = (a.variant == 2);
  const bool want_fg = epi || a.zncc != nullptr;  // sum f g: the epipolar ZNSSD, or the ZNCC
  const int count = a.qcount[bucket == 2 ? 4 : bucket];
  const int gM = fr.M - 6;
  for (int qi = blockIdx.x; qi < count; qi += gridDim.x) {
    const int* q = a.queue + 3 * ((long long)bucket * a.n + qi);
    const long long t = q[0];
    const int w = q[1];
    if (q[2] == kSlowSubset || q[2] == kMovedSubset) continue;  // solved by another pass
    const bool masked = q[2] == 1;
    const int W1 = w + 1, npx = W1 * W1;
    const int half = w / 2;
    double x0 = a.coords[t], y0 = a.coords[a.n + t];
    if (quad) {
      x0 = mround(x0);
      y0 = mround(y0);
    }
    const int seed = (int)floor((w + 1) / 2.0) - 1;
    SolveSmem<F64> s = carve<F64>(smem_raw, npx);
    // ---- load the subset window ----
    {
      const int r0 = (int)x0 - half - 1, c0 = (int)y0 - half - 1;
      for (int p = tid; p < npx; p += NT) {
        const int aa = p % W1, bb = p / W1;
        const size_t k = (size_t)(r0 + aa) + (size_t)(c0 + bb) * fr.M;
        const size_t kg = (size_t)(r0 + aa - a.crop) + (size_t)(c0 + bb - a.crop) * gM;
        float f = fr.ref[k];
        uint8_t on = 1;
        if (quad && fr.mask) {
          on = fr.mask[k] != 0;
          if (!on) f = 0.f;
        }
        s.f[p] = f;
        s.gx[p] = fr.gx[kg];
        s.gy[p] = fr.gy[kg];
        s.on[p] = on;
      }
    }
    __syncthreads();
    if (masked) {
      // bwselect(logical(mask), seed, seed, 4) restricts f, fx, fy (funICGNQuadtree.m:83-88)
      flood_select(s.on, s.lab, W1, W1, seed, seed, 4, nullptr);
      for (int p = tid; p < npx; p += NT)
        if (!s.lab[p]) {
          s.f[p] = 0.f;
          s.gx[p] = 0.f;
          s.gy[p] = 0.f;
        }
      __syncthreads();
    }
    // ---- setup sums: H (21), sum J f (6), sum J (6), f stats (3), sum |f| (1); FP64 per thread
    //      (J = gradient x integer offset is exact in FP64) ----
    {
      double v[37];
#pragma unroll
      for (int k = 0; k < 37; ++k) v[k] = 0.0;
      for (int p = tid; p < npx; p += NT) {
        const double dx = (double)(p % W1 - half), dy = (double)(p / W1 - half);
        const double gxv = s.gx[p], gyv = s.gy[p], f = s.f[p];
        const double J[6] = {gxv * dx, gyv * dx, gxv * dy, gyv * dy, gxv, gyv};
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
          for (int j = i; j < 6; ++j) {
            const int m = i * 6 - i * (i - 1) / 2 + (j - i);  // packed upper triangle by rows
            v[m] = fma(J[i], J[j], v[m]);
          }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          v[21 + i] = fma(J[i], f, v[21 + i]);
          v[27 + i] += J[i];
        }
        const bool sel = quad ? (fabs(f) > 1e-10) : true;
        if (sel) {
          v[33] += f;
          v[34] = fma(f, f, v[34]);
          v[35] += 1.0;
        }
        v[36] += fabs(f);
      }
      block_sum<37, NT>(v, red, sums);
    }
    if (tid == 0) {
      double H[36];
      int k = 0;
      for (int i = 0; i < 6; ++i)
        for (int j = i; j < 6; ++j) {
          H[i + 6 * j] = sums[k];
          H[j + 6 * i] = sums[k];
          ++k;
        }
      // packed lower triangle by columns == upper triangle by rows
      k = 0;
      for (int col = 0; col < 6; ++col)
        for (int row = col; row < 6; ++row) c.H[k++] = H[row + 6 * col];
      invert6(H, c.Hinv);
      const double n = sums[35];
      if (n > 0) {
        c.meanf = sums[33] / n;
        c.bf = sqrt(fmax(sums[34] - sums[33] * sums[33] / n, 0.0));
      } else {
        c.meanf = ALDIC_NAN;
        c.bf = ALDIC_NAN;
      }
      for (int i = 0; i < 6; ++i) {
        c.B[i] = sums[27 + i];
        c.A[i] = (sums[21 + i] - c.meanf * c.B[i]) / c.bf;
      }
      c.sabsf = sums[36];
      c.P[0] = c.P[1] = c.P[2] = c.P[3] = 0.0;
      if (a.F0 && !epi)
        for (int k = 0; k < 4; ++k) c.P[k] = a.F0[4 * t + k];  // a gradient initial guess (learned)
      if (epi) {
        c.P[4] = 0.0;
        c.P[5] = 0.0;
      } else {
        c.P[4] = a.U0[2 * t];
        c.P[5] = a.U0[2 * t + 1];
      }
      c.normNew = 1.0;
      c.normAbs = 1.0;
      c.normInit = 0.0;
      c.step = 0;
      c.status = 0;
      c.fbw8_ready = 0;
      c.done_error = 0;
      c.to_fp64 = 0;
      c.gsum_prev = 0.0;
      c.znssd = ALDIC_NAN;
    }
    __syncthreads();
    // ---- Gauss-Newton iterations ----
    const int q_nt = NT / W1, r_nt = NT % W1;
    while (true) {
      if (tid == 0) {
        int go = (!c.to_fp64 && c.step <= a.max_iter && c.normNew > a.tol && c.normAbs > a.tol) ? 1 : 0;
        if (go && !F64 && !epi && a.slow_fp64 && c.step >= a.warp_cap) {
          c.to_fp64 = 1;  // a long trajectory: the FP64 pass re-solves it from its initial guess
          go = 0;
        }
        if (go) {
          c.step += 1;
          if (quad && masked && c.step > 1) {
            // funICGNQuadtree.m:139-145 re-derives the subset size without re-slicing f
            const double w0 = a.winsize;
            const double wn = 2 * ceil(sqrt((w0 + 1) * (w0 + 1) / c.gsum_prev) * w / 2);
            if (wn != (double)w) {
              if (!window_ok(fr, x0, y0, wn, wn, false, a.crop)) {
                c.done_error = 1;
              } else if (warped_oob(fr, c.P, x0, y0, wn / 2, wn / 2)) {
                c.normNew = 1e6;
              } else {
                c.done_error = 1;  // array size mismatch in the reference
              }
              go = 0;
            }
          }
          if (go && warped_oob(fr, c.P, x0, y0, half, half)) {
            c.normNew = 1e6;
            go = 0;
          }
          if (go) prep_coeffs(c, x0, y0);
        }
        c.go = go;
      }
      __syncthreads();
      if (!c.go) break;
      // pass 1: interpolate, single-pass sums (FP64 across the threads' partials)
      double v[11];
      {
        G C[6] = {0, 0, 0, 0, 0, 0}, S1 = 0, S2 = 0, fg = 0;
        float ns = 0.f, nz = 0.f;
        int aa = tid % W1, bb = tid / W1;
        for (int p = tid; p < npx; p += NT) {
          G g;
          if constexpr (F64) {
            // u22 - (x0 + n5) in FP64, the reference's own interpolation arithmetic
            const double dx = (double)(aa - half), dy = (double)(bb - half);
            const double lx = dx + (c.P[0] * dx + (c.P[2] * dy + c.d5));
            const double ly = dy + (c.P[3] * dy + (c.P[1] * dx + c.d6));
            const double ix = floor(lx), iy = floor(ly);
            g = stencil16_ref64(fr.def, fr.M, c.base_r + (int)ix, c.base_c + (int)iy, lx - ix, ly - iy);
          } else {
            g = warp_g(fr, c, (float)(aa - half), (float)(bb - half));
          }
          s.g[p] = g;
          const G dx = (G)(aa - half), dy = (G)(bb - half);
          const G ag = (G)s.gx[p] * g, bg = (G)s.gy[p] * g;
          C[0] = fma(ag, dx, C[0]);
          C[1] = fma(bg, dx, C[1]);
          C[2] = fma(ag, dy, C[2]);
          C[3] = fma(bg, dy, C[3]);
          C[4] += ag;
          C[5] += bg;
          const bool sel = quad ? (fabs(g) > (G)1e-10) : true;
          if (sel) {
            S1 += g;
            S2 = fma(g, g, S2);
            ns += 1.f;
          }
          nz += (g == (G)0) ? 1.f : 0.f;
          if (want_fg) fg = fma((G)s.f[p], g, fg);
          aa += r_nt;
          bb += q_nt;
          if (aa >= W1) {
            aa -= W1;
            bb += 1;
          }
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = C[k];
        v[6] = S1;
        v[7] = S2;
        v[8] = ns;
        v[9] = nz;
        v[10] = fg;
      }
      block_sum<11, NT>(v, red, sums);
      const bool run_mask = quad && (masked || sums[9] > 0);
      if (run_mask) {
        // g region: bwselect(logical(g), seed, seed, 8); if it covers the window, the
        // 8-connected f-mask region instead (funICGNQuadtree.m:170-182)
        for (int p = tid; p < npx; p += NT) s.tmp[p] = (s.g[p] != (G)0);
        __syncthreads();
        flood_select(s.tmp, s.lab, W1, W1, seed, seed, 8, nullptr);
        int allon = 1;
        for (int p = tid; p < npx; p += NT) allon &= s.lab[p];
        allon = __syncthreads_and(allon);
        const uint8_t* gm = s.lab;
        if (allon) {
          if (!c.fbw8_ready) {
            flood_select(s.on, s.fbw8, W1, W1, seed, seed, 8, nullptr);
            if (tid == 0) c.fbw8_ready = 1;
          }
          gm = s.fbw8;
        }
        __syncthreads();
        G C2[6] = {0, 0, 0, 0, 0, 0}, T1 = 0, T2 = 0, TF = 0;
        float tn = 0.f, gs = 0.f;
        for (int p = tid; p < npx; p += NT) {
          const G dx = (G)(p % W1 - half), dy = (G)(p / W1 - half);
          const G g = gm[p] ? s.g[p] : (G)0;
          const G ag = (G)s.gx[p] * g, bg = (G)s.gy[p] * g;
          C2[0] = fma(ag, dx, C2[0]);
          C2[1] = fma(bg, dx, C2[1]);
          C2[2] = fma(ag, dy, C2[2]);
          C2[3] = fma(bg, dy, C2[3]);
          C2[4] += ag;
          C2[5] += bg;
          if (fabs(g) > (G)1e-10) {
            T1 += g;
            T2 = fma(g, g, T2);
            tn += 1.f;
          }
          gs += gm[p] ? 1.f : 0.f;
          if (want_fg) TF = fma((G)s.f[p], g, TF);
        }
        double v2[11] = {C2[0], C2[1], C2[2], C2[3], C2[4], C2[5], T1, T2, tn, gs, TF};
        block_sum<11, NT>(v2, red, sums);
        if (tid == 0) c.gsum_prev = sums[9];
      }
      if (tid == 0) {
        const double n = sums[8];
        double meang, bg;
        if (n > 0) {
          meang = sums[6] / n;
          bg = sqrt(fmax(sums[7] - sums[6] * sums[6] / n, 0.0));
        } else {
          meang = ALDIC_NAN;
          bg = ALDIC_NAN;
        }
        double b[6];
        for (int i = 0; i < 6; ++i) b[i] = c.bf * (c.A[i] - (sums[i] - meang * c.B[i]) / bg);
        if (want_fg) c.znssd = 2.0 - 2.0 * (sums[10] - c.meanf * sums[6]) / (c.bf * bg);
        double nn = 0;
        for (int i = 0; i < 6; ++i) nn += b[i] * b[i];
        c.normNew = sqrt(nn);
        c.normAbs = c.normNew;
        if (c.step == 1) c.normInit = c.normNew;
        if (c.normInit > a.tol) c.normNew = c.normNew / c.normInit;
        else c.normNew = 0.0;
        const double trH = c.H[0] + c.H[6] + c.H[11] + c.H[15] + c.H[18] + c.H[20];
        if (!F64 && !epi &&
            too_close_to_call(c.normNew, c.normAbs, c.normInit, a.tol, a.band,
                              fp32_noise(a.noise, c.step, c.bf, bg, trH, sums[7], n))) {
          c.to_fp64 = 1;  // leave the loop; the FP64 pass re-solves this subset
        } else if (!(c.normNew < a.tol || c.normAbs < a.tol)) {
          double dP[6];
          for (int i = 0; i < 6; ++i) {
            double acc = 0;
            for (int j = 0; j < 6; ++j) acc += c.Hinv[i + 6 * j] * b[j];
            dP[i] = -acc;
          }
          if (!compose_inverse(c.P, dP)) {
            c.step = a.max_iter + 1000;  // leave the loop (det(dP) == 0)
            c.status = 1;
          } else if (epi) {
            c.P[4] = 0.0;
            c.P[5] = 0.0;
          }
        }
      }
      __syncthreads();
    }
    // ---- finalize ----
    if (tid == 0) {
      int step = c.step;
      if (c.status == 1) step -= 1000;  // restore the count at the det == 0 break
      if (!(c.normNew < a.tol || c.normAbs < a.tol)) step = a.max_iter + 1;
      if (isnan(c.normNew)) step = a.max_iter + 1;
      if (quad && c.sabsf < 1e-6) step = a.max_iter + 3;
      if (c.to_fp64) {
        push_fp64(a, t, w, masked ? 1 : 0);
      } else if (epi) {
        a.znssd[t] = c.done_error ? ALDIC_NAN : c.znssd;
        if (a.conv) a.conv[t] = c.done_error ? -1 : step;
      } else if (c.done_error) {
        a.conv[t] = -1;
        a.U[2 * t] = ALDIC_NAN;
        a.U[2 * t + 1] = ALDIC_NAN;
        for (int k = 0; k < 4; ++k) a.F[4 * t + k] = ALDIC_NAN;
        if (a.H)
          for (int k = 0; k < 21; ++k) a.H[t + a.n * k] = 0.0;
      } else {
        a.conv[t] = step;
        a.U[2 * t] = c.P[4];
        a.U[2 * t + 1] = c.P[5];
        for (int k = 0; k < 4; ++k) a.F[4 * t + k] = c.P[k];
        if (want_fg) a.zncc[t] = 1.0 - 0.5 * c.znssd;
        if (a.H)
          for (int k = 0; k < 21; ++k) a.H[t + a.n * k] = c.H[k];
      }
    }
    __syncthreads();
  }
}

// ================================================================================
// fast 6-DOF solve for subsets at the nominal window without a mask region
// ================================================================================
// The common case (uniform variant; quadtree subsets whose window holds no masked or zero
// pixel) needs no flood fill, so a group of NW warps solves one subset with no shared image
// buffer.  Every thread walks its share of the window pixels; the sums are warp shuffles
// (FP32 per thread, FP64 across lanes) plus, for NW > 1, one fixed-order FP64 sum of the
// NW warp totals behind a named barrier of the group, so every thread holds the same
// totals and runs the same FP64 Gauss-Newton control redundantly: there is no other
// barrier per iteration.  The gradients f_x, f_y are re-read from the L1-resident gradient
// images each iteration.  The 6x6 inverse is a per-group [H | I] Gauss-Jordan elimination
// without pivoting by the group's first warp (H is the symmetric positive semi-definite
// Gauss-Newton Hessian; a zero pivot propagates Inf/NaN as the reference's singular solve
// does).
//
// The main pass (NW = 1, queue 0) gives each subset at most warp_cap iterations (8 by
// default; 6-12 measured within 1 % of each other on the stereo pass, 4 and 24 slower): the
// few subsets that need more (most never converge and run to max_iter) would otherwise
// keep single warps running long after the rest of the grid.  They go to queue 1 flagged
// kSlowSubset and continue in the multi-warp pass (NW = kSlowNW = 2) from the state the warp
// pass stored (P, the first norm, the step; without a state buffer they restart from their
// initial guess), whose iterations run about twice as fast; two warps measured faster over the whole stereo step
// than four or eight, which finish each subset sooner but crowd out the passes beside them.  A quadtree subset that meets an exact zero in g (a
// masked deformed image) needs the g-region flood fill: it is handed to the general kernel
// through queue 1 and restarted there.
constexpr int kWT = 256;  // threads per CTA: 8 / NW subset groups
constexpr int kSlowNW = 2;  // warps per subset in the pass that restarts the slow subsets
constexpr int kSub1SlowNW = 4;  // the same for the Subpb1 step

template <int NW>
__device__ __forceinline__ void group_bar(int id) {
  if (NW == 1)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(32 * NW) : "memory");
}

// Sum of v over the group, left in every thread of the group (FP64; the NW warp totals
// are added in warp order).  red holds NW * K doubles of the group.
template <int NW, int K>
__device__ __forceinline__ void group_sum(double (&v)[K], double* red, int gw, int lane, int bar) {
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  if (NW == 1) return;
  if (lane < K) {
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (lane == k) red[gw * K + k] = v[k];
  }
  group_bar<NW>(bar);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double s = red[k];
#pragma unroll
    for (int u = 1; u < NW; ++u) s += red[u * K + k];
    v[k] = s;
  }
  group_bar<NW>(bar);
}

// The one-warp pass is latency-bound on its image reads: three CTAs per SM (24 warps, 80
// registers with a few spills) measured 12 % faster than two (128 registers, no spills);
// four (64 registers) spill too much.
// Staging (STAGED): every group owns a shared-memory buffer of box_r x box_c floats (the
// box of a TMA tensor map over the deformed image, column-major) and an mbarrier.  Before an
// iteration it computes the tap footprint of the warped window (0-based image rows / columns
// from the window's corners in the pixel loop's own FP32 arithmetic, one row / column of
// margin) and, when that leaves the staged box, loads a new box whose first row is rounded
// down to a 16-byte boundary (the TMA rule for the innermost coordinate).  The stencil then
// reads shared memory with the same operations as the gather path, so values are
// bit-identical.  An iteration whose footprint exceeds the box (a large deformation) gathers
// from the image.  A wait that outlasts kTmaWaitCycles sets qcount[8] and the group gathers
// from the image from then on.
constexpr long long kTmaWaitCycles = 2000000000LL;  // ~1 s at the B200 clock
constexpr size_t kStageBytesMax = 100 * 1024;       // staging buffers of one block: two blocks per SM

struct StageGeom {
  int box_r, box_c;  // tensor-map box: rows (a multiple of 4) x columns
  int buf_floats;    // floats per group buffer (a multiple of 32: 128-byte aligned buffers)
};

// Tap footprint (0-based image rows rlo..rhi, columns clo..chi) of the warped window of an
// iteration: the window's corners in the pixel loop's own FP32 arithmetic, one row / column
// of margin on each side (an interior pixel's floor() may differ from a corner's by one).
__device__ __forceinline__ void tap_footprint(float p0, float p1, float p2, float p3, float f5, float f6, int half,
                                              int br, int bc, int& rlo, int& rhi, int& clo, int& chi) {
  float lxmin = 3.0e38f, lxmax = -3.0e38f, lymin = 3.0e38f, lymax = -3.0e38f;
#pragma unroll
  for (int cx = -1; cx <= 1; cx += 2)
#pragma unroll
    for (int cy = -1; cy <= 1; cy += 2) {
      const float dxc = (float)(cx * half), dyc = (float)(cy * half);
      const float lx = dxc + fmaf(p0, dxc, fmaf(p2, dyc, f5));
      const float ly = dyc + fmaf(p3, dyc, fmaf(p1, dxc, f6));
      lxmin = fminf(lxmin, lx);
      lxmax = fmaxf(lxmax, lx);
      lymin = fminf(lymin, ly);
      lymax = fmaxf(lymax, ly);
    }
  rlo = br + (int)floorf(lxmin) - 1;
  rhi = br + (int)floorf(lxmax) + 4;
  clo = bc + (int)floorf(lymin) - 1;
  chi = bc + (int)floorf(lymax) + 4;
}

// Issue the TMA load of the box that covers a footprint (its first row rounded down to a
// 16-byte boundary) into the group's buffer; false when the footprint does not fit a box.  The
// caller has no load in flight into this buffer.  Every thread of the group calls it.
template <int NW>
__device__ __forceinline__ bool stage_issue(const CUtensorMap& tmap, float* tile, int BR, int BC, int rlo, int rhi,
                                            int clo, int chi, uint64_t& bar_mem, int bar, int gt, int& tr0,
                                            int& tc0) {
  const int nr0 = rlo - (((rlo % 4) + 4) % 4);
  if (!(rhi - nr0 < BR && chi - clo < BC)) return false;
  fence_proxy_async_shared();  // this thread's reads of the old box before the copy writes
  group_bar<NW>(bar);
  if (gt == 0) {
    mbar_arrive_expect_tx(&bar_mem, (uint32_t)(BR * BC * 4));
    tma_load_2d(tile, &tmap, nr0, clo, &bar_mem);
  }
  tr0 = nr0;
  tc0 = clo;
  return true;
}

// Wait for the group's load in flight (every thread polls; the outcome is agreed by the group).
// On time-out the group gathers from the image from then on and flags qcount[8].
template <int NW>
__device__ __forceinline__ void stage_wait(bool& pending, bool& tile_ok, bool& broken, uint32_t& phase,
                                           uint64_t& bar_mem, int& ok_mem, int bar, int gt, int* qcount) {
  bool ok = mbar_wait(&bar_mem, phase, kTmaWaitCycles);
  if (NW == 1) {
    ok = __all_sync(0xffffffffu, ok);
  } else {
    if (gt == 0) ok_mem = 1;
    group_bar<NW>(bar);
    if (!ok) ok_mem = 0;
    group_bar<NW>(bar);
    ok = ok_mem != 0;
  }
  if (ok) {
    phase ^= 1;
    pending = false;
    tile_ok = true;
  } else {
    broken = true;  // the copy may still land: the buffer is never reused
    tile_ok = false;
    if (gt == 0) atomicOr(qcount + 8, 1);
  }
}

template <int NW, bool SLOW, bool STAGED>
__global__ void __launch_bounds__(kWT, STAGED ? 2 : (NW == 1 ? 3 : 2))
    icgn_group_kernel(IcgnArgs a, const __grid_constant__ CUtensorMap tmap, StageGeom geo) {
  constexpr int NG = kWT / (32 * NW);  // subset groups per CTA
  constexpr int GT = 32 * NW;          // threads per group
  extern __shared__ __align__(128) float s_tiles[];
  __shared__ __align__(8) uint64_t s_bar[NG];
  __shared__ int s_ok[NG];
  __shared__ double s_aug[NG][72];     // 6 x 12 row-major [H | I] -> [I | H^-1]
  __shared__ double s_ab[NG][12];      // A (0..5), B (6..11)
  __shared__ double s_h[NG][21];       // packed upper triangle by rows
  __shared__ double s_fac[NG][6];      // elimination factors of the current pivot column
  __shared__ double s_red[NG][NW * 21];
  const int lane = threadIdx.x & 31, grp = threadIdx.x / GT, gw = (threadIdx.x % GT) >> 5;
  const int gt = threadIdx.x % GT, bar = 1 + grp;
  double* aug = s_aug[grp];
  double* AB = s_ab[grp];
  double* red = s_red[grp];
  const FrameDev& fr = a.fr;
  const bool quad = (a.variant == 1);
  const bool epi = (a.variant == 2);
  const bool want_fg = epi || a.zncc != nullptr;  // sum f g: the epipolar ZNSSD, or the ZNCC
  __shared__ int s_qi[NG];
  const int count = a.qcount[SLOW ? 1 : 0];
  const int gM = fr.M - 6;
  int* next = a.qcount + (SLOW ? 3 : 2);  // work counter of this pass (zeroed with the queues)
  // staging state of the group (replicated in its threads)
  // the buffers start at the first 128-byte boundary of the dynamic shared memory (the launch
  // allocates 128 bytes more than the buffers need)
  float* tile = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(s_tiles) + 127) & ~uintptr_t(127)) +
                (STAGED ? grp * geo.buf_floats : 0);
  const int BR = geo.box_r, BC = geo.box_c;
  int tr0 = 0, tc0 = 0;
  bool tile_ok = false, pending = false, broken = false;
  uint32_t phase = 0;
  if (STAGED) {
    if (gt == 0) {
      mbar_init(&s_bar[grp], 1);
      fence_barrier_init();
    }
    group_bar<NW>(bar);
  }
  while (true) {
    // the group's next queue entry (dynamic: slow subsets do not pile up on one group)
    int qi = 0;
    if (gt == 0) qi = atomicAdd(next, 1);
    if (NW == 1) {
      qi = __shfl_sync(0xffffffffu, qi, 0);
    } else {
      if (gt == 0) s_qi[grp] = qi;
      group_bar<NW>(bar);
      qi = s_qi[grp];
    }
    if (qi >= count) {
      // a copy in flight (a prefetch never used, or one that outlasted its wait) must land
      // before the block's shared memory is released
      if (STAGED && (pending || broken)) mbar_wait(&s_bar[grp], phase, kTmaWaitCycles);
      break;
    }
    const int* q = a.queue + 3 * ((SLOW ? a.n : 0) + qi);
    if (SLOW && q[2] != kSlowSubset) {
      group_bar<NW>(bar);
      continue;
    }
    const long long t = q[0];
    const int w = q[1];
    const int W1 = w + 1, npx = W1 * W1, half = w / 2;
    double x0 = a.coords[t], y0 = a.coords[a.n + t];
    if (quad) {
      x0 = mround(x0);
      y0 = mround(y0);
    }
    const int r0 = (int)x0 - half - 1, c0 = (int)y0 - half - 1;
    const int q_nt = GT / W1, r_nt = GT % W1;
    if constexpr (STAGED) {
      // prefetch the first iteration's box (P = [0 0 0 0 U0], or the carried state) so the
      // load overlaps the set-up sums
      if (!broken && !pending) {
        double Pp[6] = {0.0, 0.0, 0.0, 0.0, epi ? 0.0 : a.U0[2 * t], epi ? 0.0 : a.U0[2 * t + 1]};
        if (a.F0 && !epi)
          for (int k = 0; k < 4; ++k) Pp[k] = a.F0[4 * t + k];
        if (SLOW && a.carry)
          for (int k = 0; k < 6; ++k) Pp[k] = a.carry[8 * t + k];
        const double m5 = mround(Pp[4]), m6 = mround(Pp[5]);
        if (isfinite(m5) && isfinite(m6) && fabs(m5) < 1e6 && fabs(m6) < 1e6) {
          int rlo, rhi, clo, chi;
          tap_footprint((float)Pp[0], (float)Pp[1], (float)Pp[2], (float)Pp[3], (float)(Pp[4] - m5),
                        (float)(Pp[5] - m6), half, (int)(x0 + m5) - 2, (int)(y0 + m6) - 2, rlo, rhi, clo, chi);
          const bool covered = tile_ok && rlo >= tr0 && rhi < tr0 + BR && clo >= tc0 && chi < tc0 + BC;
          if (!covered && stage_issue<NW>(tmap, tile, BR, BC, rlo, rhi, clo, chi, s_bar[grp], bar, gt, tr0, tc0)) {
            pending = true;
            tile_ok = false;
          }
        }
      }
    }
    // ---- set-up sums, FP64 per lane (J = gradient x integer offset is exact in FP64), in two
    //      passes over the window to bound the live accumulators ----
    double meanf, bf, sabsf;
    {
      double jf[6], jb[6], fs = 0.0, fs2 = 0.0, fab = 0.0;
      float fn = 0.f;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        jf[k] = 0.0;
        jb[k] = 0.0;
      }
      int aa = gt % W1, bb = gt / W1;
      for (int p = gt; p < npx; p += GT) {
        const int k = (r0 + aa) + (c0 + bb) * fr.M;
        const int kg = (r0 + aa - a.crop) + (c0 + bb - a.crop) * gM;
        const float ff = fr.ref[k];  // a quadtree subset here has no masked pixel
        const double f = ff, gxv = fr.gx[kg], gyv = fr.gy[kg];
        const double dx = (double)(aa - half), dy = (double)(bb - half);
        const double J[6] = {gxv * dx, gyv * dx, gxv * dy, gyv * dy, gxv, gyv};
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          jf[i] = fma(J[i], f, jf[i]);
          jb[i] += J[i];
        }
        if (!quad || fabsf(ff) > 1e-10f) {
          fs += f;
          fs2 = fma(f, f, fs2);
          fn += 1.f;
        }
        fab += fabs(f);
        aa += r_nt;
        bb += q_nt;
        if (aa >= W1) {
          aa -= W1;
          bb += 1;
        }
      }
      {
        double v[4] = {fs, fs2, (double)fn, fab};
        group_sum<NW, 4>(v, red, gw, lane, bar);
        sabsf = v[3];
        if (v[2] > 0) {
          meanf = v[0] / v[2];
          bf = sqrt(fmax(v[1] - v[0] * v[0] / v[2], 0.0));
        } else {
          meanf = ALDIC_NAN;
          bf = ALDIC_NAN;
        }
      }
      {
        double v[12];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          v[k] = jb[k];
          v[6 + k] = jf[k];
        }
        group_sum<NW, 12>(v, red, gw, lane, bar);
        if (gt < 6) {
#pragma unroll
          for (int k = 0; k < 6; ++k)
            if (gt == k) {
              AB[6 + k] = v[k];
              AB[k] = (v[6 + k] - meanf * v[k]) / bf;
            }
        }
      }
    }
    {
      double h[21];
#pragma unroll
      for (int k = 0; k < 21; ++k) h[k] = 0.0;
      int aa = gt % W1, bb = gt / W1;
      for (int p = gt; p < npx; p += GT) {
        const int kg = (r0 + aa - a.crop) + (c0 + bb - a.crop) * gM;
        const double gxv = fr.gx[kg], gyv = fr.gy[kg];
        const double dx = (double)(aa - half), dy = (double)(bb - half);
        const double J[6] = {gxv * dx, gyv * dx, gxv * dy, gyv * dy, gxv, gyv};
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
          for (int j = i; j < 6; ++j) {
            const int m = i * 6 - i * (i - 1) / 2 + (j - i);  // packed upper triangle by rows
            h[m] = fma(J[i], J[j], h[m]);
          }
        aa += r_nt;
        bb += q_nt;
        if (aa >= W1) {
          aa -= W1;
          bb += 1;
        }
      }
      group_sum<NW, 21>(h, red, gw, lane, bar);
      if (gt < 21) {
#pragma unroll
        for (int k = 0; k < 21; ++k)
          if (gt == k) s_h[grp][k] = h[k];
      }
    }
    group_bar<NW>(bar);
    if (gw == 0) {
      for (int e = lane; e < 72; e += 32) {
        const int i = e / 12, j = e % 12;
        double val;
        if (j < 6) {
          const int r = i < j ? i : j, cc = i < j ? j : i;  // packed upper-triangle index of (r, cc)
          val = s_h[grp][r * 6 - r * (r - 1) / 2 + (cc - r)];
        } else {
          val = (j - 6 == i) ? 1.0 : 0.0;
        }
        aug[e] = val;
      }
      __syncwarp();
      for (int k = 0; k < 6; ++k) {
        // partial pivoting: the row (>= k) with the largest |entry| in column k, first one on
        // ties (the mldivide of funICGN.m:288 pivots as well)
        double best = lane >= k && lane < 6 ? fabs(aug[lane * 12 + k]) : -1.0;
        int piv = lane;
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
          const double ob = __shfl_down_sync(0xffffffffu, best, o);
          const int op = __shfl_down_sync(0xffffffffu, piv, o);
          if (lane + o < 8 && (ob > best || (ob == best && op < piv))) {
            best = ob;
            piv = op;
          }
        }
        piv = __shfl_sync(0xffffffffu, piv, 0);
        if (piv != k && lane < 12) {
          const double tk = aug[k * 12 + lane];
          aug[k * 12 + lane] = aug[piv * 12 + lane];
          aug[piv * 12 + lane] = tk;
        }
        __syncwarp();
        if (lane < 6) s_fac[grp][lane] = aug[lane * 12 + k];
        const double pv = aug[k * 12 + k];
        __syncwarp();
        if (lane < 12) aug[k * 12 + lane] /= pv;
        __syncwarp();
        for (int e = lane; e < 72; e += 32) {
          const int i = e / 12, j = e % 12;
          if (i != k) aug[e] -= s_fac[grp][i] * aug[k * 12 + j];
        }
        __syncwarp();
      }
    }
    group_bar<NW>(bar);
    // ---- Gauss-Newton iterations (control replicated in every thread) ----
    const double trH = s_h[grp][0] + s_h[grp][6] + s_h[grp][11] + s_h[grp][15] + s_h[grp][18] + s_h[grp][20];
    double P[6] = {0.0, 0.0, 0.0, 0.0, epi ? 0.0 : a.U0[2 * t], epi ? 0.0 : a.U0[2 * t + 1]};
    if (a.F0 && !epi)
      for (int k = 0; k < 4; ++k) P[k] = a.F0[4 * t + k];  // a gradient initial guess (learned)
    double normNew = 1.0, normAbs = 1.0, normInit = 0.0, znssd = ALDIC_NAN;
    int step = 0, status = 0, requeue = -1;
    if (SLOW && a.carry) {  // continue from where the warp pass stopped: P, the first norm, the step
      const double* cs = a.carry + 8 * t;
#pragma unroll
      for (int k = 0; k < 6; ++k) P[k] = cs[k];
      normInit = cs[6];
      step = (int)cs[7];
    }
    while (step <= a.max_iter && normNew > a.tol && normAbs > a.tol) {
      if (!SLOW && step >= a.warp_cap) {
        // a long trajectory: FP32 rounding accumulates along it, so it is re-solved in FP64
        // from its initial guess (or, for the epipolar score, continued by the multi-warp pass)
        requeue = (a.slow_fp64 && !epi) ? kToFp64 : kSlowSubset;
        break;
      }
      step += 1;
      if (warped_oob(fr, P, x0, y0, half, half)) {
        normNew = 1e6;
        break;
      }
      const double n5 = mround(P[4]), n6 = mround(P[5]);
      const float p0 = (float)P[0], p1 = (float)P[1], p2 = (float)P[2], p3 = (float)P[3];
      const float f5 = (float)(P[4] - n5), f6 = (float)(P[5] - n6);
      const int br = (int)(x0 + n5) - 2, bc = (int)(y0 + n6) - 2;
      bool use_tile = false;
      if constexpr (STAGED) {
        if (!broken) {
          int rlo, rhi, clo, chi;
          tap_footprint(p0, p1, p2, p3, f5, f6, half, br, bc, rlo, rhi, clo, chi);
          const bool covered = rlo >= tr0 && rhi < tr0 + BR && clo >= tc0 && chi < tc0 + BC;
          if (!(covered && (tile_ok || pending))) {
            // the staged (or prefetched) box misses this footprint: load the one that covers it
            if (pending) stage_wait<NW>(pending, tile_ok, broken, phase, s_bar[grp], s_ok[grp], bar, gt, a.qcount);
            tile_ok = false;
            if (!broken && stage_issue<NW>(tmap, tile, BR, BC, rlo, rhi, clo, chi, s_bar[grp], bar, gt, tr0, tc0))
              pending = true;
          }
          if (pending) stage_wait<NW>(pending, tile_ok, broken, phase, s_bar[grp], s_ok[grp], bar, gt, a.qcount);
          use_tile = tile_ok && !broken;
        }
      }
      // per-lane sums of the pixel pairs (p, p + GT) in packed FP32 with Kahan compensation
      // (s + k is the compensated total; 3 extra packed operations per term), a last unpaired
      // pixel alone; the lane totals go to FP64 before the cross-lane sums
      double v[11];
      {
        float2 C2[6], K2[6], S12 = make_float2(0.f, 0.f), KS1 = make_float2(0.f, 0.f);
        float2 S22 = make_float2(0.f, 0.f), KS2 = make_float2(0.f, 0.f), fg2 = make_float2(0.f, 0.f);
        float S1 = 0.f, kS1 = 0.f, S2 = 0.f, kS2 = 0.f, ns = 0.f, nz = 0.f;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          C2[k] = make_float2(0.f, 0.f);
          K2[k] = make_float2(0.f, 0.f);
        }
        const float2 pp0 = make_float2(p0, p0), pp1 = make_float2(p1, p1), pp2 = make_float2(p2, p2);
        const float2 pp3 = make_float2(p3, p3), ff5 = make_float2(f5, f5), ff6 = make_float2(f6, f6);
        int aa = gt % W1, bb = gt / W1;
        int p = gt;
        for (; p + GT < npx; p += 2 * GT) {
          int ab = aa + r_nt, bbb = bb + q_nt;
          if (ab >= W1) {
            ab -= W1;
            bbb += 1;
          }
          const float2 dx = make_float2((float)(aa - half), (float)(ab - half));
          const float2 dy = make_float2((float)(bb - half), (float)(bbb - half));
          const float2 lx = fadd2(dx, ffma2(pp0, dx, ffma2(pp2, dy, ff5)));
          const float2 ly = fadd2(dy, ffma2(pp3, dy, ffma2(pp1, dx, ff6)));
          const float ixa = floorf(lx.x), ixb = floorf(lx.y), iya = floorf(ly.x), iyb = floorf(ly.y);
          const float2 tr = make_float2(lx.x - ixa, lx.y - ixb), tc = make_float2(ly.x - iya, ly.y - iyb);
          float2 g;
          if (STAGED && use_tile) {
            const int oa = (br + (int)ixa - tr0) + (bc + (int)iya - tc0) * BR;
            const int ob = (br + (int)ixb - tr0) + (bc + (int)iyb - tc0) * BR;
            g = stencil16_x2_tile(tile, BR, oa, ob, tr, tc);
          } else {
            const int ia = (br + (int)ixa) + (bc + (int)iya) * fr.M, ib = (br + (int)ixb) + (bc + (int)iyb) * fr.M;
            g = stencil16_x2(fr.def, fr.M, ia, ib, tr, tc);
          }
          const int ka = (r0 + aa - a.crop) + (c0 + bb - a.crop) * gM;
          const int kb = (r0 + ab - a.crop) + (c0 + bbb - a.crop) * gM;
          const float2 ag = fmul2(make_float2(fr.gx[ka], fr.gx[kb]), g);
          const float2 bg = fmul2(make_float2(fr.gy[ka], fr.gy[kb]), g);
          kahan2(C2[0], K2[0], ffma2(ag, dx, K2[0]));
          kahan2(C2[1], K2[1], ffma2(bg, dx, K2[1]));
          kahan2(C2[2], K2[2], ffma2(ag, dy, K2[2]));
          kahan2(C2[3], K2[3], ffma2(bg, dy, K2[3]));
          kahan2(C2[4], K2[4], fadd2(ag, K2[4]));
          kahan2(C2[5], K2[5], fadd2(bg, K2[5]));
          if (!quad) {
            kahan2(S12, KS1, fadd2(g, KS1));
            kahan2(S22, KS2, ffma2(g, g, KS2));
          } else {
            if (fabsf(g.x) > 1e-10f) {
              kahan1(S1, kS1, g.x + kS1);
              kahan1(S2, kS2, fmaf(g.x, g.x, kS2));
              ns += 1.f;
            }
            if (fabsf(g.y) > 1e-10f) {
              kahan1(S1, kS1, g.y + kS1);
              kahan1(S2, kS2, fmaf(g.y, g.y, kS2));
              ns += 1.f;
            }
            nz += (g.x == 0.f ? 1.f : 0.f) + (g.y == 0.f ? 1.f : 0.f);
          }
          if (want_fg)
            fg2 = ffma2(make_float2(fr.ref[(r0 + aa) + (c0 + bb) * fr.M], fr.ref[(r0 + ab) + (c0 + bbb) * fr.M]), g,
                        fg2);
          aa = ab + r_nt;
          bb = bbb + q_nt;
          if (aa >= W1) {
            aa -= W1;
            bb += 1;
          }
        }
#pragma unroll
        for (int k = 0; k < 6; ++k)
          v[k] = ((double)C2[k].x + (double)K2[k].x) + ((double)C2[k].y + (double)K2[k].y);
        if (!quad) {
          v[6] = ((double)S12.x + (double)KS1.x) + ((double)S12.y + (double)KS1.y);
          v[7] = ((double)S22.x + (double)KS2.x) + ((double)S22.y + (double)KS2.y);
          ns = (float)((npx - gt + GT - 1) / GT);  // pixels of this thread
        } else {
          v[6] = (double)S1 + (double)kS1;
          v[7] = (double)S2 + (double)kS2;
        }
        v[10] = (double)fg2.x + (double)fg2.y;
        if (p < npx) {  // the last, unpaired pixel
          const float dx = (float)(aa - half), dy = (float)(bb - half);
          const float lx = dx + fmaf(p0, dx, fmaf(p2, dy, f5));
          const float ly = dy + fmaf(p3, dy, fmaf(p1, dx, f6));
          const float ix = floorf(lx), iy = floorf(ly);
          const float g = (STAGED && use_tile)
                              ? stencil16_tile(tile, BR, (br + (int)ix - tr0) + (bc + (int)iy - tc0) * BR, lx - ix,
                                               ly - iy)
                              : stencil16(fr.def, fr.M, br + (int)ix, bc + (int)iy, lx - ix, ly - iy);
          const int kg = (r0 + aa - a.crop) + (c0 + bb - a.crop) * gM;
          const float ag = fr.gx[kg] * g, bg = fr.gy[kg] * g;
          v[0] += (double)(ag * dx);
          v[1] += (double)(bg * dx);
          v[2] += (double)(ag * dy);
          v[3] += (double)(bg * dy);
          v[4] += (double)ag;
          v[5] += (double)bg;
          if (quad) {
            if (fabsf(g) > 1e-10f) {
              v[6] += (double)g;
              v[7] += (double)g * (double)g;
              ns += 1.f;
            }
            if (g == 0.f) nz += 1.f;
          } else {
            v[6] += (double)g;
            v[7] += (double)g * (double)g;
          }
          if (want_fg) v[10] += (double)fr.ref[(r0 + aa) + (c0 + bb) * fr.M] * (double)g;
        }
        v[8] = ns;
        v[9] = nz;
      }
      group_sum<NW, 11>(v, red, gw, lane, bar);
      if (v[9] > 0) {  // exact zero in g: the g-region flood fill is needed
        requeue = 0;
        break;
      }
      double meang, bgn;
      if (v[8] > 0) {
        meang = v[6] / v[8];
        bgn = sqrt(fmax(v[7] - v[6] * v[6] / v[8], 0.0));
      } else {
        meang = ALDIC_NAN;
        bgn = ALDIC_NAN;
      }
      if (want_fg) znssd = 2.0 - 2.0 * (v[10] - meanf * v[6]) / (bf * bgn);
      double b[6];
      const double ibgn = 1.0 / bgn;  // one FP64 division per iteration instead of six
#pragma unroll
      for (int k = 0; k < 6; ++k) b[k] = bf * (AB[k] - (v[k] - meang * AB[6 + k]) * ibgn);
      double dP[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        double acc = 0;
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += aug[i * 12 + 6 + j] * b[j];
        dP[i] = -acc;
      }
      double nn = 0;
#pragma unroll
      for (int i = 0; i < 6; ++i) nn += b[i] * b[i];
      normNew = sqrt(nn);
      normAbs = normNew;
      if (step == 1) normInit = normNew;
      if (normInit > a.tol) normNew = normNew / normInit;
      else normNew = 0.0;
      if (!epi && too_close_to_call(normNew, normAbs, normInit, a.tol, a.band,
                                    fp32_noise(a.noise, step, bf, bgn, trH, v[7], v[8]))) {
        requeue = kToFp64;  // the FP64 pass re-solves this subset from its initial guess
        break;
      }
      if (!(normNew < a.tol || normAbs < a.tol)) {
        if (!compose_inverse(P, dP)) {
          step = a.max_iter + 1000;
          status = 1;
        } else if (epi) {
          P[4] = 0.0;
          P[5] = 0.0;
        }
      }
    }
    if (gt == 0) {
      if (requeue == kToFp64) {
        push_fp64(a, t, w, 0);  // unmasked, at the window this pass solved
        if (SLOW) const_cast<int*>(q)[2] = kMovedSubset;
        requeue = -2;
      }
      if (requeue == kSlowSubset && a.carry) {
        double* cs = a.carry + 8 * t;
#pragma unroll
        for (int k = 0; k < 6; ++k) cs[k] = P[k];
        cs[6] = normInit;
        cs[7] = (double)step;
      }
      if (requeue >= 0) {
        // hand this subset to a later pass (they run after this kernel).  A queue-0
        // subset is appended to queue 1 (at most one entry each: queue 1 never holds more
        // than n); a queue-1 subset is re-flagged in place.
        if (SLOW) {
          const_cast<int*>(q)[2] = requeue;
        } else {
          const int pos = atomicAdd(&a.qcount[1], 1);
          int* q1 = a.queue + 3 * ((long long)a.n + pos);
          q1[0] = (int)t;
          q1[1] = w;
          q1[2] = requeue;
        }
      } else if (requeue == -1) {
        if (status == 1) step -= 1000;
        if (!(normNew < a.tol || normAbs < a.tol)) step = a.max_iter + 1;
        if (isnan(normNew)) step = a.max_iter + 1;
        if (quad && sabsf < 1e-6) step = a.max_iter + 3;
        if (epi) {
          a.znssd[t] = znssd;
          if (a.conv) a.conv[t] = step;
        } else {
          a.conv[t] = step;
          a.U[2 * t] = P[4];
          a.U[2 * t + 1] = P[5];
          for (int k = 0; k < 4; ++k) a.F[4 * t + k] = P[k];
          if (want_fg) a.zncc[t] = 1.0 - 0.5 * znssd;
          if (a.H)
            for (int k = 0; k < 21; ++k) a.H[t + a.n * k] = s_h[grp][k];
        }
      }
    }
    group_bar<NW>(bar);
  }
}

// ================================================================================
// Subpb1: classify + solve
// ================================================================================
__global__ void subpb1_classify_kernel(Sub1Args a) {
  const long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= a.n) return;
  const FrameDev& fr = a.fr;
  const bool quad = (a.variant == 1);
  double x0 = a.coords[t], y0 = a.coords[a.n + t];
  double wx, wy;
  if (quad) {
    x0 = mround(x0);
    y0 = mround(y0);
    wx = a.winsize_list[t];
    wy = a.winsize_list[a.n + t];
  } else {
    wx = wy = a.winsize;
  }
  int status = 0;
  const bool ok = window_ok(fr, x0, y0, wx, wy, true, 3);
  long long cnt = 0;
  if (ok) {
    const int R = (int)wx + 1, Cc = (int)wy + 1;
    const int r0 = (int)(x0 - wx / 2) - 1, c0 = (int)(y0 - wy / 2) - 1;
    for (int p = lane; p < R * Cc; p += 32) {
      const int aa = p % R, bb = p / R;
      const size_t k = (size_t)(r0 + aa) + (size_t)(c0 + bb) * fr.M;
      if (quad) {
        const bool mk = fr.mask ? (fr.mask[k] != 0) : true;
        cnt += (!mk || fr.ref[k] == 0.f);
      } else {
        cnt += (fr.gx[(size_t)(r0 + aa - 3) + (size_t)(c0 + bb - 3) * (fr.M - 6)] == 0.f);
      }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  }
  double wxf = wx, wyf = wy;
  if (!ok) {
    status = -1;
  } else if (quad) {
    const double Nw = (wx + 1) * (wy + 1);
    if (cnt < 0.4 * Nw) {
      if (cnt > 0) {
        wxf = 2 * ceil(sqrt((wx + 1) * (wy + 1) / ((wx + 1) * (wy + 1) - (double)cnt)) * wx / 2);
        wyf = 2 * ceil(sqrt((wxf + 1) * (wy + 1) / ((wxf + 1) * (wy + 1) - (double)cnt)) * wy / 2);
        if (!window_ok(fr, x0, y0, wxf, wyf, true, 3)) status = -1;
      }
    } else {
      status = 102;
    }
  } else {
    const double Nw = (wx + 1) * (wx + 1);
    if (cnt < 0.5 * Nw) {
      if (cnt > 0.1 * Nw) {
        wxf = wyf = mround(1.4142135623730951 * wx);
        if (!window_ok(fr, x0, y0, wxf, wyf, true, 3)) status = -1;
      }
    } else {
      status = 102;
    }
  }
  if (lane != 0) return;
  if (status == 0) {
    const bool nominal = (wxf == a.winsize && wyf == a.winsize);
    const int bucket = nominal ? 0 : 1;
    const int pos = atomicAdd(&a.qcount[bucket], 1);
    int* q = a.queue + 4 * ((long long)bucket * a.n + pos);
    q[0] = (int)t;
    q[1] = (int)wxf;
    q[2] = (int)wyf;
    q[3] = (quad && cnt > 0) ? 1 : 0;
    return;
  }
  if (status == -1) {
    a.conv[t] = quad ? 0 : -1;
    a.U[2 * t] = ALDIC_NAN;
    a.U[2 * t + 1] = ALDIC_NAN;
  } else {
    a.conv[t] = 102;
    a.U[2 * t] = a.UOld[2 * t];
    a.U[2 * t + 1] = a.UOld[2 * t + 1];
  }
}

struct Sub1Ctl {
  double P[6];
  double H2[4];
  double A[2], B[2];
  double meanf, bf, sabsf;
  double normNew, normAbs, normInit;
  float pf[4], f5, f6;
  int base_r, base_c;
  int step, go, status, fbw8_ready;
};

// Shared-memory arrays of one Subpb1 subset: f (= ImgRef .* mask), fx, fy, g as floats;
// on (mask pixel set), cur (the region that currently restricts f, fx, fy: bw4 after
// set-up, the last g region after a masked iteration), tmp/glab (flood fill of g), fbw8.
struct Sub1Smem {
  float *f, *gx, *gy, *g;
  uint8_t *on, *cur, *tmp, *glab, *fbw8;
};

__device__ __forceinline__ Sub1Smem carve_sub1(unsigned char* base, int npx) {
  Sub1Smem s;
  s.f = reinterpret_cast<float*>(base);
  s.gx = s.f + npx;
  s.gy = s.gx + npx;
  s.g = s.gy + npx;
  uint8_t* u = reinterpret_cast<uint8_t*>(s.g + npx);
  s.on = u;
  s.cur = u + npx;
  s.tmp = u + 2 * npx;
  s.glab = u + 3 * npx;
  s.fbw8 = u + 4 * npx;
  return s;
}

// Derive mean_f, bf, H2, A, B from f-side sums v = [H0 H1 H2 JF0 JF1 JB0 JB1 fs fs2 fn fab].
__device__ __forceinline__ void sub1_fside(Sub1Ctl& c, const double* v, bool use_sum_h, const double* hstore,
                                           double mu) {
  const double n = v[9];
  if (n > 0) {
    c.meanf = v[7] / n;
    c.bf = sqrt(fmax(v[8] - v[7] * v[7] / n, 0.0));
  } else {
    c.meanf = ALDIC_NAN;
    c.bf = ALDIC_NAN;
  }
  const double h0 = use_sum_h ? v[0] : hstore[0];
  const double h1 = use_sum_h ? v[1] : hstore[1];
  const double h2 = use_sum_h ? v[2] : hstore[2];
  const double s2 = 2.0 / (c.bf * c.bf);
  c.H2[0] = h0 * s2 + mu;
  c.H2[1] = h1 * s2;
  c.H2[2] = h1 * s2;
  c.H2[3] = h2 * s2 + mu;
  for (int i = 0; i < 2; ++i) {
    c.B[i] = v[5 + i];
    c.A[i] = (v[3 + i] - c.meanf * c.B[i]) / c.bf;
  }
  c.sabsf = v[10];
}

__global__ void __launch_bounds__(kNT) subpb1_solve_kernel(Sub1Args a, int bucket) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ Sub1Ctl c;
  __shared__ double red[(kNT / 32) * 16];
  __shared__ double sums[16];
  const int tid = threadIdx.x;
  const FrameDev& fr = a.fr;
  const bool quad = (a.variant == 1);
  const int count = a.qcount[bucket];
  const int gM = fr.M - 6;
  for (int qi = blockIdx.x; qi < count; qi += gridDim.x) {
    const int* q = a.queue + 4 * ((long long)bucket * a.n + qi);
    const long long t = q[0];
    const int wx = q[1], wy = q[2];
    if (q[3] == 0 || q[3] == kSlowSubset) continue;  // solved by the warp-group passes
    const bool masked = q[3] == 1;
    const int R = wx + 1, Cc = wy + 1, npx = R * Cc;
    const int hx = wx / 2, hy = wy / 2;
    double x0 = a.coords[t], y0 = a.coords[a.n + t];
    if (quad) {
      x0 = mround(x0);
      y0 = mround(y0);
    }
    // bwselect(BW, c, r): column seed from winsize_x, row seed from winsize_y
    // (funICGN_Subpb1quadtree.m:93)
    const int sc = (int)floor((wx + 1) / 2.0) - 1;
    const int sr = (int)floor((wy + 1) / 2.0) - 1;
    Sub1Smem s = carve_sub1(smem_raw, npx);
    {
      const int r0 = (int)x0 - hx - 1, c0 = (int)y0 - hy - 1;
      for (int p = tid; p < npx; p += kNT) {
        const int aa = p % R, bb = p / R;
        const size_t k = (size_t)(r0 + aa) + (size_t)(c0 + bb) * fr.M;
        const size_t kg = (size_t)(r0 + aa - 3) + (size_t)(c0 + bb - 3) * gM;
        float f = fr.ref[k];
        uint8_t on = 1;
        if (quad && fr.mask) {
          on = fr.mask[k] != 0;
          if (!on) f = 0.f;
        }
        s.f[p] = f;
        s.gx[p] = fr.gx[kg];
        s.gy[p] = fr.gy[kg];
        s.on[p] = on;
        s.cur[p] = 1;
      }
    }
    __syncthreads();
    if (masked) {
      flood_select(s.on, s.cur, R, Cc, sr, sc, 4, nullptr);  // cur = bw4
      __syncthreads();
    }
    // f-side sums restricted by cur: H(3), sum J f (2), sum J (2), f stats (3), sum|f|
    {
      float h0 = 0, h1 = 0, h2 = 0, jf0 = 0, jf1 = 0, jb0 = 0, jb1 = 0, fs = 0, fs2 = 0, fn = 0, fab = 0;
      for (int p = tid; p < npx; p += kNT) {
        const float m = s.cur[p] ? 1.f : 0.f;
        const float gxv = s.gx[p] * m, gyv = s.gy[p] * m, f = s.f[p] * m;
        h0 = fmaf(gxv, gxv, h0);
        h1 = fmaf(gxv, gyv, h1);
        h2 = fmaf(gyv, gyv, h2);
        jf0 = fmaf(gxv, f, jf0);
        jf1 = fmaf(gyv, f, jf1);
        jb0 += gxv;
        jb1 += gyv;
        const bool sel = quad ? (fabsf(f) > 1e-10f) : true;
        if (sel) {
          fs += f;
          fs2 = fmaf(f, f, fs2);
          fn += 1.f;
        }
        fab += fabsf(f);
      }
      double v[11] = {h0, h1, h2, jf0, jf1, jb0, jb1, fs, fs2, fn, fab};
      block_sum<11, kNT>(v, red, sums);
    }
    if (tid == 0) {
      double hs[3] = {0, 0, 0};
      if (!quad && a.HPar) {  // stored Hessian block H(5:6,5:6) (funICGN_Subpb1.m:35)
        hs[0] = a.HPar[t + a.n * 18];
        hs[1] = a.HPar[t + a.n * 19];
        hs[2] = a.HPar[t + a.n * 20];
      }
      sub1_fside(c, sums, quad, hs, a.mu);
      c.P[0] = a.FOld[4 * t];
      c.P[1] = a.FOld[4 * t + 1];
      c.P[2] = a.FOld[4 * t + 2];
      c.P[3] = a.FOld[4 * t + 3];
      c.P[4] = a.UOld[2 * t];
      c.P[5] = a.UOld[2 * t + 1];
      c.normNew = 1.0;
      c.normAbs = 1.0;
      c.normInit = 0.0;
      c.step = 0;
      c.status = 0;
      c.fbw8_ready = 0;
    }
    __syncthreads();
    const double uo0 = a.UOld[2 * t], uo1 = a.UOld[2 * t + 1];
    const double vd0 = a.vdual[2 * t], vd1 = a.vdual[2 * t + 1];
    while (true) {
      if (tid == 0) {
        int go = (c.step <= 100 && c.normNew > a.tol && c.normAbs > a.tol) ? 1 : 0;
        if (go) {
          c.step += 1;
          if (warped_oob(fr, c.P, x0, y0, hx, hy)) {
            c.normNew = 1e6;
            go = 0;
          } else {
            const double n5 = mround(c.P[4]), n6 = mround(c.P[5]);
            c.pf[0] = (float)c.P[0];
            c.pf[1] = (float)c.P[1];
            c.pf[2] = (float)c.P[2];
            c.pf[3] = (float)c.P[3];
            c.f5 = (float)(c.P[4] - n5);
            c.f6 = (float)(c.P[5] - n6);
            c.base_r = (int)(x0 + n5) - 2;
            c.base_c = (int)(y0 + n6) - 2;
          }
        }
        c.go = go;
      }
      __syncthreads();
      if (!c.go) break;
      // pass 1: g and the g-side sums with the current f-side region
      float C0 = 0, C1 = 0, S1 = 0, S2 = 0, ns = 0, nz = 0;
      for (int p = tid; p < npx; p += kNT) {
        const float dx = (float)(p % R - hx), dy = (float)(p / R - hy);
        const float lx = dx + fmaf(c.pf[0], dx, fmaf(c.pf[2], dy, c.f5));
        const float ly = dy + fmaf(c.pf[3], dy, fmaf(c.pf[1], dx, c.f6));
        const float ix = floorf(lx), iy = floorf(ly);
        const float g = stencil16(fr.def, fr.M, c.base_r + (int)ix, c.base_c + (int)iy, lx - ix, ly - iy);
        s.g[p] = g;
        const float m = s.cur[p] ? 1.f : 0.f;
        C0 = fmaf(s.gx[p] * m, g, C0);
        C1 = fmaf(s.gy[p] * m, g, C1);
        const bool sel = quad ? (fabsf(g) > 1e-10f) : true;
        if (sel) {
          S1 += g;
          S2 = fmaf(g, g, S2);
          ns += 1.f;
        }
        nz += (g == 0.f) ? 1.f : 0.f;
      }
      double gv[6] = {C0, C1, S1, S2, ns, nz};
      block_sum<6, kNT>(gv, red, sums);
      double Cg[2] = {sums[0], sums[1]}, Sg1 = sums[2], Sg2 = sums[3], Sgn = sums[4];
      const bool run_mask = quad && (masked || sums[5] > 0);
      __syncthreads();
      if (run_mask) {
        // funICGN_Subpb1quadtree.m:158-193: 4-connected g region, fallback to the
        // 8-connected f-mask region; f, fx, fy, H, mean_f, bf recomputed on it.
        for (int p = tid; p < npx; p += kNT) s.tmp[p] = (s.g[p] != 0.f);
        __syncthreads();
        flood_select(s.tmp, s.glab, R, Cc, sr, sc, 4, nullptr);
        int allon = 1;
        for (int p = tid; p < npx; p += kNT) allon &= s.glab[p];
        allon = __syncthreads_and(allon);
        if (allon && !c.fbw8_ready) {
          flood_select(s.on, s.fbw8, R, Cc, sr, sc, 8, nullptr);
          __syncthreads();
          if (tid == 0) c.fbw8_ready = 1;
        }
        const uint8_t* gm = allon ? s.fbw8 : s.glab;
        float h0 = 0, h1 = 0, h2 = 0, jf0 = 0, jf1 = 0, jb0 = 0, jb1 = 0, fs = 0, fs2 = 0, fn = 0, fab = 0;
        float c0 = 0, c1 = 0, t1 = 0, t2 = 0, tn = 0;
        for (int p = tid; p < npx; p += kNT) {
          const uint8_t mk = gm[p];
          s.cur[p] = mk;
          const float m = mk ? 1.f : 0.f;
          const float gxv = s.gx[p] * m, gyv = s.gy[p] * m, f = s.f[p] * m, g = s.g[p] * m;
          h0 = fmaf(gxv, gxv, h0);
          h1 = fmaf(gxv, gyv, h1);
          h2 = fmaf(gyv, gyv, h2);
          jf0 = fmaf(gxv, f, jf0);
          jf1 = fmaf(gyv, f, jf1);
          jb0 += gxv;
          jb1 += gyv;
          if (fabsf(f) > 1e-10f) {
            fs += f;
            fs2 = fmaf(f, f, fs2);
            fn += 1.f;
          }
          fab += fabsf(f);
          c0 = fmaf(gxv, g, c0);
          c1 = fmaf(gyv, g, c1);
          if (fabsf(g) > 1e-10f) {
            t1 += g;
            t2 = fmaf(g, g, t2);
            tn += 1.f;
          }
        }
        double v[16] = {h0, h1, h2, jf0, jf1, jb0, jb1, fs, fs2, fn, fab, c0, c1, t1, t2, tn};
        block_sum<16, kNT>(v, red, sums);
        if (tid == 0) sub1_fside(c, sums, true, nullptr, a.mu);
        Cg[0] = sums[11];
        Cg[1] = sums[12];
        Sg1 = sums[13];
        Sg2 = sums[14];
        Sgn = sums[15];
      }
      if (tid == 0) {
        double meang, bg;
        if (Sgn > 0) {
          meang = Sg1 / Sgn;
          bg = sqrt(fmax(Sg2 - Sg1 * Sg1 / Sgn, 0.0));
        } else {
          meang = ALDIC_NAN;
          bg = ALDIC_NAN;
        }
        double b[2];
        for (int i = 0; i < 2; ++i) b[i] = c.bf * (c.A[i] - (Cg[i] - meang * c.B[i]) / bg);
        const double s2 = 2.0 / (c.bf * c.bf);
        const double tb[2] = {b[0] * s2 + a.mu * (c.P[4] - uo0 - vd0), b[1] * s2 + a.mu * (c.P[5] - uo1 - vd1)};
        const double dmax = fmax(c.H2[0], c.H2[3]);
        const double tH[4] = {c.H2[0] + 1e-3 * dmax, c.H2[1], c.H2[2], c.H2[3] + 1e-3 * dmax};
        const double nb[2] = {-tb[0], -tb[1]};
        double d56[2];
        solve_small(2, tH, nb, d56);
        c.normNew = sqrt(tb[0] * tb[0] + tb[1] * tb[1]);
        c.normAbs = c.normNew;
        if (c.step == 1) c.normInit = c.normNew;
        if (c.normInit > a.tol) c.normNew = c.normNew / c.normInit;
        else c.normNew = 0.0;
        if (!(c.normNew < a.tol || c.normAbs < a.tol)) {
          const double dP[6] = {0, 0, 0, 0, d56[0], d56[1]};
          if (!compose_inverse(c.P, dP)) {
            c.step += 1000;
            c.status = 1;
          }
        }
      }
      __syncthreads();
    }
    if (tid == 0) {
      int step = c.step;
      if (c.status == 1) step -= 1000;
      if (!(c.normNew < a.tol || c.normAbs < a.tol)) step = 101;
      if (isnan(c.normNew)) step = 101;
      if (quad && c.sabsf < 1e-6) step = 103;
      a.conv[t] = step;
      a.U[2 * t] = c.P[4];
      a.U[2 * t + 1] = c.P[5];
    }
    __syncthreads();
  }
}

// ================================================================================
// host launchers
// ================================================================================
static int occupancy_grid(const void* fn, size_t smem, int threads = kNT) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

size_t icgn_smem_bytes(int w) { return (size_t)(w + 1) * (w + 1) * (4 * sizeof(float) + 4); }
size_t icgn_smem_bytes_f64(int w) { return (size_t)(w + 1) * (w + 1) * (sizeof(double) + 3 * sizeof(float) + 4); }
size_t sub1_smem_bytes(int wx, int wy) { return (size_t)(wx + 1) * (wy + 1) * (4 * sizeof(float) + 5); }


// ================================================================================
// Subpb1 for unmasked subsets: warp groups, as icgn_group_kernel
// ================================================================================
// Every subset without a mask region (either queue; any window size) is solved by a group of
// NW warps with no shared image buffer and no block barrier; the FP64 control is replicated
// in every thread.  The main pass (NW = 1) gives a subset at most warp_cap iterations and
// hands slower ones to the 4-warp pass (queue-1 flag kSlowSubset); a quadtree subset that
// meets an exact zero in g needs the g-region flood fill and goes to the general kernel
// (flag kRestartGeneral).  Queue-1 entries are flagged 0 (unmasked: this kernel), 1 (masked:
// the general kernel), kSlowSubset or kRestartGeneral.
constexpr int kRestartGeneral = 3;

template <int NW, bool SLOW>
__global__ void __launch_bounds__(kWT, 2) subpb1_group_kernel(Sub1Args a) {
  constexpr int NG = kWT / (32 * NW);
  constexpr int GT = 32 * NW;
  __shared__ double s_red[NG][NW * 11];
  __shared__ int s_qi[NG];
  const int lane = threadIdx.x & 31, grp = threadIdx.x / GT, gw = (threadIdx.x % GT) >> 5;
  const int gt = threadIdx.x % GT, bar = 1 + grp;
  double* red = s_red[grp];
  const FrameDev& fr = a.fr;
  const bool quad = (a.variant == 1);
  const int c0n = SLOW ? 0 : a.qcount[0];
  const int count = c0n + a.qcount[1];
  const int gM = fr.M - 6;
  int* next = a.qcount + (SLOW ? 3 : 2);
  while (true) {
    int qi = 0;
    if (gt == 0) qi = atomicAdd(next, 1);
    if (NW == 1) {
      qi = __shfl_sync(0xffffffffu, qi, 0);
    } else {
      if (gt == 0) s_qi[grp] = qi;
      group_bar<NW>(bar);
      qi = s_qi[grp];
    }
    if (qi >= count) break;
    const int* q = qi < c0n ? a.queue + 4 * (long long)qi : a.queue + 4 * (a.n + (qi - c0n));
    if (q[3] != (SLOW ? kSlowSubset : 0)) {
      group_bar<NW>(bar);
      continue;
    }
    const long long t = q[0];
    const int wx = q[1], wy = q[2];
    const int R = wx + 1, Cc = wy + 1, npx = R * Cc;
    const int hx = wx / 2, hy = wy / 2;
    double x0 = a.coords[t], y0 = a.coords[a.n + t];
    if (quad) {
      x0 = mround(x0);
      y0 = mround(y0);
    }
    const int r0 = (int)x0 - hx - 1, c0 = (int)y0 - hy - 1;
    const int q_nt = GT / R, r_nt = GT % R;
    // ---- f-side sums over the whole window ----
    double H2[4], A2[2], B2[2], meanf, bf, sabsf;
    {
      float h0 = 0, h1 = 0, h2 = 0, jf0 = 0, jf1 = 0, jb0 = 0, jb1 = 0, fs = 0, fs2 = 0, fn = 0, fab = 0;
      int aa = gt % R, bb = gt / R;
      for (int p = gt; p < npx; p += GT) {
        const int k = (r0 + aa) + (c0 + bb) * fr.M;
        const int kg = (r0 + aa - 3) + (c0 + bb - 3) * gM;
        const float f = fr.ref[k], gxv = fr.gx[kg], gyv = fr.gy[kg];
        h0 = fmaf(gxv, gxv, h0);
        h1 = fmaf(gxv, gyv, h1);
        h2 = fmaf(gyv, gyv, h2);
        jf0 = fmaf(gxv, f, jf0);
        jf1 = fmaf(gyv, f, jf1);
        jb0 += gxv;
        jb1 += gyv;
        if (!quad || fabsf(f) > 1e-10f) {
          fs += f;
          fs2 = fmaf(f, f, fs2);
          fn += 1.f;
        }
        fab += fabsf(f);
        aa += r_nt;
        bb += q_nt;
        if (aa >= R) {
          aa -= R;
          bb += 1;
        }
      }
      double v[11] = {h0, h1, h2, jf0, jf1, jb0, jb1, fs, fs2, fn, fab};
      group_sum<NW, 11>(v, red, gw, lane, bar);
      Sub1Ctl c;
      double hs[3] = {0, 0, 0};
      if (!quad && a.HPar) {  // stored Hessian block H(5:6,5:6) (funICGN_Subpb1.m:35)
        hs[0] = a.HPar[t + a.n * 18];
        hs[1] = a.HPar[t + a.n * 19];
        hs[2] = a.HPar[t + a.n * 20];
      }
      sub1_fside(c, v, quad, hs, a.mu);
      for (int k = 0; k < 4; ++k) H2[k] = c.H2[k];
      A2[0] = c.A[0];
      A2[1] = c.A[1];
      B2[0] = c.B[0];
      B2[1] = c.B[1];
      meanf = c.meanf;
      bf = c.bf;
      sabsf = c.sabsf;
    }
    (void)meanf;
    double P[6] = {a.FOld[4 * t], a.FOld[4 * t + 1], a.FOld[4 * t + 2], a.FOld[4 * t + 3], a.UOld[2 * t],
                   a.UOld[2 * t + 1]};
    const double uo0 = a.UOld[2 * t], uo1 = a.UOld[2 * t + 1];
    const double vd0 = a.vdual[2 * t], vd1 = a.vdual[2 * t + 1];
    double normNew = 1.0, normAbs = 1.0, normInit = 0.0;
    int step = 0, status = 0, requeue = -1;
    while (step <= 100 && normNew > a.tol && normAbs > a.tol) {
      if (!SLOW && step >= a.warp_cap) {
        requeue = kSlowSubset;
        break;
      }
      step += 1;
      if (warped_oob(fr, P, x0, y0, hx, hy)) {
        normNew = 1e6;
        break;
      }
      const double n5 = mround(P[4]), n6 = mround(P[5]);
      const float p0 = (float)P[0], p1 = (float)P[1], p2 = (float)P[2], p3 = (float)P[3];
      const float f5 = (float)(P[4] - n5), f6 = (float)(P[5] - n6);
      const int br = (int)(x0 + n5) - 2, bc = (int)(y0 + n6) - 2;
      float C0 = 0, C1 = 0, S1 = 0, S2 = 0, ns = 0, nz = 0;
      {
        int aa = gt % R, bb = gt / R;
        for (int p = gt; p < npx; p += GT) {
          const float dx = (float)(aa - hx), dy = (float)(bb - hy);
          const float lx = dx + fmaf(p0, dx, fmaf(p2, dy, f5));
          const float ly = dy + fmaf(p3, dy, fmaf(p1, dx, f6));
          const float ix = floorf(lx), iy = floorf(ly);
          const float g = stencil16(fr.def, fr.M, br + (int)ix, bc + (int)iy, lx - ix, ly - iy);
          const int kg = (r0 + aa - 3) + (c0 + bb - 3) * gM;
          C0 = fmaf(fr.gx[kg], g, C0);
          C1 = fmaf(fr.gy[kg], g, C1);
          if (!quad || fabsf(g) > 1e-10f) {
            S1 += g;
            S2 = fmaf(g, g, S2);
            ns += 1.f;
          }
          nz += (g == 0.f) ? 1.f : 0.f;
          aa += r_nt;
          bb += q_nt;
          if (aa >= R) {
            aa -= R;
            bb += 1;
          }
        }
      }
      double v[6] = {C0, C1, S1, S2, ns, nz};
      group_sum<NW, 6>(v, red, gw, lane, bar);
      if (quad && v[5] > 0) {  // exact zero in g: the g-region flood fill of the general kernel
        requeue = kRestartGeneral;
        break;
      }
      double meang, bgn;
      if (v[4] > 0) {
        meang = v[2] / v[4];
        bgn = sqrt(fmax(v[3] - v[2] * v[2] / v[4], 0.0));
      } else {
        meang = ALDIC_NAN;
        bgn = ALDIC_NAN;
      }
      double b[2];
      for (int i = 0; i < 2; ++i) b[i] = bf * (A2[i] - (v[i] - meang * B2[i]) / bgn);
      const double s2 = 2.0 / (bf * bf);
      const double tb[2] = {b[0] * s2 + a.mu * (P[4] - uo0 - vd0), b[1] * s2 + a.mu * (P[5] - uo1 - vd1)};
      const double dmax = fmax(H2[0], H2[3]);
      const double tH[4] = {H2[0] + 1e-3 * dmax, H2[1], H2[2], H2[3] + 1e-3 * dmax};
      const double nb[2] = {-tb[0], -tb[1]};
      double d56[2];
      solve_small(2, tH, nb, d56);
      normNew = sqrt(tb[0] * tb[0] + tb[1] * tb[1]);
      normAbs = normNew;
      if (step == 1) normInit = normNew;
      if (normInit > a.tol) normNew = normNew / normInit;
      else normNew = 0.0;
      if (!(normNew < a.tol || normAbs < a.tol)) {
        const double dP[6] = {0, 0, 0, 0, d56[0], d56[1]};
        if (!compose_inverse(P, dP)) {
          step += 1000;
          status = 1;
        }
      }
    }
    if (gt == 0) {
      if (requeue >= 0) {
        // a queue-1 entry is re-flagged in place; a queue-0 subset is appended once, so
        // queue 1 never holds more than n entries
        if (qi >= c0n) {
          const_cast<int*>(q)[3] = requeue;
        } else {
          const int pos = atomicAdd(&a.qcount[1], 1);
          int* q1 = a.queue + 4 * (a.n + pos);
          q1[0] = (int)t;
          q1[1] = wx;
          q1[2] = wy;
          q1[3] = requeue;
        }
      } else {
        if (status == 1) step -= 1000;
        if (!(normNew < a.tol || normAbs < a.tol)) step = 101;
        if (isnan(normNew)) step = 101;
        if (quad && sabsf < 1e-6) step = 103;
        a.conv[t] = step;
        a.U[2 * t] = P[4];
        a.U[2 * t + 1] = P[5];
      }
    }
    group_bar<NW>(bar);
  }
}

// Tensor map of a column-major FP32 image for the staging boxes (see tma.cuh).
bool make_tmap_2d_f32(CUtensorMap* map, const float* base, int M, int N, int box_r, int box_c) {
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
  if (!encode || !base || M < 1 || N < 1) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || ((size_t)M * sizeof(float)) % 16 != 0) return false;
  if (box_r < 4 || box_r > 256 || box_r % 4 != 0 || box_c < 1 || box_c > 256) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)M, (cuuint64_t)N};
  const cuuint64_t strides[1] = {(cuuint64_t)M * sizeof(float)};  // bytes between columns
  const cuuint32_t box[2] = {(cuuint32_t)box_r, (cuuint32_t)box_c};
  const cuuint32_t estride[2] = {1, 1};
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box,
                            estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

int launch_icgn(const IcgnArgs& a, int wmax_enlarged, cudaStream_t st) {
  int launches = 0;
  // counts of buckets 0 and 1, the 2 work counters, the count of bucket 2, the staging flag
  cudaMemsetAsync(a.qcount, 0, 16 * sizeof(int), st);
  const long long threads = a.n * 32;
  const int cb = 256;
  icgn_classify_kernel<<<(unsigned)((threads + cb - 1) / cb), cb, 0, st>>>(a);
  ++launches;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  {  // nominal-window subsets without a mask region: one warp per subset, then the slow ones
    // TMA staging of the deformed window when the tensor map can describe the image and the
    // per-group boxes fit two blocks per SM; the gather path otherwise
    StageGeom geo{0, 0, 0};
    CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    bool staged = false;
    if (a.staging) {
      const int W1 = a.winsize + 1;
      geo.box_r = (W1 + 14 + 3) / 4 * 4;  // footprint W1 + 5, alignment 3, 6 rows of deformation
      geo.box_c = W1 + 11;                // footprint W1 + 5, 6 columns of deformation
      geo.buf_floats = (geo.box_r * geo.box_c + 31) / 32 * 32;
      const size_t bytes = (size_t)(kWT / 32) * geo.buf_floats * sizeof(float) + 128;
      staged = geo.box_r <= 256 && geo.box_c <= 256 && bytes <= kStageBytesMax &&
               make_tmap_2d_f32(&tmap, a.fr.def, a.fr.M, a.fr.N, geo.box_r, geo.box_c);
    }
    const int snw = a.slow_nw == 4 ? 4 : kSlowNW;
    const size_t smem1 = staged ? (size_t)(kWT / 32) * geo.buf_floats * sizeof(float) + 128 : 0;
    const size_t smem2 = staged ? (size_t)(kWT / (32 * snw)) * geo.buf_floats * sizeof(float) + 128 : 0;
    auto k1 = staged ? icgn_group_kernel<1, false, true> : icgn_group_kernel<1, false, false>;
    auto k2 = snw == 4 ? (staged ? icgn_group_kernel<4, true, true> : icgn_group_kernel<4, true, false>)
                       : (staged ? icgn_group_kernel<kSlowNW, true, true> : icgn_group_kernel<kSlowNW, true, false>);
    if (staged) {
      cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1);
      cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2);
    }
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k1, kWT, smem1);
    long long grid = (long long)sms * (per_sm < 1 ? 1 : per_sm);
    const long long need = (a.n + 7) / 8;
    if (grid > need) grid = need;
    k1<<<(unsigned)grid, kWT, smem1, st>>>(a, tmap, geo);
    ++launches;
    if (!a.slow_fp64 || a.variant == 2) {  // the FP32 multi-warp pass continues the slow subsets
      per_sm = 1;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2, kWT, smem2);
      grid = (long long)sms * (per_sm < 1 ? 1 : per_sm);
      const long long need_slow = (a.n + kWT / (32 * snw) - 1) / (kWT / (32 * snw));
      if (grid > need_slow) grid = need_slow;
      k2<<<(unsigned)grid, kWT, smem2, st>>>(a, tmap, geo);
      ++launches;
    }
  }
  {  // enlarged / masked subsets, and those handed over by the fast kernel
    const size_t smem = icgn_smem_bytes(wmax_enlarged);
    cudaFuncSetAttribute(icgn_solve_kernel<false, kNT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int grid = occupancy_grid((const void*)icgn_solve_kernel<false, kNT>, smem, kNT);
    grid = grid < 296 ? grid : 296;
    if ((long long)grid > a.n) grid = (int)a.n;
    if (grid < 1) grid = 1;
    icgn_solve_kernel<false, kNT><<<grid, kNT, smem, st>>>(a, 1);
    ++launches;
  }
  if ((a.band > 0 || a.slow_fp64) && a.variant != 2) {
    // FP64 re-solves: the subsets too close to call in FP32 and the long trajectories
    const size_t smem = icgn_smem_bytes_f64(wmax_enlarged);
    auto kf = a.fp64_threads == 512   ? icgn_solve_kernel<true, 512>
              : a.fp64_threads == 256 ? icgn_solve_kernel<true, 256>
                                      : icgn_solve_kernel<true, 128>;
    const int nt = a.fp64_threads == 512 ? 512 : (a.fp64_threads == 256 ? 256 : 128);
    cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int grid = occupancy_grid((const void*)kf, smem, nt);
    grid = grid < 4 * sms ? grid : 4 * sms;
    if ((long long)grid > a.n) grid = (int)a.n;
    if (grid < 1) grid = 1;
    kf<<<grid, nt, smem, st>>>(a, 2);
    ++launches;
  }
  return launches;
}

// ZNCC of a subset under the warp P = [F U]: one warp per subset, FP32 interpolation (the
// IC-GN stencil), FP64 sums of f, f^2, g, g^2, f g over the (w+1)^2 window.
__global__ void subset_zncc_kernel(FrameDev fr, long long n, const double* __restrict__ coords,
                                   const double* __restrict__ U, const double* __restrict__ F, int w,
                                   double* __restrict__ zncc) {
  const long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= n) return;
  const double x0 = mround(coords[t]), y0 = mround(coords[n + t]);
  const double P[6] = {F[4 * t], F[4 * t + 1], F[4 * t + 2], F[4 * t + 3], U[2 * t], U[2 * t + 1]};
  const int half = w / 2, W1 = w + 1;
  const bool finite = isfinite(P[0]) && isfinite(P[1]) && isfinite(P[2]) && isfinite(P[3]) && isfinite(P[4]) &&
                      isfinite(P[5]);
  if (!finite || !window_ok(fr, x0, y0, w, w, false, 3) || warped_oob(fr, P, x0, y0, half, half)) {
    if (lane == 0) zncc[t] = ALDIC_NAN;
    return;
  }
  const double n5 = mround(P[4]), n6 = mround(P[5]);
  const float p0 = (float)P[0], p1 = (float)P[1], p2 = (float)P[2], p3 = (float)P[3];
  const float f5 = (float)(P[4] - n5), f6 = (float)(P[5] - n6);
  const int br = (int)(x0 + n5) - 2, bc = (int)(y0 + n6) - 2;
  const int r0 = (int)x0 - half - 1, c0 = (int)y0 - half - 1;
  double sf = 0, sf2 = 0, sg = 0, sg2 = 0, sfg = 0;
  for (int p = lane; p < W1 * W1; p += 32) {
    const int aa = p % W1, bb = p / W1;
    const float dx = (float)(aa - half), dy = (float)(bb - half);
    const float lx = dx + fmaf(p0, dx, fmaf(p2, dy, f5));
    const float ly = dy + fmaf(p3, dy, fmaf(p1, dx, f6));
    const float ix = floorf(lx), iy = floorf(ly);
    const double g = stencil16(fr.def, fr.M, br + (int)ix, bc + (int)iy, lx - ix, ly - iy);
    const double f = fr.ref[(size_t)(r0 + aa) + (size_t)(c0 + bb) * fr.M];
    sf += f;
    sf2 += f * f;
    sg += g;
    sg2 += g * g;
    sfg += f * g;
  }
  sf = warp_sum(sf);
  sf2 = warp_sum(sf2);
  sg = warp_sum(sg);
  sg2 = warp_sum(sg2);
  sfg = warp_sum(sfg);
  if (lane == 0) {
    const double m = (double)W1 * W1;
    const double den = sqrt(fmax(sf2 - sf * sf / m, 0.0) * fmax(sg2 - sg * sg / m, 0.0));
    zncc[t] = den > 0 ? (sfg - sf * sg / m) / den : ALDIC_NAN;
  }
}

int launch_subset_zncc(const FrameDev& fr, long long n, const double* coords, const double* U, const double* F,
                       int winsize, double* zncc, cudaStream_t st) {
  if (n <= 0) return 0;
  subset_zncc_kernel<<<(unsigned)((n * 32 + 255) / 256), 256, 0, st>>>(fr, n, coords, U, F, winsize, zncc);
  return 1;
}

// The subsets a learned initial guess failed: IC-GN did not converge (code outside 1..100) or
// the final ZNCC is below zmin (or NaN).  Their indices are appended to list (in no fixed
// order) and counted in *count (zeroed by the caller).
__global__ void fallback_select_kernel(const int32_t* __restrict__ conv, const double* __restrict__ zncc, long long n,
                                       double zmin, int32_t* __restrict__ list, int* __restrict__ count) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int c = conv[t];
    if (c < 1 || c > 100 || !(zncc[t] >= zmin)) list[atomicAdd(count, 1)] = (int32_t)t;
  }
}

int launch_fallback_select(const int32_t* conv, const double* zncc, long long n, double zmin, int32_t* list,
                           int* count, cudaStream_t st) {
  if (n <= 0) return 0;
  cudaMemsetAsync(count, 0, sizeof(int), st);
  const long long blocks = (n + 255) / 256;
  fallback_select_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, st>>>(conv, zncc, n, zmin, list,
                                                                                           count);
  return 1;
}

int launch_subpb1(const Sub1Args& a, int wmax_x, int wmax_y, cudaStream_t st) {
  int launches = 0;
  cudaMemsetAsync(a.qcount, 0, 4 * sizeof(int), st);  // 2 queue counts, 2 work counters
  const long long threads = a.n * 32;
  const int cb = 256;
  subpb1_classify_kernel<<<(unsigned)((threads + cb - 1) / cb), cb, 0, st>>>(a);
  ++launches;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  {  // unmasked subsets (both queues): one warp per subset, then the slow ones with 4
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, subpb1_group_kernel<1, false>, kWT, 0);
    long long grid = (long long)sms * (per_sm < 1 ? 1 : per_sm);
    const long long need = (a.n + 7) / 8;
    if (grid > need) grid = need;
    subpb1_group_kernel<1, false><<<(unsigned)grid, kWT, 0, st>>>(a);
    per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, subpb1_group_kernel<kSub1SlowNW, true>, kWT, 0);
    grid = (long long)sms * (per_sm < 1 ? 1 : per_sm);
    const long long need_slow = (a.n + kWT / (32 * kSub1SlowNW) - 1) / (kWT / (32 * kSub1SlowNW));
    if (grid > need_slow) grid = need_slow;
    subpb1_group_kernel<kSub1SlowNW, true><<<(unsigned)grid, kWT, 0, st>>>(a);
    launches += 2;
  }
  {  // masked subsets and restarts: the general kernel on queue 1
    const size_t smem = sub1_smem_bytes(wmax_x, wmax_y);
    cudaFuncSetAttribute(subpb1_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int grid = occupancy_grid((const void*)subpb1_solve_kernel, smem);
    grid = grid < 296 ? grid : 296;
    if ((long long)grid > a.n) grid = (int)a.n;
    if (grid < 1) grid = 1;
    subpb1_solve_kernel<<<grid, kNT, smem, st>>>(a, 1);
    ++launches;
  }
  return launches;
}

}  // namespace aldic
