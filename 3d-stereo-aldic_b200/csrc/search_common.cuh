// Helpers shared by the two integer-search implementations (search.cu: one CTA per
// subset; search_tile.cu: shared products over tiles of subsets): the per-subset search
// geometry of funIntegerSearchWholeField (func/funIntegerSearch.m:139-152), window sums
// from the FP64 integral images, and the FP64 3 x 3 refit + findpeak (func/findpeak.m).
#pragma once
#include "common.cuh"
#include "kernels.h"

namespace aldic {

__host__ __device__ inline int round_up8(int v) { return (v + 7) & ~7; }
__host__ __device__ inline int round_up16(int v) { return (v + 15) & ~15; }

// Search extents along one image axis for a template starting at the 1-based index
// `start` (ii or jj): [lo hi] = [s0 s1] clamped as funIntegerSearch.m:139-152 does (the
// high-side clamp uses gridx(end) / gridy(end), `gend`).  `ok` is the axis part of the
// validity test: the template and the cut-out window lie inside the image.
struct AxisGeom {
  int lo, hi;      // L, R (rows) or U, D (columns), >= 0
  int d0, d1;      // 0-based inclusive extent of the cut-out window along the axis
  bool ok;
};

__host__ __device__ inline AxisGeom axis_geom(int start, int w, int s0, int s1, int size, int gend) {
  AxisGeom g;
  int lo = s0, hi = s1;
  if (start - lo < 1) lo = start - 1;
  if (start + w + hi > size) hi = gend - start - w - 1;
  g.lo = lo > 0 ? lo : 0;
  g.hi = hi > 0 ? hi : 0;
  g.d0 = start - g.lo - 1;
  g.d1 = start + w + g.hi - 1;
  g.ok = start >= 1 && start + w <= size && g.d0 >= 0 && g.d1 < size;
  return g;
}

struct SubsetGeom {
  int ii, jj;        // 1-based template top-left
  int L, R, U, D;    // search extents
  int na, nb;        // crop size
  int dr0, dr1, dc0, dc1;  // 0-based inclusive extent of the cut-out window D
  bool ok;
};

// Subset t of the nx x ny grid (t = i + j nx).
__device__ inline SubsetGeom subset_geom(const SearchArgs& a, long long t) {
  SubsetGeom s;
  const int i = (int)(t % a.nx), j = (int)(t / a.nx);
  const int w = a.winsize;
  s.ii = a.gx0 + i * a.step;
  s.jj = a.gy0 + j * a.step;
  const AxisGeom r = axis_geom(s.ii, w, a.s0, a.s1, a.M, a.gx1);
  const AxisGeom c = axis_geom(s.jj, w, a.s0, a.s1, a.N, a.gy1);
  s.L = r.lo;
  s.R = r.hi;
  s.U = c.lo;
  s.D = c.hi;
  s.na = s.L + s.R + 3;
  s.nb = s.U + s.D + 3;
  s.dr0 = r.d0;
  s.dr1 = r.d1;
  s.dc0 = c.d0;
  s.dc1 = c.d1;
  s.ok = r.ok && c.ok;
  return s;
}

// Output slot of subset t = i + j nx in the x, y, u, v, phi arrays: o = j + i ny.
__device__ __forceinline__ long long subset_out(const SearchArgs& a, long long t) {
  return t / a.nx + (t % a.nx) * (long long)a.ny;
}

// Sums of g and g^2 over the image box rows r0..r1, columns c0..c1 (inclusive, 0-based)
// from the (M+1) x (N+1) integral images.
__device__ __forceinline__ void box_sums(int r0, int r1, int c0, int c1, const double* __restrict__ I1,
                                         const double* __restrict__ I2, size_t ld, double* S1, double* S2) {
  const size_t p00 = (size_t)r0 + (size_t)c0 * ld, p10 = (size_t)(r1 + 1) + (size_t)c0 * ld;
  const size_t p01 = (size_t)r0 + (size_t)(c1 + 1) * ld, p11 = (size_t)(r1 + 1) + (size_t)(c1 + 1) * ld;
  *S1 = (I1[p11] - I1[p10]) - (I1[p01] - I1[p00]);
  *S2 = (I2[p11] - I2[p10]) - (I2[p01] - I2[p00]);
}

// Window sums of the crop shift (a, b): the (w+1)^2 window with top-left at Dpad (a, b),
// intersected with D (image rows dr0-1+a ..), from the integral images.
__device__ __forceinline__ void window_sums(const SubsetGeom& s, int w, int a, int b, const double* __restrict__ I1,
                                            const double* __restrict__ I2, size_t ld, double* S1, double* S2) {
  const int r0 = max(s.dr0, s.dr0 - 1 + a), r1 = min(s.dr1, s.dr0 - 1 + a + w);
  const int c0 = max(s.dc0, s.dc0 - 1 + b), c1 = min(s.dc1, s.dc0 - 1 + b + w);
  box_sums(r0, r1, c0, c1, I1, I2, ld, S1, S2);
}

__device__ __forceinline__ double matlab_eps_d(double x) {
  x = fabs(x);
  return nextafter(x, INFINITY) - x;
}

// Per-subset constants of the normalised cross-correlation, computed once per call.
struct SubsetPrm {
  double fm;     // template mean
  double denT;   // sqrt(sum (T - mean)^2)
  double tolz;   // normxcorr2 zero threshold on the denominator
  double tolv;   // the same threshold on the window variance sum: (tolz / denT)^2
  int valid;     // geometry inside the image and a non-constant template
  int pad;
};

// FP64 NCC at crop shift (aa, bb) from its numerator sum((T - mean) D): the normxcorr2
// zero rules (denominator threshold tolz, |C| - 1 > sqrt(eps(1)) -> 0); 0 outside the crop.
__device__ inline double ncc_at(const SearchArgs& a, const SubsetGeom& s, int aa, int bb, double num, double denT,
                                double tolz) {
  if (aa < 0 || aa >= s.na || bb < 0 || bb >= s.nb) return 0.0;
  const int w = a.winsize, W1 = w + 1;
  double S1, S2;
  window_sums(s, w, aa, bb, a.I1, a.I2, (size_t)a.M + 1, &S1, &S2);
  const double den = denT * sqrt(fmax(S2 - S1 * S1 / ((double)W1 * W1), 0.0));
  double cv = (den > tolz) ? num / den : 0.0;
  if (fabs(cv) - 1 > 1.4901161193847656e-08) cv = 0.0;
  return cv;
}

// findpeak (func/findpeak.m:27-66) on the 3 x 3 NCC values around the crop peak (pa, pb),
// cc[(row offset + 1) + 3 (column offset + 1)], and the displacement of
// funIntegerSearch.m:170-190 written to slot o.
__device__ inline void findpeak_store(const SearchArgs& a, const SubsetGeom& s, long long o, int pa, int pb,
                                      const double (&cc)[9]) {
  // xpeak = crop column, ypeak = crop row (1-based)
  double xpeak = pb + 1, ypeak = pa + 1, maxf = cc[4];
  const bool edge = (pb == 0 || pb == s.nb - 1 || pa == 0 || pa == s.na - 1);
  if (!edge) {
    // u(dx, dy) with dx = column offset, dy = row offset: cc[(dy+1) + 3 (dx+1)]
    double S = 0, Sx = 0, Sy = 0, Sx2 = 0, Sy2 = 0;
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy) {
        const double u = cc[(dy + 1) + 3 * (dx + 1)];
        S += u;
        Sx += dx * u;
        Sy += dy * u;
        if (dx != 0) Sx2 += u;
        if (dy != 0) Sy2 += u;
      }
    const double A2 = Sx / 6.0, A3 = Sy / 6.0;
    const double A4 = (cc[8] - cc[6] - cc[2] + cc[0]) / 4.0;
    const double A5 = Sx2 / 2.0 - S / 3.0, A6 = Sy2 / 2.0 - S / 3.0;
    const double A1 = (5.0 * S - 3.0 * (Sx2 + Sy2)) / 9.0;
    const double dd = A4 * A4 - 4 * A5 * A6;
    double xo = (-A3 * A4 + 2 * A6 * A2) / dd;
    double yo = -1 / dd * (A4 * A2 - 2 * A5 * A3);
    if (!(fabs(xo) > 1 || fabs(yo) > 1)) {
      xo = round(1000 * xo) / 1000;
      yo = round(1000 * yo) / 1000;
      xpeak += xo;
      ypeak += yo;
      maxf = A1 + A2 * xo + A3 * yo + A4 * xo * yo + A5 * xo * xo + A6 * yo * yo;
    }
  }
  a.u[o] = ypeak - 2 - s.L;
  a.v[o] = xpeak - 2 - s.U;
  a.phi[o] = maxf;
}

// Per-thread FP64 numerator partials of the 3 x 3 neighbourhood of (pa, pb): template
// elements p = first, first + stride, ...
__device__ __forceinline__ void peak_partials(const SearchArgs& a, const SubsetGeom& s, int pa, int pb, double tm,
                                              int first, int stride, double (&v)[9]) {
  const int W1 = a.winsize + 1;
#pragma unroll
  for (int k = 0; k < 9; ++k) v[k] = 0.0;
  int i = first % W1, j = first / W1;
  const int di = stride % W1, dj = stride / W1;
  const float* fb = a.f + (s.ii - 1) + (size_t)(s.jj - 1) * a.M;
  const float* gb = a.g + (s.dr0 - 2 + pa) + (size_t)(s.dc0 - 2 + pb) * a.M;
  if (pa >= 2 && pa <= s.na - 3 && pb >= 2 && pb <= s.nb - 3) {
    // the 3 x 3 shifts are whole windows inside D: no zero padding
    for (int p = first; p < W1 * W1; p += stride) {
      const int o = i + j * a.M;
      const double tv = (double)fb[o] - tm;
      const float* q = gb + o;
#pragma unroll
      for (int cb = 0; cb < 3; ++cb) {
        const float* qc = q + cb * a.M;
#pragma unroll
        for (int rb = 0; rb < 3; ++rb) v[rb + 3 * cb] += tv * (double)qc[rb];
      }
      i += di;
      j += dj;
      if (i >= W1) {
        i -= W1;
        ++j;
      }
    }
    return;
  }
  for (int p = first; p < W1 * W1; p += stride) {
    const double tv = (double)fb[i + (size_t)j * a.M] - tm;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const int r = s.dr0 - 2 + pa + (k % 3) + i, c = s.dc0 - 2 + pb + (k / 3) + j;
      double d = 0.0;
      if (r >= s.dr0 && r <= s.dr1 && c >= s.dc0 && c <= s.dc1) d = (double)a.g[(size_t)r + (size_t)c * a.M];
      v[k] += tv * d;
    }
    i += di;
    j += dj;
    if (i >= W1) {
      i -= W1;
      ++j;
    }
  }
}

// Warp form of the interior case of peak_partials: the same nine sums, with lane = template
// row.  A lane walks its row along the columns, keeping the taps of the 3 x 3 shift block in
// a sliding window, so each step loads (and widens to FP64) one template value and the
// three g values of the newest column instead of ten values per pixel; consecutive lanes
// read consecutive rows (coalesced).  Rows beyond the first 32 are split into column
// parts over the lanes.
__device__ __forceinline__ void peak_partials_warp_interior(const SearchArgs& a, const SubsetGeom& s, int pa, int pb,
                                                            double tm, int lane, double (&v)[9]) {
  const int W1 = a.winsize + 1;
  const size_t M = (size_t)a.M;
#pragma unroll
  for (int k = 0; k < 9; ++k) v[k] = 0.0;
  const float* fb = a.f + (s.ii - 1) + (size_t)(s.jj - 1) * M;
  const float* gb = a.g + (s.dr0 - 2 + pa) + (size_t)(s.dc0 - 2 + pb) * M;
  for (int r0 = 0; r0 < W1; r0 += 32) {
    const int nr = min(32, W1 - r0), parts = 32 / nr;
    if (lane >= parts * nr) continue;
    const int i = r0 + lane % nr, part = lane / nr;
    const int c0 = part * W1 / parts, c1 = (part + 1) * W1 / parts;
    const float* fr = fb + i;
    const float* gr = gb + i;
    double t0[3], t1[3];
#pragma unroll
    for (int rb = 0; rb < 3; ++rb) {
      t0[rb] = (double)gr[rb + (size_t)c0 * M];
      t1[rb] = (double)gr[rb + (size_t)(c0 + 1) * M];
    }
    // unrolled so that several columns' loads are in flight at once (each new column is a
    // fresh cache line for every lane)
#pragma unroll 6
    for (int j = c0; j < c1; ++j) {
      double t2[3];
#pragma unroll
      for (int rb = 0; rb < 3; ++rb) t2[rb] = (double)gr[rb + (size_t)(j + 2) * M];
      const double tv = (double)fr[(size_t)j * M] - tm;
#pragma unroll
      for (int rb = 0; rb < 3; ++rb) {
        v[rb] += tv * t0[rb];
        v[rb + 3] += tv * t1[rb];
        v[rb + 6] += tv * t2[rb];
        t0[rb] = t1[rb];
        t1[rb] = t2[rb];
      }
    }
  }
}

// Block version: every thread of the block calls it; thread 0 writes u, v, phi.
__device__ inline void refit_peak(const SearchArgs& a, const SubsetGeom& s, long long o, int pa, int pb, double tm,
                                  double denT, double tolz, double* red, double* sums) {
  {
    double v[9];
    peak_partials(a, s, pa, pb, tm, threadIdx.x, blockDim.x, v);
    block_sum_dyn<9>(v, red, sums, blockDim.x >> 5);
  }
  if (threadIdx.x == 0) {
    double cc[9];
    for (int k = 0; k < 9; ++k) cc[k] = ncc_at(a, s, pa + (k % 3) - 1, pb + (k / 3) - 1, sums[k], denT, tolz);
    findpeak_store(a, s, o, pa, pb, cc);
  }
  __syncthreads();
}

// Warp version: the 32 lanes of one warp call it; the 9 NCC values are formed by lanes
// 0..8 in parallel and lane 0 writes u, v, phi.
__device__ inline void refit_peak_warp(const SearchArgs& a, const SubsetGeom& s, long long o, int pa, int pb,
                                       double tm, double denT, double tolz) {
  const int lane = threadIdx.x & 31;
  double v[9];
  if (pa >= 2 && pa <= s.na - 3 && pb >= 2 && pb <= s.nb - 3)
    peak_partials_warp_interior(a, s, pa, pb, tm, lane, v);
  else
    peak_partials(a, s, pa, pb, tm, lane, 32, v);
#pragma unroll
  for (int k = 0; k < 9; ++k) v[k] = warp_sum(v[k]);
  double mine = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k)
    if (lane == k) mine = ncc_at(a, s, pa + (k % 3) - 1, pb + (k / 3) - 1, v[k], denT, tolz);
  double cc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) cc[k] = __shfl_sync(0xffffffffu, mine, k);
  if (lane == 0) findpeak_store(a, s, o, pa, pb, cc);
}

}  // namespace aldic
