// Whole-field integer search (funIntegerSearchWholeField, func/funIntegerSearch.m:100-203):
// per grid subset, zero-normalised cross-correlation of the (w+1)^2 template of f with the
// border-clamped search window of g (normxcorr2 semantics, Lewis 1995), cropped to the
// (L+R+3) x (U+D+3) shifts the reference keeps, then findpeak (func/findpeak.m).
//
// Direct correlation, one CTA per subset:
//   * window sums sum(D), sum(D^2) of every shift come from FP64 integral images of g
//     (computed once per call), so the partial-overlap ring of the crop (zero padding of
//     the cut-out window) is exact;
//   * the numerator sum((T - mean T) * D) is tiled over 64 x 64 shifts; each thread owns
//     8 consecutive shift rows x 2 shift columns in registers, slides a 15-value register
//     window down the template column, accumulates each template column in FP32 and
//     adds it to FP64 accumulators (41-term FP32 partial sums);
//   * argmax is the first maximum in column-major order (MATLAB max); the 3 x 3
//     neighbourhood of the peak is recomputed in FP64 for the sub-pixel fit.
#include "common.cuh"
#include "kernels.h"

namespace aldic {

constexpr int SNT = 256;  // threads per search CTA
constexpr int STA = 64;   // shift tile rows
constexpr int STB = 64;   // shift tile columns

__host__ __device__ inline int round_up8(int v) { return (v + 7) & ~7; }

// Column prefix sums: II(r+1, c+1) = sum_{r' <= r} g(r', c) (and of g^2); II is
// (M+1) x (N+1) column-major, row 0 and column 0 zero.
__global__ void integral_cols_kernel(const float* __restrict__ g, int M, int N, double* __restrict__ I1,
                                     double* __restrict__ I2) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t ld = (size_t)M + 1;
  if (c > N) return;
  if (c == 0) {
    for (int r = 0; r <= M; ++r) {
      I1[r] = 0.0;
      I2[r] = 0.0;
    }
    return;
  }
  double s1 = 0, s2 = 0;
  I1[(size_t)c * ld] = 0.0;
  I2[(size_t)c * ld] = 0.0;
  const float* col = g + (size_t)(c - 1) * M;
  for (int r = 0; r < M; ++r) {
    const double v = col[r];
    s1 += v;
    s2 += v * v;
    I1[(size_t)(r + 1) + (size_t)c * ld] = s1;
    I2[(size_t)(r + 1) + (size_t)c * ld] = s2;
  }
}

// Row prefix of the column prefixes -> full integral image.
__global__ void integral_rows_kernel(int M, int N, double* __restrict__ I1, double* __restrict__ I2) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > M) return;
  const size_t ld = (size_t)M + 1;
  double s1 = 0, s2 = 0;
  for (int c = 1; c <= N; ++c) {
    s1 += I1[r + c * ld];
    s2 += I2[r + c * ld];
    I1[r + c * ld] = s1;
    I2[r + c * ld] = s2;
  }
}

struct SubsetGeom {
  int ii, jj;        // 1-based template top-left
  int L, R, U, D;    // search extents
  int na, nb;        // crop size
  int dr0, dr1, dc0, dc1;  // 0-based inclusive extent of the cut-out window D
  bool ok;
};

__device__ inline SubsetGeom subset_geom(const SearchArgs& a, long long t) {
  SubsetGeom s;
  const int i = (int)(t % a.nx), j = (int)(t / a.nx);
  const int w = a.winsize;
  s.ii = a.gx0 + i * a.step;
  s.jj = a.gy0 + j * a.step;
  // [left right up down] = [s0 s1 s0 s1] (funIntegerSearch.m:12), clamped per subset
  // (:139-152); the right/down clamps use gridx(end)/gridy(end) as the reference does.
  int L = a.s0, R = a.s1, U = a.s0, D = a.s1;
  if (s.ii - L < 1) L = s.ii - 1;
  if (s.jj - U < 1) U = s.jj - 1;
  if (s.ii + w + R > a.M) R = a.gx1 - s.ii - w - 1;
  if (s.jj + w + D > a.N) D = a.gy1 - s.jj - w - 1;
  s.L = max(L, 0);
  s.R = max(R, 0);
  s.U = max(U, 0);
  s.D = max(D, 0);
  s.na = s.L + s.R + 3;
  s.nb = s.U + s.D + 3;
  s.dr0 = s.ii - s.L - 1;
  s.dr1 = s.ii + w + s.R - 1;
  s.dc0 = s.jj - s.U - 1;
  s.dc1 = s.jj + w + s.D - 1;
  s.ok = s.ii >= 1 && s.ii + w <= a.M && s.jj >= 1 && s.jj + w <= a.N && s.dr0 >= 0 && s.dr1 < a.M &&
         s.dc0 >= 0 && s.dc1 < a.N;
  return s;
}

// Window sums of the shift (a, b): the (w+1)^2 window with top-left at Dpad (a, b),
// intersected with D (image rows dr0-1+a ..), from the integral images.
__device__ __forceinline__ void window_sums(const SubsetGeom& s, int w, int a, int b, const double* __restrict__ I1,
                                            const double* __restrict__ I2, size_t ld, double* S1, double* S2) {
  const int r0 = max(s.dr0, s.dr0 - 1 + a), r1 = min(s.dr1, s.dr0 - 1 + a + w);
  const int c0 = max(s.dc0, s.dc0 - 1 + b), c1 = min(s.dc1, s.dc0 - 1 + b + w);
  const size_t p00 = (size_t)r0 + (size_t)c0 * ld, p10 = (size_t)(r1 + 1) + (size_t)c0 * ld;
  const size_t p01 = (size_t)r0 + (size_t)(c1 + 1) * ld, p11 = (size_t)(r1 + 1) + (size_t)(c1 + 1) * ld;
  *S1 = (I1[p11] - I1[p10]) - (I1[p01] - I1[p00]);
  *S2 = (I2[p11] - I2[p10]) - (I2[p01] - I2[p00]);
}

__device__ __forceinline__ double matlab_eps_d(double x) {
  x = fabs(x);
  return nextafter(x, INFINITY) - x;
}

__global__ void __launch_bounds__(SNT, 2) ncc_search_kernel(SearchArgs a) {
  const double* __restrict__ I1 = a.I1;
  const double* __restrict__ I2 = a.I2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[(SNT / 32) * 10];
  __shared__ double sums[10];
  __shared__ float sbest[SNT / 32];
  __shared__ int sidx[SNT / 32];
  __shared__ double s_tmean, s_denT, s_tolz;
  __shared__ int s_peak;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int w = a.winsize, W1 = w + 1;
  const int TR = round_up8(W1);
  const int DR = (STA + TR) | 1;  // odd leading dimension: conflict-free column loads
  const int DC = STB + w;
  const size_t ld = (size_t)a.M + 1;
  float* Tp = reinterpret_cast<float*>(smem_raw);  // TR x W1 (rows >= W1 are zero)
  float* Dt = Tp + TR * W1;                         // DR x DC tile of the padded window
  float* den_t = Dt + (size_t)DR * DC;              // STA x STB
  const long long n = (long long)a.nx * a.ny;
  for (long long t = blockIdx.x; t < n; t += gridDim.x) {
    const SubsetGeom s = subset_geom(a, t);
    const int oi = (int)(t % a.nx), oj = (int)(t / a.nx);
    const long long o = oj + (long long)oi * a.ny;
    if (tid == 0) {
      a.x[o] = (s.ii + s.ii + w) / 2.0;
      a.y[o] = (s.jj + s.jj + w) / 2.0;
    }
    if (!s.ok) {
      if (tid == 0) a.u[o] = a.v[o] = a.phi[o] = ALDIC_NAN;
      continue;
    }
    // ---- template: mean, centred FP32 copy, FP64 norm ----
    {
      double v[1] = {0};
      for (int p = tid; p < W1 * W1; p += SNT) {
        const int i = p % W1, j = p / W1;
        v[0] += (double)a.f[(size_t)(s.ii - 1 + i) + (size_t)(s.jj - 1 + j) * a.M];
      }
      block_sum<1, SNT>(v, red, sums);
      if (tid == 0) s_tmean = sums[0] / (double)(W1 * W1);
      __syncthreads();
      const double tm = s_tmean;
      double ss[1] = {0};
      for (int p = tid; p < TR * W1; p += SNT) {
        const int i = p % TR, j = p / TR;
        float tv = 0.f;
        if (i < W1) {
          const double d = (double)a.f[(size_t)(s.ii - 1 + i) + (size_t)(s.jj - 1 + j) * a.M] - tm;
          ss[0] += d * d;
          tv = (float)d;
        }
        Tp[i + j * TR] = tv;
      }
      block_sum<1, SNT>(ss, red, sums);
      if (tid == 0) s_denT = sqrt(sums[0]);
      __syncthreads();
    }
    const double denT = s_denT;
    if (!(denT != 0)) {  // constant template: normxcorr2 throws
      if (tid == 0) a.u[o] = a.v[o] = a.phi[o] = ALDIC_NAN;
      __syncthreads();
      continue;
    }
    const double nwin = (double)W1 * W1;
    // ---- pre-pass: largest denominator over the crop (normxcorr2 zero threshold) ----
    {
      double dmax = 0;
      for (int k = tid; k < s.na * s.nb; k += SNT) {
        double S1, S2;
        window_sums(s, w, k % s.na, k / s.na, I1, I2, ld, &S1, &S2);
        dmax = fmax(dmax, denT * sqrt(fmax(S2 - S1 * S1 / nwin, 0.0)));
      }
      for (int off = 16; off > 0; off >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
      if (lane == 0) red[warp] = dmax;
      __syncthreads();
      if (tid == 0) {
        double m = 0;
        for (int i = 0; i < SNT / 32; ++i) m = fmax(m, red[i]);
        s_tolz = sqrt(matlab_eps_d(m));
      }
      __syncthreads();
    }
    const double tolz = s_tolz;
    const float one_tol = 1.4901161193847656e-08f;  // sqrt(eps(1))
    float best = -INFINITY;
    int bidx = 0x7fffffff;
    // task of this thread inside a 64 x 64 tile: 8 shift rows x shift columns (b, b+8)
    const int la = lane & 3, lb = lane >> 2;
    const int wa = warp & 1, wb = warp >> 1;
    const int a0 = (wa * 4 + la) * 8;
    const int b0 = wb * 16 + lb;
    for (int ta0 = 0; ta0 < s.na; ta0 += STA)
      for (int tb0 = 0; tb0 < s.nb; tb0 += STB) {
        // load the tile of the padded window: Dpad(p, q) = g at image (dr0-1+p, dc0-1+q)
        // inside D, zero outside
        for (int k = tid; k < DR * DC; k += SNT) {
          const int p = ta0 + k % DR, q = tb0 + k / DR;
          const int r = s.dr0 - 1 + p, c = s.dc0 - 1 + q;
          float v = 0.f;
          if (r >= s.dr0 && r <= s.dr1 && c >= s.dc0 && c <= s.dc1) v = __ldg(a.g + (size_t)r + (size_t)c * a.M);
          Dt[k] = v;
        }
        for (int k = tid; k < STA * STB; k += SNT) {
          const int aa = ta0 + k % STA, bb = tb0 + k / STA;
          float dv = -1.f;
          if (aa < s.na && bb < s.nb) {
            double S1, S2;
            window_sums(s, w, aa, bb, I1, I2, ld, &S1, &S2);
            const double den = denT * sqrt(fmax(S2 - S1 * S1 / nwin, 0.0));
            dv = (den > tolz) ? (float)den : -1.f;
          }
          den_t[k] = dv;
        }
        __syncthreads();
        if (ta0 + a0 < s.na && tb0 + b0 < s.nb) {
          double acc0[8], acc1[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            acc0[k] = 0.0;
            acc1[k] = 0.0;
          }
          for (int j = 0; j < W1; ++j) {
            const float* c0 = Dt + (size_t)(b0 + j) * DR + a0;
            const float* c1 = c0 + 8 * (size_t)DR;
            const float* tj = Tp + j * TR;
            float p0[8], p1[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              p0[k] = 0.f;
              p1[k] = 0.f;
            }
            for (int i0 = 0; i0 < TR; i0 += 8) {
              float w0[15], w1[15];
#pragma unroll
              for (int m = 0; m < 15; ++m) {
                w0[m] = c0[i0 + m];
                w1[m] = c1[i0 + m];
              }
#pragma unroll
              for (int sidx8 = 0; sidx8 < 8; ++sidx8) {
                const float tv = tj[i0 + sidx8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                  p0[k] = fmaf(tv, w0[k + sidx8], p0[k]);
                  p1[k] = fmaf(tv, w1[k + sidx8], p1[k]);
                }
              }
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              acc0[k] += (double)p0[k];
              acc1[k] += (double)p1[k];
            }
          }
          // NCC, zero rules, running first-max in column-major crop order
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const int bb = tb0 + b0 + 8 * half;
            if (bb >= s.nb) continue;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const int aa = ta0 + a0 + k;
              if (aa >= s.na) continue;
              const float dv = den_t[(a0 + k) + (b0 + 8 * half) * STA];
              float cval = 0.f;
              if (dv > 0.f) cval = (float)((half ? acc1[k] : acc0[k]) / (double)dv);
              if (fabsf(cval) - 1.f > one_tol) cval = 0.f;
              const int lin = aa + bb * s.na;
              if (cval > best || (cval == best && lin < bidx)) {
                best = cval;
                bidx = lin;
              }
            }
          }
        }
        __syncthreads();
      }
    // ---- block argmax (max value, then smallest column-major index) ----
    for (int off = 16; off > 0; off >>= 1) {
      const float ob = __shfl_xor_sync(0xffffffffu, best, off);
      const int oidx = __shfl_xor_sync(0xffffffffu, bidx, off);
      if (ob > best || (ob == best && oidx < bidx)) {
        best = ob;
        bidx = oidx;
      }
    }
    if (lane == 0) {
      sbest[warp] = best;
      sidx[warp] = bidx;
    }
    __syncthreads();
    if (tid == 0) {
      float b = sbest[0];
      int bi = sidx[0];
      for (int i = 1; i < SNT / 32; ++i)
        if (sbest[i] > b || (sbest[i] == b && sidx[i] < bi)) {
          b = sbest[i];
          bi = sidx[i];
        }
      s_peak = bi;
    }
    __syncthreads();
    // ---- FP64 NCC of the 3 x 3 neighbourhood of the peak ----
    const int pa = s_peak % s.na, pb = s_peak / s.na;
    {
      double v[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) v[k] = 0.0;
      const double tm = s_tmean;
      for (int p = tid; p < W1 * W1; p += SNT) {
        const int i = p % W1, j = p / W1;
        const double tv = (double)a.f[(size_t)(s.ii - 1 + i) + (size_t)(s.jj - 1 + j) * a.M] - tm;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          const int aa = pa + (k % 3) - 1, bb = pb + (k / 3) - 1;
          const int r = s.dr0 - 1 + aa + i, c = s.dc0 - 1 + bb + j;
          double d = 0.0;
          if (r >= s.dr0 && r <= s.dr1 && c >= s.dc0 && c <= s.dc1) d = (double)a.g[(size_t)r + (size_t)c * a.M];
          v[k] += tv * d;
        }
      }
      block_sum<9, SNT>(v, red, sums);
    }
    if (tid == 0) {
      double cc[9];
      for (int k = 0; k < 9; ++k) {
        const int aa = pa + (k % 3) - 1, bb = pb + (k / 3) - 1;
        cc[k] = 0.0;
        if (aa < 0 || aa >= s.na || bb < 0 || bb >= s.nb) continue;
        double S1, S2;
        window_sums(s, w, aa, bb, I1, I2, ld, &S1, &S2);
        const double den = denT * sqrt(fmax(S2 - S1 * S1 / nwin, 0.0));
        double cv = (den > tolz) ? sums[k] / den : 0.0;
        if (fabs(cv) - 1 > 1.4901161193847656e-08) cv = 0.0;
        cc[k] = cv;
      }
      // findpeak (func/findpeak.m:27-66); xpeak = crop column, ypeak = crop row (1-based)
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
        const double A4 = (cc[2 + 6] - cc[0 + 6] - cc[2 + 0] + cc[0 + 0]) / 4.0;
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
    __syncthreads();
  }
}

size_t search_smem_bytes(int winsize, int s0, int s1) {
  (void)s0;
  (void)s1;
  const int W1 = winsize + 1;
  const int TR = round_up8(W1);
  const int DR = (STA + TR) | 1;
  const int DC = STB + winsize;
  return sizeof(float) * ((size_t)TR * W1 + (size_t)DR * DC + (size_t)STA * STB);
}

int launch_search(const SearchArgs& a, cudaStream_t st) {
  const long long n = (long long)a.nx * a.ny;
  if (n <= 0) return 0;
  integral_cols_kernel<<<(a.N + 1 + 127) / 128, 128, 0, st>>>(a.g, a.M, a.N, a.I1, a.I2);
  integral_rows_kernel<<<(a.M + 1 + 127) / 128, 128, 0, st>>>(a.M, a.N, a.I1, a.I2);
  const size_t smem = search_smem_bytes(a.winsize, a.s0, a.s1);
  cudaFuncSetAttribute(ncc_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ncc_search_kernel, SNT, smem);
  if (per_sm < 1) per_sm = 1;
  long long grid = (long long)sms * per_sm;
  if (grid > n) grid = n;
  ncc_search_kernel<<<(unsigned)grid, SNT, smem, st>>>(a);
  return 3;
}

}  // namespace aldic
