// Whole-field integer search with shared products: the same results as the per-subset
// normxcorr2 of funIntegerSearchWholeField (func/funIntegerSearch.m:100-203, findpeak at
// :170-190), computed for tiles of grid subsets at once.
//
// The numerator of the NCC of subset s at the shift d = (da, db) is
//     sum over the (w+1)^2 window W_s of (f - fm_s)(x) g(x + d),
// and the windows of neighbouring grid subsets overlap ((w+1) / step times along each axis
// for w = 40, step = 10).  For a tile of TI x 8 subsets and one shift, every product
// f(x) g(x + d) of the tile is formed once and summed in blocks of `step` columns and rows
// (each window is Q = (w+1) / step whole blocks plus REM = (w+1) mod step leading rows /
// columns of the next block), instead of once per overlapping window:
//   pass 1  each thread owns one tile row x and 8 consecutive shift columns db and walks the
//           tile's columns with a sliding register window of g (128-bit shared loads); the
//           block sums give, per row, the row-band sums RB(x, j, d) over the columns of
//           window j;
//   pass 2  each thread owns (window column j, shift column db) and walks the rows of half
//           of the tile's window rows; block sums over rows give the window sums N(i, j, d).
// The window mean and variance sums of g come from a per-position map (full windows) and a
// per-subset table (the ring of partial windows at the crop border, where normxcorr2 zero-
// pads the cut-out window), both built from the FP64 integral images.  A ring shift drops
// the excluded template row (one RB value) and / or column (a per-subset table of column
// products) from the window sum.  The argmax (first maximum in column-major crop order) is
// refit in FP64 on the 3 x 3 neighbourhood, as the per-subset kernel does.
#include "search_common.cuh"

namespace aldic {

namespace {

constexpr int kTJ = 8;     // subset columns per tile
constexpr int kRing = 128; // rows of the circular g buffer

// Smallest m >= n with m = 4 (mod 8): row strides of 128-bit loads across consecutive
// rows then hit 8 distinct 16-byte bank groups per quarter warp.
constexpr int pad4odd(int n) { return ((n + 3) / 4 % 2 == 1) ? (n + 3) / 4 * 4 : (n + 3) / 4 * 4 + 4; }

// Dynamic shared memory of a tile: f tile, g ring, RB (the same sums as TileShape below; a
// plain function so that sizing candidate tiles instantiates no shape).
constexpr size_t tile_dyn_smem(int ST, int W1, int TI, int DBC) {
  return sizeof(float) * ((size_t)((TI - 1) * ST + W1) * pad4odd((kTJ - 1) * ST + W1) +
                          (size_t)kRing * pad4odd((kTJ - 1) * ST + W1 + DBC + 2) +
                          (size_t)kTJ * DBC * pad4odd((TI - 1) * ST + W1));
}

// DBC shift columns per chunk, in groups of 8 (one pass-1 thread group of 128 rows each).
template <int ST, int W1, int TI, int DBC>
struct TileShape {
  static constexpr int Q = W1 / ST;
  static constexpr int NT = DBC / 8 * 128;           // threads per CTA
  static constexpr int FR = (TI - 1) * ST + W1;      // tile rows
  static constexpr int FC = (kTJ - 1) * ST + W1;     // tile columns
  static constexpr int FCP = pad4odd(FC);            // row stride of F (row-major)
  static constexpr int GCP = pad4odd(FC + DBC + 2);  // row stride of the g ring (row-major)
  static constexpr int FRP = pad4odd(FR);            // row stride of RB (one row per (j, d))
  static constexpr int H0 = (TI + 1) / 2;            // subset rows of the first pass-2 half
  static constexpr int NSUB = TI * kTJ;
  static constexpr size_t smem_bytes =
      sizeof(float) * ((size_t)FR * FCP + (size_t)kRing * GCP + (size_t)kTJ * DBC * FRP);
  static_assert(smem_bytes == tile_dyn_smem(ST, W1, TI, DBC), "one shared-memory size");
  static_assert(DBC % 8 == 0 && DBC >= 16, "chunks hold whole groups of 8 shift columns");
  static_assert(Q >= 1, "step must not exceed the window");
  static_assert(FR <= kRing - 1, "tile rows must leave one free ring row");
};

// Shared memory per CTA: the dynamic buffers plus the static per-subset arrays (a bound).
template <int ST, int W1, int TI, int DBC>
constexpr size_t tile_total_smem() {
  return tile_dyn_smem(ST, W1, TI, DBC) + (size_t)TI * kTJ * 64 + 1024;
}

// Subset rows per tile: as many as fit 127 tile rows and the 227 KB of shared memory a CTA
// may use.
template <int ST, int W1, int DBC>
struct TileFor {
  static constexpr int TI0 = (kRing - 1 - W1) / ST + 1;
  static constexpr int TI = tile_total_smem<ST, W1, TI0, DBC>() <= 232448 ? TI0
                            : tile_total_smem<ST, W1, TI0 - 1, DBC>() <= 232448 ? TI0 - 1
                                                                               : TI0 - 2;
  static_assert(tile_total_smem<ST, W1, TI, DBC>() <= 232448, "tile does not fit shared memory");
};

struct TileScratch {
  float2* map;       // MW x NW row-major (x * NW + y): (window mean of g, 1 / sqrt(variance sum))
  double* V;         // MW x NW row-major: window variance sum S2 - S1^2 / n
  double* H;         // MW x ny: max of V over the non-ring shift columns of grid column j
  SubsetPrm* prm;    // nx * ny
  float2* ringv;     // nx * ny x 4 NDA: (mean, 1/sqrt(variance sum)) of the partial windows
  float* cx;         // nx * ny x 2 NDA: products of the excluded template column
  int* best;         // nx * ny: crop index of the first maximum
  float* cf;         // one centring constant per tile
  double* rr;        // nx x 2 sides x 4 x (N+1): integral-image rows of the top / bottom ring windows
};

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

inline size_t scratch_layout(int M, int N, int W1, int nx, int ny, int nda, char* base, TileScratch* sc) {
  const size_t MW = (size_t)(M - W1 + 1), NW = (size_t)(N - W1 + 1), n = (size_t)nx * ny;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + off : nullptr;
    off += align256(bytes);
    return p;
  };
  char* pm = take(MW * NW * sizeof(float2));
  char* pv = take(MW * NW * sizeof(double));
  char* ph = take(MW * (size_t)ny * sizeof(double));
  char* pp = take(n * sizeof(SubsetPrm));
  char* pr = take(n * 4 * (size_t)nda * sizeof(float2));
  char* pc = take(n * 2 * (size_t)nda * sizeof(float));
  char* pb = take(n * sizeof(int));
  char* pf = take(n * sizeof(float));  // >= the number of tiles
  char* prr = take((size_t)nx * 8 * (size_t)(N + 1) * sizeof(double));
  if (sc) {
    sc->rr = (double*)prr;
    sc->cf = (float*)pf;
    sc->map = (float2*)pm;
    sc->V = (double*)pv;
    sc->H = (double*)ph;
    sc->prm = (SubsetPrm*)pp;
    sc->ringv = (float2*)pr;
    sc->cx = (float*)pc;
    sc->best = (int*)pb;
  }
  return off;
}

__device__ __forceinline__ float rsqrt_from(double v) { return v > 0 ? (float)(1.0 / sqrt(v)) : INFINITY; }

}  // namespace

// Window mean and variance sum of g for every full (w+1)^2 window position (x, y) (top-left,
// 0-based), with the same integral-image expression as window_sums.
__global__ void window_map_kernel(const double* __restrict__ I1, const double* __restrict__ I2, int M, int N,
                                  int W1, float2* __restrict__ map, double* __restrict__ V) {
  const int MW = M - W1 + 1, NW = N - W1 + 1;
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= (long long)MW * NW) return;
  const int x = (int)(p / NW), y = (int)(p % NW);  // row-major: consecutive shift columns adjacent
  double S1, S2;
  box_sums(x, x + W1 - 1, y, y + W1 - 1, I1, I2, (size_t)M + 1, &S1, &S2);
  const double nwin = (double)W1 * W1;
  const double v = S2 - S1 * S1 / nwin;
  V[p] = v;
  map[p] = make_float2((float)(S1 / nwin), rsqrt_from(v));
}

// H(x, j) = max(0, max over the non-ring shift columns db in [-U_j, D_j] of V(x, jj-1+db)).
__global__ void window_rowmax_kernel(SearchArgs a, const double* __restrict__ V, double* __restrict__ H) {
  const int W1 = a.winsize + 1, MW = a.M - W1 + 1, NW = a.N - W1 + 1;
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= (long long)MW * a.ny) return;
  const int x = (int)(p % MW), j = (int)(p / MW);
  const int jj = a.gy0 + j * a.step;
  const AxisGeom c = axis_geom(jj, a.winsize, a.s0, a.s1, a.N, a.gy1);
  double m = 0.0;
  if (c.ok)
    for (int db = -c.lo; db <= c.hi; ++db) m = fmax(m, V[(size_t)x * NW + (jj - 1 + db)]);
  H[p] = m;
}

// Rows r0 and r1 + 1 of both integral images for the top (a = 0) and bottom (a = na-1)
// ring windows of grid row i, whose rows [r0, r1] depend on i alone: stored contiguously
// so that the window sums along a ring row read consecutive addresses.
__global__ void ring_rows_kernel(SearchArgs a, double* __restrict__ rr) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int N1 = a.N + 1;
  if (p >= (long long)a.nx * 2 * N1) return;
  const int c = (int)(p % N1), side = (int)((p / N1) % 2), i = (int)(p / (2 * (long long)N1));
  const int w = a.winsize;
  const AxisGeom g = axis_geom(a.gx0 + i * a.step, w, a.s0, a.s1, a.M, a.gx1);
  if (!g.ok) return;
  const int na = g.lo + g.hi + 3, aa = side ? na - 1 : 0;
  const int r0 = max(g.d0, g.d0 - 1 + aa), r1 = min(g.d1, g.d0 - 1 + aa + w);
  const size_t ld = (size_t)a.M + 1;
  double* out = rr + ((size_t)i * 2 + side) * 4 * N1;
  out[c] = a.I1[(size_t)r0 + c * ld];
  out[N1 + c] = a.I1[(size_t)(r1 + 1) + c * ld];
  out[2 * N1 + c] = a.I2[(size_t)r0 + c * ld];
  out[3 * N1 + c] = a.I2[(size_t)(r1 + 1) + c * ld];
}

// One warp per subset: template mean and norm, the window sums of the ring of partial
// windows, the largest window variance sum over the crop (normxcorr2 zero threshold) and
// validity; writes x, y and the NaN outputs of invalid subsets.
__global__ void __launch_bounds__(256, 4) subset_prep_kernel(SearchArgs a, const double* __restrict__ H, const double* __restrict__ rr,
                                   SubsetPrm* __restrict__ prm, float2* __restrict__ ringv) {
  const int lane = threadIdx.x & 31;
  const long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long n = (long long)a.nx * a.ny;
  if (t >= n) return;
  const SubsetGeom s = subset_geom(a, t);
  const long long o = subset_out(a, t);
  const int w = a.winsize, W1 = w + 1;
  const int nda = a.s0 + a.s1 + 3;
  if (lane == 0) {
    a.x[o] = (s.ii + s.ii + w) / 2.0;
    a.y[o] = (s.jj + s.jj + w) / 2.0;
  }
  SubsetPrm P;
  P.fm = P.denT = P.tolz = P.tolv = 0.0;
  P.valid = 0;
  P.pad = 0;
  if (s.ok) {
    double sum = 0.0;
    for (int p = lane; p < W1 * W1; p += 32)
      sum += (double)a.f[(size_t)(s.ii - 1 + p % W1) + (size_t)(s.jj - 1 + p / W1) * a.M];
    const double fm = warp_sum(sum) / (double)(W1 * W1);
    double ss = 0.0;
    for (int p = lane; p < W1 * W1; p += 32) {
      const double d = (double)a.f[(size_t)(s.ii - 1 + p % W1) + (size_t)(s.jj - 1 + p / W1) * a.M] - fm;
      ss += d * d;
    }
    const double denT = sqrt(warp_sum(ss));
    if (denT != 0) {
      const int MW = a.M - W1 + 1;
      const int j = (int)(t / a.nx);
      const size_t ld = (size_t)a.M + 1;
      const double nwin = (double)W1 * W1;
      float2* rv = ringv + t * 4 * (long long)nda;
      double m = 0.0;
      for (int da = -s.L + lane; da <= s.R; da += 32) m = fmax(m, H[(size_t)(s.ii - 1 + da) + (size_t)j * MW]);
      // the ring of partial windows: a in {0, na-1} for every b, b in {0, nb-1} for every a
      const int N1 = a.N + 1;
      const int i = (int)(t % a.nx);
      for (int side = 0; side < 2; ++side) {
        // the same expression as window_sums, from the extracted rows r0 and r1 + 1
        const double* R = rr + ((size_t)i * 2 + side) * 4 * N1;
        for (int bb = lane; bb < s.nb; bb += 32) {
          const int c0 = max(s.dc0, s.dc0 - 1 + bb), c1 = min(s.dc1, s.dc0 - 1 + bb + w);
          const double S1 = (R[N1 + c1 + 1] - R[N1 + c0]) - (R[c1 + 1] - R[c0]);
          const double S2 = (R[3 * N1 + c1 + 1] - R[3 * N1 + c0]) - (R[2 * N1 + c1 + 1] - R[2 * N1 + c0]);
          const double v = S2 - S1 * S1 / nwin;
          m = fmax(m, v);
          rv[side * nda + bb] = make_float2((float)(S1 / nwin), rsqrt_from(v));
        }
      }
      for (int k = lane; k < 2 * s.na; k += 32) {
        double S1, S2;
        const int side = k & 1, aa = k >> 1;
        window_sums(s, w, aa, side ? s.nb - 1 : 0, a.I1, a.I2, ld, &S1, &S2);
        const double v = S2 - S1 * S1 / nwin;
        m = fmax(m, v);
        rv[(2 + side) * nda + aa] = make_float2((float)(S1 / nwin), rsqrt_from(v));
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
      P.fm = fm;
      P.denT = denT;
      P.tolz = sqrt(matlab_eps_d(denT * sqrt(fmax(m, 0.0))));
      P.tolv = (P.tolz / denT) * (P.tolz / denT);
      P.valid = 1;
    }
  }
  if (lane == 0) {
    prm[t] = P;
    if (!P.valid) a.u[o] = a.v[o] = a.phi[o] = ALDIC_NAN;
  }
}

// One warp per subset: for the two ring shift columns (b = 0: db = -U-1, template column 0;
// b = nb-1: db = D+1, template column w) and every shift row, the sum over the template
// rows of (f - cf) g at that column — the products a ring window drops.  f is centred by
// the tile constant cf and g is zero outside the image, exactly as the tile kernel holds
// them.
__global__ void ring_column_kernel(SearchArgs a, const SubsetPrm* __restrict__ prm, int TI,
                                   const float* __restrict__ tcf, float* __restrict__ cx) {
  const int lane = threadIdx.x & 31;
  const long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long n = (long long)a.nx * a.ny;
  if (t >= n || !prm[t].valid) return;
  const int i = (int)(t % a.nx), j = (int)(t / a.nx);
  const SubsetGeom s = subset_geom(a, t);
  const float cf = tcf[i / TI + (j / kTJ) * ((a.nx + TI - 1) / TI)];
  const int W1 = a.winsize + 1, DA0 = -a.s0 - 1, nda = a.s0 + a.s1 + 3;
  const int X = s.ii - 1, Y = s.jj - 1;
  float* out = cx + t * 2 * (long long)nda;
  for (int side = 0; side < 2; ++side) {
    const int c = Y + (side ? W1 - 1 : 0);
    const int cg = c + (side ? s.D + 1 : -s.U - 1);
    for (int k = lane; k < nda; k += 32) {
      const int aa = DA0 + k + s.L + 1;
      if (aa < 0 || aa >= s.na) continue;
      float acc = 0.f;
      for (int r = 0; r < W1; ++r) {
        const float fv = __ldg(a.f + (size_t)(X + r) + (size_t)c * a.M) - cf;
        const int xg = X + r + DA0 + k;
        float gv = 0.f;
        if (xg >= 0 && xg < a.M && cg >= 0 && cg < a.N) gv = __ldg(a.g + (size_t)xg + (size_t)cg * a.M);
        acc = fmaf(fv, gv, acc);
      }
      out[side * nda + k] = acc;
    }
  }
}

// Pass 1 for one tile row: row-band sums RB(x, j, t) = sum over the columns c of window j
// of F(x, c) G(x + da, c + db0 + t), t = 0..7.  frow = F row x, grow = ring row of x + da
// at column db0 (both 16-byte aligned), rbx = RB at (j = 0, t = 0) for row x.
template <int ST, int W1, int FC, int FRP, int DBC>
__host__ __device__ __forceinline__ void row_band_sums(const float* __restrict__ frow, const float* __restrict__ grow,
                                              float* __restrict__ rbx) {
  constexpr int Q = W1 / ST, REM = W1 % ST, NB = (FC + ST - 1) / ST;
  constexpr int NGG = (FC + 7 + 3) / 4;  // 4-column groups of g covering columns 0 .. FC+6
  constexpr int NFG = (FC + 3) / 4;
  float g[4 * NGG], f[4 * NFG];
  float Bk[NB][8];
  float acc[8], P[8];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const float4 q = *reinterpret_cast<const float4*>(grow + 4 * u);
    g[4 * u] = q.x;
    g[4 * u + 1] = q.y;
    g[4 * u + 2] = q.z;
    g[4 * u + 3] = q.w;
  }
#pragma unroll
  for (int c = 0; c < FC; ++c) {
    const int kc = c / ST, cc = c % ST;
    if (c % 4 == 0) {
      const float4 q = *reinterpret_cast<const float4*>(frow + c);
      f[c] = q.x;
      f[c + 1] = q.y;
      f[c + 2] = q.z;
      f[c + 3] = q.w;
    }
    if ((c + 7) % 4 == 0 && (c + 7) / 4 >= 2) {
      const int u = (c + 7) / 4;
      const float4 q = *reinterpret_cast<const float4*>(grow + 4 * u);
      g[4 * u] = q.x;
      g[4 * u + 1] = q.y;
      g[4 * u + 2] = q.z;
      g[4 * u + 3] = q.w;
    }
    if (cc == 0) {
#pragma unroll
      for (int t = 0; t < 8; ++t) acc[t] = P[t] = 0.f;
    }
    const float fv = f[c];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if (cc < REM)
        P[t] = fmaf(fv, g[c + t], P[t]);
      else
        acc[t] = fmaf(fv, g[c + t], acc[t]);
    }
    if (cc == ST - 1 || c == FC - 1) {
#pragma unroll
      for (int t = 0; t < 8; ++t) Bk[kc][t] = acc[t] + P[t];
      if (REM > 0) {
        // window j = kc - Q: Q whole blocks j..j+Q-1 and the first REM columns of block kc
        if (kc >= Q && kc - Q < kTJ) {
          const int j = kc - Q;
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            float s = Bk[j][t];
#pragma unroll
            for (int b = 1; b < Q; ++b) s += Bk[j + b][t];
            rbx[(j * DBC + t) * FRP] = s + P[t];
          }
        }
      } else {
        if (kc >= Q - 1 && kc - Q + 1 < kTJ) {
          const int j = kc - Q + 1;
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            float s = Bk[j][t];
#pragma unroll
            for (int b = 1; b < Q; ++b) s += Bk[j + b][t];
            rbx[(j * DBC + t) * FRP] = s;
          }
        }
      }
    }
  }
}

// Pass 2 walk: window sums N[e] of NS consecutive window rows starting at tile row R0, from
// one RB row (rb = RB + (j, d) row, 16-byte aligned) by block sums over rows.
template <int ST, int W1, int NS, int R0>
__host__ __device__ __forceinline__ void column_sums(const float* __restrict__ rb, float (&N)[NS]) {
  constexpr int Q = W1 / ST, REM = W1 % ST;
  constexpr int NBV = NS - 1 + Q + (REM > 0 ? 1 : 0);
  constexpr int ROWS = (NS - 1) * ST + W1;
  float v[ROWS + 3];
#pragma unroll
  for (int i = 0; i < ROWS; ++i) {
    const int r = R0 + i, m = r & 3, j0 = i - m;
    const bool in4 = (j0 >= 0) && (j0 + 3 < ROWS);  // covered by an aligned 128-bit load at j0
    if (in4) {
      if (m == 0) {
        const float4 q = *reinterpret_cast<const float4*>(rb + r);
        v[i] = q.x;
        v[i + 1] = q.y;
        v[i + 2] = q.z;
        v[i + 3] = q.w;
      }
    } else {
      v[i] = rb[r];
    }
  }
  float BV[NBV], PV[NBV];
#pragma unroll
  for (int k = 0; k < NBV; ++k) BV[k] = PV[k] = 0.f;
#pragma unroll
  for (int r = 0; r < ROWS; ++r) {
    if (r % ST < REM)
      PV[r / ST] += v[r];
    else
      BV[r / ST] += v[r];
  }
#pragma unroll
  for (int e = 0; e < NS; ++e) {
    float s = BV[e] + PV[e];
#pragma unroll
    for (int b = 1; b < Q; ++b) s += BV[e + b] + PV[e + b];
    if (REM > 0) s += PV[e + Q];
    N[e] = s;
  }
}

// Pass 1 with packed FP32 pairs (even steps): the same row-band sums as row_band_sums.
// At an even column c the 8 products f(c) g(c + t) are 4 pairs t = (0,1) .. (6,7) of
// aligned g pairs; at an odd column, t = (1,2) .. (5,6) are aligned pairs and t = 0, 7
// scalars.  Even and odd columns accumulate separately (E and O) and are added at the
// block end; the first REM columns of a block (P) seed the remaining columns' sums.
template <int ST, int W1, int FC, int FRP, int DBC>
__host__ __device__ __forceinline__ void row_band_sums_x2(const float* __restrict__ frow, const float* __restrict__ grow,
                                                 float* __restrict__ rbx) {
  static_assert(ST % 2 == 0, "blocks must start on even columns");
  constexpr int Q = W1 / ST, REM = W1 % ST, NB = (FC + ST - 1) / ST;
  constexpr int NGG = (FC + 7 + 3) / 4;  // 4-column groups of g covering columns 0 .. FC+6
  constexpr int NFG = (FC + 3) / 4;
  constexpr int E_A0 = (REM + 1) / 2 * 2;  // first even column of a block outside P
  constexpr int O_A0 = REM / 2 * 2 + 1;    // first odd column of a block outside P
  float2 gp[2 * NGG];                      // gp[m] = (g(2m), g(2m+1))
  float f[4 * NFG];
  float2 B[NB][4], S2[NB][4];              // block sums and sums of consecutive block pairs, t pairs
  float2 PE[4], AE[4], PO[3], AO[3];
  float PO0 = 0.f, PO7 = 0.f, AO0 = 0.f, AO7 = 0.f;
  float2 ffn;
  // loads run one 4-column group ahead of their first use
#pragma unroll
  for (int u = 0; u < 3 && u < NGG; ++u) {
    const float4 q = *reinterpret_cast<const float4*>(grow + 4 * u);
    gp[2 * u] = make_float2(q.x, q.y);
    gp[2 * u + 1] = make_float2(q.z, q.w);
  }
#pragma unroll
  for (int u = 0; u < 2 && u < NFG; ++u) {
    const float4 q = *reinterpret_cast<const float4*>(frow + 4 * u);
    f[4 * u] = q.x;
    f[4 * u + 1] = q.y;
    f[4 * u + 2] = q.z;
    f[4 * u + 3] = q.w;
  }
  ffn = make_float2(f[0], f[0]);
#pragma unroll
  for (int c = 0; c < FC; ++c) {
    const int kc = c / ST, cc = c % ST;
    if (c % 4 == 0 && c / 4 + 2 < NFG) {  // f group needed at column c + 8
      const int u = c / 4 + 2;
      const float4 q = *reinterpret_cast<const float4*>(frow + 4 * u);
      f[4 * u] = q.x;
      f[4 * u + 1] = q.y;
      f[4 * u + 2] = q.z;
      f[4 * u + 3] = q.w;
    }
    if ((c + 11) % 4 == 0 && (c + 11) / 4 >= 3 && (c + 11) / 4 < NGG) {  // g group first needed at column c + 4
      const int u = (c + 11) / 4;
      const float4 q = *reinterpret_cast<const float4*>(grow + 4 * u);
      gp[2 * u] = make_float2(q.x, q.y);
      gp[2 * u + 1] = make_float2(q.z, q.w);
    }
    // (f, f) pair of this column, built one column ahead
    const float2 ff = ffn;
    if (c + 1 < FC) ffn = make_float2(f[c + 1], f[c + 1]);
    if (cc % 2 == 0) {
      const int m = c / 2;  // gp[m + i] = (g(c + 2i), g(c + 2i + 1))
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (cc < REM)
          PE[i] = (cc == 0) ? fmul2(ff, gp[m + i]) : ffma2(ff, gp[m + i], PE[i]);
        else if (cc == E_A0)
          AE[i] = (REM > 0) ? ffma2(ff, gp[m + i], PE[i]) : fmul2(ff, gp[m + i]);
        else
          AE[i] = ffma2(ff, gp[m + i], AE[i]);
      }
    } else {
      const int m = (c + 1) / 2;  // gp[m + i] = (g(c + 1 + 2i), g(c + 2 + 2i))
      const float g0 = gp[m - 1].y, g7 = gp[m + 3].x;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        if (cc < REM)
          PO[i] = (cc == 1) ? fmul2(ff, gp[m + i]) : ffma2(ff, gp[m + i], PO[i]);
        else if (cc == O_A0)
          AO[i] = (REM > 1) ? ffma2(ff, gp[m + i], PO[i]) : fmul2(ff, gp[m + i]);
        else
          AO[i] = ffma2(ff, gp[m + i], AO[i]);
      }
      if (cc < REM) {
        PO0 = (cc == 1) ? f[c] * g0 : fmaf(f[c], g0, PO0);
        PO7 = (cc == 1) ? f[c] * g7 : fmaf(f[c], g7, PO7);
      } else if (cc == O_A0) {
        AO0 = (REM > 1) ? fmaf(f[c], g0, PO0) : f[c] * g0;
        AO7 = (REM > 1) ? fmaf(f[c], g7, PO7) : f[c] * g7;
      } else {
        AO0 = fmaf(f[c], g0, AO0);
        AO7 = fmaf(f[c], g7, AO7);
      }
    }
    if (cc == ST - 1 || c == FC - 1) {
      // P of this block (first REM columns) as t pairs
      float2 P[4];
      if (REM > 1) {
        P[0] = make_float2(PE[0].x + PO0, PE[0].y + PO[0].x);
        P[1] = make_float2(PE[1].x + PO[0].y, PE[1].y + PO[1].x);
        P[2] = make_float2(PE[2].x + PO[1].y, PE[2].y + PO[2].x);
        P[3] = make_float2(PE[3].x + PO[2].y, PE[3].y + PO7);
      } else if (REM == 1) {
#pragma unroll
        for (int i = 0; i < 4; ++i) P[i] = PE[i];
      }
      if (cc == ST - 1) {  // a whole block: its sum (P alone where no column of a parity follows it)
        float2 e[4], o[3];
#pragma unroll
        for (int i = 0; i < 4; ++i) e[i] = (E_A0 < ST) ? AE[i] : PE[i];
#pragma unroll
        for (int i = 0; i < 3; ++i) o[i] = (O_A0 < ST) ? AO[i] : PO[i];
        const float o0 = (O_A0 < ST) ? AO0 : PO0, o7 = (O_A0 < ST) ? AO7 : PO7;
        B[kc][0] = make_float2(e[0].x + o0, e[0].y + o[0].x);
        B[kc][1] = make_float2(e[1].x + o[0].y, e[1].y + o[1].x);
        B[kc][2] = make_float2(e[2].x + o[1].y, e[2].y + o[2].x);
        B[kc][3] = make_float2(e[3].x + o[2].y, e[3].y + o7);
        if (kc >= 1) {
#pragma unroll
          for (int i = 0; i < 4; ++i) S2[kc - 1][i] = fadd2(B[kc - 1][i], B[kc][i]);
        }
      }
      // window j ends in this block: Q whole blocks j..j+Q-1 (+ the first REM columns of block kc)
      const int j = REM > 0 ? kc - Q : kc - Q + 1;
      if (j >= 0 && j < kTJ) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          float2 s = (Q >= 2) ? S2[j][i] : B[j][i];
#pragma unroll
          for (int b = 2; b < Q; b += 2) s = fadd2(s, (b + 1 < Q) ? S2[j + b][i] : B[j + b][i]);
          if (REM > 0) s = fadd2(s, P[i]);
          rbx[(j * DBC + 2 * i) * FRP] = s.x;
          rbx[(j * DBC + 2 * i + 1) * FRP] = s.y;
        }
      }
    }
  }
}

// Pass 2 with packed pairs of rows (even steps; R0 even): window sums as column_sums.
template <int ST, int W1, int NS, int R0>
__host__ __device__ __forceinline__ void column_sums_x2(const float* __restrict__ rb, float (&N)[NS]) {
  static_assert(ST % 2 == 0 && R0 % 2 == 0, "row pairs must align with blocks");
  constexpr int Q = W1 / ST, REM = W1 % ST;
  constexpr int NBV = NS - 1 + Q + (REM > 0 ? 1 : 0);
  constexpr int ROWS = (NS - 1) * ST + W1;
  constexpr int NP = (ROWS + 1) / 2;
  float2 v[NP + 2];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    const int r = R0 + 2 * p;  // even
    if (r % 4 == 0 && 2 * p + 3 < ROWS) {
      const float4 q = *reinterpret_cast<const float4*>(rb + r);
      v[p] = make_float2(q.x, q.y);
      v[p + 1] = make_float2(q.z, q.w);
    } else if (r % 4 == 2 && p >= 1 && 2 * (p - 1) + 3 < ROWS) {
      // loaded with the previous 128-bit load
    } else if (2 * p + 1 < ROWS) {
      v[p] = *reinterpret_cast<const float2*>(rb + r);
    } else {
      v[p] = make_float2(rb[r], 0.f);
    }
  }
  float Bs[NBV], Ps[NBV];
#pragma unroll
  for (int kb = 0; kb < NBV; ++kb) {
    const int r0 = kb * ST;  // even
    float pv = 0.f;          // first REM rows
#pragma unroll
    for (int r = 0; r < REM; ++r) {
      const float x = ((r0 + r) % 2) ? v[(r0 + r) / 2].y : v[(r0 + r) / 2].x;
      pv = (r == 0) ? x : pv + x;
    }
    Ps[kb] = pv;
    if (r0 + ST <= ROWS) {  // whole block: pair tree over ST / 2 row pairs
      float2 t[ST / 2];
#pragma unroll
      for (int i = 0; i < ST / 2; ++i) t[i] = v[r0 / 2 + i];
#pragma unroll
      for (int h = 1; h < ST / 2; h *= 2)
#pragma unroll
        for (int i = 0; i + h < ST / 2; i += 2 * h) t[i] = fadd2(t[i], t[i + h]);
      Bs[kb] = t[0].x + t[0].y;
    } else {
      Bs[kb] = 0.f;
    }
  }
#pragma unroll
  for (int e = 0; e < NS; ++e) {
    float s = Bs[e];
#pragma unroll
    for (int b = 1; b < Q; ++b) s += Bs[e + b];
    if (REM > 0) s += Ps[e + Q];
    N[e] = s;
  }
}

template <int ST, int W1, int TI, int DBC>
__global__ void __launch_bounds__(TileShape<ST, W1, TI, DBC>::NT, 1)
    ncc_tile_kernel(SearchArgs a, const float2* __restrict__ map, const double* __restrict__ Vmap,
                    const SubsetPrm* __restrict__ prm, const float2* __restrict__ ringv,
                    const float* __restrict__ cxv, const float* __restrict__ tcf, int* __restrict__ best) {
  using S = TileShape<ST, W1, TI, DBC>;
  constexpr int FR = S::FR, FC = S::FC, FCP = S::FCP, GCP = S::GCP, FRP = S::FRP, H0 = S::H0, NSUB = S::NSUB;
  constexpr int NT = S::NT;
  constexpr int GC = FC + DBC - 1;  // g columns a chunk needs
  extern __shared__ __align__(16) float smf[];
  float* Ft = smf;                  // FR x FCP: f - cf, row-major
  float* Gt = Ft + FR * FCP;        // kRing x GCP: g, ring over rows, row-major
  float* RB = Gt + kRing * GCP;     // (kTJ * DBC) x FRP: one row per (window column, shift column)
  __shared__ float p_kf[NSUB], p_invden[NSUB], p_sqtolv[NSUB];
  __shared__ double p_tolv[NSUB];
  __shared__ int p_ok[NSUB];
  __shared__ int r_L[TI], r_na[TI], r_d0[TI], r_d1[TI], c_U[kTJ], c_nb[kTJ], c_d0[kTJ], c_d1[kTJ];
  __shared__ int r_aoff[TI];   // crop row of shift row k: aa = k + r_aoff
  __shared__ int p_na[NSUB];   // crop rows of a valid subset, 0 for an invalid one
  __shared__ float4 p_c[NSUB]; // (kf, 1 / denT, sqrt(tolv), 0): the fast epilogue's operands, one load
  __shared__ int2 p_g[NSUB];   // (crop row offset r_aoff, crop rows p_na): the prefetch's operands, one load
  __shared__ float s_cf;

  const int tid = threadIdx.x;
  const int w = W1 - 1;
  const int ntx = (a.nx + TI - 1) / TI;
  const int i0 = (int)(blockIdx.x % ntx) * TI, j0 = (int)(blockIdx.x / ntx) * kTJ;
  const int X0 = a.gx0 - 1 + i0 * ST, Y0 = a.gy0 - 1 + j0 * ST;  // 0-based tile origin
  const int DA0 = -a.s0 - 1, NDA = a.s0 + a.s1 + 3;               // shifts, both axes
  const int NW = a.N - W1 + 1;
  const double nwin = (double)W1 * W1;
  const size_t ld = (size_t)a.M + 1;

  // ---- per-subset constants and geometry ----
  if (tid == 0) s_cf = tcf[blockIdx.x];
  if (tid >= 32 && tid < 32 + TI) {
    const int il = tid - 32, i = i0 + il;
    const AxisGeom r = axis_geom(a.gx0 + i * a.step, w, a.s0, a.s1, a.M, a.gx1);
    r_L[il] = r.lo;
    r_na[il] = i < a.nx ? r.lo + r.hi + 3 : 0;
    r_aoff[il] = DA0 + r.lo + 1;
    r_d0[il] = r.d0;
    r_d1[il] = r.d1;
  } else if (tid >= 64 && tid < 64 + kTJ) {
    const int jl = tid - 64, j = j0 + jl;
    const AxisGeom c = axis_geom(a.gy0 + j * a.step, w, a.s0, a.s1, a.N, a.gy1);
    c_U[jl] = c.lo;
    c_nb[jl] = j < a.ny ? c.lo + c.hi + 3 : 0;
    c_d0[jl] = c.d0;
    c_d1[jl] = c.d1;
  }
  __syncthreads();
  const float cf = s_cf;
  for (int q = tid; q < NSUB; q += NT) {
    const int i = i0 + q % TI, j = j0 + q / TI;
    int ok = 0;
    if (i < a.nx && j < a.ny) {
      const SubsetPrm P = prm[i + (long long)j * a.nx];
      ok = P.valid;
      p_tolv[q] = P.tolv;
      p_kf[q] = (float)(nwin * (P.fm - (double)cf));
      p_invden[q] = ok ? (float)(1.0 / P.denT) : 0.f;
      p_sqtolv[q] = (float)sqrt(P.tolv);
    }
    p_ok[q] = ok;
  }
  __syncthreads();
  for (int q = tid; q < NSUB; q += NT) {
    p_na[q] = p_ok[q] ? r_na[q % TI] : 0;
    p_c[q] = make_float4(p_kf[q], p_invden[q], p_sqtolv[q], 0.f);
    p_g[q] = make_int2(r_aoff[q % TI], p_ok[q] ? r_na[q % TI] : 0);
  }
  // ---- f tile, centred ----
  // consecutive threads take consecutive tile rows x: contiguous in the column-major image
  for (int idx = tid; idx < FR * FCP; idx += NT) {
    const int x = idx % FR, c = idx / FR;
    float v = 0.f;
    if (c < FC && X0 + x < a.M && Y0 + c < a.N) v = __ldg(a.f + (size_t)(X0 + x) + (size_t)(Y0 + c) * a.M) - cf;
    Ft[x * FCP + c] = v;
  }

  // pass-2 roles and running first maxima
  const int half = tid / (kTJ * DBC), jl = (tid / DBC) % kTJ, dl = tid % DBC;
  const int il0 = half ? H0 : 0, ns = half ? TI - H0 : H0;
  const float* rbrow = RB + (jl * DBC + dl) * FRP;
  float bv[H0];
  int bl[H0];
#pragma unroll
  for (int e = 0; e < H0; ++e) {
    bv[e] = -INFINITY;
    bl[e] = 0x7fffffff;
  }

  for (int dbc = 0; dbc < NDA; dbc += DBC) {
    __syncthreads();
    // g buffer for this chunk: ring rows 0..FR-1 = tile rows DA0 + rel, columns from db = DA0 + dbc
    const int gy0 = Y0 + DA0 + dbc;
    for (int idx = tid; idx < FR * GCP; idx += NT) {
      const int rel = idx % FR, col = idx / FR;  // consecutive threads: consecutive image rows
      const int x = X0 + DA0 + rel, y = gy0 + col;
      float v = 0.f;
      if (col < GC && x >= 0 && x < a.M && y >= 0 && y < a.N) v = __ldg(a.g + (size_t)x + (size_t)y * a.M);
      Gt[rel * GCP + col] = v;
    }
    for (int idx = FR * GCP + tid; idx < kRing * GCP; idx += NT) Gt[idx] = 0.f;
    __syncthreads();
    // this thread's shift column for the chunk: crop column bb of its window column jl
    const int dbr = dbc + dl, db = DA0 + dbr;
    const int bb = db + c_U[jl] + 1, nbv = c_nb[jl];
    const bool bok = dbr < NDA && bb >= 0 && bb < nbv;
    const bool rbg = bb == 0 || bb == nbv - 1;
    const long long mcol = (long long)(X0 + DA0) * NW + (Y0 + jl * ST + db);  // map index of (il = 0, k = 0)
    // crop index of shift row k of subset row e is k + lbase[e] (lin = aa + bb na)
    int lbase[H0];
#pragma unroll
    for (int e = 0; e < H0; ++e) {
      const int2 gq = p_g[(il0 + e < TI ? il0 + e : TI - 1) + jl * TI];
      lbase[e] = gq.x + bb * gq.y;
    }
    for (int k = 0; k < NDA; ++k) {
      // ---- epilogue operands of this shift, fetched before pass 1 hides their latency ----
      int st[H0];
      float2 pf[H0];
      float pcx[H0];
#pragma unroll
      for (int e = 0; e < H0; ++e) {
        st[e] = 0;
        pf[e] = make_float2(0.f, 0.f);
        pcx[e] = 0.f;
        if (!bok || e >= ns) continue;
        const int il = il0 + e;
        const int2 gq = p_g[il + jl * TI];
        const int na = gq.y, aa = k + gq.x;
        if ((unsigned)aa >= (unsigned)na) continue;
        const bool ra = aa == 0 || aa == na - 1;
        if (!ra && !rbg) {
          pf[e] = __ldg(map + (mcol + (long long)(il * ST + k) * NW));
          st[e] = 1;
        } else {
          const long long t = (long long)(i0 + il) + (long long)(j0 + jl) * a.nx;
          const float2* rv = ringv + t * 4 * NDA;
          pf[e] = ra ? __ldg(rv + (aa == 0 ? 0 : NDA) + bb) : __ldg(rv + (bb == 0 ? 2 : 3) * NDA + aa);
          if (rbg) pcx[e] = __ldg(cxv + t * 2 * NDA + (bb == 0 ? 0 : NDA) + k);
          st[e] = 2 | (ra ? 4 : 0) | (rbg ? 8 : 0) | (aa == 0 ? 16 : 0) | (bb == 0 ? 32 : 0);
        }
      }
      // the ring row of shift row k + 1 goes to the one slot pass 1 does not read
      float nrow = 0.f;
      if (k + 1 < NDA && tid < GC) {
        const int x = X0 + DA0 + k + FR, y = gy0 + tid;
        if (x >= 0 && x < a.M && y >= 0 && y < a.N) nrow = __ldg(a.g + (size_t)x + (size_t)y * a.M);
      }
      // ---- pass 1 ----
      {
        const int grp = tid >> 7, x = tid & 127;
        if (x < FR) {
          if constexpr (ST % 2 == 0)
            row_band_sums_x2<ST, W1, FC, FRP, DBC>(Ft + x * FCP, Gt + ((x + k) & (kRing - 1)) * GCP + grp * 8,
                                              RB + (grp * 8) * FRP + x);
          else
            row_band_sums<ST, W1, FC, FRP, DBC>(Ft + x * FCP, Gt + ((x + k) & (kRing - 1)) * GCP + grp * 8,
                                           RB + (grp * 8) * FRP + x);
        }
      }
      if (k + 1 < NDA && tid < GCP) Gt[((k + FR) & (kRing - 1)) * GCP + tid] = nrow;
      __syncthreads();
      // ---- pass 2 ----
      if (dbr < NDA) {
        float N[H0];
        if (half == 0) {
          if constexpr (ST % 2 == 0)
            column_sums_x2<ST, W1, H0, 0>(rbrow, N);
          else
            column_sums<ST, W1, H0, 0>(rbrow, N);
        } else {
          float N1[TI - H0 > 0 ? TI - H0 : 1];
          if constexpr (ST % 2 == 0)
            column_sums_x2<ST, W1, (TI - H0 > 0 ? TI - H0 : 1), H0 * ST>(rbrow, N1);
          else
            column_sums<ST, W1, (TI - H0 > 0 ? TI - H0 : 1), H0 * ST>(rbrow, N1);
#pragma unroll
          for (int e = 0; e < TI - H0; ++e) N[e] = N1[e];
        }
        // fast path, branch-free: interior shifts whose variance sum is well above the
        // zero threshold; the others (ring shifts, near-threshold variance) are flagged
        unsigned slow = 0;
#pragma unroll
        for (int e = 0; e < H0; ++e) {
          if (e >= ns) break;  // the second half has TI - H0 subset rows
          const int q = il0 + e + jl * TI;
          const float2 v = pf[e];
          const float4 c = p_c[q];
          const bool fast = st[e] == 1 && v.y * c.z < 0.5f;
          if (st[e] != 0 && !fast) slow |= 1u << e;
          float cval = (N[e] - c.x * v.x) * v.y * c.y;
          if (fabsf(cval) - 1.f > 1.4901161193847656e-08f) cval = 0.f;
          // a thread meets each subset's crop indices lin = aa + bb na in increasing order
          // (aa grows with k, bb with the chunk), so the first maximum is the first strict one
          if (fast && cval > bv[e]) {
            bv[e] = cval;
            bl[e] = k + lbase[e];
          }
        }
        if (slow) {
#pragma unroll
          for (int e = 0; e < H0; ++e) {
            if (!((slow >> e) & 1u)) continue;
            const int sf = st[e];
            const int il = il0 + e, q = il + jl * TI;
            float C = N[e];
            if (sf & 2) {  // partial window: drop the template row / column whose partner is outside D
              const int rx = (sf & 16) ? il * ST : il * ST + W1 - 1;
              const int cxc = (sf & 32) ? jl * ST : jl * ST + W1 - 1;
              if (sf & 4) C -= rbrow[rx];
              if (sf & 8) {
                C -= pcx[e];
                if (sf & 4) C += Ft[rx * FCP + cxc] * Gt[((rx + k) & (kRing - 1)) * GCP + cxc + dl];
              }
            }
            const float2 v = pf[e];
            const float num = C - p_kf[q] * v.x;
            float cval;
            if (v.y * p_sqtolv[q] < 0.5f) {
              cval = num * v.y * p_invden[q];
            } else {  // near the zero threshold: decide it on the FP64 variance sum
              const int aa = k + r_aoff[il];
              double var;
              if (sf & 2) {
                SubsetGeom sg;
                sg.dr0 = r_d0[il];
                sg.dr1 = r_d1[il];
                sg.dc0 = c_d0[jl];
                sg.dc1 = c_d1[jl];
                double S1, S2;
                window_sums(sg, w, aa, bb, a.I1, a.I2, ld, &S1, &S2);
                var = fmax(S2 - S1 * S1 / nwin, 0.0);
              } else {
                var = fmax(Vmap[mcol + (long long)(il * ST + k) * NW], 0.0);
              }
              cval = var > p_tolv[q] ? num * (float)(1.0 / sqrt(var)) * p_invden[q] : 0.f;
            }
            if (fabsf(cval) - 1.f > 1.4901161193847656e-08f) cval = 0.f;
            if (cval > bv[e]) {
              bv[e] = cval;
              bl[e] = (k + r_aoff[il]) + bb * p_na[q];
            }
          }
        }
      }
      __syncthreads();
    }
  }
  // ---- first maximum per subset over the 16 shift-column lanes ----
  float* rv = RB;
  int* ri = reinterpret_cast<int*>(RB + NSUB * DBC);
#pragma unroll
  for (int e = 0; e < H0; ++e) {
    if (e >= ns) break;
    const int q = (il0 + e) + jl * TI;
    rv[q * DBC + dl] = bv[e];
    ri[q * DBC + dl] = bl[e];
  }
  __syncthreads();
  for (int q = tid; q < NSUB; q += NT) {
    if (!p_ok[q]) continue;
    float b = rv[q * DBC];
    int bi = ri[q * DBC];
    for (int l = 1; l < DBC; ++l) {
      const float v = rv[q * DBC + l];
      const int li = ri[q * DBC + l];
      if (v > b || (v == b && li < bi)) {
        b = v;
        bi = li;
      }
    }
    const int i = i0 + q % TI, j = j0 + q / TI;
    best[i + (long long)j * a.nx] = bi == 0x7fffffff ? 0 : bi;
  }
}

// FP64 refit + findpeak at the argmax of every valid subset (one warp per subset).
// Three CTAs per SM (80 registers) and, for subset_prep_kernel, four (64): both warp-per-subset
// FP64 kernels are latency-bound, and the extra warps measured 0.2 ms off the stereo step.
__global__ void __launch_bounds__(256, 3) subset_refit_kernel(SearchArgs a, const SubsetPrm* __restrict__ prm,
                                                           const int* __restrict__ best) {
  const long long t = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  if (t >= (long long)a.nx * a.ny) return;
  const SubsetPrm P = prm[t];
  if (!P.valid) return;
  const SubsetGeom s = subset_geom(a, t);
  const int bi = best[t];
  refit_peak_warp(a, s, subset_out(a, t), bi % s.na, bi / s.na, P.fm, P.denT, P.tolz);
}

// Centring constant of every tile: the mean of its valid template means (one warp per
// tile; the lanes' partial sums are added in lane order by lane 0, a fixed order shared by
// every launch).
__global__ void tile_centre_kernel(int nx, int ny, int TI, const SubsetPrm* __restrict__ prm, float* __restrict__ cf) {
  const int ntx = (nx + TI - 1) / TI, nty = (ny + kTJ - 1) / kTJ;
  const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (b >= ntx * nty) return;
  const int i0 = (b % ntx) * TI, j0 = (b / ntx) * kTJ;
  double s = 0.0;
  int c = 0;
  for (int q = lane; q < TI * kTJ; q += 32) {
    const int i = i0 + q % TI, j = j0 + q / TI;
    if (i < nx && j < ny) {
      const SubsetPrm& P = prm[i + (long long)j * nx];
      if (P.valid) {
        s += P.fm;
        ++c;
      }
    }
  }
  double ts = 0.0;
  int tc = 0;
  for (int l = 0; l < 32; ++l) {
    ts += __shfl_sync(0xffffffffu, s, l);
    tc += __shfl_sync(0xffffffffu, c, l);
  }
  if (lane == 0) cf[b] = tc ? (float)(ts / tc) : 0.f;
}

namespace {

struct TileEntry {
  int TI;
  int (*launch)(const SearchArgs&, const TileScratch&, cudaStream_t);
  bool (*fits)();
};

template <int ST, int W1, int DBC>
int launch_tile(const SearchArgs& a, const TileScratch& sc, cudaStream_t st) {
  constexpr int TI = TileFor<ST, W1, DBC>::TI;
  using S = TileShape<ST, W1, TI, DBC>;
  auto kern = ncc_tile_kernel<ST, W1, TI, DBC>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem_bytes) != cudaSuccess)
    return -1;
  const long long tiles = (long long)((a.nx + TI - 1) / TI) * ((a.ny + kTJ - 1) / kTJ);
  kern<<<(unsigned)tiles, S::NT, S::smem_bytes, st>>>(a, sc.map, sc.V, sc.prm, sc.ringv, sc.cx, sc.cf, sc.best);
  return 0;
}

// Whether the tile kernel's shared memory (static + dynamic) fits this device.
template <int ST, int W1, int DBC>
bool tile_fits() {
  constexpr int TI = TileFor<ST, W1, DBC>::TI;
  cudaFuncAttributes fa;
  int dev = 0, optin = 0;
  return cudaFuncGetAttributes(&fa, ncc_tile_kernel<ST, W1, TI, DBC>) == cudaSuccess &&
         cudaGetDevice(&dev) == cudaSuccess &&
         cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess &&
         fa.sharedSizeBytes + TileShape<ST, W1, TI, DBC>::smem_bytes <= (size_t)optin;
}

template <int ST, int W1, int DBC = 16>
TileEntry entry() {
  return TileEntry{TileFor<ST, W1, DBC>::TI, launch_tile<ST, W1, DBC>, tile_fits<ST, W1, DBC>};
}

// The step / window pairs with a tile kernel (others use the per-subset kernel), each with
// 16 or 24 shift columns per pass (chunk); chunk 0 takes the shape's measured default (24 for
// the stereo shape (10, 41), 16 for the others).
bool tile_entry(int step, int W1, int chunk, TileEntry* e) {
  if (chunk != 0 && chunk != 16 && chunk != 24) return false;
  const bool c24 = chunk == 24 || (chunk == 0 && step == 10 && W1 == 41);
  switch (step * 1000 + W1) {
    case 10 * 1000 + 41: *e = c24 ? entry<10, 41, 24>() : entry<10, 41, 16>(); return true;
    case 16 * 1000 + 31: *e = c24 ? entry<16, 31, 24>() : entry<16, 31>(); return true;
    case 16 * 1000 + 33: *e = c24 ? entry<16, 33, 24>() : entry<16, 33>(); return true;
    case 12 * 1000 + 21: *e = c24 ? entry<12, 21, 24>() : entry<12, 21>(); return true;
    case 9 * 1000 + 17: *e = c24 ? entry<9, 17, 24>() : entry<9, 17>(); return true;
    case 8 * 1000 + 33: *e = c24 ? entry<8, 33, 24>() : entry<8, 33>(); return true;
    default: return false;
  }
}

}  // namespace

bool search_tile_available(int step, int winsize, int chunk) {
  TileEntry e;
  return tile_entry(step, winsize + 1, chunk, &e) && e.fits();
}

size_t search_tile_bytes(int M, int N, int winsize, int step, int nx, int ny, int s0, int s1, int chunk) {
  const int W1 = winsize + 1;
  TileEntry e;
  if (!tile_entry(step, W1, chunk, &e) || M < W1 || N < W1 || nx <= 0 || ny <= 0) return 0;
  return scratch_layout(M, N, W1, nx, ny, s0 + s1 + 3, nullptr, nullptr);
}

int launch_search_tile(const SearchArgs& a, cudaStream_t st) {
  const int W1 = a.winsize + 1;
  TileEntry e;
  if (a.impl == 2 || !tile_entry(a.step, W1, a.chunk, &e) || !a.tile_scratch || a.M < W1 || a.N < W1 || !e.fits())
    return -1;
  const int nda = a.s0 + a.s1 + 3;
  TileScratch sc;
  scratch_layout(a.M, a.N, W1, a.nx, a.ny, nda, (char*)a.tile_scratch, &sc);
  const long long n = (long long)a.nx * a.ny;
  const long long npos = (long long)(a.M - W1 + 1) * (a.N - W1 + 1);
  window_map_kernel<<<(unsigned)((npos + 255) / 256), 256, 0, st>>>(a.I1, a.I2, a.M, a.N, W1, sc.map, sc.V);
  const long long nh = (long long)(a.M - W1 + 1) * a.ny;
  window_rowmax_kernel<<<(unsigned)((nh + 255) / 256), 256, 0, st>>>(a, sc.V, sc.H);
  const long long nrr = (long long)a.nx * 2 * (a.N + 1);
  ring_rows_kernel<<<(unsigned)((nrr + 255) / 256), 256, 0, st>>>(a, sc.rr);
  subset_prep_kernel<<<(unsigned)((n * 32 + 255) / 256), 256, 0, st>>>(a, sc.H, sc.rr, sc.prm, sc.ringv);
  const int ntiles = ((a.nx + e.TI - 1) / e.TI) * ((a.ny + kTJ - 1) / kTJ);
  tile_centre_kernel<<<(ntiles * 32 + 255) / 256, 256, 0, st>>>(a.nx, a.ny, e.TI, sc.prm, sc.cf);
  ring_column_kernel<<<(unsigned)((n * 32 + 255) / 256), 256, 0, st>>>(a, sc.prm, e.TI, sc.cf, sc.cx);
  if (a.ev_start) cudaEventRecord(a.ev_start, st);
  if (e.launch(a, sc, st) != 0) return -1;
  if (a.ev_stop) cudaEventRecord(a.ev_stop, st);
  subset_refit_kernel<<<(unsigned)((n * 32 + 255) / 256), 256, 0, st>>>(a, sc.prm, sc.best);
  return 8;
}

}  // namespace aldic
