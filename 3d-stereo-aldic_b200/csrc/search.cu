// Whole-field integer search (funIntegerSearchWholeField, func/funIntegerSearch.m:100-203):
// per grid subset, zero-normalised cross-correlation of the (w+1)^2 template of f with the
// border-clamped search window of g (normxcorr2 semantics, Lewis 1995), cropped to the
// (L+R+3) x (U+D+3) shifts the reference keeps, then findpeak (func/findpeak.m).
//
// Direct correlation, one CTA per subset:
//   * window sums sum(D), sum(D^2) of every shift come from FP64 integral images of g
//     (computed once per call), so the partial-overlap ring of the crop (zero padding of
//     the cut-out window) is exact;
//   * the numerator sum((T - mean T) * D): the whole zero-padded window of the subset (or a
//     strip of its shift columns) sits in shared memory; each thread owns
//     8 consecutive shift rows x 2 shift columns in registers, slides a 16-value register
//     window (four 128-bit shared loads) down the template column, accumulates each template column in FP32 and
//     adds it to FP64 accumulators (41-term FP32 partial sums);
//   * argmax is the first maximum in column-major order (MATLAB max); the 3 x 3
//     neighbourhood of the peak is recomputed in FP64 for the sub-pixel fit.
#include "search_common.cuh"

namespace aldic {


// Integral images of g and g^2 in FP64: II(r, c) = sum over rows < r and columns < c;
// (M+1) x (N+1) column-major, row 0 and column 0 zero.
//
// Pass 1 (one warp per image column, coalesced): column prefix sums by warp scans.
__global__ void integral_cols_kernel(const float* __restrict__ g, int M, int N, double* __restrict__ I1,
                                     double* __restrict__ I2) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const size_t ld = (size_t)M + 1;
  if (warp > N) return;
  double* c1 = I1 + (size_t)warp * ld;
  double* c2 = I2 + (size_t)warp * ld;
  if (warp == 0) {  // column 0 is zero
    for (int r = lane; r <= M; r += 32) {
      c1[r] = 0.0;
      c2[r] = 0.0;
    }
    return;
  }
  const float* col = g + (size_t)(warp - 1) * M;
  if (lane == 0) {
    c1[0] = 0.0;
    c2[0] = 0.0;
  }
  double carry1 = 0.0, carry2 = 0.0;
  for (int r0 = 0; r0 < M; r0 += 32) {
    const int r = r0 + lane;
    const double v = r < M ? (double)col[r] : 0.0;
    double s1 = v, s2 = v * v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double t1 = __shfl_up_sync(0xffffffffu, s1, o), t2 = __shfl_up_sync(0xffffffffu, s2, o);
      if (lane >= o) {
        s1 += t1;
        s2 += t2;
      }
    }
    s1 += carry1;
    s2 += carry2;
    if (r < M) {
      c1[r + 1] = s1;
      c2[r + 1] = s2;
    }
    carry1 = __shfl_sync(0xffffffffu, s1, 31);
    carry2 = __shfl_sync(0xffffffffu, s2, 31);
  }
}

constexpr int kRowChunk = 64;  // columns per thread in the row pass

// Pass 2a: within each chunk of kRowChunk columns, prefix along the row (one thread per
// (row, chunk); consecutive threads take consecutive rows: coalesced).  Chunk totals go
// to tot (nchunk x (M+1)).
__global__ void integral_rows_local_kernel(int M, int N, double* __restrict__ I1, double* __restrict__ I2,
                                           double* __restrict__ tot) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int rows = M + 1;
  const int nchunk = (N + kRowChunk - 1) / kRowChunk;
  if (t >= (long long)rows * nchunk) return;
  const int r = (int)(t % rows), ch = (int)(t / rows);
  const size_t ld = (size_t)M + 1;
  const int c0 = 1 + ch * kRowChunk, c1 = min(N, c0 + kRowChunk - 1);
  double s1 = 0, s2 = 0;
  for (int c = c0; c <= c1; ++c) {
    s1 += I1[r + c * ld];
    s2 += I2[r + c * ld];
    I1[r + c * ld] = s1;
    I2[r + c * ld] = s2;
  }
  tot[2 * ((size_t)ch * rows + r)] = s1;
  tot[2 * ((size_t)ch * rows + r) + 1] = s2;
}

// Pass 2b: add the totals of the preceding chunks of the row.
__global__ void integral_rows_fix_kernel(int M, int N, double* __restrict__ I1, double* __restrict__ I2,
                                         const double* __restrict__ tot) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int rows = M + 1;
  const int nchunk = (N + kRowChunk - 1) / kRowChunk;
  if (t >= (long long)rows * nchunk) return;
  const int r = (int)(t % rows), ch = (int)(t / rows);
  if (ch == 0) return;
  double o1 = 0, o2 = 0;
  for (int k = 0; k < ch; ++k) {
    o1 += tot[2 * ((size_t)k * rows + r)];
    o2 += tot[2 * ((size_t)k * rows + r) + 1];
  }
  const size_t ld = (size_t)M + 1;
  const int c0 = 1 + ch * kRowChunk, c1 = min(N, c0 + kRowChunk - 1);
  for (int c = c0; c <= c1; ++c) {
    I1[r + c * ld] += o1;
    I2[r + c * ld] += o2;
  }
}

// Shared-memory layout of one subset: the centred template (TR x W1, rows >= W1 zero)
// and the padded search window Dpad restricted to the current strip of shift columns
// (DR x DC, zero outside the cut-out window D).
struct SearchLayout {
  int W1, TR, DR, DC, strip_b;  // strip_b = shift columns covered per strip
};

__host__ __device__ inline SearchLayout search_layout(int w, int na_max, int strip_b) {
  SearchLayout L;
  L.W1 = w + 1;
  L.TR = round_up8(L.W1);
  // rows a0 .. a0 + TR + 7 of every 8-row block, leading dimension = 4 (mod 32): each
  // quarter-warp phase of a 128-bit column load (4 row blocks x 2 columns) covers all 32
  // banks exactly once
  const int need = round_up8(na_max) + L.TR;
  L.DR = need + ((4 - need) % 32 + 32) % 32;
  L.strip_b = strip_b;
  L.DC = round_up16(strip_b) + w;               // columns b + j for b < round_up16(strip_b)
  return L;
}

// One CTA per subset (grid-stride).  Each warp task covers 32 shift rows (4 lanes x 8
// consecutive rows) x 16 shift columns (8 lanes x the column pair b, b + 8); the window
// column of a thread is read as four 128-bit loads per 8 template rows.
template <int TRC>
__global__ void __launch_bounds__(512, 1) ncc_search_kernel(SearchArgs a, int strip_b, int na_max) {
  const double* __restrict__ I1 = a.I1;
  const double* __restrict__ I2 = a.I2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[16 * 10];
  __shared__ double sums[10];
  __shared__ float sbest[16];
  __shared__ int sidx[16];
  __shared__ double s_tmean, s_denT, s_tolz;
  __shared__ int s_peak;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const int w = a.winsize;
  const SearchLayout Ly = search_layout(w, na_max, strip_b);
  const int W1 = Ly.W1, DR = Ly.DR, DC = Ly.DC;
  constexpr int TR = TRC;  // == Ly.TR (checked on the host)
  const size_t ld = (size_t)a.M + 1;
  float* Tp = reinterpret_cast<float*>(smem_raw);
  float* Dt = Tp + TR * W1;
  const long long n = a.list ? a.nlist : (long long)a.nx * a.ny;
  for (long long q = blockIdx.x; q < n; q += gridDim.x) {
    const long long t = a.list ? (long long)a.list[q] : q;
    const SubsetGeom s = subset_geom(a, t);
    const long long o = a.list ? q : subset_out(a, t);
    if (tid == 0) {
      a.x[o] = (s.ii + s.ii + w) / 2.0;
      a.y[o] = (s.jj + s.jj + w) / 2.0;
    }
    if (!s.ok || s.na > na_max) {
      if (tid == 0) a.u[o] = a.v[o] = a.phi[o] = ALDIC_NAN;
      continue;
    }
    // ---- template: mean, centred FP32 copy, FP64 norm ----
    {
      double v[1] = {0};
      for (int p = tid; p < W1 * W1; p += blockDim.x) {
        const int i = p % W1, j = p / W1;
        v[0] += (double)a.f[(size_t)(s.ii - 1 + i) + (size_t)(s.jj - 1 + j) * a.M];
      }
      block_sum_dyn<1>(v, red, sums, nwarps);
      if (tid == 0) s_tmean = sums[0] / (double)(W1 * W1);
      __syncthreads();
      const double tm = s_tmean;
      double ss[1] = {0};
      for (int p = tid; p < TR * W1; p += blockDim.x) {
        const int i = p % TR, j = p / TR;
        float tv = 0.f;
        if (i < W1) {
          const double d = (double)a.f[(size_t)(s.ii - 1 + i) + (size_t)(s.jj - 1 + j) * a.M] - tm;
          ss[0] += d * d;
          tv = (float)d;
        }
        Tp[i + j * TR] = tv;
      }
      block_sum_dyn<1>(ss, red, sums, nwarps);
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
    // ---- largest denominator over the crop (normxcorr2 zero threshold) ----
    {
      double dmax = 0;  // largest window variance sum; sqrt is monotone
      for (int k = tid; k < s.na * s.nb; k += blockDim.x) {
        double S1, S2;
        window_sums(s, w, k % s.na, k / s.na, I1, I2, ld, &S1, &S2);
        dmax = fmax(dmax, S2 - S1 * S1 / nwin);
      }
      for (int off = 16; off > 0; off >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
      if (lane == 0) red[warp] = dmax;
      __syncthreads();
      if (tid == 0) {
        double m = 0;
        for (int i = 0; i < nwarps; ++i) m = fmax(m, red[i]);
        s_tolz = sqrt(matlab_eps_d(denT * sqrt(fmax(m, 0.0))));
      }
      __syncthreads();
    }
    const double tolz = s_tolz;
    const double tolv = (tolz / denT) * (tolz / denT);
    const float inv_denT = (float)(1.0 / denT);
    float best = -INFINITY;
    int bidx = 0x7fffffff;
    const int la = lane & 3, lb = lane >> 2;
    const int ablocks = (s.na + 31) / 32;
    for (int tb0 = 0; tb0 < s.nb; tb0 += Ly.strip_b) {
      const int nbs = min(Ly.strip_b, s.nb - tb0);
      // padded window for this strip: Dpad(p, tb0 + q) = g at image (dr0-1+p, dc0-1+tb0+q)
      for (int k = tid; k < DR * DC; k += blockDim.x) {
        const int p = k % DR, q = tb0 + k / DR;
        const int r = s.dr0 - 1 + p, c = s.dc0 - 1 + q;
        float v = 0.f;
        if (r >= s.dr0 && r <= s.dr1 && c >= s.dc0 && c <= s.dc1) v = __ldg(a.g + (size_t)r + (size_t)c * a.M);
        Dt[k] = v;
      }
      __syncthreads();
      const int bgroups = (nbs + 15) / 16;
      for (int task = warp; task < ablocks * bgroups; task += nwarps) {
        const int a0 = (task % ablocks) * 32 + la * 8;
        const int bl = (task / ablocks) * 16 + lb;  // strip-local shift column
        if (a0 >= s.na || bl >= nbs) continue;
        double acc0[8], acc1[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          acc0[k] = 0.0;
          acc1[k] = 0.0;
        }
        for (int j = 0; j < W1; ++j) {
          const float* c0 = Dt + (size_t)(bl + j) * DR + a0;
          const float* c1 = c0 + 8 * (size_t)DR;
          const float* tj = Tp + j * TR;
          float p0[8], p1[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            p0[k] = 0.f;
            p1[k] = 0.f;
          }
#pragma unroll
          for (int i0 = 0; i0 < TR; i0 += 8) {
            float w0[16], w1[16];
            const float4* v0 = reinterpret_cast<const float4*>(c0 + i0);
            const float4* v1 = reinterpret_cast<const float4*>(c1 + i0);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float4 x0 = v0[q], x1 = v1[q];
              w0[4 * q] = x0.x;
              w0[4 * q + 1] = x0.y;
              w0[4 * q + 2] = x0.z;
              w0[4 * q + 3] = x0.w;
              w1[4 * q] = x1.x;
              w1[4 * q + 1] = x1.y;
              w1[4 * q + 2] = x1.z;
              w1[4 * q + 3] = x1.w;
            }
            const float4 ta = *reinterpret_cast<const float4*>(tj + i0);
            const float4 tb = *reinterpret_cast<const float4*>(tj + i0 + 4);
            const float tv[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
#pragma unroll
            for (int s8 = 0; s8 < 8; ++s8) {
#pragma unroll
              for (int k = 0; k < 8; ++k) {
                p0[k] = fmaf(tv[s8], w0[k + s8], p0[k]);
                p1[k] = fmaf(tv[s8], w1[k + s8], p1[k]);
              }
            }
          }
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            acc0[k] += (double)p0[k];
            acc1[k] += (double)p1[k];
          }
        }
        // NCC with the zero rules, running first maximum in column-major crop order
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          const int bb = tb0 + bl + 8 * half;
          if (bl + 8 * half >= nbs) continue;
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int aa = a0 + k;
            if (aa >= s.na) continue;
            double S1, S2;
            window_sums(s, w, aa, bb, I1, I2, ld, &S1, &S2);
            // den = denT * sqrt(var); den > tolz  <=>  var > (tolz / denT)^2
            const double var = fmax(S2 - S1 * S1 / nwin, 0.0);
            float cval = 0.f;
            if (var > tolv) {
              const float vf = (float)var;
              float r = rsqrtf(vf);
              r = r * fmaf(-0.5f * vf * r, r, 1.5f);  // one Newton step: ~1 ulp
              cval = (float)(half ? acc1[k] : acc0[k]) * r * inv_denT;
            }
            if (fabsf(cval) - 1.f > 1.4901161193847656e-08f) cval = 0.f;
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
      for (int i = 1; i < nwarps; ++i)
        if (sbest[i] > b || (sbest[i] == b && sidx[i] < bi)) {
          b = sbest[i];
          bi = sidx[i];
        }
      s_peak = bi;
    }
    __syncthreads();
    refit_peak(a, s, o, s_peak % s.na, s_peak / s.na, s_tmean, denT, tolz, red, sums);
  }
}

// Largest crop size of any subset: interior subsets have na = s0 + s1 + 3.
static int crop_max(int s0, int s1) { return s0 + s1 + 3; }

// Columns of shifts per strip so that template + window fit in `budget` bytes.
static int strip_columns(int w, int na_max, int nb_max, size_t budget) {
  int sb = round_up16(nb_max);
  while (sb > 16) {
    const SearchLayout L = search_layout(w, na_max, sb);
    const size_t bytes = sizeof(float) * ((size_t)L.TR * L.W1 + (size_t)L.DR * L.DC);
    if (bytes <= budget) break;
    sb -= 16;
  }
  return sb;
}

size_t search_smem_bytes(int winsize, int s0, int s1) {
  const int na = crop_max(s0, s1);
  const int sb = strip_columns(winsize, na, na, 200 * 1024);
  const SearchLayout L = search_layout(winsize, na, sb);
  return sizeof(float) * ((size_t)L.TR * L.W1 + (size_t)L.DR * L.DC);
}

size_t search_tot_bytes(int M, int N) {
  const int nchunk = (N + kRowChunk - 1) / kRowChunk;
  return (size_t)nchunk * (M + 1) * 2 * sizeof(double);
}

int launch_search(const SearchArgs& a, cudaStream_t st) {
  const long long n = a.list ? a.nlist : (long long)a.nx * a.ny;
  if (n <= 0) return 0;
  integral_cols_kernel<<<(unsigned)(((long long)(a.N + 1) * 32 + 255) / 256), 256, 0, st>>>(a.g, a.M, a.N, a.I1,
                                                                                          a.I2);
  const long long rt = (long long)(a.M + 1) * ((a.N + kRowChunk - 1) / kRowChunk);
  integral_rows_local_kernel<<<(unsigned)((rt + 255) / 256), 256, 0, st>>>(a.M, a.N, a.I1, a.I2, a.tot);
  integral_rows_fix_kernel<<<(unsigned)((rt + 255) / 256), 256, 0, st>>>(a.M, a.N, a.I1, a.I2, a.tot);
  // shared products over tiles of subsets where a tile kernel exists for (step, w + 1) (a
  // subset list takes the direct kernel)
  const int tl = a.list ? -1 : launch_search_tile(a, st);
  if (tl >= 0) return 3 + tl;
  const int na = crop_max(a.s0, a.s1);
  const int sb = strip_columns(a.winsize, na, na, 200 * 1024);
  const SearchLayout L = search_layout(a.winsize, na, sb);
  const size_t smem = sizeof(float) * ((size_t)L.TR * L.W1 + (size_t)L.DR * L.DC);
  // warps: one per 32 x 16 block of shifts of an interior subset, at most 16
  int nw = ((na + 31) / 32) * ((min(sb, na) + 15) / 16);
  nw = nw < 2 ? 2 : (nw > 16 ? 16 : nw);
  const int threads = nw * 32;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto go = [&](auto kern) {
    int per_sm = 1;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (per_sm < 1) per_sm = 1;
    long long grid = (long long)sms * per_sm;
    if (grid > n) grid = n;
    if (a.ev_start) cudaEventRecord(a.ev_start, st);
    kern<<<(unsigned)grid, threads, smem, st>>>(a, sb, na);
    if (a.ev_stop) cudaEventRecord(a.ev_stop, st);
  };
  switch (L.TR) {  // template rows rounded up to 8: compile-time for full unrolling
    case 8: go(ncc_search_kernel<8>); break;
    case 16: go(ncc_search_kernel<16>); break;
    case 24: go(ncc_search_kernel<24>); break;
    case 32: go(ncc_search_kernel<32>); break;
    case 40: go(ncc_search_kernel<40>); break;
    case 48: go(ncc_search_kernel<48>); break;
    case 56: go(ncc_search_kernel<56>); break;
    case 64: go(ncc_search_kernel<64>); break;
    case 72: go(ncc_search_kernel<72>); break;
    case 80: go(ncc_search_kernel<80>); break;
    case 88: go(ncc_search_kernel<88>); break;
    case 96: go(ncc_search_kernel<96>); break;
    case 104: go(ncc_search_kernel<104>); break;
    case 112: go(ncc_search_kernel<112>); break;
    case 120: go(ncc_search_kernel<120>); break;
    default: return -1;
  }
  return 4;
}

}  // namespace aldic
