// Initial-guess assembly of the stereo / temporal drivers: Init(u, v, Phi, x, y, 0)
// (func/Init.m:1-2 and :85-92), i.e. inpaint_nans(u, 4) and inpaint_nans(v, 4) of the
// integer-search grids, then U0 interleaved in mesh order.
//
// inpaint_nans method 4 (func/inpaint_nans.m:369-398, the "spring analogy"): every NaN
// entry is tied by a spring of unit stiffness to each of its horizontal and vertical
// neighbours inside the grid (each pair once), and the NaN entries take the least-squares
// solution of "every spring at rest" with the known entries fixed.  The normal equations of
// that system are, for every unknown i with in-grid 4-neighbours N(i),
//     |N(i)| x_i - sum over unknown j in N(i) of x_j = sum over known j in N(i) of A_j,
// a symmetric positive definite system (a graph Laplacian with Dirichlet values) whenever
// every connected NaN region touches a known entry.  It is solved here by conjugate
// gradients in FP64, matrix-free on the grid, by one CTA per grid (the unknowns are the
// search's few failed subsets); the residual is driven to 1e-13 of the right-hand side.
// A NaN region with no known neighbour has no unique solution: CG leaves it at 0.
#include "common.cuh"
#include "kernels.h"

namespace aldic {

namespace {

constexpr int kInitThreads = 1024;

// Grid neighbours (row-1, row+1, col-1, col+1) of linear index g in an m x n column-major grid.
__device__ __forceinline__ int nbr(int g, int k, int m, int n) {
  const int r = g % m, c = g / m;
  switch (k) {
    case 0: return r > 0 ? g - 1 : -1;
    case 1: return r < m - 1 ? g + 1 : -1;
    case 2: return c > 0 ? g - m : -1;
    default: return c < n - 1 ? g + m : -1;
  }
}

}  // namespace

// One CTA per grid, blockIdx.x selecting the grid: the NaN entries of A_c (m x n,
// column-major) are solved and written to the same entries of O_c (O_c may be A_c for an
// in-place fill; no other entry of O_c is written).  Scratch per grid (stride bytes apart):
// map (m n ints), list (m n ints), x, r, p, q (m n doubles each).  hint (optional): the
// grid is skipped when hint[c] + hint[2] == 0, i.e. a caller-side count of its NaN entries
// is zero.  status[3 c + 0] = unknowns, [3 c + 1] = CG iterations, [3 c + 2] = 1 when the
// residual target was met.
__global__ void __launch_bounds__(kInitThreads) inpaint_springs_kernel(const double* A0, const double* A1, double* O0,
                                                                       double* O1, int m, int n, char* scratch,
                                                                       size_t stride, const int* __restrict__ hint,
                                                                       int* __restrict__ status) {
  __shared__ double red[32];
  __shared__ int s_count;
  __shared__ int s_warp[32];
  const int comp = blockIdx.x;
  const double* A = comp ? A1 : A0;
  double* O = comp ? O1 : O0;
  status += 3 * comp;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  if (hint && hint[comp] + hint[2] == 0) {  // no NaN entry: nothing to read
    if (tid == 0) {
      status[0] = 0;
      status[1] = 0;
      status[2] = 1;
    }
    return;
  }
  const int mn = m * n;
  char* sc = scratch + (size_t)comp * stride;
  int* map = (int*)sc;
  int* list = map + mn;
  double* x = (double*)(((uintptr_t)(list + mn) + 255) & ~(uintptr_t)255);
  double* r = x + mn;
  double* p = r + mn;
  double* q = p + mn;
  // ---- compaction of the NaN entries, in grid order: every thread counts a contiguous
  // range, one block scan gives the offsets, the same ranges are written ----
  const int per = (mn + (int)blockDim.x - 1) / (int)blockDim.x;
  const int g0 = min(mn, tid * per), g1 = min(mn, g0 + per);
  int cnt = 0;
  for (int g = g0; g < g1; ++g) cnt += isnan(A[g]) ? 1 : 0;
  int incl = cnt;  // inclusive scan within the warp
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += y;
  }
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (tid == 0) {
    int run = 0;
    for (int k = 0; k < nw; ++k) {
      const int t = s_warp[k];
      s_warp[k] = run;
      run += t;
    }
    s_count = run;
  }
  __syncthreads();
  const int nu = s_count;
  if (nu == 0) {  // nothing to fill: one read of the grid
    if (tid == 0) {
      status[0] = 0;
      status[1] = 0;
      status[2] = 1;
    }
    return;
  }
  int pos = s_warp[wid] + incl - cnt;  // exclusive offset of this thread's range
  for (int g = g0; g < g1; ++g) {
    const bool unk = isnan(A[g]);
    map[g] = unk ? pos : -1;
    if (unk) list[pos++] = g;
  }
  __syncthreads();
  // ---- right-hand side and the CG start x = 0, r = p = b ----
  double bb_local = 0.0;
  for (int u = tid; u < nu; u += blockDim.x) {
    const int g = list[u];
    double b = 0.0;
    for (int k = 0; k < 4; ++k) {
      const int h = nbr(g, k, m, n);
      if (h >= 0 && map[h] < 0) b += A[h];
    }
    x[u] = 0.0;
    r[u] = b;
    p[u] = b;
    bb_local += b * b;
  }
  const double bb = block_sum_all(bb_local, red);
  double rr = bb;
  const double target = 1e-26 * bb;  // |r| <= 1e-13 |b|
  const int maxit = nu + 200 < 100000 ? nu + 200 : 100000;
  int it = 0;
  bool met = rr <= target;
  while (!met && it < maxit) {
    __syncthreads();  // p complete
    double pq_local = 0.0;
    for (int u = tid; u < nu; u += blockDim.x) {
      const int g = list[u];
      double s = 0.0;
      int deg = 0;
      for (int k = 0; k < 4; ++k) {
        const int h = nbr(g, k, m, n);
        if (h < 0) continue;
        ++deg;
        const int j = map[h];
        if (j >= 0) s += p[j];
      }
      const double v = deg * p[u] - s;
      q[u] = v;
      pq_local += p[u] * v;
    }
    const double pq = block_sum_all(pq_local, red);
    if (!(pq > 0.0)) break;  // singular direction (a region with no known neighbour)
    const double alpha = rr / pq;
    double rr_local = 0.0;
    for (int u = tid; u < nu; u += blockDim.x) {
      x[u] += alpha * p[u];
      const double rn = r[u] - alpha * q[u];
      r[u] = rn;
      rr_local += rn * rn;
    }
    const double rr_new = block_sum_all(rr_local, red);
    ++it;
    met = rr_new <= target;
    const double beta = rr_new / rr;
    rr = rr_new;
    for (int u = tid; u < nu; u += blockDim.x) p[u] = r[u] + beta * p[u];
  }
  __syncthreads();  // every read of A done before an in-place write
  for (int u = tid; u < nu; u += blockDim.x) O[list[u]] = x[u];
  if (tid == 0) {
    status[0] = nu;
    status[1] = it;
    status[2] = met ? 1 : 0;
  }
}

// U0 in mesh order from the inpainted grids (ny x nx column-major, the search's output
// layout): U0(2 i - 1) = u'(i), U0(2 i) = v'(i) with i running over the transposed grid,
// XList fastest (func/Init.m:86-92); u' is u where finite and the fill fu (written at the
// NaN entries only) where NaN, v' likewise.
__global__ void interleave_u0_kernel(const double* __restrict__ u, const double* __restrict__ v,
                                     const double* __restrict__ fu, const double* __restrict__ fv, int ny, int nx,
                                     double* __restrict__ U0) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nx * ny) return;
  const int ix = (int)(i % nx), iy = (int)(i / nx);
  const long long g = iy + (long long)ix * ny;
  const double a = u[g], b = v[g];
  U0[2 * i] = isnan(a) ? fu[g] : a;
  U0[2 * i + 1] = isnan(b) ? fv[g] : b;
}

// MATLAB std(x, 'omitnan') of k values in order (mean first, then the squared deviations),
// every operation rounded on its own as MATLAB's are (no fused multiply-adds).
__device__ __forceinline__ double std_omitnan(const double* x, int k) {
  double m = 0.0;
  int c = 0;
  for (int t = 0; t < k; ++t)
    if (!isnan(x[t])) {
      m = __dadd_rn(m, x[t]);
      ++c;
    }
  if (c < 2) return c == 1 ? 0.0 : (double)NAN;
  m = __ddiv_rn(m, (double)c);
  double ss = 0.0;
  for (int t = 0; t < k; ++t)
    if (!isnan(x[t])) {
      const double d = __dsub_rn(x[t], m);
      ss = __dadd_rn(ss, __dmul_rn(d, d));
    }
  return __dsqrt_rn(__ddiv_rn(ss, (double)(c - 1)));
}

// One spring outlier pass of Init index 1 (func/Init.m:31-62, :76-105, :119-150) over the
// interior nodes of the m x n grids: ut, vt are the pass's (inpainted) inputs, ui, vi their
// copies that receive the NaN marks (a node failing the test for u or for v is set NaN in
// both, with its neighbourhood; overlapping marks write the same NaN).  mode 0: the 8
// neighbours, average (sum of the 4 edge neighbours / 8 + sum of the 4 corners / 16) / (3/4),
// 3 standard deviations, 8-neighbourhood marked; mode 1: the 4 edge neighbours, their mean,
// 2 standard deviations, 4-neighbourhood; mode 2: as mode 0 with 2 standard deviations.
__global__ void spring_mark_kernel(const double* __restrict__ ut, const double* __restrict__ vt, double* ui,
                                   double* vi, int m, int n, int mode) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m < 3 || n < 3 || idx >= (long long)(m - 2) * (n - 2)) return;
  const int i = 1 + (int)(idx % (m - 2)), j = 1 + (int)(idx / (m - 2));
  const long long g = i + (long long)j * m;
  // neighbour order of the reference: (i-1,j) (i+1,j) (i,j-1) (i,j+1) (i-1,j-1) (i+1,j-1)
  // (i+1,j+1) (i-1,j+1)
  const long long nb[8] = {g - 1, g + 1, g - m, g + m, g - 1 - m, g + 1 - m, g + 1 + m, g - 1 + m};
  const double kk = mode == 0 ? 3.0 : 2.0;
  bool bad = false;
  for (int comp = 0; comp < 2; ++comp) {
    const double* t = comp ? vt : ut;
    double x[8];
    for (int q = 0; q < 8; ++q) x[q] = t[nb[q]];
    double avg, sd;
    if (mode == 1) {
      double acc = 0.0;
      int c = 0;
      for (int q = 0; q < 4; ++q)
        if (!isnan(x[q])) {
          acc = __dadd_rn(acc, x[q]);
          ++c;
        }
      avg = c ? __ddiv_rn(acc, (double)c) : (double)NAN;
      sd = std_omitnan(x, 4);
    } else {
      const double se = __dadd_rn(__dadd_rn(__dadd_rn(x[0], x[1]), x[2]), x[3]);
      const double sc = __dadd_rn(__dadd_rn(__dadd_rn(x[4], x[5]), x[6]), x[7]);
      avg = __ddiv_rn(__dadd_rn(__dmul_rn(0.125, se), __dmul_rn(0.0625, sc)), 0.75);
      sd = std_omitnan(x, 8);
    }
    const double err = __dsub_rn(fabs(__dsub_rn(t[g], avg)), __dmul_rn(kk, sd));
    if (err > 0.0) bad = true;
  }
  if (!bad) return;
  const int cnt = mode == 1 ? 4 : 8;
  ui[g] = (double)NAN;
  vi[g] = (double)NAN;
  for (int q = 0; q < cnt; ++q) {
    ui[nb[q]] = (double)NAN;
    vi[nb[q]] = (double)NAN;
  }
}

// The border rows and columns of both grids set NaN (func/Init.m:62-63 and the same lines
// after each pass).
__global__ void border_nan_kernel(double* ui, double* vi, int m, int n) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = 2LL * m + 2LL * n;
  if (idx >= per) return;
  long long g;
  if (idx < m) g = idx;                                          // column 1
  else if (idx < 2LL * m) g = (idx - m) + (long long)(n - 1) * m;  // column n
  else if (idx < 2LL * m + n) g = (idx - 2LL * m) * m;            // row 1
  else g = (m - 1) + (idx - 2LL * m - n) * m;                     // row m
  ui[g] = (double)NAN;
  vi[g] = (double)NAN;
}

int launch_spring_pass(const double* ut, const double* vt, double* ui, double* vi, int m, int n, int mode,
                       cudaStream_t st) {
  const long long interior = (m >= 3 && n >= 3) ? (long long)(m - 2) * (n - 2) : 0;
  int l = 0;
  if (interior > 0) {
    spring_mark_kernel<<<(unsigned)((interior + 255) / 256), 256, 0, st>>>(ut, vt, ui, vi, m, n, mode);
    ++l;
  }
  const long long per = 2LL * m + 2LL * n;
  border_nan_kernel<<<(unsigned)((per + 255) / 256), 256, 0, st>>>(ui, vi, m, n);
  return l + 1;
}

size_t inpaint_scratch_bytes(long long mn) { return (size_t)mn * (2 * sizeof(int) + 4 * sizeof(double)) + 1024; }

int launch_inpaint(double* A, int m, int n, void* scratch, int* status, cudaStream_t st) {
  inpaint_springs_kernel<<<1, kInitThreads, 0, st>>>(A, A, A, A, m, n, (char*)scratch, 0, nullptr, status);
  return 1;
}

int launch_inpaint2(const double* A0, const double* A1, double* O0, double* O1, int m, int n, void* scratch,
                    const int* hint, int* status, cudaStream_t st) {
  const size_t stride = (inpaint_scratch_bytes((long long)m * n) + 255) & ~(size_t)255;
  inpaint_springs_kernel<<<2, kInitThreads, 0, st>>>(A0, A1, O0, O1, m, n, (char*)scratch, stride, hint, status);
  return 1;
}

int launch_interleave_u0(const double* u, const double* v, const double* fu, const double* fv, int ny, int nx,
                         double* U0, cudaStream_t st) {
  const long long n = (long long)nx * ny;
  interleave_u0_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(u, v, fu, fv, ny, nx, U0);
  return 1;
}

}  // namespace aldic
