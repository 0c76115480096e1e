// The integer search's bad-point removal: funRemoveOutliers(u, v, cc, 0, Thr0) with a
// threshold Thr0 > 0 (func/funRemoveOutliers.m:16, :44-87), the call that ends
// IntegerSearchQuadtree's whole-field branch (func_quadtree/IntegerSearchQuadtree.m:158-160).
//
// For each of u and v (m x n column-major grids) funMedRemoveOutliers (:374-390):
//   1. the NaN holes are filled with inpaint_nans(., 3) (func/inpaint_nans.m:255-325): the
//      least-squares solution of del^4 = 0 around the holes (del^2 / [1 -2 1] near the
//      grid edges) with the finite entries fixed;
//   2. medFilt2(., [2 2], 'symmetric', 2) (:393-441): per entry the median of itself, the
//      entry below and the entry below-right (the last row and column repeated past the
//      edge), in MATLAB's single precision (the neighbour stack is single, :413);
//   3. the normalised fluctuation |u - median| / (median of |u - median| + 0.1), single.
// Entries whose sqrt(nfu^2 + nfv^2) exceeds Thr0 are set NaN in both grids (:64-68), both
// are filled with inpaint_nans(., 4) (:69, init.cu's spring solver) and the entries that
// were NaN in u on entry are NaN again (:72).
//
// Method 3 is solved by CGLS (conjugate gradients on the normal equations, matrix-free on
// the grid) in FP64 by one CTA per grid, started from the method-4 fill of the same grid
// (close to the method-3 surface, so the slowly converging smooth modes start small) and
// run until |A^T r| <= 1e-12 |A^T b| or the iteration limit.  Its result feeds only the
// median test: outside the holes it is never written back.
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace aldic {

namespace {

constexpr int kDel4Threads = 1024;

__host__ __device__ inline bool is_nan_hd(double x) { return x != x; }

// MATLAB single arithmetic, each operation rounded on its own.
__host__ __device__ inline float f_add(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
__host__ __device__ inline float f_sub(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
__host__ __device__ inline float f_mul(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
__host__ __device__ inline float f_div(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fdiv_rn(a, b);
#else
  return a / b;
#endif
}
__host__ __device__ inline float f_sqrt(float a) {
#ifdef __CUDA_ARCH__
  return __fsqrt_rn(a);
#else
  return sqrtf(a);
#endif
}

}  // namespace

// ---------------------------------------------------------------------------------------
// inpaint_nans method 3: the operator, row by row
// ---------------------------------------------------------------------------------------

// The 13 taps a row of the method-3 operator can have, as (row, column) offsets.
__host__ __device__ inline void del4_tap(int o, int& dr, int& dc) {
  const int R[13] = {0, -1, 1, 0, 0, -2, 2, 0, 0, -1, 1, -1, 1};
  const int C[13] = {0, 0, 0, -1, 1, 0, 0, -2, 2, -1, -1, 1, 1};
  dr = R[o];
  dc = C[o];
}

// Coefficient of tap (dr, dc) in the row of entry (r, c) (0-based) of an m x n grid: the sum
// of the four stencil sets of func/inpaint_nans.m:268-321 that apply to the entry -- del^4
// (20 centre, -8 edge, 2 diagonal, 1 at distance 2) for rows and columns 3..end-2 (1-based),
// the 5-point del^2 on the second / second-last row or column, [1 -2 1] along the first /
// last row (between columns) and the first / last column (between rows).  As in the
// reference, a tap is the column-major linear index g + dr + dc m: on grids of at least 3 x 3
// every non-zero coefficient's tap is the entry at (r + dr, c + dc); on a grid of 2 rows the
// second-row stencil wraps into the neighbouring column exactly as the reference's sparse()
// indices do, and a tap outside 0..m n - 1 (where the reference stops with an index error)
// is skipped.
__host__ __device__ inline double del4_coef(int r, int c, int m, int n, int dr, int dc) {
  const int R = r + 1, C = c + 1;
  const int ar = dr < 0 ? -dr : dr, ac = dc < 0 ? -dc : dc;
  const bool centre = dr == 0 && dc == 0;
  double w = 0.0;
  if (R >= 3 && R <= m - 2 && C >= 3 && C <= n - 2) {
    if (centre) w += 20.0;
    else if (ar + ac == 1) w += -8.0;
    else if ((ar == 2 && dc == 0) || (ac == 2 && dr == 0)) w += 1.0;
    else if (ar == 1 && ac == 1) w += 2.0;
  }
  if (((R == 2 || R == m - 1) && C >= 2 && C <= n - 1) || ((C == 2 || C == n - 1) && R >= 2 && R <= m - 1)) {
    if (centre) w += -4.0;
    else if (ar + ac == 1) w += 1.0;
  }
  if ((R == 1 || R == m) && C >= 2 && C <= n - 1) {
    if (centre) w += -2.0;
    else if (dr == 0 && ac == 1) w += 1.0;
  }
  if ((C == 1 || C == n) && R >= 2 && R <= m - 1) {
    if (centre) w += -2.0;
    else if (dc == 0 && ar == 1) w += 1.0;
  }
  return w;
}

// Whether the row of entry g has a non-zero coefficient on a NaN entry of A (the rows the
// reference keeps, func/inpaint_nans.m:324).
__host__ __device__ inline bool del4_touches_nan(int g, int m, int n, const double* A) {
  const int r = g % m, c = g / m, mn = m * n;
  for (int o = 0; o < 13; ++o) {
    int dr, dc;
    del4_tap(o, dr, dc);
    const int h = g + dr + dc * m;
    if (h < 0 || h >= mn) continue;
    if (del4_coef(r, c, m, n, dr, dc) != 0.0 && is_nan_hd(A[h])) return true;
  }
  return false;
}

// Right-hand side of row g: minus the row's coefficients times the finite entries.
__host__ __device__ inline double del4_rhs(int g, int m, int n, const double* A) {
  const int r = g % m, c = g / m, mn = m * n;
  double s = 0.0;
  for (int o = 0; o < 13; ++o) {
    int dr, dc;
    del4_tap(o, dr, dc);
    const int h = g + dr + dc * m;
    if (h < 0 || h >= mn) continue;
    const double w = del4_coef(r, c, m, n, dr, dc);
    const double a = A[h];
    if (w != 0.0 && !is_nan_hd(a)) s -= w * a;
  }
  return s;
}

// (A p) at row g: p holds the unknowns, map[h] the unknown index of grid entry h (-1 known).
__host__ __device__ inline double del4_row(int g, int m, int n, const int* map, const double* p) {
  const int r = g % m, c = g / m, mn = m * n;
  double s = 0.0;
  for (int o = 0; o < 13; ++o) {
    int dr, dc;
    del4_tap(o, dr, dc);
    const int h = g + dr + dc * m;
    if (h < 0 || h >= mn) continue;
    const double w = del4_coef(r, c, m, n, dr, dc);
    const int j = map[h];
    if (w != 0.0 && j >= 0) s += w * p[j];
  }
  return s;
}

// (A^T r) at unknown entry g: the rows e whose tap lands on g (e = g - dr - dc m), emap[e]
// the row index of grid entry e (-1 for entries without a kept row).
__host__ __device__ inline double del4_col(int g, int m, int n, const int* emap, const double* rv) {
  const int mn = m * n;
  double s = 0.0;
  for (int o = 0; o < 13; ++o) {
    int dr, dc;
    del4_tap(o, dr, dc);
    const int e = g - dr - dc * m;
    if (e < 0 || e >= mn) continue;
    const double w = del4_coef(e % m, e / m, m, n, dr, dc);
    const int t = emap[e];
    if (w != 0.0 && t >= 0) s += w * rv[t];
  }
  return s;
}

// ---------------------------------------------------------------------------------------
// the median test, per entry
// ---------------------------------------------------------------------------------------

__host__ __device__ inline float med3f(float a, float b, float c) {
  return fmaxf(fminf(a, b), fminf(fmaxf(a, b), c));
}

// u - medFilt2(u) at entry (r, c) in single: the median of (r, c), (r+1, c), (r+1, c+1), the
// last row / column repeated.
__host__ __device__ inline float med_fluct(const double* U, int m, int n, int r, int c) {
  const int r1 = r + 1 < m ? r + 1 : m - 1, c1 = c + 1 < n ? c + 1 : n - 1;
  const float a = (float)U[r + (long long)c * m];
  const float b = (float)U[r1 + (long long)c * m];
  const float d = (float)U[r1 + (long long)c1 * m];
  return f_sub(a, med3f(a, b, d));
}

// As med_fluct on the grid whose NaN entries take the values of F (F is read there only).
__host__ __device__ inline float med_fluct_filled(const double* U, const double* F, int m, int n, int r, int c) {
  const int r1 = r + 1 < m ? r + 1 : m - 1, c1 = c + 1 < n ? c + 1 : n - 1;
  const long long ga = r + (long long)c * m, gb = r1 + (long long)c * m, gd = r1 + (long long)c1 * m;
  const float a = (float)(is_nan_hd(U[ga]) ? F[ga] : U[ga]);
  const float b = (float)(is_nan_hd(U[gb]) ? F[gb] : U[gb]);
  const float d = (float)(is_nan_hd(U[gd]) ? F[gd] : U[gd]);
  return f_sub(a, med3f(a, b, d));
}

// |fl / (medFilt2(|fl|) + 0.1)| at entry (r, c), single.
__host__ __device__ inline float norm_fluct(const float* fl, int m, int n, int r, int c) {
  const int r1 = r + 1 < m ? r + 1 : m - 1, c1 = c + 1 < n ? c + 1 : n - 1;
  const float x = fl[r + (long long)c * m];
  const float res = med3f(fabsf(x), fabsf(fl[r1 + (long long)c * m]), fabsf(fl[r1 + (long long)c1 * m]));
  return fabsf(f_div(x, f_add(res, 0.1f)));
}

__host__ __device__ inline float norm_fluct_mag(const float* fu, const float* fv, int m, int n, int r, int c) {
  const float a = norm_fluct(fu, m, n, r, c), b = norm_fluct(fv, m, n, r, c);
  return f_sqrt(f_add(f_mul(a, a), f_mul(b, b)));
}

namespace {

// Stream compaction of the grid entries g < mn with pred(g), in grid order: map[g] = the
// entry's position (-1 when pred is false), list[pos] = g; returns the count to every
// thread.  Every thread takes a contiguous range, one block scan gives the offsets.
// s_warp holds 33 ints.  The caller synchronises before reading map / list.
template <class Pred>
__device__ int block_compact(int mn, Pred pred, int* map, int* list, int* s_warp) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  const int per = (mn + (int)blockDim.x - 1) / (int)blockDim.x;
  const int g0 = min(mn, tid * per), g1 = min(mn, g0 + per);
  int cnt = 0;
  for (int g = g0; g < g1; ++g) cnt += pred(g) ? 1 : 0;
  int incl = cnt;
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += y;
  }
  __syncthreads();  // s_warp may still be read from a previous call
  if (lane == 31) s_warp[wid] = incl;
  __syncthreads();
  if (tid == 0) {
    int run = 0;
    for (int k = 0; k < nw; ++k) {
      const int t = s_warp[k];
      s_warp[k] = run;
      run += t;
    }
    s_warp[32] = run;
  }
  __syncthreads();
  const int total = s_warp[32];
  int pos = s_warp[wid] + incl - cnt;
  for (int g = g0; g < g1; ++g) {
    const bool k = pred(g);
    map[g] = k ? pos : -1;
    if (k) list[pos++] = g;
  }
  return total;
}

}  // namespace

// One CTA per grid, blockIdx.x selecting the grid: the method-3 least-squares values of the
// NaN entries of A_c (m x n column-major) are written to the same entries of O_c (no other
// entry is written), CGLS started from X0_c (read at the NaN entries only).  hint: the grid
// is skipped when hint[c] + hint[2] == 0 (a caller-side NaN count of zero).
// status[3 c + 0] = unknowns, [3 c + 1] = iterations, [3 c + 2] = 1 when the target was met.
__global__ void __launch_bounds__(kDel4Threads) inpaint_del4_kernel(
    const double* A0, const double* A1, const double* X00, const double* X01, double* O0, double* O1, int m,
    int n, int maxit, char* scratch, size_t stride, const int* __restrict__ hint, int* __restrict__ status) {
  __shared__ double red[32];
  __shared__ int s_warp[33];
  const int comp = blockIdx.x;
  const double* A = comp ? A1 : A0;
  const double* X0 = comp ? X01 : X00;
  double* O = comp ? O1 : O0;
  status += 3 * comp;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (hint && hint[comp] + hint[2] == 0) {
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
  int* emap = list + mn;
  int* elist = emap + mn;
  double* x = (double*)(((uintptr_t)(elist + mn) + 255) & ~(uintptr_t)255);
  double* s = x + mn;
  double* p = s + mn;
  double* rv = p + mn;
  double* q = rv + mn;
  const int nu = block_compact(mn, [&](int g) { return is_nan_hd(A[g]); }, map, list, s_warp);
  if (nu == 0) {  // nothing to fill: one read of the grid
    if (tid == 0) {
      status[0] = 0;
      status[1] = 0;
      status[2] = 1;
    }
    return;
  }
  const int ne = block_compact(mn, [&](int g) { return del4_touches_nan(g, m, n, A); }, emap, elist, s_warp);
  __syncthreads();  // map, list, emap, elist complete
  for (int t = tid; t < ne; t += nt) rv[t] = del4_rhs(elist[t], m, n, A);
  for (int u = tid; u < nu; u += nt) x[u] = X0[list[u]];
  __syncthreads();
  double loc = 0.0;
  for (int u = tid; u < nu; u += nt) {
    const double v = del4_col(list[u], m, n, emap, rv);
    loc += v * v;
  }
  const double atb = block_sum_all(loc, red);  // |A^T b|^2
  for (int t = tid; t < ne; t += nt) rv[t] -= del4_row(elist[t], m, n, map, x);  // r = b - A x0
  __syncthreads();
  loc = 0.0;
  for (int u = tid; u < nu; u += nt) {
    const double v = del4_col(list[u], m, n, emap, rv);
    s[u] = v;
    p[u] = v;
    loc += v * v;
  }
  double gamma = block_sum_all(loc, red);
  const double target = 1e-24 * atb;  // |A^T r| <= 1e-12 |A^T b|
  int it = 0;
  bool met = gamma <= target;
  while (!met && it < maxit) {
    __syncthreads();  // p complete
    loc = 0.0;
    for (int t = tid; t < ne; t += nt) {
      const double v = del4_row(elist[t], m, n, map, p);
      q[t] = v;
      loc += v * v;
    }
    const double qq = block_sum_all(loc, red);
    if (!(qq > 0.0)) break;  // no direction left (rank-deficient system)
    const double alpha = gamma / qq;
    for (int u = tid; u < nu; u += nt) x[u] += alpha * p[u];
    for (int t = tid; t < ne; t += nt) rv[t] -= alpha * q[t];
    __syncthreads();  // r complete
    loc = 0.0;
    for (int u = tid; u < nu; u += nt) {
      const double v = del4_col(list[u], m, n, emap, rv);
      s[u] = v;
      loc += v * v;
    }
    const double gn = block_sum_all(loc, red);
    ++it;
    met = gn <= target;
    const double beta = gn / gamma;
    gamma = gn;
    for (int u = tid; u < nu; u += nt) p[u] = s[u] + beta * p[u];
  }
  __syncthreads();
  for (int u = tid; u < nu; u += nt) O[list[u]] = x[u];
  if (tid == 0) {
    status[0] = nu;
    status[1] = it;
    status[2] = met ? 1 : 0;
  }
}

// NaN entries of u and v: counts[0] += #NaN(u), counts[1] += #NaN(v) (warp ballots, one
// atomic per warp and grid).
__global__ void nan_count_kernel(const double* __restrict__ u, const double* __restrict__ v, long long mn,
                                 int* __restrict__ counts) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool in = g < mn;
  const unsigned bu = __ballot_sync(0xffffffffu, in && is_nan_hd(u[in ? g : 0]));
  const unsigned bv = __ballot_sync(0xffffffffu, in && is_nan_hd(v[in ? g : 0]));
  if ((threadIdx.x & 31) == 0) {
    if (bu) atomicAdd(counts, __popc(bu));
    if (bv) atomicAdd(counts + 1, __popc(bv));
  }
}

// u - medFilt2(u) and v - medFilt2(v), single, of the method-3 filled grids: the grid's own
// value where finite, the fill (uf, vf, written at the NaN entries only) where NaN.
__global__ void median_fluct_kernel(const double* __restrict__ u, const double* __restrict__ v,
                                    const double* __restrict__ uf, const double* __restrict__ vf, int m, int n,
                                    float* __restrict__ fu, float* __restrict__ fv) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= (long long)m * n) return;
  const int r = (int)(g % m), c = (int)(g / m);
  fu[g] = med_fluct_filled(u, uf, m, n, r, c);
  fv[g] = med_fluct_filled(v, vf, m, n, r, c);
}

// The median test: entries with |normalised fluctuation| > thr set NaN in u and v; hole
// records the entries of u that were NaN on entry; count receives the number removed.
__global__ void outlier_mark_kernel(const float* __restrict__ fu, const float* __restrict__ fv, int m, int n,
                                    float thr, double* __restrict__ u, double* __restrict__ v,
                                    unsigned char* __restrict__ hole, int* __restrict__ count) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= (long long)m * n) return;
  const int r = (int)(g % m), c = (int)(g / m);
  hole[g] = is_nan_hd(u[g]) ? 1 : 0;
  if (norm_fluct_mag(fu, fv, m, n, r, c) > thr) {
    u[g] = (double)NAN;
    v[g] = (double)NAN;
    atomicAdd(count, 1);
  }
}

__global__ void restore_holes_kernel(const unsigned char* __restrict__ hole, long long mn, double* __restrict__ u,
                                     double* __restrict__ v) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= mn || !hole[g]) return;
  u[g] = (double)NAN;
  v[g] = (double)NAN;
}

size_t del4_scratch_bytes(long long mn) { return (size_t)mn * (4 * sizeof(int) + 5 * sizeof(double)) + 2048; }

int launch_inpaint_del4(const double* A0, const double* A1, const double* X00, const double* X01, double* O0,
                        double* O1, int m, int n, int maxit, void* scratch, const int* hint, int* status,
                        cudaStream_t st) {
  const size_t stride = (del4_scratch_bytes((long long)m * n) + 255) & ~(size_t)255;
  inpaint_del4_kernel<<<2, kDel4Threads, 0, st>>>(A0, A1, X00, X01, O0, O1, m, n, maxit, (char*)scratch, stride,
                                                 hint, status);
  return 1;
}

int launch_nan_count(const double* u, const double* v, int m, int n, int* counts, cudaStream_t st) {
  const long long mn = (long long)m * n;
  nan_count_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, st>>>(u, v, mn, counts);
  return 1;
}

int launch_median_fluct(const double* u, const double* v, const double* uf, const double* vf, int m, int n,
                        float* fu, float* fv, cudaStream_t st) {
  const long long mn = (long long)m * n;
  median_fluct_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, st>>>(u, v, uf, vf, m, n, fu, fv);
  return 1;
}

int launch_outlier_mark(const float* fu, const float* fv, int m, int n, float thr, double* u, double* v,
                        unsigned char* hole, int* count, cudaStream_t st) {
  const long long mn = (long long)m * n;
  outlier_mark_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, st>>>(fu, fv, m, n, thr, u, v, hole, count);
  return 1;
}

int launch_restore_holes(const unsigned char* hole, int m, int n, double* u, double* v, cudaStream_t st) {
  const long long mn = (long long)m * n;
  restore_holes_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, st>>>(hole, mn, u, v);
  return 1;
}

}  // namespace aldic
