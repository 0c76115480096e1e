// FP64 CPU oracle for the 3D-Stereo-ALDIC per-subset hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++ double precision, the
// algorithms of the reference MATLAB/MEX code so that the CUDA path can be checked
// against it.  Nothing in the product (the CUDA library and its host mirror) links or
// calls this code; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// load it, as the checker.
//
// Every function cites the reference file:line it follows.  Conventions are the
// reference's: images are column-major M x Nc (dim 1 = image x after the
// transposed imread), pixel coordinates are 1-based, U is interleaved [u1 v1 u2 v2 ...],
// F is interleaved [F11 F21 F12 F22 ...], H is n x 21 column-major.
//
// Parity pin: the interpolation restatement is pinned against the reference's own
// ba_interp2_spline.cpp compiled under oracle/_ref (golden vectors in tests/golden/).
// The MATLAB parts (IC-GN control flow, normxcorr2, findpeak, bwselect) cannot be run
// here (no MATLAB/Octave); they are restated from the reference source and from the
// published definitions of the toolbox functions they call.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

// ---------------------------------------------------------------------------------
// Local 4x4 B-spline stencil (ba_interp2_spline.cpp:235-331).
// The interpolant is A = BC * Q * BC^T on the 4x4 neighbourhood Q, evaluated as
// sum_ij a_ij tr^i tc^j with tr the fraction along dim 1 and tc along dim 2
// (ba_interp2_spline.cpp:145-148 swaps the roles of X and Y).  Row i of BC is
// sign_i * scale_i * K[i]; the reference's double path multiplies each a_ij by a scale
// constant that is first rounded to float (ba_interp2_spline.cpp:310-325), and the
// restatement keeps that rounding so that its values track the reference to ~1e-13.
// ---------------------------------------------------------------------------------
const int kK[4][4] = {{0, 1, 0, 0}, {11, 1, -15, 3}, {19, -39, 25, -5}, {-3, 8, -8, 3}};
const double kSign[4] = {1.0, -1.0, 1.0, 1.0};

struct StencilScale {
  double c[4][4];
  StencilScale() {
    volatile float f356 = 3.0f / 56.0f;       // a10,a20,a01,a02
    volatile float f17 = 1.0f / 7.0f;         // a30,a03
    volatile float f9 = (1.0f / 3136.0f) * 9.0f;  // a11,a12,a21,a22
    volatile float f3392 = 3.0f / 392.0f;     // a13,a31,a23,a32
    volatile float f149 = 1.0f / 49.0f;       // a33
    double one_d[4] = {1.0, (double)f356, (double)f356, (double)f17};
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        double s;
        if (i == 0 || j == 0) s = (i == 0) ? one_d[j] : one_d[i];
        else if (i == 3 && j == 3) s = (double)f149;
        else if (i == 3 || j == 3) s = (double)f3392;
        else s = (double)f9;
        c[i][j] = kSign[i] * kSign[j] * s;
      }
  }
};
const StencilScale kScale;

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// F: M x N column-major.  X = dim-2 coordinate, Y = dim-1 coordinate, both 1-based
// (the argument order of ba_interp2_spline(F, X, Y)).
inline double interp_local(const double* F, int M, int N, double X, double Y) {
  const double fX = std::floor(X), fY = std::floor(Y);
  const double tr = Y - fY;  // fraction along dim 1
  const double tc = X - fX;  // fraction along dim 2
  // 0-based first tap: one before floor()-1 (ba_interp2_spline.cpp:172,89-118).
  const int r0 = (int)(fY - 1.0) - 1;
  const int c0 = (int)(fX - 1.0) - 1;
  double Q[4][4];
  for (int c = 0; c < 4; ++c) {
    const int cc = clampi(c0 + c, 0, N - 1);
    for (int r = 0; r < 4; ++r) Q[r][c] = F[(size_t)clampi(r0 + r, 0, M - 1) + (size_t)cc * M];
  }
  // T_ij = sum_rc K_i[r] K_j[c] Q[r][c]
  double rowc[4][4];  // rowc[i][c] = sum_r K_i[r] Q[r][c]
  for (int i = 0; i < 4; ++i)
    for (int c = 0; c < 4; ++c) {
      double s = 0;
      for (int r = 0; r < 4; ++r) s += kK[i][r] * Q[r][c];
      rowc[i][c] = s;
    }
  const double pr[4] = {1.0, tr, tr * tr, tr * tr * tr};
  const double pc[4] = {1.0, tc, tc * tc, tc * tc * tc};
  double val = 0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double t = 0;
      for (int c = 0; c < 4; ++c) t += kK[j][c] * rowc[i][c];
      val += kScale.c[i][j] * t * pr[i] * pc[j];
    }
  return val;
}

// ---------------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------------
inline double matlab_eps(double x) {
  x = std::fabs(x);
  if (!(x < std::numeric_limits<double>::infinity())) return kNaN;
  return std::nextafter(x, std::numeric_limits<double>::infinity()) - x;
}

// mean and sqrt((n-1)*var) of the selected values (MATLAB mean/var semantics:
// empty -> NaN, single value -> var 0).
inline void mean_bottom(const std::vector<double>& v, const std::vector<uint8_t>* sel, double thr_abs,
                        double* mean, double* bottom) {
  double s = 0;
  long n = 0;
  for (size_t k = 0; k < v.size(); ++k) {
    if (sel && !(*sel)[k]) continue;
    if (thr_abs >= 0 && !(std::fabs(v[k]) > thr_abs)) continue;
    s += v[k];
    ++n;
  }
  if (n == 0) {
    *mean = kNaN;
    *bottom = kNaN;
    return;
  }
  const double m = s / n;
  double ss = 0;
  for (size_t k = 0; k < v.size(); ++k) {
    if (sel && !(*sel)[k]) continue;
    if (thr_abs >= 0 && !(std::fabs(v[k]) > thr_abs)) continue;
    ss += (v[k] - m) * (v[k] - m);
  }
  *mean = m;
  *bottom = std::sqrt(ss);
}

// bwselect(BW, c, r, conn): the connected component of `on` pixels that contains the
// seed (row sr, col sc, 0-based), under 4- or 8-connectivity; empty if the seed is off
// or outside.  (Image Processing Toolbox bwselect, as used at
// func_quadtree/funICGNQuadtree.m:83,174,179.)
void bwselect(const std::vector<uint8_t>& bw, int rows, int cols, int sr, int sc, int conn,
              std::vector<uint8_t>* out) {
  out->assign(bw.size(), 0);
  if (sr < 0 || sr >= rows || sc < 0 || sc >= cols) return;
  if (!bw[sr + (size_t)sc * rows]) return;
  std::vector<int> stack;
  stack.push_back(sr + sc * rows);
  (*out)[sr + (size_t)sc * rows] = 1;
  while (!stack.empty()) {
    const int p = stack.back();
    stack.pop_back();
    const int r = p % rows, c = p / rows;
    for (int dc = -1; dc <= 1; ++dc)
      for (int dr = -1; dr <= 1; ++dr) {
        if (dr == 0 && dc == 0) continue;
        if (conn == 4 && dr != 0 && dc != 0) continue;
        const int rr = r + dr, cc = c + dc;
        if (rr < 0 || rr >= rows || cc < 0 || cc >= cols) continue;
        const size_t q = rr + (size_t)cc * rows;
        if (bw[q] && !(*out)[q]) {
          (*out)[q] = 1;
          stack.push_back((int)q);
        }
      }
  }
}

// Solve A x = b (n x n, column-major) by Gaussian elimination with partial pivoting,
// the general path of mldivide.  A singular pivot divides by zero (Inf/NaN), as
// mldivide's LU does after its singularity warning.
void solve_dense(int n, const double* A_in, const double* b_in, double* x) {
  double A[36], b[6];
  std::memcpy(A, A_in, sizeof(double) * n * n);
  std::memcpy(b, b_in, sizeof(double) * n);
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = std::fabs(A[k + k * n]);
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[i + k * n]) > best) {
        best = std::fabs(A[i + k * n]);
        piv = i;
      }
    if (piv != k) {
      for (int j = 0; j < n; ++j) std::swap(A[k + j * n], A[piv + j * n]);
      std::swap(b[k], b[piv]);
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

// Inverse-compositional update (func/funICGN.m:289-307): P <- P o dP^-1.
// Returns false when det(dP) == 0 (the reference breaks out of the loop).
bool compose_inverse(double P[6], const double d[6]) {
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

struct Frame {
  const double* ref;
  const double* def;
  const double* mask;  // may be null (treated as all ones)
  const double* dfdx;  // (M-6) x (N-6)
  const double* dfdy;
  int M, N;
  int crop;  // gradient array offset: Df.DfCropWidth (3), or Df.DfAxis start (4) for epipolar
};

// A rectangular window rows [r0, r1] x cols [c0, c1] (1-based inclusive) sliced from the
// frame.  Returns false when MATLAB indexing would throw (out of range / non-integer).
struct Window {
  int r0, r1, c0, c1, rows, cols;
  std::vector<double> f, fmask, gx, gy;
};

bool is_int(double v) { return std::floor(v) == v && std::isfinite(v); }

bool slice(const Frame& fr, double r0d, double r1d, double c0d, double c1d, bool need_grad, Window* w) {
  if (!is_int(r0d) || !is_int(r1d) || !is_int(c0d) || !is_int(c1d)) return false;
  const int r0 = (int)r0d, r1 = (int)r1d, c0 = (int)c0d, c1 = (int)c1d;
  if (r1 < r0 || c1 < c0) return false;
  if (r0 < 1 || r1 > fr.M || c0 < 1 || c1 > fr.N) return false;
  if (need_grad) {
    const int gM = fr.M - 6, gN = fr.N - 6;
    if (r0 - fr.crop < 1 || r1 - fr.crop > gM || c0 - fr.crop < 1 || c1 - fr.crop > gN) return false;
  }
  w->r0 = r0;
  w->r1 = r1;
  w->c0 = c0;
  w->c1 = c1;
  w->rows = r1 - r0 + 1;
  w->cols = c1 - c0 + 1;
  const size_t n = (size_t)w->rows * w->cols;
  w->f.resize(n);
  w->fmask.resize(n);
  if (need_grad) {
    w->gx.resize(n);
    w->gy.resize(n);
  }
  const int gM = fr.M - 6;
  for (int b = 0; b < w->cols; ++b)
    for (int a = 0; a < w->rows; ++a) {
      const int i = r0 - 1 + a, j = c0 - 1 + b;  // 0-based image index
      const size_t k = a + (size_t)b * w->rows;
      w->f[k] = fr.ref[i + (size_t)j * fr.M];
      w->fmask[k] = fr.mask ? fr.mask[i + (size_t)j * fr.M] : 1.0;
      if (need_grad) {
        const int gi = i - fr.crop, gj = j - fr.crop;
        w->gx[k] = fr.dfdx[gi + (size_t)gj * gM];
        w->gy[k] = fr.dfdy[gi + (size_t)gj * gM];
      }
    }
  return true;
}

// Warp every window pixel with P and interpolate g; returns false when any warped
// coordinate leaves [3, M-2] x [3, N-2] (func/funICGN.m:116-124) or is not finite.
bool warp_interp(const Frame& fr, const Window& w, double x0, double y0, const double P[6],
                 std::vector<double>* g) {
  g->resize((size_t)w.rows * w.cols);
  std::vector<double> U((size_t)w.rows * w.cols), V((size_t)w.rows * w.cols);
  bool oob = false;
  for (int b = 0; b < w.cols; ++b)
    for (int a = 0; a < w.rows; ++a) {
      const double dx = (w.r0 + a) - x0, dy = (w.c0 + b) - y0;
      const double u22 = (1 + P[0]) * dx + P[2] * dy + (x0 + P[4]);
      const double v22 = P[1] * dx + (1 + P[3]) * dy + (y0 + P[5]);
      const size_t k = a + (size_t)b * w.rows;
      U[k] = u22;
      V[k] = v22;
      // Non-finite warps are treated as out of image: the MEX would index with an
      // undefined integer conversion of NaN.
      if (!(u22 >= 3 && u22 <= fr.M - 2 && v22 >= 3 && v22 <= fr.N - 2)) oob = true;
    }
  if (oob) return false;
  for (size_t k = 0; k < g->size(); ++k) (*g)[k] = interp_local(fr.def, fr.M, fr.N, V[k], U[k]);
  return true;
}

// 6x6 Gauss-Newton Hessian sum J^T J with J = [fx dx, fy dx, fx dy, fy dy, fx, fy]
// (func/funICGN.m:70-82).
void hessian6(const Window& w, double x0, double y0, double H[36]) {
  double acc[6][6] = {};
  for (int b = 0; b < w.cols; ++b)
    for (int a = 0; a < w.rows; ++a) {
      const size_t k = a + (size_t)b * w.rows;
      const double dx = (w.r0 + a) - x0, dy = (w.c0 + b) - y0;
      const double J[6] = {w.gx[k] * dx, w.gy[k] * dx, w.gx[k] * dy, w.gy[k] * dy, w.gx[k], w.gy[k]};
      for (int p = 0; p < 6; ++p)
        for (int q = p; q < 6; ++q) acc[p][q] += J[p] * J[q];
    }
  for (int p = 0; p < 6; ++p)
    for (int q = 0; q < 6; ++q) H[p + 6 * q] = (p <= q) ? acc[p][q] : acc[q][p];
}

void pack_h21(const double H[36], double* out, long n, long idx) {
  int t = 0;
  for (int c = 0; c < 6; ++c)
    for (int r = c; r < 6; ++r) out[idx + n * (t++)] = H[r + 6 * c];
}

struct IcgnOut {
  double P[6];
  double H[36];
  int conv;
  bool error;  // a MATLAB error inside the solver (driver stores -1 / NaN)
};

// b vector of the 6-DOF step (func/funICGN.m:257-266).
void bvec6(const Window& w, double x0, double y0, const std::vector<double>& f, double meanf, double bf,
           const std::vector<double>& g, double meang, double bg, double b[6]) {
  double acc[6] = {};
  for (int bb = 0; bb < w.cols; ++bb)
    for (int a = 0; a < w.rows; ++a) {
      const size_t k = a + (size_t)bb * w.rows;
      const double dx = (w.r0 + a) - x0, dy = (w.c0 + bb) - y0;
      const double r = (f[k] - meanf) / bf - (g[k] - meang) / bg;
      acc[0] += dx * w.gx[k] * r;
      acc[1] += dx * w.gy[k] * r;
      acc[2] += dy * w.gx[k] * r;
      acc[3] += dy * w.gy[k] * r;
      acc[4] += w.gx[k] * r;
      acc[5] += w.gy[k] * r;
    }
  for (int i = 0; i < 6; ++i) b[i] = bf * acc[i];
}

inline double norm6(const double* b, int n) {
  double s = 0;
  for (int i = 0; i < n; ++i) s += b[i] * b[i];
  return std::sqrt(s);
}

// funICGN (func/funICGN.m:1-347): uniform-mesh 6-DOF IC-GN, Gauss-Newton.
// `zero_fix_p56` and `max_iter` give epipolar_ICGN1 (func/epipolar_ICGN1.m:49,134-135).
// F0 (optional): an initial displacement gradient [F11 F21 F12 F22] in place of the reference's
// zero start (the learned initial guess; not part of the reference).
void fun_icgn(const Frame& fr, const double U0[2], double x0, double y0, int winsize, double tol, int max_iter,
              bool zero_fix_p56, IcgnOut* out, std::vector<double>* znssd_out = nullptr, const double* F0 = nullptr) {
  out->error = false;
  std::memset(out->H, 0, sizeof(out->H));
  double P[6] = {0, 0, 0, 0, U0[0], U0[1]};
  if (F0)
    for (int k = 0; k < 4; ++k) P[k] = F0[k];
  std::memcpy(out->P, P, sizeof(P));
  double w = winsize;
  Window W;
  if (!slice(fr, x0 - w / 2, x0 + w / 2, y0 - w / 2, y0 + w / 2, true, &W)) {
    out->error = true;
    return;
  }
  const double Nw = (w + 1) * (w + 1);
  long zc = 0;
  for (double v : W.gx) zc += (v == 0);
  if (zc < 0.50 * Nw) {
    if (zc > 0.1 * Nw) {
      w = std::round(std::sqrt(2.0) * w);
      if (!slice(fr, x0 - w / 2, x0 + w / 2, y0 - w / 2, y0 + w / 2, true, &W)) {
        out->error = true;
        return;
      }
    }
    double H[36];
    hessian6(W, x0, y0, H);
    double meanf, bf;
    mean_bottom(W.f, nullptr, -1, &meanf, &bf);
    double normNew = 1, normAbs = 1, normInit = 0;
    int step = 0;
    std::vector<double> g;
    while (step <= max_iter && normNew > tol && normAbs > tol) {
      ++step;
      if (!warp_interp(fr, W, x0, y0, P, &g)) {
        normNew = 1e6;
        break;
      }
      double meang, bg;
      mean_bottom(g, nullptr, -1, &meang, &bg);
      double b[6];
      bvec6(W, x0, y0, W.f, meanf, bf, g, meang, bg, b);
      normNew = norm6(b, 6);
      normAbs = normNew;
      if (step == 1) normInit = normNew;
      if (normInit > tol) normNew = normNew / normInit;
      else normNew = 0;
      if (znssd_out) {
        double z = 0;
        for (size_t k = 0; k < g.size(); ++k) {
          const double r = (W.f[k] - meanf) / bf - (g[k] - meang) / bg;
          z += r * r;
        }
        znssd_out->push_back(z);
      }
      if (normNew < tol || normAbs < tol) break;
      double dP[6], nb[6];
      for (int i = 0; i < 6; ++i) nb[i] = -b[i];
      solve_dense(6, H, nb, dP);
      if (!compose_inverse(P, dP)) break;
      if (zero_fix_p56) {
        P[4] = 0;
        P[5] = 0;
      }
    }
    if (!(normNew < tol || normAbs < tol)) step = max_iter + 1;
    if (std::isnan(normNew)) step = max_iter + 1;
    out->conv = step;
    std::memcpy(out->H, H, sizeof(H));
  } else {
    out->conv = max_iter + 2;
  }
  std::memcpy(out->P, P, sizeof(P));
}

// funICGNQuadtree (func_quadtree/funICGNQuadtree.m:1-454): masked 6-DOF IC-GN.
void fun_icgn_quadtree(const Frame& fr, const double U0[2], double x0, double y0, int winsize, double tol,
                       IcgnOut* out, const double* F0 = nullptr) {
  const int maxIter = 100;
  out->error = false;
  std::memset(out->H, 0, sizeof(out->H));
  double P[6] = {0, 0, 0, 0, U0[0], U0[1]};
  if (F0)
    for (int k = 0; k < 4; ++k) P[k] = F0[k];
  std::memcpy(out->P, P, sizeof(P));
  const double w0 = winsize;
  double w = winsize;
  Window W;
  if (!slice(fr, x0 - w / 2, x0 + w / 2, y0 - w / 2, y0 + w / 2, true, &W)) {
    out->error = true;
    return;
  }
  // tempf = ImgRef .* mask; zero count (:52-61)
  std::vector<double> tf(W.f.size());
  for (size_t k = 0; k < tf.size(); ++k) tf[k] = W.f[k] * W.fmask[k];
  long cnt = 0;
  for (double v : tf) {
    if (std::isnan(v)) {
      out->error = true;
      return;
    }
    cnt += (v == 0);
  }
  if (cnt < 0.4 * (w + 1) * (w + 1)) {
    if (cnt > 0) {
      const double N0 = (w + 1) * (w + 1);
      w = 2 * std::ceil(std::sqrt(N0 / (N0 - cnt)) * w / 2);
      if (!slice(fr, x0 - w / 2, x0 + w / 2, y0 - w / 2, y0 + w / 2, true, &W)) {
        out->error = true;
        return;
      }
      tf.resize(W.f.size());
      for (size_t k = 0; k < tf.size(); ++k) tf[k] = W.f[k] * W.fmask[k];
    }
    // 4-connected region of the f mask at the seed (:83-88)
    const int seed = (int)std::floor((w + 1) / 2) - 1;
    std::vector<uint8_t> mbw(W.fmask.size()), bw4;
    for (size_t k = 0; k < mbw.size(); ++k) mbw[k] = (W.fmask[k] != 0);
    bwselect(mbw, W.rows, W.cols, seed, seed, 4, &bw4);
    for (size_t k = 0; k < tf.size(); ++k) {
      tf[k] *= bw4[k];
      W.gx[k] *= bw4[k];
      W.gy[k] *= bw4[k];
    }
    double H[36];
    hessian6(W, x0, y0, H);
    double meanf, bf;
    mean_bottom(tf, nullptr, 1e-10, &meanf, &bf);
    double normNew = 1, normAbs = 1, normInit = 0;
    int step = 0;
    std::vector<double> g;
    std::vector<uint8_t> gbw;
    double gsum_prev = 0;
    Window Wn = W;  // window geometry used for warping (may regrow)
    while (step <= maxIter && normNew > tol && normAbs > tol) {
      ++step;
      if (step > 1 && cnt > 0) {
        // :139-145 re-derives the subset size from the g region without re-slicing f.
        const double wn = 2 * std::ceil(std::sqrt((w0 + 1) * (w0 + 1) / gsum_prev) * w / 2);
        if (wn != w) {
          w = wn;
          Window tmp;
          if (!slice(fr, x0 - w / 2, x0 + w / 2, y0 - w / 2, y0 + w / 2, false, &tmp)) {
            out->error = true;  // index error while re-slicing the mask (:144)
            std::memcpy(out->P, P, sizeof(P));
            return;
          }
          // Warp with the regrown grid; an out-of-image warp breaks first (:154-157),
          // otherwise the size mismatch at :366 throws.
          std::vector<double> gg;
          if (!warp_interp(fr, tmp, x0, y0, P, &gg)) {
            normNew = 1e6;
            break;
          }
          out->error = true;
          std::memcpy(out->P, P, sizeof(P));
          return;
        }
      }
      if (!warp_interp(fr, Wn, x0, y0, P, &g)) {
        normNew = 1e6;
        break;
      }
      long gcnt = 0;
      for (double v : g) {
        if (std::isnan(v)) {
          out->error = true;
          std::memcpy(out->P, P, sizeof(P));
          return;
        }
        gcnt += (v == 0);
      }
      if (cnt > 0 || gcnt > 0) {
        std::vector<uint8_t> gl(g.size());
        for (size_t k = 0; k < g.size(); ++k) gl[k] = (g[k] != 0);
        bwselect(gl, Wn.rows, Wn.cols, seed, seed, 8, &gbw);
        bool all_on = true;
        for (uint8_t v : gbw) all_on = all_on && v;
        if (all_on) bwselect(mbw, Wn.rows, Wn.cols, seed, seed, 8, &gbw);
        double s = 0;
        for (size_t k = 0; k < g.size(); ++k) {
          g[k] *= gbw[k];
          s += gbw[k];
        }
        gsum_prev = s;
      }
      double meang, bg;
      mean_bottom(g, nullptr, 1e-10, &meang, &bg);
      double b[6];
      bvec6(Wn, x0, y0, tf, meanf, bf, g, meang, bg, b);
      normNew = norm6(b, 6);
      normAbs = normNew;
      if (step == 1) normInit = normNew;
      if (normInit > tol) normNew = normNew / normInit;
      else normNew = 0;
      if (normNew < tol || normAbs < tol) break;
      double dP[6], nb[6];
      for (int i = 0; i < 6; ++i) nb[i] = -b[i];
      solve_dense(6, H, nb, dP);
      if (!compose_inverse(P, dP)) break;
    }
    if (!(normNew < tol || normAbs < tol)) step = maxIter + 1;
    if (std::isnan(normNew)) step = maxIter + 1;
    double sabs = 0;
    for (double v : tf) sabs += std::fabs(v);
    if (sabs < 1e-6) step = maxIter + 3;
    out->conv = step;
    std::memcpy(out->H, H, sizeof(H));
  } else {
    out->conv = maxIter + 2;
  }
  std::memcpy(out->P, P, sizeof(P));
}

struct Sub1Out {
  double U[2];
  int conv;
  bool error;
};

// funICGN_Subpb1quadtree (func_quadtree/funICGN_Subpb1quadtree.m:1-476): ALDIC
// augmented-Lagrangian local step, translation only, F fixed at FOld.
void fun_subpb1_quadtree(const Frame& fr, double x0, double y0, int wx_in, int wy_in, double mu,
                         const double vdual[2], const double UOld[2], const double FOld[4], double tol,
                         Sub1Out* out) {
  const int maxIter = 100;
  out->error = false;
  double P[6] = {FOld[0], FOld[1], FOld[2], FOld[3], UOld[0], UOld[1]};
  out->U[0] = P[4];
  out->U[1] = P[5];
  double wx = wx_in, wy = wy_in;
  Window W;
  if (!slice(fr, x0 - wx / 2, x0 + wx / 2, y0 - wy / 2, y0 + wy / 2, true, &W)) {
    out->error = true;
    return;
  }
  std::vector<double> tf(W.f.size());
  for (size_t k = 0; k < tf.size(); ++k) tf[k] = W.f[k] * W.fmask[k];
  long cnt = 0;
  for (double v : tf) {
    if (std::isnan(v)) {
      out->error = true;
      return;
    }
    cnt += (v == 0);
  }
  if (cnt < 0.4 * (wx + 1) * (wy + 1)) {
    if (cnt > 0) {
      // :78-79 (the second line uses the already-updated winsize_x)
      wx = 2 * std::ceil(std::sqrt((wx + 1) * (wy + 1) / ((wx + 1) * (wy + 1) - cnt)) * wx / 2);
      wy = 2 * std::ceil(std::sqrt((wx + 1) * (wy + 1) / ((wx + 1) * (wy + 1) - cnt)) * wy / 2);
      if (!slice(fr, x0 - wx / 2, x0 + wx / 2, y0 - wy / 2, y0 + wy / 2, true, &W)) {
        out->error = true;
        return;
      }
      tf.resize(W.f.size());
      for (size_t k = 0; k < tf.size(); ++k) tf[k] = W.f[k] * W.fmask[k];
    }
    // bwselect(BW, c, r, n): column seed from winsize_x, row seed from winsize_y (:93).
    const int sc = (int)std::floor((wx + 1) / 2) - 1;
    const int sr = (int)std::floor((wy + 1) / 2) - 1;
    std::vector<uint8_t> mbw(W.fmask.size()), bw4;
    for (size_t k = 0; k < mbw.size(); ++k) mbw[k] = (W.fmask[k] != 0);
    bwselect(mbw, W.rows, W.cols, sr, sc, 4, &bw4);
    std::vector<double> gx = W.gx, gy = W.gy;
    for (size_t k = 0; k < tf.size(); ++k) {
      tf[k] *= bw4[k];
      gx[k] *= bw4[k];
      gy[k] *= bw4[k];
    }
    auto hess2 = [&](const std::vector<double>& ax, const std::vector<double>& ay, double Hm[4]) {
      double a = 0, b = 0, c = 0;
      for (size_t k = 0; k < ax.size(); ++k) {
        a += ax[k] * ax[k];
        b += ax[k] * ay[k];
        c += ay[k] * ay[k];
      }
      Hm[0] = a;
      Hm[1] = b;
      Hm[2] = b;
      Hm[3] = c;
    };
    double H[4];
    hess2(gx, gy, H);
    double meanf, bf;
    mean_bottom(tf, nullptr, 1e-10, &meanf, &bf);
    double H2[4] = {H[0] * 2 / (bf * bf) + mu, H[1] * 2 / (bf * bf), H[2] * 2 / (bf * bf), H[3] * 2 / (bf * bf) + mu};
    double normNew = 1, normAbs = 1, normInit = 0;
    int step = 0;
    std::vector<double> g;
    std::vector<uint8_t> gbw;
    while (step <= 100 && normNew > tol && normAbs > tol) {
      ++step;
      if (!warp_interp(fr, W, x0, y0, P, &g)) {
        normNew = 1e6;
        break;
      }
      long gcnt = 0;
      for (double v : g) {
        if (std::isnan(v)) {
          out->error = true;
          out->U[0] = P[4];
          out->U[1] = P[5];
          return;
        }
        gcnt += (v == 0);
      }
      if (cnt > 0 || gcnt > 0) {
        std::vector<uint8_t> gl(g.size());
        for (size_t k = 0; k < g.size(); ++k) gl[k] = (g[k] != 0);
        bwselect(gl, W.rows, W.cols, sr, sc, 4, &gbw);
        bool all_on = true;
        for (uint8_t v : gbw) all_on = all_on && v;
        if (all_on) bwselect(mbw, W.rows, W.cols, sr, sc, 8, &gbw);
        for (size_t k = 0; k < g.size(); ++k) {
          g[k] *= gbw[k];
          tf[k] = W.f[k] * W.fmask[k] * gbw[k];
          gx[k] = W.gx[k] * gbw[k];
          gy[k] = W.gy[k] * gbw[k];
        }
        hess2(gx, gy, H);
        mean_bottom(tf, nullptr, 1e-10, &meanf, &bf);
        H2[0] = H[0] * 2 / (bf * bf) + mu;
        H2[1] = H[1] * 2 / (bf * bf);
        H2[2] = H[2] * 2 / (bf * bf);
        H2[3] = H[3] * 2 / (bf * bf) + mu;
      }
      double meang, bg;
      mean_bottom(g, nullptr, 1e-10, &meang, &bg);
      double b2[2] = {0, 0};
      for (size_t k = 0; k < g.size(); ++k) {
        const double r = (tf[k] - meanf) / bf - (g[k] - meang) / bg;
        b2[0] += gx[k] * r;
        b2[1] += gy[k] * r;
      }
      const double b[2] = {bf * b2[0], bf * b2[1]};
      double tb[2] = {b[0] * 2 / (bf * bf) + mu * (P[4] - UOld[0] - vdual[0]),
                      b[1] * 2 / (bf * bf) + mu * (P[5] - UOld[1] - vdual[1])};
      const double delta = 1e-3 * std::max(H2[0], H2[3]);
      double tH[4] = {H2[0] + delta, H2[1], H2[2], H2[3] + delta};
      double nb[2] = {-tb[0], -tb[1]}, d56[2];
      solve_dense(2, tH, nb, d56);
      normNew = norm6(tb, 2);
      normAbs = normNew;
      if (step == 1) normInit = normNew;
      if (normInit > tol) normNew = normNew / normInit;
      else normNew = 0;
      if (normNew < tol || normAbs < tol) break;
      const double dP[6] = {0, 0, 0, 0, d56[0], d56[1]};
      if (!compose_inverse(P, dP)) break;
    }
    if (!(normNew < tol || normAbs < tol)) step = maxIter + 1;
    if (std::isnan(normNew)) step = maxIter + 1;
    double sabs = 0;
    for (double v : tf) sabs += std::fabs(v);
    if (sabs < 1e-6) step = maxIter + 3;
    out->conv = step;
  } else {
    out->conv = 102;
  }
  out->U[0] = P[4];
  out->U[1] = P[5];
}

// funICGN_Subpb1 (func/funICGN_Subpb1.m): uniform-mesh ALDIC local step; H2 from the
// stored Hessian block H(5:6,5:6).
void fun_subpb1_uniform(const Frame& fr, double x0, double y0, int winsize, double mu, const double H56[3],
                        const double vdual[2], const double UOld[2], const double FOld[4], double tol,
                        Sub1Out* out) {
  out->error = false;
  double P[6] = {FOld[0], FOld[1], FOld[2], FOld[3], UOld[0], UOld[1]};
  out->U[0] = P[4];
  out->U[1] = P[5];
  double w = winsize;
  Window W;
  if (!slice(fr, x0 - w / 2, x0 + w / 2, y0 - w / 2, y0 + w / 2, true, &W)) {
    out->error = true;
    return;
  }
  const double Nw = (w + 1) * (w + 1);
  long zc = 0;
  for (double v : W.gx) zc += (v == 0);
  if (zc < 0.5 * Nw) {
    if (zc > 0.1 * Nw) {
      w = std::round(std::sqrt(2.0) * w);
      if (!slice(fr, x0 - w / 2, x0 + w / 2, y0 - w / 2, y0 + w / 2, true, &W)) {
        out->error = true;
        return;
      }
    }
    double meanf, bf;
    mean_bottom(W.f, nullptr, -1, &meanf, &bf);
    double normNew = 1, normAbs = 1, normInit = 0;
    int step = 0;
    std::vector<double> g;
    while (step <= 100 && normNew > tol && normAbs > tol) {
      ++step;
      if (!warp_interp(fr, W, x0, y0, P, &g)) {
        normNew = 1e6;
        break;
      }
      double meang, bg;
      mean_bottom(g, nullptr, -1, &meang, &bg);
      double b2[2] = {0, 0};
      for (size_t k = 0; k < g.size(); ++k) {
        const double r = (W.f[k] - meanf) / bf - (g[k] - meang) / bg;
        b2[0] += W.gx[k] * r;
        b2[1] += W.gy[k] * r;
      }
      const double b[2] = {bf * b2[0], bf * b2[1]};
      double tb[2] = {b[0] * 2 / (bf * bf) + mu * (P[4] - UOld[0] - vdual[0]),
                      b[1] * 2 / (bf * bf) + mu * (P[5] - UOld[1] - vdual[1])};
      const double H2[4] = {H56[0] * 2 / (bf * bf) + mu, H56[1] * 2 / (bf * bf), H56[1] * 2 / (bf * bf),
                            H56[2] * 2 / (bf * bf) + mu};
      const double delta = 1e-3 * std::max(H2[0], H2[3]);
      double tH[4] = {H2[0] + delta, H2[1], H2[2], H2[3] + delta};
      double nb[2] = {-tb[0], -tb[1]}, d56[2];
      solve_dense(2, tH, nb, d56);
      normNew = norm6(tb, 2);
      normAbs = normNew;
      if (step == 1) normInit = normNew;
      if (normInit > tol) normNew = normNew / normInit;
      else normNew = 0;
      if (normNew < tol || normAbs < tol) break;
      const double dP[6] = {0, 0, 0, 0, d56[0], d56[1]};
      if (!compose_inverse(P, dP)) break;
    }
    if (!(normNew < tol || normAbs < tol)) step = 101;
    if (std::isnan(normNew)) step = 101;
    out->conv = step;
  } else {
    out->conv = 102;
  }
  out->U[0] = P[4];
  out->U[1] = P[5];
}

// ---------------------------------------------------------------------------------
// normxcorr2 (Image Processing Toolbox; Lewis, "Fast Normalized Cross-Correlation",
// 1995) restated from its published definition: full-size output, A zero-padded,
// numerator sum(T.*A_w) - sum(A_w)*sum(T)/mn, denominator
// sqrt(sum((T-Tbar)^2)) * sqrt(max(sum(A_w^2) - sum(A_w)^2/mn, 0)); entries whose
// denominator is <= sqrt(eps(max denominator)) are 0, and |C| > 1 + sqrt(eps(1)) -> 0.
// T: m x n, A: ma x na, out: (ma+m-1) x (na+n-1) column-major.
// ---------------------------------------------------------------------------------
bool normxcorr2(const double* T, int m, int n, const double* A, int ma, int na, std::vector<double>* out) {
  if (m > ma || n > na) return false;
  const double mn = (double)m * n;
  double sT = 0;
  for (int k = 0; k < m * n; ++k) sT += T[k];
  const double Tbar = sT / mn;
  double ssT = 0;
  for (int k = 0; k < m * n; ++k) ssT += (T[k] - Tbar) * (T[k] - Tbar);
  const double denomT = std::sqrt(ssT);
  if (!(denomT != 0)) return false;  // constant template: normxcorr2 throws
  const int R = ma + m - 1, C = na + n - 1;
  out->assign((size_t)R * C, 0.0);
  std::vector<double> num((size_t)R * C), den((size_t)R * C);
  double dmax = 0;
  for (int oc = 0; oc < C; ++oc)
    for (int orr = 0; orr < R; ++orr) {
      // template top-left at A(orr - m + 1, oc - n + 1)
      const int ar0 = orr - m + 1, ac0 = oc - n + 1;
      double sTA = 0, sA = 0, sAA = 0;
      for (int j = 0; j < n; ++j) {
        const int ac = ac0 + j;
        if (ac < 0 || ac >= na) continue;
        for (int i = 0; i < m; ++i) {
          const int ar = ar0 + i;
          if (ar < 0 || ar >= ma) continue;
          const double a = A[ar + (size_t)ac * ma];
          sTA += T[i + (size_t)j * m] * a;
          sA += a;
          sAA += a * a;
        }
      }
      const size_t k = orr + (size_t)oc * R;
      num[k] = sTA - sA * sT / mn;
      const double dA = std::sqrt(std::max(sAA - sA * sA / mn, 0.0));
      den[k] = denomT * dA;
      dmax = std::max(dmax, std::fabs(den[k]));
    }
  const double tolz = std::sqrt(matlab_eps(dmax));
  const double one_tol = std::sqrt(matlab_eps(1.0));
  for (size_t k = 0; k < num.size(); ++k) {
    double c = 0;
    if (den[k] > tolz) c = num[k] / den[k];
    if (std::fabs(c) - 1 > one_tol) c = 0;
    (*out)[k] = c;
  }
  return true;
}

// findpeak (func/findpeak.m:27-66) with subpixel = 1.  f: r x c column-major.
// Returns 1-based (xpeak = column, ypeak = row) and max_f.
void findpeak(const double* f, int r, int c, double* xpeak, double* ypeak, double* max_f) {
  long imax = 0;
  double best = f[0];
  for (long k = 1; k < (long)r * c; ++k)
    if (f[k] > best || (std::isnan(best) && !std::isnan(f[k]))) {
      best = f[k];
      imax = k;
    }
  const int row = (int)(imax % r) + 1, col = (int)(imax / r) + 1;
  *max_f = best;
  *xpeak = col;
  *ypeak = row;
  if (col == 1 || col == c || row == 1 || row == r) return;
  // 9 samples u(dx, dy), dx = column offset, dy = row offset (:37-40)
  auto U = [&](int dx, int dy) { return f[(row - 1 + dy) + (size_t)(col - 1 + dx) * r]; };
  double S = 0, Sx2 = 0, Sy2 = 0, Sx = 0, Sy = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy) {
      const double u = U(dx, dy);
      S += u;
      Sx += dx * u;
      Sy += dy * u;
      if (dx != 0) Sx2 += u;
      if (dy != 0) Sy2 += u;
    }
  // least-squares fit u = A1 + A2 x + A3 y + A4 xy + A5 x^2 + A6 y^2 on the 3x3 grid
  const double A2 = Sx / 6.0, A3 = Sy / 6.0;
  const double A4 = (U(1, 1) - U(1, -1) - U(-1, 1) + U(-1, -1)) / 4.0;
  const double A5 = Sx2 / 2.0 - S / 3.0, A6 = Sy2 / 2.0 - S / 3.0;
  const double A1 = (5.0 * S - 3.0 * (Sx2 + Sy2)) / 9.0;
  const double den = A4 * A4 - 4 * A5 * A6;
  double xo = (-A3 * A4 + 2 * A6 * A2) / den;
  double yo = -1 / den * (A4 * A2 - 2 * A5 * A3);
  if (std::fabs(xo) > 1 || std::fabs(yo) > 1) return;
  xo = std::round(1000 * xo) / 1000;
  yo = std::round(1000 * yo) / 1000;
  *xpeak = col + xo;
  *ypeak = row + yo;
  *max_f = A1 + A2 * xo + A3 * yo + A4 * xo * yo + A5 * xo * xo + A6 * yo * yo;
}

// q-factors of one cross-correlation map (func/funIntegerSearch.m:211-264): PCE and PPE.
// PPE uses 30 equal-width bins over [0, max]; MATLAB's histcounts places "nice" edges,
// which is not reproduced (PPE parity is unpinned).
void qfactors(const std::vector<double>& cc, double* pce, double* ppe) {
  double mn = cc[0];
  for (double v : cc) mn = std::min(mn, v);
  std::vector<double> m(cc.size());
  double peak = 0, s2 = 0;
  for (size_t k = 0; k < cc.size(); ++k) {
    m[k] = cc[k] - mn;
    peak = std::max(peak, m[k]);
    s2 += m[k] * m[k];
  }
  *pce = peak * peak / (s2 / cc.size());
  long hist[30] = {};
  for (double v : m) {
    int b = (peak > 0) ? (int)std::floor(v / peak * 30) : 0;
    if (b >= 30) b = 29;
    if (b < 0) b = 0;
    hist[b]++;
  }
  double ent = 0;
  for (int b = 0; b < 30; ++b) {
    const double p = (double)hist[b] / cc.size();
    if (p > 0) ent += p * std::log(1 / p);
  }
  *ppe = 1 / ent;
}

}  // namespace

extern "C" {

int orc_abi_version() { return 1; }

// Interpolate F (M x N) at (X = dim-2, Y = dim-1) 1-based coordinates
// (ba_interp2_spline.cpp:235-331, called as ba_interp2_spline(F, v22, u22)).
void orc_interp(const double* F, int M, int N, const double* X, const double* Y, long n, double* out) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) out[i] = interp_local(F, M, N, X[i], Y[i]);
}

// funNormalizeImg (func/funNormalizeImg.m:109-127): ROI clamp, mean/std (N-1) over the
// ROI, out = (img - mean) / std.  gridx/gridy are 1-based inclusive ROI ranges.
void orc_normalize(const double* img, int M, int N, const int* gridx_in, const int* gridy_in, double* out,
                   double* mean_std) {
  int gx0 = gridx_in[0], gx1 = gridx_in[1], gy0 = gridy_in[0], gy1 = gridy_in[1];
  if (gx0 < 1) gx0 = 1;
  if (gx1 > M) gx1 = M;
  if (gy0 < 1) gy0 = 1;
  if (gy1 > N) gy1 = N;
  double s = 0;
  long cnt = 0;
  for (int j = gy0 - 1; j < gy1; ++j)
    for (int i = gx0 - 1; i < gx1; ++i) {
      s += img[i + (size_t)j * M];
      ++cnt;
    }
  const double mean = s / cnt;
  double ss = 0;
  for (int j = gy0 - 1; j < gy1; ++j)
    for (int i = gx0 - 1; i < gx1; ++i) {
      const double d = img[i + (size_t)j * M] - mean;
      ss += d * d;
    }
  const double sd = std::sqrt(ss / (cnt - 1));
  for (size_t k = 0; k < (size_t)M * N; ++k) out[k] = (img[k] - mean) / sd;
  if (mean_std) {
    mean_std[0] = mean;
    mean_std[1] = sd;
  }
}

// funImgGradient (func/funImgGradient.m:50-78): 7-tap central difference
// [-1/60 3/20 -3/4 0 3/4 -3/20 1/60] along dim 1 (dfdx) and dim 2 (dfdy), cropped by 3,
// times mask(4:M-3, 4:N-3).  Outputs are (M-6) x (N-6).
void orc_gradient(const double* img, const double* mask, int M, int N, double* dfdx, double* dfdy) {
  const double h[7] = {-1.0 / 60, 3.0 / 20, -3.0 / 4, 0.0, 3.0 / 4, -3.0 / 20, 1.0 / 60};
  const int gM = M - 6, gN = N - 6;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < gN; ++j)
    for (int i = 0; i < gM; ++i) {
      const int ci = i + 3, cj = j + 3;
      double sx = 0, sy = 0;
      for (int k = 0; k < 7; ++k) {
        sx += h[k] * img[(ci - 3 + k) + (size_t)cj * M];
        sy += h[k] * img[ci + (size_t)(cj - 3 + k) * M];
      }
      const double mk = mask ? mask[ci + (size_t)cj * M] : 1.0;
      dfdx[i + (size_t)j * gM] = sx * mk;
      dfdy[i + (size_t)j * gM] = sy * mk;
    }
}

// Batched local IC-GN over n subsets, i.e. the loop bodies of
//   variant 0: LocalICGN         (func/LocalICGN.m:64-164, solver func/funICGN.m)
//   variant 1: LocalICGNQuadtree (func_quadtree/LocalICGNQuadtree.m:67-164, solver
//              func_quadtree/funICGNQuadtree.m)
// coords: n x 2 column-major; U0/U: 2n interleaved; F: 4n interleaved; H: n x 21
// column-major; conv: n; markHole (variant 1 only, may be null): n.
// A solver error gives conv = -1 and U = F = NaN, as the drivers' catch blocks do.
void orc_local_icgn_guess(int variant, const double* ref, const double* def, const double* mask, const double* dfdx,
                          const double* dfdy, int M, int N, long n, const double* coords, const double* U0,
                          const double* F0, int winsize, double tol, double* U, double* F, double* H, int* conv,
                          uint8_t* markHole, int nthreads);

void orc_local_icgn(int variant, const double* ref, const double* def, const double* mask, const double* dfdx,
                    const double* dfdy, int M, int N, long n, const double* coords, const double* U0, int winsize,
                    double tol, double* U, double* F, double* H, int* conv, uint8_t* markHole, int nthreads) {
  orc_local_icgn_guess(variant, ref, def, mask, dfdx, dfdy, M, N, n, coords, U0, nullptr, winsize, tol, U, F, H, conv,
                       markHole, nthreads);
}

// orc_local_icgn from the initial guesses [F0 U0] (F0 4n, or null for the reference's zero).
void orc_local_icgn_guess(int variant, const double* ref, const double* def, const double* mask, const double* dfdx,
                          const double* dfdy, int M, int N, long n, const double* coords, const double* U0,
                          const double* F0, int winsize, double tol, double* U, double* F, double* H, int* conv,
                          uint8_t* markHole, int nthreads) {
  Frame fr{ref, def, mask, dfdx, dfdy, M, N, 3};
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 4)
  for (long t = 0; t < n; ++t) {
    double x0 = coords[t], y0 = coords[n + t];
    if (variant == 1) {
      x0 = std::round(x0);
      y0 = std::round(y0);
      if (markHole) {
        // :73-86 hole-strain mark from the uniform window
        const double w = winsize;
        Window Wm;
        uint8_t mk = 0;
        if (!slice(fr, x0 - w / 2, x0 + w / 2, y0 - w / 2, y0 + w / 2, false, &Wm)) mk = 1;
        else {
          long c = 0;
          for (size_t k = 0; k < Wm.f.size(); ++k) c += (Wm.f[k] * Wm.fmask[k] == 0);
          if (c > 0.6 * (w + 1) * (w + 1)) mk = 1;
        }
        markHole[t] = mk;
      }
    }
    IcgnOut o;
    const double u0[2] = {U0[2 * t], U0[2 * t + 1]};
    const double* f0 = F0 ? F0 + 4 * t : nullptr;
    if (variant == 1) fun_icgn_quadtree(fr, u0, x0, y0, winsize, tol, &o, f0);
    else fun_icgn(fr, u0, x0, y0, winsize, tol, 100, false, &o, nullptr, f0);
    if (o.error) {
      conv[t] = -1;
      U[2 * t] = U[2 * t + 1] = kNaN;
      for (int k = 0; k < 4; ++k) F[4 * t + k] = kNaN;
      for (int k = 0; k < 21; ++k) H[t + n * k] = 0;  // HtempPar row keeps its zeros
    } else {
      conv[t] = o.conv;
      U[2 * t] = o.P[4];
      U[2 * t + 1] = o.P[5];
      F[4 * t + 0] = o.P[0];
      F[4 * t + 1] = o.P[1];
      F[4 * t + 2] = o.P[2];
      F[4 * t + 3] = o.P[3];
      pack_h21(o.H, H, n, t);
    }
  }
}

// Batched ALDIC Subpb1 local step, the loop bodies of
//   variant 0: Subpb1          (func/Subpb1.m, solver func/funICGN_Subpb1.m); H56 from
//              HPar (n x 21, entries (5,5),(6,5),(6,6)); error -> conv -1, U NaN
//   variant 1: Subpb1Quadtree  (func_quadtree/Subpb1Quadtree.m:71-126, solver
//              func_quadtree/funICGN_Subpb1quadtree.m); error -> conv 0, U NaN
// winsize_xy: n x 2 column-major (winsize_List) for variant 1.
void orc_subpb1(int variant, const double* ref, const double* def, const double* mask, const double* dfdx,
                const double* dfdy, int M, int N, long n, const double* coords, const double* UOld,
                const double* FOld, const double* vdual, const int* winsize_xy, int winsize, const double* HPar,
                double mu, double tol, double* U, int* conv, int nthreads) {
  Frame fr{ref, def, mask, dfdx, dfdy, M, N, 3};
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 4)
  for (long t = 0; t < n; ++t) {
    double x0 = coords[t], y0 = coords[n + t];
    Sub1Out o;
    const double uo[2] = {UOld[2 * t], UOld[2 * t + 1]};
    const double fo[4] = {FOld[4 * t], FOld[4 * t + 1], FOld[4 * t + 2], FOld[4 * t + 3]};
    const double vd[2] = {vdual[2 * t], vdual[2 * t + 1]};
    if (variant == 1) {
      x0 = std::round(x0);
      y0 = std::round(y0);
      fun_subpb1_quadtree(fr, x0, y0, winsize_xy[t], winsize_xy[n + t], mu, vd, uo, fo, tol, &o);
    } else {
      double h56[3] = {0, 0, 0};
      if (HPar) {
        h56[0] = HPar[t + n * 18];
        h56[1] = HPar[t + n * 19];
        h56[2] = HPar[t + n * 20];
      }
      fun_subpb1_uniform(fr, x0, y0, winsize, mu, h56, vd, uo, fo, tol, &o);
    }
    if (o.error) {
      conv[t] = (variant == 1) ? 0 : -1;
      U[2 * t] = U[2 * t + 1] = kNaN;
    } else {
      conv[t] = o.conv;
      U[2 * t] = o.U[0];
      U[2 * t + 1] = o.U[1];
    }
  }
}

// epipolar_ICGN1 (func/epipolar_ICGN1.m:1-253) for n candidate points: IC-GN from P = 0
// with P5 = P6 held at 0, at most 30 iterations, gradient offset Df.DfAxis start (4);
// returns the ZNSSD of the final iteration (NaN when the solver errors or leaves the image).
void orc_epipolar_icgn(const double* ref, const double* def, const double* dfdx, const double* dfdy, int M, int N,
                       long n, const double* pts, int winsize, double tol, double* znssd, int* conv, int nthreads) {
  Frame fr{ref, def, nullptr, dfdx, dfdy, M, N, 4};
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 4)
  for (long t = 0; t < n; ++t) {
    IcgnOut o;
    const double u0[2] = {0, 0};
    std::vector<double> z;
    fun_icgn(fr, u0, pts[t], pts[n + t], winsize, tol, 30, true, &o, &z);
    conv[t] = o.error ? -1 : o.conv;
    znssd[t] = (o.error || z.empty()) ? kNaN : z.back();
  }
}

// Grid of funIntegerSearchWholeField (func/funIntegerSearch.m:106-107).
void orc_search_grid(const int* gridx, const int* gridy, int winsize, int step, int* nx, int* ny) {
  const int ex = gridx[1] - winsize - step, ey = gridy[1] - winsize - step;
  *nx = ex >= gridx[0] ? (ex - gridx[0]) / step + 1 : 0;
  *ny = ey >= gridy[0] ? (ey - gridy[0]) / step + 1 : 0;
}

// funIntegerSearchWholeField (func/funIntegerSearch.m:100-203): per grid subset
// normxcorr2 of the template f(ii:ii+w, jj:jj+w) against the border-clamped window of g,
// crop [w : end-w+1], findpeak; search = tempSizeOfSearchRegion as passed (length 2,
// expanded to [left right up down] = [s0 s1 s0 s1] at :12).  Outputs are nY x nX
// column-major (x, y, u, v, phi) and qf (nX*nY x 2, normalised as :184-187).
// One subset of funIntegerSearchWholeField (func/funIntegerSearch.m:134-176): template
// top-left (ii, jj) 1-based; gridx_end/gridy_end are gridx(end)/gridy(end) used by the
// right/down clamps.  out5 = [u v phi pce ppe] (NaN / Inf on failure).
static void search_one(const double* f, const double* g, int M, int N, const int* search, int gridx_end,
                       int gridy_end, int ii, int jj, int w, double* out5) {
  int L = search[0], R = search[1], Uu = search[0], D = search[1];
  if (ii - L < 1) L = ii - 1;
  if (jj - Uu < 1) Uu = jj - 1;
  if (ii + w + R > M) R = gridx_end - ii - w - 1;
  if (jj + w + D > N) D = gridy_end - jj - w - 1;
  L = std::max(L, 0);
  R = std::max(R, 0);
  Uu = std::max(Uu, 0);
  D = std::max(D, 0);
  out5[0] = out5[1] = out5[2] = kNaN;
  out5[3] = out5[4] = INFINITY;
  const int m = w + 1;
  const int ar0 = ii - L, ar1 = ii + w + R, ac0 = jj - Uu, ac1 = jj + w + D;
  if (!(ii >= 1 && ii + w <= M && jj >= 1 && jj + w <= N && ar0 >= 1 && ar1 <= M && ac0 >= 1 && ac1 <= N)) return;
  std::vector<double> T((size_t)m * m), A((size_t)(ar1 - ar0 + 1) * (ac1 - ac0 + 1));
  for (int b = 0; b < m; ++b)
    for (int a = 0; a < m; ++a) T[a + (size_t)b * m] = f[(ii - 1 + a) + (size_t)(jj - 1 + b) * M];
  const int ma = ar1 - ar0 + 1, na = ac1 - ac0 + 1;
  for (int b = 0; b < na; ++b)
    for (int a = 0; a < ma; ++a) A[a + (size_t)b * ma] = g[(ar0 - 1 + a) + (size_t)(ac0 - 1 + b) * M];
  std::vector<double> cc;
  if (!normxcorr2(T.data(), m, m, A.data(), ma, na, &cc)) return;
  qfactors(cc, &out5[3], &out5[4]);
  const int R2 = ma + m - 1, C2 = na + m - 1;
  const int cr = R2 - 2 * w + 2, ccn = C2 - 2 * w + 2;
  std::vector<double> crop((size_t)cr * ccn);
  for (int b = 0; b < ccn; ++b)
    for (int a = 0; a < cr; ++a) crop[a + (size_t)b * cr] = cc[(w - 1 + a) + (size_t)(w - 1 + b) * R2];
  double xp, yp, mf;
  findpeak(crop.data(), cr, ccn, &xp, &yp, &mf);
  out5[0] = yp - 2 - L;
  out5[1] = xp - 2 - Uu;
  out5[2] = mf;
}

// The same subset as search_one for whole-grid checks, computed only where the result needs
// it: normxcorr2's numerator and local sums over the crop (func/funIntegerSearch.m:166) in
// the same summation order as normxcorr2() above (template column outer, row inner; zero
// padding adds exact zeros where the overlap is partial), so u, v and phi are bit-identical
// to search_one's; the zero threshold takes the largest denominator of the full output from
// box sums (it enters only through eps(dmax), a power of two).  Eight consecutive shifts of
// a crop column are independent accumulators held together (no sum is reordered).
// out4 = [u v phi margin], margin = the crop's largest NCC minus its second largest.
namespace {
// num / sa / saa of crop rows d0 .. d0 + 7 of one crop column: per shift the sums over the
// template in normxcorr2()'s order; the 8 shifts are independent accumulators.
__attribute__((target_clones("avx2", "default"))) void crop_block8(const double* P, int Pm, const double* T, int m,
                                                                  int row0, int col0, double* num, double* sa,
                                                                  double* saa) {
  double na[8] = {0, 0, 0, 0, 0, 0, 0, 0}, s1[8] = {0, 0, 0, 0, 0, 0, 0, 0}, s2[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) {
      const double t = T[i + (size_t)j * m];
      const double* a = P + (row0 + i) + (size_t)(col0 + j) * Pm;
      for (int k = 0; k < 8; ++k) {
        const double v = a[k];
        na[k] += t * v;
        s1[k] += v;
        s2[k] += v * v;
      }
    }
  for (int k = 0; k < 8; ++k) {
    num[k] = na[k];
    sa[k] = s1[k];
    saa[k] = s2[k];
  }
}
}  // namespace

static void search_fast_one(const double* f, const double* g, int M, int N, const int* search, int gridx_end,
                            int gridy_end, int ii, int jj, int w, double* out4) {
  int L = search[0], R = search[1], Uu = search[0], D = search[1];
  if (ii - L < 1) L = ii - 1;
  if (jj - Uu < 1) Uu = jj - 1;
  if (ii + w + R > M) R = gridx_end - ii - w - 1;
  if (jj + w + D > N) D = gridy_end - jj - w - 1;
  L = std::max(L, 0);
  R = std::max(R, 0);
  Uu = std::max(Uu, 0);
  D = std::max(D, 0);
  out4[0] = out4[1] = out4[2] = out4[3] = kNaN;
  const int m = w + 1;
  const int ar0 = ii - L, ar1 = ii + w + R, ac0 = jj - Uu, ac1 = jj + w + D;
  if (!(ii >= 1 && ii + w <= M && jj >= 1 && jj + w <= N && ar0 >= 1 && ar1 <= M && ac0 >= 1 && ac1 <= N)) return;
  const int ma = ar1 - ar0 + 1, na = ac1 - ac0 + 1;
  if (m > ma || m > na) return;
  std::vector<double> T((size_t)m * m);
  for (int b = 0; b < m; ++b)
    for (int a = 0; a < m; ++a) T[a + (size_t)b * m] = f[(ii - 1 + a) + (size_t)(jj - 1 + b) * M];
  const double mn = (double)m * m;
  double sT = 0;
  for (int k = 0; k < m * m; ++k) sT += T[k];
  const double Tbar = sT / mn;
  double ssT = 0;
  for (int k = 0; k < m * m; ++k) ssT += (T[k] - Tbar) * (T[k] - Tbar);
  const double denomT = std::sqrt(ssT);
  if (!(denomT != 0)) return;
  // window zero-padded by m - 1 on every side: full-output position (r, c) has its template
  // top-left at padded (r, c)
  const int R2 = ma + m - 1, C2 = na + m - 1;
  const int Pm = ma + 2 * (m - 1), Pn = na + 2 * (m - 1);
  std::vector<double> Pd((size_t)Pm * Pn + 8, 0.0);  // + 8: the last block of 8 shifts reads past the end
  for (int b = 0; b < na; ++b)
    for (int a = 0; a < ma; ++a)
      Pd[(m - 1 + a) + (size_t)(m - 1 + b) * Pm] = g[(ar0 - 1 + a) + (size_t)(ac0 - 1 + b) * M];
  // largest denominator over the full output (box sums: column sums, then across columns)
  double dmax = 0;
  {
    std::vector<double> cs((size_t)R2 * Pn), cs2((size_t)R2 * Pn);
    for (int c = 0; c < Pn; ++c)
      for (int r = 0; r < R2; ++r) {
        double s1 = 0, s2 = 0;
        for (int i = 0; i < m; ++i) {
          const double v = Pd[(r + i) + (size_t)c * Pm];
          s1 += v;
          s2 += v * v;
        }
        cs[r + (size_t)c * R2] = s1;
        cs2[r + (size_t)c * R2] = s2;
      }
    for (int c = 0; c < C2; ++c)
      for (int r = 0; r < R2; ++r) {
        double s1 = 0, s2 = 0;
        for (int j = 0; j < m; ++j) {
          s1 += cs[r + (size_t)(c + j) * R2];
          s2 += cs2[r + (size_t)(c + j) * R2];
        }
        dmax = std::max(dmax, std::fabs(denomT * std::sqrt(std::max(s2 - s1 * s1 / mn, 0.0))));
      }
  }
  const double tolz = std::sqrt(matlab_eps(dmax));
  const double one_tol = std::sqrt(matlab_eps(1.0));
  // the crop: full-output rows / columns w-1 .. (its first and last are partial overlaps)
  const int cr = R2 - 2 * w + 2, ccn = C2 - 2 * w + 2;
  const int crp = (cr + 7) / 8 * 8;
  std::vector<double> crop((size_t)cr * ccn), num(crp), sa(crp), saa(crp);
  for (int b = 0; b < ccn; ++b) {
    for (int d0 = 0; d0 < cr; d0 += 8)
      crop_block8(Pd.data(), Pm, T.data(), m, w - 1 + d0, w - 1 + b, &num[d0], &sa[d0], &saa[d0]);
    for (int a = 0; a < cr; ++a) {
      const double nm = num[a] - sa[a] * sT / mn;
      const double den = denomT * std::sqrt(std::max(saa[a] - sa[a] * sa[a] / mn, 0.0));
      double c = 0;
      if (den > tolz) c = nm / den;
      if (std::fabs(c) - 1 > one_tol) c = 0;
      crop[a + (size_t)b * cr] = c;
    }
  }
  double xp, yp, mf;
  findpeak(crop.data(), cr, ccn, &xp, &yp, &mf);
  // margin: the largest crop value minus the second largest
  double b1 = -INFINITY, b2 = -INFINITY;
  for (double v : crop) {
    if (v > b1) {
      b2 = b1;
      b1 = v;
    } else if (v > b2) {
      b2 = v;
    }
  }
  out4[0] = yp - 2 - L;
  out4[1] = xp - 2 - Uu;
  out4[2] = mf;
  out4[3] = b1 - b2;
}

void orc_search_check(const double* f, const double* g, int M, int N, const int* search, int gridx_end, int gridy_end,
                      long n, const int* ii, const int* jj, int w, double* out, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 2)
  for (long k = 0; k < n; ++k) search_fast_one(f, g, M, N, search, gridx_end, gridy_end, ii[k], jj[k], w, out + 4 * k);
}

// A list of grid subsets (template top-lefts ii[k], jj[k]) searched in parallel, for
// sampled checks and CPU timing; out is n x 5 row-major [u v phi pce ppe].
void orc_search_list(const double* f, const double* g, int M, int N, const int* search, int gridx_end,
                     int gridy_end, long n, const int* ii, const int* jj, int w, double* out, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (long k = 0; k < n; ++k) search_one(f, g, M, N, search, gridx_end, gridy_end, ii[k], jj[k], w, out + 5 * k);
}

void orc_integer_search(const double* f, const double* g, int M, int N, const int* search, const int* gridx,
                        const int* gridy, int winsize, int step, double* x, double* y, double* u, double* v,
                        double* phi, double* qf, int nthreads) {
  int nX, nY;
  orc_search_grid(gridx, gridy, winsize, step, &nX, &nY);
  const long n = (long)nX * nY;
  const int w = winsize;
  std::vector<double> q0(n), q1(n);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 2)
  for (long t = 0; t < n; ++t) {
    const int i = (int)(t % nX), j = (int)(t / nX);
    const int ii = gridx[0] + i * step, jj = gridy[0] + j * step;
    double r5[5];
    search_one(f, g, M, N, search, gridx[1], gridy[1], ii, jj, w, r5);
    const double uu = r5[0], vv = r5[1], pp = r5[2], qa = r5[3], qb = r5[4];
    const long o = j + (long)i * nY;
    u[o] = uu;
    v[o] = vv;
    phi[o] = pp;
    x[o] = (ii + ii + w) / 2.0;
    y[o] = (jj + jj + w) / 2.0;
    q0[t] = qa;
    q1[t] = qb;
  }
  if (qf) {
    for (int k = 0; k < 2; ++k) {
      std::vector<double>& q = k ? q1 : q0;
      double mn = INFINITY;
      for (double vq : q)
        if (!std::isnan(vq)) mn = std::min(mn, vq);
      double mx = -INFINITY;
      for (double vq : q)
        if (!std::isnan(vq)) mx = std::max(mx, vq - mn);
      for (long t = 0; t < n; ++t) qf[t + n * k] = (q[t] - mn) / mx;
    }
  }
}

// findpeak on an arbitrary map, exposed for tests.
void orc_findpeak(const double* f, int r, int c, double* out3) { findpeak(f, r, c, out3, out3 + 1, out3 + 2); }

// normxcorr2 exposed for tests.  out must hold (ma+m-1)*(na+n-1) values.
int orc_normxcorr2(const double* T, int m, int n, const double* A, int ma, int na, double* out) {
  std::vector<double> o;
  if (!normxcorr2(T, m, n, A, ma, na, &o)) return -1;
  std::memcpy(out, o.data(), sizeof(double) * o.size());
  return 0;
}

// bwselect exposed for tests: bw (rows x cols, 0/1) -> out.
void orc_bwselect(const uint8_t* bw, int rows, int cols, int sr, int sc, int conn, uint8_t* out) {
  std::vector<uint8_t> b(bw, bw + (size_t)rows * cols), o;
  bwselect(b, rows, cols, sr, sc, conn, &o);
  std::memcpy(out, o.data(), o.size());
}

}  // extern "C"
