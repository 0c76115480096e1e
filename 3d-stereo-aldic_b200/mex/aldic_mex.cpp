// aldic_mex -- MATLAB MEX gateway to the B200 library (include/aldic_b200.h).
//
// One MEX file dispatching on a command string.  Each command replaces one per-subset loop
// (or one whole function) of the reference's MATLAB drivers with a batched library call, so
// the MATLAB code around it (bad-point rules, NaN fills, meshing) is unchanged.  The MEX ABI
// is the reference's own boundary (ba_interp2_spline.cpp:418-435): read-only prhs owned by
// MATLAB, outputs created with mxCreate* and handed to MATLAB, errors raised through
// mexErrMsgIdAndTxt.  One library context lives for the MATLAB session (freed at mexAtExit),
// so the frame loaded for LocalICGNQuadtree is reused by the Subpb1Quadtree calls after it.
//
// Built in MATLAB (R2018a interleaved API) with
//   mex -R2018a aldic_mex.cpp -I<repo>/include -L<repo>/3d-stereo-aldic_b200/aldic_b200 -laldic_b200
//
// Commands (arrays in the reference's layouts; masks may be logical or double):
//   [U, F, HtempPar, ConvItPerEle, markHole] = aldic_mex('local_icgn_quadtree', U0, coordinatesFEM,
//        DfDx, DfDy, ImgRefMask, ImgRef, ImgDef, winsize, tol)   % LocalICGNQuadtree.m:67-157
//   [U, F, HtempPar, ConvItPerEle] = aldic_mex('local_icgn', U0, coordinatesFEM, DfDx, DfDy,
//        ImgRef, ImgDef, winsize, tol)                           % LocalICGN.m:64-162
//   [U, ConvItPerEle] = aldic_mex('subpb1_quadtree', UOld, FOld, vdual, coordinatesFEM, DfDx,
//        DfDy, ImgRefMask, ImgRef, ImgDef, mu, winsize_List, tol)  % Subpb1Quadtree.m:71-123
//   [U, ConvItPerEle] = aldic_mex('subpb1', UOld, FOld, vdual, coordinatesFEM, DfDx, DfDy,
//        ImgRef, ImgDef, mu, HPar, winsize, tol)                 % Subpb1.m loop
//   [x, y, u, v, phi] = aldic_mex('integer_search', f, g, searchRegion, gridx, gridy, winsize,
//        winstepsize)                                            % funIntegerSearch.m:100-203
//   U0 = aldic_mex('init', u, v, index)                           % Init.m
//   [u, v] = aldic_mex('remove_outliers', u, v, Thr0)             % funRemoveOutliers.m:16-87
//   USubpb2 = aldic_mex('subpb2', coordinatesFEM, elementsFEM, dirichlet, GaussPtOrder, beta,
//        mu, U, F, alpha)                                        % Subpb2Quadtree.m
//   ptsOut = aldic_mex('undistort', pts, K, RadialDistortion, TangentialDistortion)
//                                                                % funUndistortPoints.m:8-39
//   [xyz, reprojErr] = aldic_mex('triangulate', matchedPairs, K_L, K_R, R, T)
//                                                                % stereoReconstruction_quadtree.m:30-52
//   Z = aldic_mex('interp2', F, X, Y)                             % ba_interp2_spline(F, X, Y)
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "aldic_b200.h"
#include "mex.h"

namespace {

aldic_ctx* g_ctx = nullptr;

void release_context() {
  if (g_ctx) aldic_destroy(g_ctx);
  g_ctx = nullptr;
}

void check(int rc, const char* what) {
  if (rc != ALDIC_OK) mexErrMsgIdAndTxt("aldic:library", "%s: %s", what, aldic_last_error(g_ctx));
}

void need(bool ok, const char* msg) {
  if (!ok) mexErrMsgIdAndTxt("aldic:argument", "%s", msg);
}

const double* doubles(const mxArray* a, const char* name) {
  if (!mxIsDouble(a) || mxIsComplex(a)) mexErrMsgIdAndTxt("aldic:argument", "%s must be a real double array", name);
  return mxGetDoubles(a);
}

// A mask as doubles (nonzero = inside): logical masks, as the reference builds them
// (logical(...), func_quadtree/funICGNQuadtree.m:83), and double masks are both accepted.
std::vector<double> mask_values(const mxArray* a) {
  const size_t n = mxGetNumberOfElements(a);
  std::vector<double> m(n);
  if (mxIsLogical(a)) {
    const mxLogical* p = mxGetLogicals(a);
    for (size_t i = 0; i < n; ++i) m[i] = p[i] ? 1.0 : 0.0;
  } else {
    const double* p = doubles(a, "ImgRefMask");
    std::memcpy(m.data(), p, n * sizeof(double));
  }
  return m;
}

std::vector<int32_t> int32s(const mxArray* a, const char* name) {
  const double* p = doubles(a, name);
  const size_t n = mxGetNumberOfElements(a);
  std::vector<int32_t> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = (int32_t)p[i];
  return v;
}

int scalar_int(const mxArray* a) { return (int)mxGetScalar(a); }

// Frame state of the IC-GN commands: normalised images, gradients, optional mask.
void load_frame(const mxArray* ref, const mxArray* def, const mxArray* dfdx, const mxArray* dfdy, const mxArray* mask) {
  const int M = (int)mxGetM(ref), N = (int)mxGetN(ref);
  need((int)mxGetM(def) == M && (int)mxGetN(def) == N, "ImgRef and ImgDef must have the same size");
  need((int)mxGetM(dfdx) == M - 6 && (int)mxGetN(dfdx) == N - 6, "DfDx must be (M-6) x (N-6) (Df.DfCropWidth 3)");
  need((int)mxGetM(dfdy) == M - 6 && (int)mxGetN(dfdy) == N - 6, "DfDy must be (M-6) x (N-6)");
  check(aldic_load_image(g_ctx, ALDIC_SLOT_REF, doubles(ref, "ImgRef"), M, N), "ImgRef");
  check(aldic_load_image(g_ctx, ALDIC_SLOT_DEF, doubles(def, "ImgDef"), M, N), "ImgDef");
  if (mask) {
    need((int)mxGetM(mask) == M && (int)mxGetN(mask) == N, "ImgRefMask must be M x N");
    const std::vector<double> m = mask_values(mask);
    check(aldic_set_mask(g_ctx, m.data(), M, N), "ImgRefMask");
  } else {
    check(aldic_set_mask(g_ctx, nullptr, M, N), "mask");
  }
  check(aldic_set_gradients(g_ctx, doubles(dfdx, "DfDx"), doubles(dfdy, "DfDy"), M - 6, N - 6), "gradients");
}

void local_icgn(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[], bool quad) {
  need(nrhs == (quad ? 10 : 9), quad ? "local_icgn_quadtree takes 9 arguments" : "local_icgn takes 8 arguments");
  const mxArray* U0 = prhs[1];
  const mxArray* coords = prhs[2];
  const int o = quad ? 1 : 0;
  load_frame(prhs[5 + o], prhs[6 + o], prhs[3], prhs[4], quad ? prhs[5] : nullptr);
  const int64_t n = (int64_t)mxGetM(coords);
  need(mxGetN(coords) == 2, "coordinatesFEM must be n x 2");
  need((int64_t)mxGetNumberOfElements(U0) == 2 * n, "U0 must hold 2n values");
  plhs[0] = mxCreateDoubleMatrix(2 * n, 1, mxREAL);
  plhs[1] = mxCreateDoubleMatrix(4 * n, 1, mxREAL);
  plhs[2] = mxCreateDoubleMatrix(n, 21, mxREAL);
  plhs[3] = mxCreateNumericMatrix(n, 1, mxINT32_CLASS, mxREAL);
  if (quad) plhs[4] = mxCreateNumericMatrix(n, 1, mxUINT8_CLASS, mxREAL);
  check(aldic_local_icgn(g_ctx, quad ? ALDIC_QUADTREE : ALDIC_UNIFORM, n, doubles(coords, "coordinatesFEM"),
                         doubles(U0, "U0"), scalar_int(prhs[7 + o]), mxGetScalar(prhs[8 + o]), mxGetDoubles(plhs[0]),
                         mxGetDoubles(plhs[1]), mxGetDoubles(plhs[2]), (int32_t*)mxGetData(plhs[3]),
                         quad ? (uint8_t*)mxGetData(plhs[4]) : nullptr),
        "aldic_local_icgn");
  (void)nlhs;
}

void subpb1(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[], bool quad) {
  need(nrhs == (quad ? 13 : 13), "subpb1 / subpb1_quadtree take 12 arguments");
  const mxArray *UOld = prhs[1], *FOld = prhs[2], *vdual = prhs[3], *coords = prhs[4];
  const int64_t n = (int64_t)mxGetM(coords);
  need(mxGetN(coords) == 2, "coordinatesFEM must be n x 2");
  std::vector<int32_t> wl;
  const double* hpar = nullptr;
  int winsize = 0;
  if (quad) {
    load_frame(prhs[8], prhs[9], prhs[5], prhs[6], prhs[7]);
    wl = int32s(prhs[11], "winsize_List");
    need((int64_t)wl.size() == 2 * n, "winsize_List must be n x 2");
  } else {
    load_frame(prhs[7], prhs[8], prhs[5], prhs[6], nullptr);
    if (mxGetNumberOfElements(prhs[10])) hpar = doubles(prhs[10], "HPar");
    winsize = scalar_int(prhs[11]);
  }
  const double mu = mxGetScalar(prhs[quad ? 10 : 9]);
  plhs[0] = mxCreateDoubleMatrix(2 * n, 1, mxREAL);
  plhs[1] = mxCreateNumericMatrix(n, 1, mxINT32_CLASS, mxREAL);
  check(aldic_subpb1(g_ctx, quad ? ALDIC_QUADTREE : ALDIC_UNIFORM, n, doubles(coords, "coordinatesFEM"),
                     doubles(UOld, "UOld"), doubles(FOld, "FOld"), doubles(vdual, "vdual"),
                     quad ? wl.data() : nullptr, winsize, hpar, mu, mxGetScalar(prhs[12]), mxGetDoubles(plhs[0]),
                     (int32_t*)mxGetData(plhs[1])),
        "aldic_subpb1");
  (void)nlhs;
}

void integer_search(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need(nrhs == 8, "integer_search takes 7 arguments");
  const mxArray *f = prhs[1], *g = prhs[2];
  const int M = (int)mxGetM(f), N = (int)mxGetN(f);
  need((int)mxGetM(g) == M && (int)mxGetN(g) == N, "f and g must have the same size");
  check(aldic_load_image(g_ctx, ALDIC_SLOT_REF, doubles(f, "f"), M, N), "f");
  check(aldic_load_image(g_ctx, ALDIC_SLOT_DEF, doubles(g, "g"), M, N), "g");
  const std::vector<int32_t> s = int32s(prhs[3], "searchRegion");
  const std::vector<int32_t> gx = int32s(prhs[4], "gridx"), gy = int32s(prhs[5], "gridy");
  need(gx.size() == 2 && gy.size() == 2, "gridx and gridy take 2 values");
  const int search[2] = {s.empty() ? 0 : s[0], s.size() > 1 ? s[1] : (s.empty() ? 0 : s[0])};
  const int w = scalar_int(prhs[6]), step = scalar_int(prhs[7]);
  int nx = 0, ny = 0;
  check(aldic_search_grid(gx.data(), gy.data(), w, step, &nx, &ny), "aldic_search_grid");
  for (int k = 0; k < 5; ++k) plhs[k] = mxCreateDoubleMatrix(ny, nx, mxREAL);
  check(aldic_integer_search(g_ctx, search, gx.data(), gy.data(), w, step, mxGetDoubles(plhs[0]),
                             mxGetDoubles(plhs[1]), mxGetDoubles(plhs[2]), mxGetDoubles(plhs[3]),
                             mxGetDoubles(plhs[4])),
        "aldic_integer_search");
  (void)nlhs;
}

void init(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need(nrhs == 4, "init takes 3 arguments (u, v, index)");
  const int ny = (int)mxGetM(prhs[1]), nx = (int)mxGetN(prhs[1]);
  need((int)mxGetM(prhs[2]) == ny && (int)mxGetN(prhs[2]) == nx, "u and v must have the same size");
  plhs[0] = mxCreateDoubleMatrix(2 * (size_t)nx * ny, 1, mxREAL);
  check(aldic_init_u0(g_ctx, ny, nx, doubles(prhs[1], "u"), doubles(prhs[2], "v"), scalar_int(prhs[3]),
                      mxGetDoubles(plhs[0])),
        "aldic_init_u0");
}

void remove_outliers(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need(nrhs == 4, "remove_outliers takes 3 arguments (u, v, Thr0)");
  const int m = (int)mxGetM(prhs[1]), n = (int)mxGetN(prhs[1]);
  need((int)mxGetM(prhs[2]) == m && (int)mxGetN(prhs[2]) == n, "u and v must have the same size");
  plhs[0] = mxCreateDoubleMatrix(m, n, mxREAL);
  plhs[1] = mxCreateDoubleMatrix(m, n, mxREAL);
  std::memcpy(mxGetDoubles(plhs[0]), doubles(prhs[1], "u"), sizeof(double) * (size_t)m * n);
  std::memcpy(mxGetDoubles(plhs[1]), doubles(prhs[2], "v"), sizeof(double) * (size_t)m * n);
  check(aldic_remove_outliers(g_ctx, m, n, mxGetDoubles(plhs[0]), mxGetDoubles(plhs[1]), mxGetScalar(prhs[3]), 0,
                              nullptr),
        "aldic_remove_outliers");
}

void subpb2(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need(nrhs == 10, "subpb2 takes 9 arguments");
  const mxArray *coords = prhs[1], *elems = prhs[2], *dir = prhs[3];
  const int64_t n = (int64_t)mxGetM(coords), n_el = (int64_t)mxGetM(elems);
  need(mxGetN(elems) == 8, "elementsFEM must be n_el x 8");
  const std::vector<int32_t> E = int32s(elems, "elementsFEM"), D = int32s(dir, "dirichlet");
  plhs[0] = mxCreateDoubleMatrix(2 * n, 1, mxREAL);
  check(aldic_subpb2(g_ctx, n, doubles(coords, "coordinatesFEM"), n_el, E.data(), scalar_int(prhs[4]),
                     mxGetScalar(prhs[5]), mxGetScalar(prhs[6]), mxGetScalar(prhs[9]), doubles(prhs[7], "U"),
                     doubles(prhs[8], "F"), (int64_t)D.size(), D.empty() ? nullptr : D.data(), 0.0, 0,
                     mxGetDoubles(plhs[0]), nullptr),
        "aldic_subpb2");
}

void undistort(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need(nrhs == 5, "undistort takes 4 arguments (pts, K, radial, tangential)");
  const int64_t n = (int64_t)mxGetM(prhs[1]);
  need(mxGetN(prhs[1]) == 2, "pts must be n x 2");
  const int nr = (int)mxGetNumberOfElements(prhs[3]);
  need(nr == 2 || nr == 3, "RadialDistortion takes 2 or 3 values");
  const double* tan = mxGetNumberOfElements(prhs[4]) == 2 ? doubles(prhs[4], "TangentialDistortion") : nullptr;
  plhs[0] = mxCreateDoubleMatrix(n, 2, mxREAL);
  check(aldic_undistort_points(g_ctx, n, doubles(prhs[1], "pts"), doubles(prhs[2], "K"),
                               doubles(prhs[3], "RadialDistortion"), nr, tan, mxGetDoubles(plhs[0])),
        "aldic_undistort_points");
}

void triangulate(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need(nrhs == 6, "triangulate takes 5 arguments (matchedPairs, K_L, K_R, R, T)");
  const int64_t n = (int64_t)mxGetM(prhs[1]);
  need(mxGetN(prhs[1]) == 4, "matchedPairs must be n x 4");
  plhs[0] = mxCreateDoubleMatrix(n, 3, mxREAL);
  plhs[1] = mxCreateDoubleMatrix(n, 1, mxREAL);
  check(aldic_triangulate(g_ctx, n, doubles(prhs[1], "matchedPairs"), doubles(prhs[2], "K_L"),
                          doubles(prhs[3], "K_R"), doubles(prhs[4], "R"), doubles(prhs[5], "T"),
                          mxGetDoubles(plhs[0]), mxGetDoubles(plhs[1])),
        "aldic_triangulate");
}

void interp2(mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  need(nrhs == 4, "interp2 takes 3 arguments (F, X, Y)");
  const int M = (int)mxGetM(prhs[1]), N = (int)mxGetN(prhs[1]);
  const size_t n = mxGetNumberOfElements(prhs[2]);
  need(mxGetNumberOfElements(prhs[3]) == n, "X and Y must have the same number of elements");
  check(aldic_load_image(g_ctx, ALDIC_SLOT_DEF, doubles(prhs[1], "F"), M, N), "F");
  plhs[0] = mxCreateDoubleMatrix(mxGetM(prhs[2]), mxGetN(prhs[2]), mxREAL);
  check(aldic_interp2(g_ctx, ALDIC_SLOT_DEF, (int64_t)n, doubles(prhs[2], "X"), doubles(prhs[3], "Y"),
                      mxGetDoubles(plhs[0])),
        "aldic_interp2");
}

}  // namespace

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs < 1 || !mxIsChar(prhs[0])) mexErrMsgIdAndTxt("aldic:argument", "first argument: a command string");
  if (!g_ctx) {
    if (aldic_create(&g_ctx, 0) != ALDIC_OK) {
      g_ctx = nullptr;
      mexErrMsgIdAndTxt("aldic:library", "aldic_create failed (no CUDA device?)");
    }
    mexAtExit(release_context);
  }
  char* c = mxArrayToString(prhs[0]);
  const std::string cmd = c ? c : "";
  mxFree(c);
  if (cmd == "local_icgn_quadtree") return local_icgn(nlhs, plhs, nrhs, prhs, true);
  if (cmd == "local_icgn") return local_icgn(nlhs, plhs, nrhs, prhs, false);
  if (cmd == "subpb1_quadtree") return subpb1(nlhs, plhs, nrhs, prhs, true);
  if (cmd == "subpb1") return subpb1(nlhs, plhs, nrhs, prhs, false);
  if (cmd == "integer_search") return integer_search(nlhs, plhs, nrhs, prhs);
  if (cmd == "init") return init(plhs, nrhs, prhs);
  if (cmd == "remove_outliers") return remove_outliers(plhs, nrhs, prhs);
  if (cmd == "subpb2") return subpb2(plhs, nrhs, prhs);
  if (cmd == "undistort") return undistort(plhs, nrhs, prhs);
  if (cmd == "triangulate") return triangulate(plhs, nrhs, prhs);
  if (cmd == "interp2") return interp2(plhs, nrhs, prhs);
  mexErrMsgIdAndTxt("aldic:argument", "unknown command '%s'", cmd.c_str());
}
