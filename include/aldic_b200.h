/*
 * aldic_b200.h -- C ABI of the B200 (sm_100a) implementation of the 3D-Stereo-ALDIC
 * per-subset hot path: image preparation, whole-field integer (ZNCC) search, local
 * IC-GN with the local bicubic B-spline stencil (uniform and quadtree/masked), the
 * ALDIC Subpb1 augmented-Lagrangian local step, the epipolar IC-GN candidate score and
 * per-point stereo triangulation.
 *
 * Conventions follow the MATLAB reference so that a MEX shim can pass mxArray data
 * pointers straight through:
 *   - images are column-major M x N (dim 1 = image x, because the reference transposes
 *     images at load), element (i, j) at i + j*M;
 *   - pixel coordinates are 1-based;
 *   - coordinatesFEM is n x 2 column-major; U is 2n interleaved [u1 v1 u2 v2 ...];
 *     F is 4n interleaved [F11 F21 F12 F22 ...]; H is n x 21 column-major (the packed
 *     lower triangle [H(1:6) H(8:12) H(15:18) H(22:24) H(29:30) H(36)]).
 *
 * Every array argument may be host or device memory (checked with
 * cudaPointerGetAttributes).  A call whose outputs are all device memory is
 * asynchronous on the context's stream; a call with any host output returns after the
 * results are in host memory.  The library never frees caller memory.
 *
 * Return value: ALDIC_OK or an error code; aldic_last_error() gives the message.
 * Per-subset outcomes are in-band as in the reference: the iteration count when
 * converged, 101 (not converged / out of image / NaN), 102 (too much of the subset
 * masked), 103 (all-zero reference subset), -1 (the reference solver raised an error).
 */
#ifndef ALDIC_B200_H
#define ALDIC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALDIC_OK 0
#define ALDIC_ERR_ARG 1
#define ALDIC_ERR_CUDA 2
#define ALDIC_ERR_TIMEOUT 3
#define ALDIC_ERR_STATE 4

/* element types of raw images */
#define ALDIC_U8 0
#define ALDIC_U16 1
#define ALDIC_F32 2
#define ALDIC_F64 3

/* image slots of a context */
#define ALDIC_SLOT_REF 0
#define ALDIC_SLOT_DEF 1

/* solver variants */
#define ALDIC_UNIFORM 0  /* LocalICGN / Subpb1 (func/funICGN.m, func/funICGN_Subpb1.m) */
#define ALDIC_QUADTREE 1 /* LocalICGNQuadtree / Subpb1Quadtree (masked solvers) */

typedef struct aldic_ctx aldic_ctx;
typedef struct aldic_net aldic_net;

/* Create a context on CUDA device `device`; it owns a stream and device buffers. */
int aldic_create(aldic_ctx** ctx, int device);
void aldic_destroy(aldic_ctx* ctx);
const char* aldic_last_error(const aldic_ctx* ctx);
/* Run subsequent work on `stream` (a cudaStream_t); NULL restores the context's own. */
int aldic_set_stream(aldic_ctx* ctx, void* stream);
int aldic_synchronize(aldic_ctx* ctx);
/* Number of kernels this context has launched since creation. */
int64_t aldic_launch_count(const aldic_ctx* ctx);
int aldic_abi_version(void);

/* ---------------------------------------------------------------- frame state ---- */
/* funNormalizeImg (func/funNormalizeImg.m:109-127) of a raw image into `slot`:
 * (img - mean_ROI) / std_ROI, FP64 statistics over gridx x gridy (1-based inclusive,
 * clamped to the image), stored as FP32 on the device.  If `mask` (M x N, nonzero = in)
 * is given the stored image is additionally multiplied by it, as TemporalMatch
 * (func/TemporalMatch_quadtree_ST1.m:47-48) does.  mean_std (2 doubles, may be NULL)
 * receives the statistics. */
int aldic_load_image_raw(aldic_ctx* ctx, int slot, const void* img, int dtype, int M, int N, const int* gridx,
                         const int* gridy, const double* mask, double* mean_std);
/* Store an already-normalised image (the ImgRef / ImgDef arguments of the MATLAB
 * solvers) into `slot`. */
int aldic_load_image(aldic_ctx* ctx, int slot, const double* img, int M, int N);
/* Df.ImgRefMask (M x N; NULL = all ones).  Values are binarised (nonzero -> 1). */
int aldic_set_mask(aldic_ctx* ctx, const double* mask, int M, int N);
/* funImgGradient (func/funImgGradient.m:50-78) of the REF slot on the device:
 * 7-tap central differences, crop 3, times the mask. */
int aldic_compute_gradients(aldic_ctx* ctx);
/* Df.DfDx / Df.DfDy given by the caller, (M-6) x (N-6). */
int aldic_set_gradients(aldic_ctx* ctx, const double* dfdx, const double* dfdy, int M6, int N6);
/* Read back device state as doubles: what = 0 REF image, 1 DEF image, 2 DfDx, 3 DfDy. */
int aldic_get_state(aldic_ctx* ctx, int what, double* out);

/* ---------------------------------------------------------- interpolation ------- */
/* ba_interp2_spline(F, X, Y) (ba_interp2_spline.cpp:418-435, local 4x4 stencil
 * :235-331) on the image in `slot`: X is the dim-2 and Y the dim-1 coordinate. */
int aldic_interp2(aldic_ctx* ctx, int slot, int64_t n, const double* X, const double* Y, double* Z);

/* ------------------------------------------------------- integer search --------- */
/* Grid size of funIntegerSearchWholeField (func/funIntegerSearch.m:106-107). */
int aldic_search_grid(const int* gridx, const int* gridy, int winsize, int step, int* nx, int* ny);
/* funIntegerSearch(f, g, search, gridx, gridy, winsize, step, 0)
 * (func/funIntegerSearch.m:2-98,100-203) with f = REF slot and g = DEF slot:
 * per grid subset ZNCC (normxcorr2) over the border-clamped search window, crop, and
 * findpeak (func/findpeak.m) with the 1e-3 px rounding.  search = [s0 s1]
 * (tempSizeOfSearchRegion; expanded to [left right up down] = [s0 s1 s0 s1]).
 * Outputs x, y, u, v, phi are nY x nX column-major; failed subsets give NaN. */
int aldic_integer_search(aldic_ctx* ctx, const int* search, const int* gridx, const int* gridy, int winsize,
                         int step, double* x, double* y, double* u, double* v, double* phi);

/* --------------------------------------------------------- local IC-GN ---------- */
/* Loop body of LocalICGN (variant ALDIC_UNIFORM; func/LocalICGN.m:64-164 with
 * func/funICGN.m) or LocalICGNQuadtree (ALDIC_QUADTREE;
 * func_quadtree/LocalICGNQuadtree.m:67-164 with func_quadtree/funICGNQuadtree.m):
 * first-order IC-GN, Gauss-Newton, maxIter 100, on the REF/DEF slots, gradients and
 * mask of the context.  H (n x 21) and markHole (n, quadtree only) may be NULL.
 * Interpolation and sums run in FP32 (Kahan-compensated per thread, FP64 across threads)
 * for up to the iteration cap; a subset whose convergence test |b|/|b_1| < tol or |b| < tol
 * (func/funICGN.m:268-282) falls within the FP32 noise of |b| plus a relative margin of tol
 * (aldic_set_fp64_band) is re-solved from its initial guess in FP64 with the reference's own
 * interpolation arithmetic, so that its iteration count, and with it U, is the FP64
 * reference's (ALDIC_OPT_SLOW_FP64 sends every long trajectory there too). */
int aldic_local_icgn(aldic_ctx* ctx, int variant, int64_t n, const double* coords, const double* U0, int winsize,
                     double tol, double* U, double* F, double* H, int32_t* conv, uint8_t* markHole);

/* Loop body of Subpb1 (ALDIC_UNIFORM; func/Subpb1.m with func/funICGN_Subpb1.m, Hessian
 * block H(5:6,5:6) from HPar n x 21) or Subpb1Quadtree (ALDIC_QUADTREE;
 * func_quadtree/Subpb1Quadtree.m:71-126 with func_quadtree/funICGN_Subpb1quadtree.m,
 * per-subset winsize_List n x 2): the ALDIC augmented-Lagrangian translation step with
 * F fixed at FOld.  vdual is 2n interleaved.  A solver error gives U = NaN and
 * conv = -1 (uniform) or 0 (quadtree), as the two drivers store. */
int aldic_subpb1(aldic_ctx* ctx, int variant, int64_t n, const double* coords, const double* UOld,
                 const double* FOld, const double* vdual, const int32_t* winsize_list, int winsize,
                 const double* HPar, double mu, double tol, double* U, int32_t* conv);

/* epipolar_ICGN1 (func/epipolar_ICGN1.m:1-253) for n candidate points pts (n x 2):
 * IC-GN from P = 0 with the translation held at 0, at most 30 iterations, gradient
 * offset Df.DfAxis(1) = 4; znssd = ZNSSD of the final iteration (NaN on failure). */
int aldic_epipolar_icgn(aldic_ctx* ctx, int64_t n, const double* pts, int winsize, double tol, double* znssd);

/* ---------------------------------------------------- ALDIC global step ------- */
/* [Uhat] = Subpb2Quadtree(DICmesh, GaussPtOrder, beta, mu, U, F, udual, vdual, alpha,
 * winstepsize, 0) (func_quadtree/Subpb2Quadtree.m) with an empty neumann list: the global
 * finite-element step of the augmented Lagrangian on a quadtree mesh of n nodes (coords n x 2
 * column-major) and n_el elements (elements n_el x 8 column-major, 1-based: corners 1-4,
 * mid-side hanging nodes 5-8 on the right / top / left / bottom edge, 0 where absent).
 * Element matrices sum_g |J| w ((beta + alpha) DN' DN + mu N' N) at gauss_order^2 points
 * (2..5), right-hand side from U (2n interleaved) and F (4n, F11 F21 F12 F22 per node); the
 * duals do not enter (the reference multiplies them by 0).  Nodes of the elements (but the
 * first entry of unique(elementsFEM), as the reference) are free, the n_dirichlet
 * dirichlet nodes (1-based) hold U, all other nodes get 0.  Solved by Jacobi-preconditioned
 * conjugate gradients in FP64 to |r| <= tol |r0| (tol <= 0: 1e-12) within maxit iterations
 * (<= 0: min(20 n + 1000, 200000)); the reference solves the free block directly.
 * Uhat: 2n.  info (optional, host, 2 ints): iterations, 1 when the tolerance was met.
 * elements = NULL solves on the mesh of the last aldic_subpb2_set_mesh (same n and n_el;
 * n_dirichlet 0: the resident mesh carries its dirichlet nodes). */
int aldic_subpb2(aldic_ctx* ctx, int64_t n, const double* coords, int64_t n_el, const int32_t* elements,
                 int gauss_order, double beta, double mu, double alpha, const double* U, const double* F,
                 int64_t n_dirichlet, const int32_t* dirichlet, double tol, int maxit, double* Uhat,
                 int32_t* info);

/* Keeps a global-step mesh resident in the context (no reference counterpart: the drivers
 * call Subpb2Quadtree four to six times per frame on one mesh): the element table's checks,
 * the node -> element lists and the free / dirichlet kinds are built once, on the host, and
 * held on the device until the next call or aldic_destroy. */
int aldic_subpb2_set_mesh(aldic_ctx* ctx, int64_t n, int64_t n_el, const int32_t* elements, int64_t n_dirichlet,
                          const int32_t* dirichlet);

/* ------------------------------------------------- bad-point fill (host) ------- */
/* Sibson (natural-neighbour) weights of m queries Q (m x 2, row-major (x, y) pairs) with
 * respect to k source points P (k x 2, row-major), for MATLAB's scatteredInterpolant
 * 'natural' in the drivers' fill of bad points (func/LocalICGN.m:199-220,
 * func_quadtree/LocalICGNQuadtree.m:212-325).  Host code; no context, no device.  The
 * caller supplies a Delaunay triangulation of P: simplices and neighbors (ntri x 3,
 * row-major; neighbour e lies opposite vertex e, -1 on the hull), circumcentres cc (ntri x 2)
 * and squared circumradii r2, the containing triangle of each query (qsimplex, -1 outside)
 * and the point set's extent (scale, for the in-circle tolerance).  Per query: idx / w
 * (cap entries each) receive the natural neighbours and their weights, count the number
 * used, or -2 outside the hull, -1 where the cavity reaches the hull, is not a simple ring
 * or has more than cap vertices (the caller computes those another way). */
int aldic_sibson_weights(int64_t k, const double* P, int64_t ntri, const int32_t* simplices, const int32_t* neighbors,
                         const double* cc, const double* r2, double scale, int64_t m, const double* Q,
                         const int32_t* qsimplex, int32_t cap, int32_t* idx, double* w, int32_t* count);

/* ------------------------------------------------------ initial guess --------- */
/* inpaint_nans(A, 4) (func/inpaint_nans.m:369-398, spring analogy), in place on an m x n
 * column-major grid: the NaN entries become the least-squares solution of unit springs
 * to their in-grid horizontal / vertical neighbours with the finite entries fixed (FP64
 * conjugate gradients to 1e-13 of the right-hand side; a NaN region with no finite
 * neighbour becomes 0).  info (optional, host, 3 ints): NaN entries, CG iterations,
 * 1 when the residual target was met; passing it makes the call wait for the device. */
int aldic_inpaint_nans(aldic_ctx* ctx, int m, int n, double* A, int32_t* info);

/* funRemoveOutliers(u, v, cc, 0, Thr0) with Thr0 = thr > 0 (func/funRemoveOutliers.m:16,
 * :44-87; the call of func_quadtree/IntegerSearchQuadtree.m:158-160 uses 100), in place on
 * the search's m x n column-major u and v grids: the median test of funMedRemoveOutliers
 * (:374-390; inpaint_nans(., 3) of each grid, medFilt2 [2 2] 'symmetric' skipping the
 * second neighbour, |u - median| / (median |u - median| + 0.1) in single precision) marks
 * the entries whose sqrt(nfu^2 + nfv^2) > thr; they are set NaN in both grids, both are
 * filled with inpaint_nans(., 4), and the entries NaN in u on entry are NaN again.
 * maxit <= 0 takes the default limit of the method-3 solver (min(8 m n + 200, 20000)
 * iterations).  info (optional, host, 4 ints): entries removed, NaN holes of u, the
 * method-3 solver's iterations (larger of u and v), 1 when both met their residual
 * target; passing it makes the call wait for the device.  The qDIC branch and the manual
 * (prompting) branches of the reference are not implemented (thr <= 0 is an error). */
int aldic_remove_outliers(aldic_ctx* ctx, int m, int n, double* u, double* v, double thr, int maxit,
                          int32_t* info);

/* Init(u, v, Phi, x, y, index) (func/Init.m): inpaint_nans(., 4) of the search's u and v
 * grids (ny x nx column-major, as aldic_integer_search returns them; left unchanged) (:13);
 * index 1 adds the three spring outlier passes (:29-166: nodes whose value departs from
 * their neighbours' average by more than 3 / 2 / 2 standard deviations are set NaN with
 * their neighbourhood, the border rows and columns too, and the grids inpainted again);
 * U0 (2 nx ny) interleaved [u1 v1 u2 v2 ...] in mesh order (XList fastest) (:169-177).
 * The stereo and temporal drivers call index 0. */
int aldic_init_u0(aldic_ctx* ctx, int ny, int nx, const double* u, const double* v, int index, double* U0);

/* funUndistortPoints (func/funUndistortPoints.m:8-39; MATLAB undistortPoints of one camera):
 * n points pts (n x 2 column-major, 1-based pixels) through the inverse of the
 * cameraParameters lens model -- radial (k1, k2 [, k3]: n_radial = 2 or 3) and tangential
 * (p1, p2; NULL = none) distortion in normalised coordinates K^-1 (u, v, 1) -- solved by
 * FP64 fixed-point iteration to 1e-15, mapped back through K (3 x 3 column-major) into out
 * (n x 2).  Non-finite rows give NaN. */
int aldic_undistort_points(aldic_ctx* ctx, int64_t n, const double* pts, const double* K, const double* radial,
                           int n_radial, const double* tangential, double* out);

/* -------------------------------------------------------- triangulation --------- */
/* triangulatePoints (func_quadtree/stereoReconstruction_quadtree.m:30-52): per row of
 * pairs (n x 4 column-major [xL yL xR yR]) the DLT of P_L = K_L [I | 0] and
 * P_R = K_R [R | T], solved in FP64 by SVD; xyz (n x 3) and the mean two-view
 * reprojection error; rows with non-finite input give NaN.  KL, KR, R are 3 x 3
 * column-major (MATLAB), T has 3 entries. */
int aldic_triangulate(aldic_ctx* ctx, int64_t n, const double* pairs, const double* KL, const double* KR,
                      const double* R, const double* T, double* xyz, double* reproj_err);

/* ------------------------------------------------------ allocation-free IC-GN ---- */
/* No counterpart in the reference.  aldic_local_icgn for callers that cannot allocate
 * device memory (a host that owns every allocation: gpuArray buffers handed over by a
 * MEX, a fixed memory budget or pool).  No context and no cudaMalloc/cudaFree: the work
 * queue lives in a fixed file-scope device array sized for ALDIC_NOALLOC_MAX_SUBSETS
 * subsets (~2.4 MB, held by every GPU that loads the library until exit).  Every array
 * must be device memory on the current device: ref/def are the normalised FP32 images
 * (M x N), mask is u8 (may be NULL), dfdx/dfdy are FP32 (M-6) x (N-6); the rest as
 * aldic_local_icgn.  Work is queued on `stream` (NULL = legacy default stream) and not
 * waited for.  n > ALDIC_NOALLOC_MAX_SUBSETS returns ALDIC_ERR_ARG.  All calls share the
 * array, so calls that overlap on the GPU race and must be serialised by the caller; the
 * first call on a device looks the array up (cudaGetSymbolAddress) and should come
 * before any stream capture. */
#define ALDIC_NOALLOC_MAX_SUBSETS 65536
int aldic_local_icgn_noalloc(int variant, const float* ref, const float* def, const uint8_t* mask, const float* dfdx,
                             const float* dfdy, int M, int N, int64_t n, const double* coords, const double* U0,
                             int winsize, double tol, double* U, double* F, double* H, int32_t* conv,
                             uint8_t* markHole, void* stream);

/* ------------------------------------------------- learned initial guess ------- */
/* No counterpart in the reference, whose initial guess is the integer search
 * (func/funIntegerSearch.m:132-180); that search stays the fallback and the judge.
 *
 * A proposal network: a 32 x 32 reference subset and the 64 x 64 deformed window around it
 * -> the subset's (u, v, du/dx, dv/dx, du/dy, dv/dy).  The same two 3 x 3 stride-2
 * convolutions (1 -> 32 -> 32 channels) turn the subset into 8 x 8 and the window into
 * 16 x 16 feature maps, their correlation over 9 x 9 offsets (+-16 px) gives an 8 x 8 x 81
 * volume, then a 3 x 3 stride-2 and a 3 x 3 stride-1 convolution (81 -> 64 -> 64 channels,
 * 4 x 4) and two fully connected layers (1024 -> 128 -> 6), ReLU between: 227 152 FP32
 * parameters with BF16 copies; every layer, data gradient and weight gradient is a BF16 x
 * BF16 -> FP32 tensor-core GEMM (tcgen05, TMA-staged operands).  Outputs are scaled (u / 8,
 * v / 8, gradients x 20).  Inputs x: batch x 72 x 72 x 2 BF16 (NHWC; the window with 4 px of
 * context each side in channel 1, the subset with 4 px of context, 40 x 40, in the centre of
 * channel 0, zero elsewhere), device memory; targets t: batch x 6 FP32 (device), scaled as the
 * outputs.  batch a multiple of 8, at most max_batch. */
int aldic_net_create(aldic_net** net, int device, int max_batch);
void aldic_net_destroy(aldic_net* net);
const char* aldic_net_last_error(const aldic_net* net);
int aldic_net_set_stream(aldic_net* net, void* stream);
int64_t aldic_net_launch_count(const aldic_net* net);
/* Number of FP32 parameters and their flat layout: per layer W (rows x cols, row-major) then
 * b: conv 32 x 16 (K = 9 taps, padded to 16 with zeros), 32 x 288, 64 x 736 (K = 729 padded),
 * 64 x 576 (K ordered (ky, kx, channel)); FC 128 x 1024 (input ordered (y, x, channel) of the
 * 4 x 4 x 64 map), 16 x 128 (rows 6..15 zero, as biases 6..15). */
int64_t aldic_net_param_count(void);
/* Parameters in (host or device FP32); resets the Adam moments. */
int aldic_net_set_params(aldic_net* net, const float* params);
int aldic_net_get_params(aldic_net* net, float* params);
/* y (device, batch x 6 FP32) = the network's scaled outputs for x. */
int aldic_net_forward(aldic_net* net, int batch, const void* x, float* y);
/* Gradients of the mean squared error of the outputs against t (grads: param_count FP32,
 * host or device) and the loss (host or device, 1 FP32); waits for the device. */
int aldic_net_gradients(aldic_net* net, int batch, const void* x, const float* t, float* grads, float* loss);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) at learning rate lr on the batch; loss (host,
 * optional) receives the batch's loss before the step (then the call waits). */
int aldic_net_train_step(aldic_net* net, int batch, const void* x, const float* t, float lr, float* loss);
/* ALDIC_OK, or ALDIC_ERR_TIMEOUT if a GEMM's bounded wait timed out since creation. */
int aldic_net_status(aldic_net* net);
/* Initial guesses of n subsets (coords n x 2, 1-based) on the frame of ctx (REF and DEF
 * slots): U0 (2n interleaved) and F0 (4n, [F11 F21 F12 F22] = [du/dx dv/dx du/dy dv/dy]) for
 * aldic_local_icgn_guess.  The two shared convolutions run once over each whole image; each
 * subset reads its feature crops at the nearest centre with x, y = 1 (mod 4) (equal to the
 * per-window network there) and its U0 is moved to its own centre along F0.  U0 is NaN where
 * the crops leave the feature maps (centres nearer than 32 px to the first row or column, or
 * than about 26 px to the last).  Runs on the context's stream. */
int aldic_net_predict(aldic_net* net, aldic_ctx* ctx, int64_t n, const double* coords, double* U0, double* F0);
/* The network input of n subsets (coords n x 2, 1-based, rounded) on the frame of ctx: X
 * (device, n x 72 x 72 x 2 BF16), channel 1 the normalised deformed image over rows x0-36 ..
 * x0+35 and columns y0-36 .. y0+35, channel 0 the normalised reference image over the centre
 * 40 x 40 (x0-20 .. x0+19, y0-20 .. y0+19), zero elsewhere and outside the image.  For
 * training sets and checks of aldic_net_predict. */
int aldic_net_extract(aldic_ctx* ctx, int64_t n, const double* coords, void* X);
/* aldic_local_icgn from the initial guess P = [F0 U0] instead of [0 U0] (the reference starts
 * from F = 0, func/funICGN.m:46); everything else as aldic_local_icgn.  zncc (n, optional)
 * receives each subset's zero-normalised cross-correlation of REF with DEF under the last
 * warp IC-GN evaluated, which for a converged subset is the returned [F U] (its last
 * iteration stops without an update): that iteration's sums, no extra pass (the acceptance
 * test of a learned initial guess).  NaN where no pass solved the subset. */
int aldic_local_icgn_guess(aldic_ctx* ctx, int variant, int64_t n, const double* coords, const double* U0,
                           const double* F0, int winsize, double tol, double* U, double* F, double* H, int32_t* conv,
                           uint8_t* markHole, double* zncc);
/* The fallback of a learned initial guess: the subsets whose IC-GN from it did not converge
 * (conv outside 1..100) or whose final ZNCC is below zncc_min (or NaN).  Their indices (0-based,
 * in no fixed order) go to list (n entries of room, host or device) and their number to
 * *count: with a host count the call waits for the device; with a device count (and a
 * device list) it is queued on the context's stream and returns at once, so a caller can
 * queue the next frame before it reads the count.  No counterpart in the reference. */
int aldic_fallback_select(aldic_ctx* ctx, int64_t n, const int32_t* conv, const double* zncc, double zncc_min,
                          int32_t* list, int64_t* count);
/* Zero-normalised cross-correlation of each subset's (winsize+1)^2 window of REF with DEF under
 * the warp [F U] (the acceptance test of a learned initial guess); NaN where the warped window
 * leaves the image. */
int aldic_subset_zncc(aldic_ctx* ctx, int64_t n, const double* coords, const double* U, const double* F, int winsize,
                      double* zncc);
/* aldic_integer_search on the n grid subsets list[k] = i + j nX (0-based grid column i, row j)
 * only, with the direct correlation kernel; outputs n entries each, in list order (the
 * fallback search of the subsets a learned initial guess fails). */
int aldic_integer_search_list(aldic_ctx* ctx, const int* search, const int* gridx, const int* gridy, int winsize,
                              int step, int64_t n, const int32_t* list, double* x, double* y, double* u, double* v,
                              double* phi);

/* C (M x N FP32, row pitch ldc) = A (M x K) * B (N x K)^T on the tensor cores (tcgen05, the
 * proposal network's GEMM): A and B device BF16, row-major with pitches lda / ldb (multiples
 * of 8), 16-byte aligned; splits > 1 adds split-K partial sums into C (which the caller
 * zeroes).  Queued on stream (a cudaStream_t; NULL = legacy default).  A test and tuning
 * entry; not part of the reference. */
int aldic_gemm_bf16(const void* A, int64_t lda, const void* B, int64_t ldb, int64_t M, int64_t N, int64_t K, float* C,
                    int64_t ldc, int splits, void* stream);

/* ------------------------------------------------------------- diagnostics ------- */
/* Measured FP32 FMA throughput of the current device (TFLOP/s): the faster of a scalar
 * FFMA loop and a packed FFMA2 (fma.rn.f32x2) loop, the denominator the library's
 * compute-bound kernels are reported against.  Not part of the reference. */
int aldic_measure_fp32_peak(aldic_ctx* ctx, double* tflops);
/* Tuning options of a context (no reference counterpart; results do not depend on them
 * beyond FP32 summation order, and with the FP64 re-solve not at all in the codes):
 *   ALDIC_OPT_ITERATION_CAP  as aldic_set_iteration_cap (1..1000, default 8);
 *   ALDIC_OPT_STAGING        1: the IC-GN warp passes stage each subset's deformed window in
 *                            shared memory by TMA 2-D tile loads when the image layout allows
 *                            (rows a multiple of 4, 16-byte aligned) and the window is small
 *                            enough; 0 (default): they gather from the image through L1;
 *   ALDIC_OPT_SLOW_WARPS     warps per subset of the pass that continues the subsets still
 *                            iterating after the iteration cap: 2 (default) or 4;
 *   ALDIC_OPT_SEARCH_IMPL    aldic_integer_search: 0 (default) the shared-product tile kernel
 *                            where one is compiled for (step, winsize + 1), else the direct
 *                            per-subset correlation; 1 the tile kernel; 2 the direct kernel;
 *   ALDIC_OPT_SEARCH_CHUNK   shift columns per pass of the tile kernel: 16, 24 or 0 (the
 *                            shape's default);
 *   ALDIC_OPT_AUTOTUNE       1: the first call of every call shape (IC-GN: variant, winsize, n
 *                            to a power of two; search: image, winsize, step, search region,
 *                            grid) times every candidate of the options above on its own
 *                            inputs, checks that all candidates' results agree, and keeps the
 *                            fastest for that shape (that call waits for the device);
 *                            aldic_tuning_report gives the choices and timings as JSON. */
#define ALDIC_OPT_ITERATION_CAP 0
#define ALDIC_OPT_STAGING 1
#define ALDIC_OPT_SLOW_WARPS 2
#define ALDIC_OPT_SEARCH_IMPL 3
#define ALDIC_OPT_SEARCH_CHUNK 4
#define ALDIC_OPT_AUTOTUNE 5
/*   ALDIC_OPT_SLOW_FP64      1: aldic_local_icgn re-solves every subset still iterating after
 *                            the iteration cap from its initial guess in FP64; 0 (default): an
 *                            FP32 multi-warp pass continues them (ALDIC_OPT_SLOW_WARPS warps
 *                            each), its convergence tests checked against the band like the
 *                            first pass's;
 *   ALDIC_OPT_FP64_THREADS   threads per subset of the FP64 re-solve: 128 (default), 256 or
 *                            512. */
#define ALDIC_OPT_SLOW_FP64 6
#define ALDIC_OPT_FP64_THREADS 7
/* Read-only statistics of the last aldic_local_icgn (aldic_get_option; waits for the call):
 * subsets re-solved in FP64, and 1 if a staging load outlasted its wait (the warp group then
 * gathered from the image). */
#define ALDIC_STAT_FP64_RESOLVES 100
#define ALDIC_STAT_STAGING_TIMEOUT 101
int aldic_set_option(aldic_ctx* ctx, int option, int value);
int aldic_get_option(aldic_ctx* ctx, int option, int* value);
/* The autotuner's choices so far as a JSON object {shape key: {"choice": {...}, "ms":
 * {candidate: time, ...}}} (a negative time marks a candidate whose results differed) into
 * buf (len bytes, NUL-terminated). */
int aldic_tuning_report(aldic_ctx* ctx, char* buf, int64_t len);
/* Margin around tol within which aldic_local_icgn re-decides an FP32 convergence test by an
 * FP64 re-solve of the subset: band x tol (default band 1e-3; a huge value re-solves every
 * subset in FP64) plus noise x 2^-24 x (bf / bg) x sqrt(tr(H) sum(g^2) / n) x the iteration
 * number, an estimate of the FP32 rounding noise of |b| (default noise 4), which decides
 * when |b| itself is near tol.  band = 0 turns the re-solve off.  A precision setting; not
 * part of the reference. */
int aldic_set_fp64_band(aldic_ctx* ctx, double band, double noise);
/* Iterations the one-warp-per-subset solver pass of aldic_local_icgn / aldic_subpb1 spends
 * on a subset before a multi-warp pass restarts it from its initial guess (default 8, 1..1000).
 * Results do not depend on it beyond FP32 summation order; it trades the tail of slow
 * subsets against repeated work.  A tuning setting; not part of the reference. */
int aldic_set_iteration_cap(aldic_ctx* ctx, int cap);
/* Device time of the correlation kernel of every aldic_integer_search call while profiling
 * is on (CUDA events recorded on the context's stream around that one launch; up to 256
 * calls are kept).  aldic_profile_read waits for the recorded events, returns their total
 * time and count, and clears the record.  A measurement hook; not part of the reference. */
int aldic_set_profiling(aldic_ctx* ctx, int on);
int aldic_profile_read(aldic_ctx* ctx, double* total_ms, int* launches);

#ifdef __cplusplus
}
#endif
#endif /* ALDIC_B200_H */
