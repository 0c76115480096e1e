// Internal kernel interfaces of the ALDIC B200 library (not part of the public C ABI).
#pragma once
#include <cuda_runtime.h>

#include <vector>
#include <stddef.h>
#include <stdint.h>

struct aldic_net;

namespace aldic {

// Device-resident frame: normalised images (FP32, column-major M x N), binary mask
// (u8, may be null = all ones) and the cropped gradients ((M-6) x (N-6), FP32).
struct FrameDev {
  const float* ref;
  const float* def;
  const uint8_t* mask;
  const float* gx;
  const float* gy;
  int M, N;
};

struct IcgnArgs {
  FrameDev fr;
  int variant;  // 0 uniform (funICGN), 1 quadtree (funICGNQuadtree), 2 epipolar (epipolar_ICGN1)
  long long n;
  const double* coords;  // n x 2
  const double* U0;      // 2n
  int winsize;
  double tol;
  int max_iter;  // 100, or 30 for the epipolar variant
  int warp_cap;  // iterations the one-warp pass spends on a subset before the multi-warp pass restarts it
  int crop;      // gradient offset: 3 (DfCropWidth) or 4 (DfAxis start)
  double* U;     // 2n
  double* F;     // 4n
  double* H;     // n x 21 or null
  int* conv;     // n
  uint8_t* mark; // n or null
  double* znssd; // n (epipolar)
  int* queue;    // 3 buckets x n x 3 ints: nominal window; enlarged / masked / handed over; FP64 re-solve
  int* qcount;   // 16 ints (cleared per call): counts of buckets 0 and 1, work counters of the 2
                 // warp-group passes, count of bucket 2; [8] set when a staging wait timed out
  double* carry; // n x 8 or null: where the warp pass left a subset it hands to the multi-warp pass
  double band;   // relative margin around tol, added to the FP32 noise of |b|, within which an
                 // FP32 convergence test is re-decided by an FP64 re-solve of the subset (0: never)
  double noise;  // factor of the FP32 noise estimate of |b| added to the band
  int staging;   // 1: the warp passes stage the deformed window by TMA when they can; 0: gathers
  int slow_nw;   // warps per subset of the FP32 pass that continues the slow subsets: 2 or 4
  const double* F0;  // 4n initial displacement gradients [F11 F21 F12 F22] or null (the reference's 0)
  int slow_fp64; // 1: subsets still iterating after warp_cap are re-solved in FP64 (not the epipolar
                 // variant, whose slow subsets always take the FP32 multi-warp pass)
  int fp64_threads;  // threads per subset of the FP64 re-solve kernel: 128 or 256
  double* zncc;  // n or null (not epipolar): ZNCC of the window under the last evaluated warp,
                 // which is the returned [F U] for a converged subset (the acceptance test of a
                 // learned initial guess; sums of the last iteration, so no extra pass)
};
constexpr double kDefaultFp64Band = 1e-3;  // default IcgnArgs::band (plus the FP32 noise of |b|)
constexpr double kDefaultFp64Noise = 4.0;  // default IcgnArgs::noise (2x the calibrated need)

struct Sub1Args {
  FrameDev fr;
  int variant;  // 0 uniform (funICGN_Subpb1), 1 quadtree (funICGN_Subpb1quadtree)
  long long n;
  const double* coords;
  const double* UOld;
  const double* FOld;
  const double* vdual;
  const int* winsize_list;  // n x 2 (quadtree)
  int winsize;              // uniform winsize / nominal bucket size
  const double* HPar;       // n x 21 (uniform)
  double mu, tol;
  int warp_cap;  // as IcgnArgs::warp_cap
  double* U;
  int* conv;
  int* queue;   // 2 buckets x n x 4 ints
  int* qcount;  // 4: queue counts of the 2 buckets, work counters of the 2 warp-group passes
};

struct SearchArgs {
  const float* f;  // normalised REF
  const float* g;  // normalised DEF
  int M, N;
  int s0, s1;      // tempSizeOfSearchRegion
  int gx0, gx1, gy0, gy1;  // gridx, gridy (1-based)
  int winsize, step;
  int nx, ny;
  double* x;
  double* y;
  double* u;
  double* v;
  double* phi;
  double* I1;   // (M+1) x (N+1) integral images of g and g^2 (scratch)
  double* I2;
  double* tot;  // row-pass chunk totals (scratch, search_tot_bytes)
  void* tile_scratch;  // shared-product search scratch (search_tile_bytes bytes), or null
  cudaEvent_t ev_start, ev_stop;  // recorded around the correlation kernel when non-null
  int impl;   // 0: the shared-product tile kernel where one exists for (step, w + 1), else direct;
              // 1: the tile kernel (falls back to direct without one); 2: the direct kernel
  int chunk;  // tile kernel shift columns per pass: 16 or 24 (0: the shape's default)
  const int* list;  // grid subsets (i + j nx) to search, or null for the whole grid; with a list
                    // the direct kernel runs and writes the outputs compactly (slot k = list[k])
  long long nlist;
};
// Whether a shared-product tile kernel exists for (step, w + 1) and fits this device.
bool search_tile_available(int step, int winsize, int chunk);

// launchers return the number of kernels they enqueued (or < 0 on argument errors)
int launch_normalize(const void* img, int dtype, int M, int N, int gx0, int gx1, int gy0, int gy1,
                     const uint8_t* mask, float* out, double* stats, double* partials, int npartials,
                     unsigned int* counter, cudaStream_t st);
int launch_f64_to_f32(const double* in, long long n, float* out, cudaStream_t st);
int launch_f32_to_f64(const float* in, long long n, double* out, cudaStream_t st);
int launch_mask_binarize(const double* in, long long n, uint8_t* out, cudaStream_t st);
int launch_gradient(const float* img, const uint8_t* mask, int M, int N, float* gx, float* gy, cudaStream_t st);
int launch_interp_points(const float* img, int M, int N, long long n, const double* X, const double* Y, double* Z,
                         cudaStream_t st);
size_t icgn_smem_bytes(int w);       // FP32 general solve kernel, window w
size_t icgn_smem_bytes_f64(int w);   // FP64 re-solve kernel
constexpr int kIcgnQueueBuckets = 3;
size_t sub1_smem_bytes(int wx, int wy);
int launch_icgn(const IcgnArgs& a, int wmax_enlarged, cudaStream_t st);
// ZNCC of each subset's (w+1)^2 window of REF against DEF warped by P = [F U] (NaN where the
// warped window leaves [3, M-2] x [3, N-2]); FP32 interpolation, FP64 sums.
int launch_fallback_select(const int32_t* conv, const double* zncc, long long n, double zmin, int32_t* list,
                           int* count, cudaStream_t st);
int launch_subset_zncc(const FrameDev& fr, long long n, const double* coords, const double* U, const double* F,
                       int winsize, double* zncc, cudaStream_t st);
// Proposal network (cnn.cu): the network input of n subsets (n x 64 x 64 x 2 BF16) from frame fr.
int launch_net_patches(const FrameDev& fr, const double* coords, long long n, void* X, cudaStream_t st);
// Proposal network (cnn.cu): initial guesses of n subsets on frame fr.
int net_predict(struct ::aldic_net* net, const FrameDev& fr, const double* coords_dev, long long n, double* U0,
                double* F0);
int launch_subpb1(const Sub1Args& a, int wmax_x, int wmax_y, cudaStream_t st);
size_t search_smem_bytes(int winsize, int s0, int s1);
size_t search_tot_bytes(int M, int N);
int launch_search(const SearchArgs& a, cudaStream_t st);
// Shared-product search (search_tile.cu): scratch size (0 when the step / window pair has
// no tile kernel), and the launcher (returns the launch count, or -1 when not available).
constexpr int kDefaultWarpCap = 8;   // default IcgnArgs / Sub1Args warp_cap
size_t search_tile_bytes(int M, int N, int winsize, int step, int nx, int ny, int s0, int s1, int chunk = 0);
int launch_search_tile(const SearchArgs& a, cudaStream_t st);
struct CamPair {
  double P[24];  // P_L = K_L [I | 0] then P_R = K_R [R | T], each 3x4 row-major
};
size_t inpaint_scratch_bytes(long long mn);
int launch_inpaint(double* A, int m, int n, void* scratch, int* status, cudaStream_t st);
// Two grids in one launch (one CTA each): NaN entries of A0 / A1 solved into O0 / O1;
// scratch holds 2 x inpaint_scratch_bytes (each rounded up to 256); hint as the kernel's.
int launch_inpaint2(const double* A0, const double* A1, double* O0, double* O1, int m, int n, void* scratch,
                    const int* hint, int* status, cudaStream_t st);
int launch_interleave_u0(const double* u, const double* v, const double* fu, const double* fv, int ny, int nx,
                         double* U0, cudaStream_t st);
size_t del4_scratch_bytes(long long mn);
int launch_inpaint_del4(const double* A0, const double* A1, const double* X00, const double* X01, double* O0,
                        double* O1, int m, int n, int maxit, void* scratch, const int* hint, int* status,
                        cudaStream_t st);
int launch_nan_count(const double* u, const double* v, int m, int n, int* counts, cudaStream_t st);
int launch_median_fluct(const double* u, const double* v, const double* uf, const double* vf, int m, int n,
                        float* fu, float* fv, cudaStream_t st);
int launch_outlier_mark(const float* fu, const float* fv, int m, int n, float thr, double* u, double* v,
                        unsigned char* hole, int* count, cudaStream_t st);
int launch_restore_holes(const unsigned char* hole, int m, int n, double* u, double* v, cudaStream_t st);
// ALDIC's global step (Subpb2Quadtree), subpb2.cu
struct Subpb2Scalars;
size_t subpb2_scalars_bytes();
int subpb2_blocks(long long n);
int launch_subpb2_setup(int n_el, const int* elem, const double* coords, long long n, const double* U,
                        const double* F, int order, double beta, double mu, double alpha, const int* adj_ptr,
                        const int* adj, const unsigned char* free_, double* Ke, double* be, double* b, double* D,
                        double* x, double* r, double* z, double* p, double* part, Subpb2Scalars* sc,
                        cudaStream_t st);
int launch_subpb2_iterations(int iters, int n_el, const int* elem, long long n, const int* adj_ptr, const int* adj,
                             const double* Ke, const unsigned char* free_, const double* D, double* x, double* r,
                             double* z, double* p, double* q, double* part, double tol2, int maxit,
                             Subpb2Scalars* sc, cudaStream_t st);
// Host: the mesh tables of a Subpb2 call from the element table E (n_el x 8 column-major,
// 1-based, 0 = absent mid-side node) and the dirichlet node numbers: ptr / adj, each node's
// (element * 8 + slot) entries in element order; kind per node, 1 free, 2 dirichlet, 0
// neither.  Returns non-zero with a message for a bad node number.
int subpb2_mesh_tables(long long n, long long n_el, const int* E, long long n_dir, const int* dir,
                       std::vector<int>& ptr, std::vector<int>& adj, std::vector<unsigned char>& kind, char* msg,
                       size_t msg_len);
// (iterations, done, converged) of the last solve, from the device scalars (host copy).
void subpb2_read_status(const void* host_copy, int* it, int* done, int* ok);
int launch_spring_pass(const double* ut, const double* vt, double* ui, double* vi, int m, int n, int mode,
                       cudaStream_t st);
// dist = (k1, k2, k3, p1, p2); K 3 x 3 column-major (MATLAB)
int launch_undistort_points(long long n, const double* pts, const double* K, const double* dist, double* out,
                            cudaStream_t st);
int launch_triangulate(long long n, const double* pairs, const CamPair& cams, double* xyz, double* err,
                       cudaStream_t st);
int launch_fp32_probe(int blocks, int threads, int iters, float* out, bool packed, cudaStream_t st);

}  // namespace aldic
