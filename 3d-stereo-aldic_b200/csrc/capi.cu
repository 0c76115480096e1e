// C ABI of the ALDIC B200 library: context (stream, device frame, scratch), argument
// staging between host and device memory, and the batched entry points declared in
// include/aldic_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "../../include/aldic_b200.h"
#include "kernels.h"

using namespace aldic;

namespace {

// Device scratch arena: bump allocation per call, reset at the start of every call.
// Growth synchronises the stream first, so earlier work never sees freed memory.
struct Arena {
  char* base = nullptr;
  size_t cap = 0, used = 0;
};

}  // namespace

struct aldic_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t launches = 0;
  // device frame
  int M = 0, N = 0;
  float* img[2] = {nullptr, nullptr};
  bool img_ok[2] = {false, false};
  uint8_t* mask = nullptr;
  bool has_mask = false;
  float* gx = nullptr;
  float* gy = nullptr;
  bool grad_ok = false;
  bool grad_from_mask = false;  // gradients computed here (they depend on the mask)
  // persistent scratch
  double* stats = nullptr;  // 4 doubles: sum, sum sq dev, mean, std
  double* partials = nullptr;
  unsigned int* counter = nullptr;
  int npartials = 0;
  int* qcount = nullptr;
  int* sel_count = nullptr;  // aldic_fallback_select's counter
  double* I1 = nullptr;
  double* I2 = nullptr;
  double* iitot = nullptr;
  size_t ii_cap = 0;
  void* tscratch = nullptr;  // shared-product search scratch
  size_t tscratch_cap = 0;
  int warp_cap = kDefaultWarpCap;  // aldic_set_iteration_cap
  double fp64_band = kDefaultFp64Band;  // aldic_set_fp64_band
  double fp64_noise = kDefaultFp64Noise;  // aldic_set_fp64_band
  // tuning options (aldic_set_option); with autotune on, each call shape takes the winner of
  // its first call's candidate runs instead (tuned below)
  int staging = 0;      // ALDIC_OPT_STAGING
  int slow_nw = 2;      // ALDIC_OPT_SLOW_WARPS (FP32 slow pass, with ALDIC_OPT_SLOW_FP64 0)
  int slow_fp64 = 0;    // ALDIC_OPT_SLOW_FP64
  int fp64_threads = 128;  // ALDIC_OPT_FP64_THREADS
  int search_impl = 0;  // ALDIC_OPT_SEARCH_IMPL
  int search_chunk = 0; // ALDIC_OPT_SEARCH_CHUNK
  int autotune = 0;     // ALDIC_OPT_AUTOTUNE
  struct Tuned {
    std::string choice;                    // the winner, as JSON
    std::vector<std::pair<std::string, double>> ms;  // every candidate's time (ms; < 0: results differed)
    int a = 0, b = 0, c = 0, d = 0;        // the winner's settings
  };
  std::map<std::string, Tuned> tuned;  // call-shape key -> winner
  // aldic_subpb2_set_mesh: the resident global-step mesh tables (element table, node ->
  // element lists, node kinds) in one device buffer
  char* sp2 = nullptr;
  size_t sp2_cap = 0;
  int64_t sp2_n = 0, sp2_nel = 0;
  size_t sp2_nadj = 0;
  // profiling: event pairs around the correlation kernel of each integer search
  bool prof = false;
  std::vector<cudaEvent_t> prof_ev;  // 2 per record
  int prof_n = 0;
  Arena arena;
  // outputs to copy back at the end of a call
  struct Back {
    void* host;
    const void* dev;
    size_t bytes;
  };
  std::vector<Back> back;
};

namespace {

int fail(aldic_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

int cuda_fail(aldic_ctx* c, cudaError_t e, const char* what) {
  return fail(c, ALDIC_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                         \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
  } while (0)

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

int arena_reserve(aldic_ctx* c, size_t bytes) {
  if (c->arena.cap >= bytes) return ALDIC_OK;
  CK(cudaStreamSynchronize(c->stream));
  if (c->arena.base) CK(cudaFree(c->arena.base));
  c->arena.base = nullptr;
  size_t cap = bytes + bytes / 2 + (1 << 20);
  CK(cudaMalloc(&c->arena.base, cap));
  c->arena.cap = cap;
  return ALDIC_OK;
}

void* arena_take(aldic_ctx* c, size_t bytes) {
  const size_t off = (c->arena.used + 255) & ~size_t(255);
  c->arena.used = off + bytes;
  return c->arena.base + off;
}

// Staging plan: the caller lists every array argument with its size, then the arena is
// sized once and host arrays are copied in (inputs) or scheduled for copy-back (outputs).
struct Arg {
  const void* user;
  size_t bytes;
  bool output;
  void* dev;
};

int stage(aldic_ctx* c, std::vector<Arg*> args) {
  c->arena.used = 0;
  c->back.clear();
  size_t need = 0;
  for (Arg* a : args)
    if (a->user && !is_device_ptr(a->user) && a->bytes) need += ((a->bytes + 255) & ~size_t(255)) + 256;
  int rc = arena_reserve(c, need);
  if (rc) return rc;
  for (Arg* a : args) {
    if (!a->user || a->bytes == 0) {
      a->dev = nullptr;
      continue;
    }
    if (is_device_ptr(a->user)) {
      a->dev = const_cast<void*>(a->user);
      continue;
    }
    a->dev = arena_take(c, a->bytes);
    if (a->output) {
      c->back.push_back({const_cast<void*>(a->user), a->dev, a->bytes});
    } else {
      CK(cudaMemcpyAsync(a->dev, a->user, a->bytes, cudaMemcpyHostToDevice, c->stream));
    }
  }
  return ALDIC_OK;
}

// Copy host outputs back and wait for them; otherwise leave the work in flight.
int finish(aldic_ctx* c, int launched) {
  c->launches += launched;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
  for (auto& b : c->back) CK(cudaMemcpyAsync(b.host, b.dev, b.bytes, cudaMemcpyDeviceToHost, c->stream));
  if (!c->back.empty()) CK(cudaStreamSynchronize(c->stream));
  c->back.clear();
  return ALDIC_OK;
}

int ensure_frame(aldic_ctx* c, int M, int N) {
  if (M < 8 || N < 8) return fail(c, ALDIC_ERR_ARG, "image must be at least 8 x 8 (got %d x %d)", M, N);
  if (c->M == M && c->N == N && c->img[0]) return ALDIC_OK;
  CK(cudaStreamSynchronize(c->stream));
  for (int s = 0; s < 2; ++s)
    if (c->img[s]) CK(cudaFree(c->img[s]));
  if (c->mask) CK(cudaFree(c->mask));
  if (c->gx) CK(cudaFree(c->gx));
  if (c->gy) CK(cudaFree(c->gy));
  const size_t npx = (size_t)M * N, ng = (size_t)(M - 6) * (N - 6);
  for (int s = 0; s < 2; ++s) CK(cudaMalloc(&c->img[s], npx * sizeof(float)));
  CK(cudaMalloc(&c->mask, npx));
  CK(cudaMalloc(&c->gx, ng * sizeof(float)));
  CK(cudaMalloc(&c->gy, ng * sizeof(float)));
  c->M = M;
  c->N = N;
  c->img_ok[0] = c->img_ok[1] = false;
  c->has_mask = false;
  c->grad_ok = false;
  return ALDIC_OK;
}

int need_frame(aldic_ctx* c, bool grads) {
  if (!c->img_ok[0] || !c->img_ok[1]) return fail(c, ALDIC_ERR_STATE, "reference and deformed images must be loaded");
  if (grads && !c->grad_ok) return fail(c, ALDIC_ERR_STATE, "gradients not set (aldic_compute_gradients / aldic_set_gradients)");
  return ALDIC_OK;
}

FrameDev frame_of(aldic_ctx* c) {
  FrameDev f;
  f.ref = c->img[0];
  f.def = c->img[1];
  f.mask = c->has_mask ? c->mask : nullptr;
  f.gx = c->gx;
  f.gy = c->gy;
  f.M = c->M;
  f.N = c->N;
  return f;
}

size_t dtype_size(int dt) {
  switch (dt) {
    case ALDIC_U8: return 1;
    case ALDIC_U16: return 2;
    case ALDIC_F32: return 4;
    case ALDIC_F64: return 8;
    default: return 0;
  }
}

}  // namespace

extern "C" {

int aldic_abi_version(void) { return 1; }

int aldic_create(aldic_ctx** out, int device) {
  if (!out) return ALDIC_ERR_ARG;
  *out = nullptr;
  aldic_ctx* c = new aldic_ctx();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    c->stream = c->own;
    c->npartials = 148 * 8;
    e = cudaMalloc(&c->stats, 8 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&c->partials, c->npartials * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&c->counter, 64);
    if (e == cudaSuccess) e = cudaMemset(c->counter, 0, 64);
    if (e == cudaSuccess) e = cudaMalloc(&c->qcount, 64);
  }
  if (e != cudaSuccess) {
    delete c;
    return ALDIC_ERR_CUDA;
  }
  *out = c;
  return ALDIC_OK;
}

void aldic_destroy(aldic_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  void* bufs[] = {c->img[0], c->img[1], c->mask, c->gx, c->gy, c->stats, c->partials, c->counter, c->qcount,
                  c->I1, c->I2, c->iitot, c->tscratch, c->arena.base, c->sp2, c->sel_count};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
}

const char* aldic_last_error(const aldic_ctx* c) { return c ? c->err.c_str() : "null context"; }

int aldic_set_stream(aldic_ctx* c, void* stream) {
  if (!c) return ALDIC_ERR_ARG;
  c->stream = stream ? (cudaStream_t)stream : c->own;
  return ALDIC_OK;
}

int aldic_synchronize(aldic_ctx* c) {
  if (!c) return ALDIC_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  return ALDIC_OK;
}

int64_t aldic_launch_count(const aldic_ctx* c) { return c ? c->launches : -1; }

int aldic_load_image_raw(aldic_ctx* c, int slot, const void* img, int dtype, int M, int N, const int* gridx,
                         const int* gridy, const double* mask, double* mean_std) {
  if (!c) return ALDIC_ERR_ARG;
  if (slot != 0 && slot != 1) return fail(c, ALDIC_ERR_ARG, "slot must be ALDIC_SLOT_REF or ALDIC_SLOT_DEF");
  const size_t es = dtype_size(dtype);
  if (!img || !es) return fail(c, ALDIC_ERR_ARG, "image pointer or dtype invalid");
  if (!gridx || !gridy) return fail(c, ALDIC_ERR_ARG, "gridx/gridy required");
  int rc = ensure_frame(c, M, N);
  if (rc) return rc;
  // ROI clamp (funNormalizeImg.m:112-115)
  int gx0 = gridx[0] < 1 ? 1 : gridx[0], gx1 = gridx[1] > M ? M : gridx[1];
  int gy0 = gridy[0] < 1 ? 1 : gridy[0], gy1 = gridy[1] > N ? N : gridy[1];
  if (gx1 < gx0 || gy1 < gy0 || (long long)(gx1 - gx0 + 1) * (gy1 - gy0 + 1) < 2)
    return fail(c, ALDIC_ERR_ARG, "ROI must hold at least two pixels");
  const size_t npx = (size_t)M * N;
  Arg ai{img, npx * es, false, nullptr}, am{mask, mask ? npx * sizeof(double) : 0, false, nullptr};
  Arg ams{mean_std, mean_std ? 2 * sizeof(double) : 0, true, nullptr};
  rc = stage(c, {&ai, &am, &ams});
  if (rc) return rc;
  int launched = 0;
  uint8_t* mk = nullptr;
  if (am.dev) {
    mk = (uint8_t*)arena_take(c, npx);
    launched += launch_mask_binarize((const double*)am.dev, (long long)npx, mk, c->stream);
  }
  launched += launch_normalize(ai.dev, dtype, M, N, gx0 - 1, gx1, gy0 - 1, gy1, mk, c->img[slot], c->stats,
                               c->partials, c->npartials, c->counter, c->stream);
  if (ams.dev) CK(cudaMemcpyAsync(ams.dev, c->stats + 2, 2 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  c->img_ok[slot] = true;
  if (slot == 0) c->grad_ok = false;
  return finish(c, launched);
}

int aldic_load_image(aldic_ctx* c, int slot, const double* img, int M, int N) {
  if (!c) return ALDIC_ERR_ARG;
  if (slot != 0 && slot != 1) return fail(c, ALDIC_ERR_ARG, "slot must be ALDIC_SLOT_REF or ALDIC_SLOT_DEF");
  if (!img) return fail(c, ALDIC_ERR_ARG, "image pointer is NULL");
  int rc = ensure_frame(c, M, N);
  if (rc) return rc;
  const size_t npx = (size_t)M * N;
  Arg ai{img, npx * sizeof(double), false, nullptr};
  rc = stage(c, {&ai});
  if (rc) return rc;
  const int l = launch_f64_to_f32((const double*)ai.dev, (long long)npx, c->img[slot], c->stream);
  c->img_ok[slot] = true;
  if (slot == 0) c->grad_ok = false;
  return finish(c, l);
}

int aldic_set_mask(aldic_ctx* c, const double* mask, int M, int N) {
  if (!c) return ALDIC_ERR_ARG;
  if (c->M != M || c->N != N) return fail(c, ALDIC_ERR_ARG, "mask size %d x %d differs from the frame", M, N);
  if (!mask) {
    c->has_mask = false;
    if (c->grad_from_mask) c->grad_ok = false;
    return ALDIC_OK;
  }
  const size_t npx = (size_t)M * N;
  Arg am{mask, npx * sizeof(double), false, nullptr};
  int rc = stage(c, {&am});
  if (rc) return rc;
  const int l = launch_mask_binarize((const double*)am.dev, (long long)npx, c->mask, c->stream);
  c->has_mask = true;
  if (c->grad_from_mask) c->grad_ok = false;  // device-computed gradients carry the old mask
  return finish(c, l);
}

int aldic_compute_gradients(aldic_ctx* c) {
  if (!c) return ALDIC_ERR_ARG;
  if (!c->img_ok[0]) return fail(c, ALDIC_ERR_STATE, "reference image not loaded");
  c->arena.used = 0;
  c->back.clear();
  const int l = launch_gradient(c->img[0], c->has_mask ? c->mask : nullptr, c->M, c->N, c->gx, c->gy, c->stream);
  c->grad_ok = true;
  c->grad_from_mask = true;
  return finish(c, l);
}

int aldic_set_gradients(aldic_ctx* c, const double* dfdx, const double* dfdy, int M6, int N6) {
  if (!c) return ALDIC_ERR_ARG;
  if (!dfdx || !dfdy) return fail(c, ALDIC_ERR_ARG, "gradient pointers are NULL");
  if (M6 != c->M - 6 || N6 != c->N - 6)
    return fail(c, ALDIC_ERR_ARG, "gradients must be (M-6) x (N-6) = %d x %d", c->M - 6, c->N - 6);
  const size_t ng = (size_t)M6 * N6;
  Arg ax{dfdx, ng * sizeof(double), false, nullptr}, ay{dfdy, ng * sizeof(double), false, nullptr};
  int rc = stage(c, {&ax, &ay});
  if (rc) return rc;
  int l = launch_f64_to_f32((const double*)ax.dev, (long long)ng, c->gx, c->stream);
  l += launch_f64_to_f32((const double*)ay.dev, (long long)ng, c->gy, c->stream);
  c->grad_ok = true;
  c->grad_from_mask = false;
  return finish(c, l);
}

int aldic_get_state(aldic_ctx* c, int what, double* out) {
  if (!c || !out) return ALDIC_ERR_ARG;
  const float* src = nullptr;
  size_t n = 0;
  if (what == 0 || what == 1) {
    if (!c->img_ok[what]) return fail(c, ALDIC_ERR_STATE, "image slot %d not loaded", what);
    src = c->img[what];
    n = (size_t)c->M * c->N;
  } else if (what == 2 || what == 3) {
    if (!c->grad_ok) return fail(c, ALDIC_ERR_STATE, "gradients not set");
    src = what == 2 ? c->gx : c->gy;
    n = (size_t)(c->M - 6) * (c->N - 6);
  } else {
    return fail(c, ALDIC_ERR_ARG, "unknown state %d", what);
  }
  Arg ao{out, n * sizeof(double), true, nullptr};
  int rc = stage(c, {&ao});
  if (rc) return rc;
  return finish(c, launch_f32_to_f64(src, (long long)n, (double*)ao.dev, c->stream));
}

int aldic_interp2(aldic_ctx* c, int slot, int64_t n, const double* X, const double* Y, double* Z) {
  if (!c) return ALDIC_ERR_ARG;
  if (slot != 0 && slot != 1) return fail(c, ALDIC_ERR_ARG, "bad slot");
  if (!c->img_ok[slot]) return fail(c, ALDIC_ERR_STATE, "image slot %d not loaded", slot);
  if (n < 0 || (n > 0 && (!X || !Y || !Z))) return fail(c, ALDIC_ERR_ARG, "bad point arrays");
  if (n == 0) return ALDIC_OK;
  Arg ax{X, n * sizeof(double), false, nullptr}, ay{Y, n * sizeof(double), false, nullptr};
  Arg az{Z, n * sizeof(double), true, nullptr};
  int rc = stage(c, {&ax, &ay, &az});
  if (rc) return rc;
  const int l = launch_interp_points(c->img[slot], c->M, c->N, n, (const double*)ax.dev, (const double*)ay.dev,
                                     (double*)az.dev, c->stream);
  return finish(c, l);
}

int aldic_search_grid(const int* gridx, const int* gridy, int winsize, int step, int* nx, int* ny) {
  if (!gridx || !gridy || !nx || !ny || step <= 0 || winsize < 0) return ALDIC_ERR_ARG;
  const int ex = gridx[1] - winsize - step, ey = gridy[1] - winsize - step;
  *nx = ex >= gridx[0] ? (ex - gridx[0]) / step + 1 : 0;
  *ny = ey >= gridy[0] ? (ey - gridy[0]) / step + 1 : 0;
  return ALDIC_OK;
}

static int tune_search(aldic_ctx* c, SearchArgs& a);  // the autotuner (below)
static int search_common(aldic_ctx* c, const int* search, const int* gridx, const int* gridy, int winsize, int step,
                         int64_t nlist, const int32_t* list, double* x, double* y, double* u, double* v, double* phi);

int aldic_integer_search(aldic_ctx* c, const int* search, const int* gridx, const int* gridy, int winsize, int step,
                         double* x, double* y, double* u, double* v, double* phi) {
  return search_common(c, search, gridx, gridy, winsize, step, -1, nullptr, x, y, u, v, phi);
}

int aldic_integer_search_list(aldic_ctx* c, const int* search, const int* gridx, const int* gridy, int winsize,
                              int step, int64_t n, const int32_t* list, double* x, double* y, double* u, double* v,
                              double* phi) {
  if (!c) return ALDIC_ERR_ARG;
  if (n < 0 || (n > 0 && !list)) return fail(c, ALDIC_ERR_ARG, "a list of n >= 0 grid subsets is required");
  return search_common(c, search, gridx, gridy, winsize, step, n, list, x, y, u, v, phi);
}

static int search_common(aldic_ctx* c, const int* search, const int* gridx, const int* gridy, int winsize, int step,
                         int64_t nlist, const int32_t* list, double* x, double* y, double* u, double* v, double* phi) {
  if (!c) return ALDIC_ERR_ARG;
  int rc = need_frame(c, false);
  if (rc) return rc;
  if (!search || !gridx || !gridy) return fail(c, ALDIC_ERR_ARG, "search/gridx/gridy required");
  if (winsize < 2 || step < 1) return fail(c, ALDIC_ERR_ARG, "winsize >= 2 and step >= 1 required");
  if (search[0] < 0 || search[1] < 0) return fail(c, ALDIC_ERR_ARG, "search region must be non-negative");
  if (winsize > 120) return fail(c, ALDIC_ERR_ARG, "winsize %d too large for the device search", winsize);
  if (search[0] + search[1] > 2000) return fail(c, ALDIC_ERR_ARG, "search region too large");
  int nx, ny;
  aldic_search_grid(gridx, gridy, winsize, step, &nx, &ny);
  const size_t ngrid = (size_t)nx * ny;
  const size_t n = nlist >= 0 ? (size_t)nlist : ngrid;  // output slots
  if (n == 0 || ngrid == 0) return ALDIC_OK;
  if (!x || !y || !u || !v || !phi) return fail(c, ALDIC_ERR_ARG, "output arrays required");
  const size_t iin = (size_t)(c->M + 1) * (c->N + 1);
  if (c->ii_cap < iin) {
    CK(cudaStreamSynchronize(c->stream));
    if (c->I1) CK(cudaFree(c->I1));
    if (c->I2) CK(cudaFree(c->I2));
    if (c->iitot) CK(cudaFree(c->iitot));
    c->I1 = c->I2 = c->iitot = nullptr;
    CK(cudaMalloc(&c->I1, iin * sizeof(double)));
    CK(cudaMalloc(&c->I2, iin * sizeof(double)));
    CK(cudaMalloc(&c->iitot, search_tot_bytes(c->M, c->N)));
    c->ii_cap = iin;
  }
  // scratch for the tile kernel whenever one exists (the autotuner may choose either chunk)
  const size_t tbytes = list ? 0 : search_tile_bytes(c->M, c->N, winsize, step, nx, ny, search[0], search[1], 0);
  if (tbytes > c->tscratch_cap) {
    CK(cudaStreamSynchronize(c->stream));
    if (c->tscratch) CK(cudaFree(c->tscratch));
    c->tscratch = nullptr;
    c->tscratch_cap = 0;
    CK(cudaMalloc(&c->tscratch, tbytes));
    c->tscratch_cap = tbytes;
  }
  Arg ox{x, n * 8, true, nullptr}, oy{y, n * 8, true, nullptr}, ou{u, n * 8, true, nullptr};
  Arg ov{v, n * 8, true, nullptr}, op{phi, n * 8, true, nullptr};
  Arg al{list, list ? n * 4 : 0, false, nullptr};
  rc = stage(c, {&ox, &oy, &ou, &ov, &op, &al});
  if (rc) return rc;
  if (list) {  // every entry a grid subset
    std::vector<int32_t> hl(n);
    if (is_device_ptr(list)) {
      CK(cudaMemcpyAsync(hl.data(), list, n * 4, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    } else {
      std::memcpy(hl.data(), list, n * 4);
    }
    for (int32_t t : hl)
      if (t < 0 || (size_t)t >= ngrid) return fail(c, ALDIC_ERR_ARG, "list entry %d outside the grid of %zu", (int)t, ngrid);
  }
  SearchArgs a;
  a.f = c->img[0];
  a.g = c->img[1];
  a.M = c->M;
  a.N = c->N;
  a.s0 = search[0];
  a.s1 = search[1];
  a.gx0 = gridx[0];
  a.gx1 = gridx[1];
  a.gy0 = gridy[0];
  a.gy1 = gridy[1];
  a.winsize = winsize;
  a.step = step;
  a.nx = nx;
  a.ny = ny;
  a.x = (double*)ox.dev;
  a.y = (double*)oy.dev;
  a.u = (double*)ou.dev;
  a.v = (double*)ov.dev;
  a.phi = (double*)op.dev;
  a.I1 = c->I1;
  a.I2 = c->I2;
  a.tot = c->iitot;
  a.tile_scratch = tbytes ? c->tscratch : nullptr;
  a.ev_start = a.ev_stop = nullptr;
  a.impl = c->search_impl;
  a.chunk = c->search_chunk;
  a.list = (const int*)al.dev;
  a.nlist = list ? (long long)n : 0;
  if (c->autotune && !list) {
    rc = tune_search(c, a);
    if (rc) return rc;
  }
  if (c->prof && 2 * (c->prof_n + 1) <= (int)c->prof_ev.size()) {
    a.ev_start = c->prof_ev[2 * c->prof_n];
    a.ev_stop = c->prof_ev[2 * c->prof_n + 1];
    ++c->prof_n;
  }
  return finish(c, launch_search(a, c->stream));
}

// ------------------------------------------------------------------------ autotuner
// The first call of each call shape (with ALDIC_OPT_AUTOTUNE on) runs every candidate
// configuration on its own inputs, each twice (the second run timed with CUDA events on the
// context's stream), checks that every candidate's results agree with the first's, and keeps
// the fastest agreeing one for that shape; later calls of the shape take it without timing.
// The call itself then runs (returns) the winner's results.  Keys bucket n by powers of two.
static std::string shape_key(const char* kind, std::initializer_list<long long> v) {
  std::string k = kind;
  for (long long x : v) k += ":" + std::to_string(x);
  return k;
}

static int log2_bucket(long long n) {
  int b = 0;
  while ((1LL << (b + 1)) <= n) ++b;
  return b;
}

static int time_on_stream(aldic_ctx* c, const std::function<int()>& run, double* ms) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  c->launches += run();  // warm-up run (first-use attribute set-up, caches)
  CK(cudaEventRecord(e0, c->stream));
  c->launches += run();
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaGetLastError());
  *ms = t;
  return ALDIC_OK;
}

static int tune_icgn(aldic_ctx* c, IcgnArgs& a, int wmax) {
  const std::string key = shape_key("icgn", {a.variant, a.winsize, log2_bucket(a.n)});
  auto it = c->tuned.find(key);
  if (it == c->tuned.end()) {
    aldic_ctx::Tuned tn;
    std::vector<int32_t> conv0((size_t)a.n), conv1((size_t)a.n);
    std::vector<double> U0v((size_t)a.n * 2), U1v((size_t)a.n * 2);
    double best = 1e300;
    bool first = true;
    // staging x warps per subset of the FP32 slow pass x threads per subset of the FP64
    // re-solve x the warp pass's iteration cap
    for (int staging = 0; staging <= 1; ++staging)
      for (int snw : {2, 4})
        for (int f64t : {128, 512})
          for (int cap : {8, 16}) {
            IcgnArgs b = a;
            b.staging = staging;
            b.slow_nw = snw;
            b.fp64_threads = f64t;
            b.warp_cap = cap;
          double ms = 0;
          int rc = time_on_stream(c, [&] { return launch_icgn(b, wmax, c->stream); }, &ms);
          if (rc) return rc;
          // results of this candidate against the first: the codes exactly (the FP64 re-solve of
          // near-threshold tests makes them independent of summation order), U to 1e-5 px where
          // the subset converged (a non-converged subset's U is whatever its 100 iterations left)
          std::vector<int32_t>& cv = first ? conv0 : conv1;
          std::vector<double>& uv = first ? U0v : U1v;
          CK(cudaMemcpyAsync(cv.data(), b.conv, cv.size() * 4, cudaMemcpyDeviceToHost, c->stream));
          CK(cudaMemcpyAsync(uv.data(), b.U, uv.size() * 8, cudaMemcpyDeviceToHost, c->stream));
          CK(cudaStreamSynchronize(c->stream));
          bool agree = true;
          if (!first) {
            for (size_t i = 0; i < conv0.size() && agree; ++i) agree = conv0[i] == conv1[i];
            for (size_t i = 0; i < U0v.size() && agree; ++i) {
              const int cd = conv0[i / 2];
              if (cd < 1 || cd > 100) continue;
              agree = (std::isnan(U0v[i]) && std::isnan(U1v[i])) || std::fabs(U0v[i] - U1v[i]) <= 1e-5;
            }
          }
          first = false;
          char name[80];
          std::snprintf(name, sizeof(name), "staging%d_slow%d_fp64threads%d_cap%d", staging, snw, f64t, cap);
          tn.ms.push_back({name, agree ? ms : -ms});
          if (agree && ms < best) {
            best = ms;
            tn.a = staging;
            tn.b = snw;
            tn.c = cap;
            tn.d = f64t;
          }
        }
    char ch[200];
    std::snprintf(ch, sizeof(ch),
                  "{\"staging\": %d, \"slow_warps\": %d, \"fp64_threads\": %d, \"iteration_cap\": %d}", tn.a, tn.b,
                  tn.d, tn.c);
    tn.choice = ch;
    it = c->tuned.emplace(key, tn).first;
  }
  a.staging = it->second.a;
  a.slow_nw = it->second.b;
  a.fp64_threads = it->second.d;
  a.warp_cap = it->second.c;
  return ALDIC_OK;
}

static int tune_search(aldic_ctx* c, SearchArgs& a) {
  const std::string key = shape_key("search", {a.M, a.N, a.winsize, a.step, a.s0, a.s1, a.nx, a.ny});
  auto it = c->tuned.find(key);
  if (it == c->tuned.end()) {
    aldic_ctx::Tuned tn;
    const size_t n = (size_t)a.nx * a.ny;
    std::vector<double> u0(n), v0(n), p0(n), u1(n), v1(n), p1(n);
    double best = 1e300;
    bool first = true;
    struct Cand {
      int impl, chunk;
      const char* name;
    };
    const Cand cands[] = {{1, 24, "tile24"}, {1, 16, "tile16"}, {2, 0, "direct"}};
    for (const Cand& cd : cands) {
      if (cd.impl == 1 && (!a.tile_scratch || !search_tile_available(a.step, a.winsize, cd.chunk))) continue;
      SearchArgs b = a;
      b.impl = cd.impl;
      b.chunk = cd.chunk;
      b.ev_start = b.ev_stop = nullptr;
      double ms = 0;
      int rc = time_on_stream(c, [&] { return launch_search(b, c->stream); }, &ms);
      if (rc) return rc;
      CK(cudaMemcpyAsync((first ? u0 : u1).data(), b.u, n * 8, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync((first ? v0 : v1).data(), b.v, n * 8, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync((first ? p0 : p1).data(), b.phi, n * 8, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      bool agree = true;
      if (!first)  // u, v identical (both implementations match the FP64 search exactly), phi to 1e-5
        for (size_t i = 0; i < n && agree; ++i) {
          const bool un = std::isnan(u0[i]) && std::isnan(u1[i]), vn = std::isnan(v0[i]) && std::isnan(v1[i]);
          const bool pn = std::isnan(p0[i]) && std::isnan(p1[i]);
          agree = (un || u0[i] == u1[i]) && (vn || v0[i] == v1[i]) && (pn || std::fabs(p0[i] - p1[i]) <= 1e-5);
        }
      first = false;
      tn.ms.push_back({cd.name, agree ? ms : -ms});
      if (agree && ms < best) {
        best = ms;
        tn.a = cd.impl;
        tn.b = cd.chunk;
      }
    }
    char ch[160];
    std::snprintf(ch, sizeof(ch), "{\"search\": \"%s\"}",
                  tn.a == 2 ? "direct" : (tn.b == 16 ? "tile16" : "tile24"));
    tn.choice = ch;
    it = c->tuned.emplace(key, tn).first;
  }
  a.impl = it->second.a;
  a.chunk = it->second.b;
  return ALDIC_OK;
}

static int icgn_common(aldic_ctx* c, int variant, int64_t n, const double* coords, const double* U0, int winsize,
                       double tol, double* U, double* F, double* H, int32_t* conv, uint8_t* mark, double* znssd,
                       const double* F0 = nullptr, double* zncc = nullptr) {
  int rc = need_frame(c, true);
  if (rc) return rc;
  if (n < 0) return fail(c, ALDIC_ERR_ARG, "n < 0");
  if (n == 0) return ALDIC_OK;
  if (n > (1LL << 30)) return fail(c, ALDIC_ERR_ARG, "too many subsets");
  if (winsize < 2 || winsize > 200) return fail(c, ALDIC_ERR_ARG, "winsize %d out of range [2, 200]", winsize);
  if (!coords) return fail(c, ALDIC_ERR_ARG, "coords required");
  const bool epi = (variant == 2);
  if (!epi && (!U0 || !U || !F || !conv)) return fail(c, ALDIC_ERR_ARG, "U0, U, F and conv are required");
  if (epi && !znssd) return fail(c, ALDIC_ERR_ARG, "znssd output required");
  // largest enlarged window (funICGN.m:61 / funICGNQuadtree.m:70)
  int wmax;
  const double w = winsize, Nw = (w + 1) * (w + 1);
  if (variant == 1) {
    // masked count < 0.4 (w+1)^2, so the growth factor is below sqrt(1/0.6)
    wmax = (int)(2 * std::ceil(std::sqrt(1.0 / 0.6) * w / 2)) + 2;
  } else {
    wmax = (int)std::round(std::sqrt(2.0) * w);
  }
  if (wmax < winsize) wmax = winsize;
  if (icgn_smem_bytes(wmax) > 200 * 1024) return fail(c, ALDIC_ERR_ARG, "winsize %d too large for shared memory", winsize);
  const size_t qbytes = (size_t)kIcgnQueueBuckets * n * 3 * sizeof(int);
  Arg ac{coords, (size_t)n * 2 * 8, false, nullptr}, au0{epi ? nullptr : U0, epi ? 0 : (size_t)n * 2 * 8, false, nullptr};
  Arg au{U, epi ? 0 : (size_t)n * 2 * 8, true, nullptr}, af{F, epi ? 0 : (size_t)n * 4 * 8, true, nullptr};
  Arg ah{H, H ? (size_t)n * 21 * 8 : 0, true, nullptr};
  Arg acv{conv, conv ? (size_t)n * 4 : 0, true, nullptr};
  Arg am{mark, mark ? (size_t)n : 0, true, nullptr};
  Arg az{znssd, znssd ? (size_t)n * 8 : 0, true, nullptr};
  Arg af0{F0, F0 ? (size_t)n * 4 * 8 : 0, false, nullptr};
  Arg azc{zncc, zncc ? (size_t)n * 8 : 0, true, nullptr};
  // the work queue comes from the arena too: reserve room for it with the staged arguments
  c->arena.used = 0;
  rc = arena_reserve(c, qbytes + 4096 + (size_t)n * (2 + 2 + 2 + 4 + 4 + 21 + 1 + 1 + 1 + 8) * 8 + 8192);
  if (rc) return rc;
  rc = stage(c, {&ac, &au0, &au, &af, &ah, &acv, &am, &az, &af0, &azc});
  if (rc) return rc;
  // subsets that no pass solves (their window leaves the image) keep a NaN ZNCC (all-ones bits)
  if (zncc) CK(cudaMemsetAsync(azc.dev, 0xFF, (size_t)n * 8, c->stream));
  IcgnArgs a;
  a.fr = frame_of(c);
  a.variant = variant;
  a.n = n;
  a.coords = (const double*)ac.dev;
  a.U0 = (const double*)au0.dev;
  a.winsize = winsize;
  a.tol = tol;
  a.max_iter = epi ? 30 : 100;
  a.warp_cap = c->warp_cap;
  a.crop = epi ? 4 : 3;
  a.U = (double*)au.dev;
  a.F = (double*)af.dev;
  a.H = (double*)ah.dev;
  a.conv = (int*)acv.dev;
  a.mark = (uint8_t*)am.dev;
  a.znssd = (double*)az.dev;
  a.queue = (int*)arena_take(c, qbytes);
  a.qcount = c->qcount;
  a.carry = (double*)arena_take(c, (size_t)n * 8 * sizeof(double));
  // the FP64 re-solve needs its (larger) shared-memory window; beyond that, FP32 decides alone
  a.band = icgn_smem_bytes_f64(wmax) <= 200 * 1024 ? c->fp64_band : 0.0;
  a.noise = c->fp64_noise;
  a.F0 = (const double*)af0.dev;
  a.staging = c->staging;
  a.slow_nw = c->slow_nw;
  a.slow_fp64 = c->slow_fp64;
  a.fp64_threads = c->fp64_threads;
  a.zncc = (double*)azc.dev;
  if (c->autotune && !epi) {
    rc = tune_icgn(c, a, wmax);
    if (rc) return rc;
  }
  return finish(c, launch_icgn(a, wmax, c->stream));
}

int aldic_local_icgn(aldic_ctx* c, int variant, int64_t n, const double* coords, const double* U0, int winsize,
                     double tol, double* U, double* F, double* H, int32_t* conv, uint8_t* markHole) {
  if (!c) return ALDIC_ERR_ARG;
  if (variant != ALDIC_UNIFORM && variant != ALDIC_QUADTREE) return fail(c, ALDIC_ERR_ARG, "bad variant %d", variant);
  return icgn_common(c, variant, n, coords, U0, winsize, tol, U, F, H, conv,
                     variant == ALDIC_QUADTREE ? markHole : nullptr, nullptr);
}

int aldic_local_icgn_guess(aldic_ctx* c, int variant, int64_t n, const double* coords, const double* U0,
                           const double* F0, int winsize, double tol, double* U, double* F, double* H, int32_t* conv,
                           uint8_t* markHole, double* zncc) {
  if (!c) return ALDIC_ERR_ARG;
  if (variant != ALDIC_UNIFORM && variant != ALDIC_QUADTREE) return fail(c, ALDIC_ERR_ARG, "bad variant %d", variant);
  if (!F0) return fail(c, ALDIC_ERR_ARG, "F0 required (aldic_local_icgn starts from F = 0)");
  return icgn_common(c, variant, n, coords, U0, winsize, tol, U, F, H, conv,
                     variant == ALDIC_QUADTREE ? markHole : nullptr, nullptr, F0, zncc);
}

int aldic_subset_zncc(aldic_ctx* c, int64_t n, const double* coords, const double* U, const double* F, int winsize,
                      double* zncc) {
  if (!c) return ALDIC_ERR_ARG;
  int rc = need_frame(c, false);
  if (rc) return rc;
  if (n < 0 || winsize < 2 || winsize > 200) return fail(c, ALDIC_ERR_ARG, "bad n or winsize");
  if (n == 0) return ALDIC_OK;
  if (!coords || !U || !F || !zncc) return fail(c, ALDIC_ERR_ARG, "coords, U, F and zncc are required");
  Arg ac{coords, (size_t)n * 16, false, nullptr}, au{U, (size_t)n * 16, false, nullptr};
  Arg af{F, (size_t)n * 32, false, nullptr}, az{zncc, (size_t)n * 8, true, nullptr};
  rc = stage(c, {&ac, &au, &af, &az});
  if (rc) return rc;
  return finish(c, launch_subset_zncc(frame_of(c), n, (const double*)ac.dev, (const double*)au.dev,
                                      (const double*)af.dev, winsize, (double*)az.dev, c->stream));
}

int aldic_fallback_select(aldic_ctx* c, int64_t n, const int32_t* conv, const double* zncc, double zncc_min,
                          int32_t* list, int64_t* count) {
  if (!c) return ALDIC_ERR_ARG;
  if (n < 0 || !count) return fail(c, ALDIC_ERR_ARG, "n >= 0 and count are required");
  CK(cudaSetDevice(c->device));
  const bool dev_count = is_device_ptr(count);
  if (!dev_count) *count = 0;
  if (n == 0) {
    if (dev_count) CK(cudaMemsetAsync(count, 0, sizeof(int64_t), c->stream));
    return ALDIC_OK;
  }
  if (!conv || !zncc || !list) return fail(c, ALDIC_ERR_ARG, "conv, zncc and list are required");
  if (!c->sel_count) CK(cudaMalloc(&c->sel_count, sizeof(int)));
  Arg acv{conv, (size_t)n * 4, false, nullptr}, az{zncc, (size_t)n * 8, false, nullptr};
  Arg al{list, (size_t)n * 4, true, nullptr};
  int rc = stage(c, {&acv, &az, &al});
  if (rc) return rc;
  c->launches += launch_fallback_select((const int32_t*)acv.dev, (const double*)az.dev, n, zncc_min,
                                        (int32_t*)al.dev, c->sel_count, c->stream);
  if (dev_count) {
    // the count stays on the device (little-endian: the int32 count is the int64's low word)
    CK(cudaMemsetAsync(count, 0, sizeof(int64_t), c->stream));
    CK(cudaMemcpyAsync(count, c->sel_count, sizeof(int), cudaMemcpyDeviceToDevice, c->stream));
    return finish(c, 0);  // waits only to copy a host list back
  }
  int h = 0;
  CK(cudaMemcpyAsync(&h, c->sel_count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  rc = finish(c, 0);  // copies a host list back and waits
  CK(cudaStreamSynchronize(c->stream));
  *count = h;
  return rc;
}

int aldic_net_predict(aldic_net* net, aldic_ctx* c, int64_t n, const double* coords, double* U0, double* F0) {
  if (!c || !net) return ALDIC_ERR_ARG;
  int rc = need_frame(c, false);
  if (rc) return rc;
  if (n < 0) return fail(c, ALDIC_ERR_ARG, "n < 0");
  if (n == 0) return ALDIC_OK;
  if (!coords || !U0 || !F0) return fail(c, ALDIC_ERR_ARG, "coords, U0 and F0 are required");
  Arg ac{coords, (size_t)n * 16, false, nullptr}, au{U0, (size_t)n * 16, true, nullptr};
  Arg af{F0, (size_t)n * 32, true, nullptr};
  rc = stage(c, {&ac, &au, &af});
  if (rc) return rc;
  // the network runs on the context's stream so that the frame and the results are ordered
  aldic_net_set_stream(net, c->stream);
  const long long before = aldic_net_launch_count(net);
  rc = net_predict(net, frame_of(c), (const double*)ac.dev, n, (double*)au.dev, (double*)af.dev);
  if (rc) return fail(c, rc, "proposal network: %s", aldic_net_last_error(net));
  c->launches += aldic_net_launch_count(net) - before;
  return finish(c, 0);
}

int aldic_net_extract(aldic_ctx* c, int64_t n, const double* coords, void* X) {
  if (!c) return ALDIC_ERR_ARG;
  int rc = need_frame(c, false);
  if (rc) return rc;
  if (n < 0) return fail(c, ALDIC_ERR_ARG, "n < 0");
  if (n == 0) return ALDIC_OK;
  if (!coords || !X || !is_device_ptr(X)) return fail(c, ALDIC_ERR_ARG, "coords and a device array X are required");
  Arg ac{coords, (size_t)n * 16, false, nullptr};
  rc = stage(c, {&ac});
  if (rc) return rc;
  return finish(c, launch_net_patches(frame_of(c), (const double*)ac.dev, n, X, c->stream));
}

int aldic_epipolar_icgn(aldic_ctx* c, int64_t n, const double* pts, int winsize, double tol, double* znssd) {
  if (!c) return ALDIC_ERR_ARG;
  return icgn_common(c, 2, n, pts, nullptr, winsize, tol, nullptr, nullptr, nullptr, nullptr, nullptr, znssd);
}

int aldic_subpb1(aldic_ctx* c, int variant, int64_t n, const double* coords, const double* UOld, const double* FOld,
                 const double* vdual, const int32_t* winsize_list, int winsize, const double* HPar, double mu,
                 double tol, double* U, int32_t* conv) {
  if (!c) return ALDIC_ERR_ARG;
  int rc = need_frame(c, true);
  if (rc) return rc;
  if (variant != ALDIC_UNIFORM && variant != ALDIC_QUADTREE) return fail(c, ALDIC_ERR_ARG, "bad variant %d", variant);
  if (n < 0) return fail(c, ALDIC_ERR_ARG, "n < 0");
  if (n == 0) return ALDIC_OK;
  if (!coords || !UOld || !FOld || !vdual || !U || !conv) return fail(c, ALDIC_ERR_ARG, "missing array argument");
  if (variant == ALDIC_QUADTREE && !winsize_list) return fail(c, ALDIC_ERR_ARG, "winsize_list required (quadtree)");
  // nominal bucket size and the largest enlarged window
  int wl_max = winsize;
  if (variant == ALDIC_QUADTREE) {
    std::vector<int32_t> wl((size_t)n * 2);
    if (is_device_ptr(winsize_list)) {
      CK(cudaMemcpyAsync(wl.data(), winsize_list, wl.size() * 4, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    } else {
      std::memcpy(wl.data(), winsize_list, wl.size() * 4);
    }
    wl_max = 0;
    for (int32_t v : wl) {
      if (v < 2 || v > 200) return fail(c, ALDIC_ERR_ARG, "winsize_list entry %d out of range [2, 200]", (int)v);
      wl_max = v > wl_max ? v : wl_max;
    }
    if (winsize < 2) winsize = wl_max;
  }
  if (winsize < 2 || winsize > 200) return fail(c, ALDIC_ERR_ARG, "winsize %d out of range", winsize);
  int wmx, wmy;
  {
    const double w = wl_max, Nw = (w + 1) * (w + 1);
    (void)Nw;
    if (variant == ALDIC_QUADTREE) {
      // both enlargement factors are below sqrt(1/0.6) (masked count < 0.4 of the window)
      wmx = wmy = (int)(2 * std::ceil(std::sqrt(1.0 / 0.6) * w / 2)) + 2;
    } else {
      wmx = wmy = (int)std::round(std::sqrt(2.0) * w);
    }
    if (wmx < wl_max) wmx = wl_max;
    if (wmy < wl_max) wmy = wl_max;
  }
  if (sub1_smem_bytes(wmx, wmy) > 200 * 1024) return fail(c, ALDIC_ERR_ARG, "winsize too large for shared memory");
  const size_t qbytes = (size_t)2 * n * 4 * sizeof(int);
  Arg ac{coords, (size_t)n * 16, false, nullptr}, auo{UOld, (size_t)n * 16, false, nullptr};
  Arg afo{FOld, (size_t)n * 32, false, nullptr}, avd{vdual, (size_t)n * 16, false, nullptr};
  Arg awl{variant == ALDIC_QUADTREE ? winsize_list : nullptr, variant == ALDIC_QUADTREE ? (size_t)n * 8 : 0, false,
          nullptr};
  Arg ahp{variant == ALDIC_UNIFORM ? HPar : nullptr, (variant == ALDIC_UNIFORM && HPar) ? (size_t)n * 21 * 8 : 0,
          false, nullptr};
  Arg au{U, (size_t)n * 16, true, nullptr}, acv{conv, (size_t)n * 4, true, nullptr};
  c->arena.used = 0;
  rc = arena_reserve(c, qbytes + (size_t)n * (2 + 2 + 4 + 2 + 1 + 21 + 2 + 1) * 8 + 16384);
  if (rc) return rc;
  rc = stage(c, {&ac, &auo, &afo, &avd, &awl, &ahp, &au, &acv});
  if (rc) return rc;
  Sub1Args a;
  a.fr = frame_of(c);
  a.variant = variant;
  a.n = n;
  a.coords = (const double*)ac.dev;
  a.UOld = (const double*)auo.dev;
  a.FOld = (const double*)afo.dev;
  a.vdual = (const double*)avd.dev;
  a.winsize_list = (const int*)awl.dev;
  a.winsize = winsize;
  a.HPar = (const double*)ahp.dev;
  a.mu = mu;
  a.warp_cap = c->warp_cap;
  a.tol = tol;
  a.U = (double*)au.dev;
  a.conv = (int*)acv.dev;
  a.queue = (int*)arena_take(c, qbytes);
  a.qcount = c->qcount;
  return finish(c, launch_subpb1(a, wmx, wmy, c->stream));
}

int aldic_inpaint_nans(aldic_ctx* c, int m, int n, double* A, int32_t* info) {
  if (!c) return ALDIC_ERR_ARG;
  if (m < 0 || n < 0) return fail(c, ALDIC_ERR_ARG, "grid size %d x %d", m, n);
  if ((long long)m * n > (1LL << 30)) return fail(c, ALDIC_ERR_ARG, "grid of %d x %d entries too large", m, n);
  if (info) {
    info[0] = 0;
    info[1] = 0;
    info[2] = 1;
  }
  if (m == 0 || n == 0) return ALDIC_OK;
  if (!A) return fail(c, ALDIC_ERR_ARG, "grid pointer is NULL");
  CK(cudaSetDevice(c->device));
  const long long mn = (long long)m * n;
  const size_t bytes = (size_t)mn * sizeof(double);
  // A is both input and output: staged in, copied back
  Arg aa{A, bytes, false, nullptr};
  c->arena.used = 0;
  c->back.clear();
  const bool host = !is_device_ptr(A);
  int rc = arena_reserve(c, (host ? bytes + 256 : 0) + inpaint_scratch_bytes(mn) + 256 + 64);
  if (rc) return rc;
  if (host) {
    aa.dev = arena_take(c, bytes);
    CK(cudaMemcpyAsync(aa.dev, A, bytes, cudaMemcpyHostToDevice, c->stream));
    c->back.push_back({A, aa.dev, bytes});
  } else {
    aa.dev = A;
  }
  void* scratch = arena_take(c, inpaint_scratch_bytes(mn));
  int* status = (int*)arena_take(c, 64);
  const int l = launch_inpaint((double*)aa.dev, m, n, scratch, status, c->stream);
  if (info) {
    int st[3];
    CK(cudaMemcpyAsync(st, status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
    rc = finish(c, l);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    info[0] = st[0];
    info[1] = st[1];
    info[2] = st[2];
    return ALDIC_OK;
  }
  return finish(c, l);
}

int aldic_remove_outliers(aldic_ctx* c, int m, int n, double* u, double* v, double thr, int maxit,
                          int32_t* info) {
  if (!c) return ALDIC_ERR_ARG;
  if (m < 0 || n < 0) return fail(c, ALDIC_ERR_ARG, "grid size %d x %d", m, n);
  if ((long long)m * n > (1LL << 30)) return fail(c, ALDIC_ERR_ARG, "grid of %d x %d entries too large", m, n);
  if (!(thr > 0.0)) return fail(c, ALDIC_ERR_ARG, "threshold must be > 0 (the reference prompts for 0)");
  if (info)
    for (int k = 0; k < 4; ++k) info[k] = k == 3 ? 1 : 0;
  if (m == 0 || n == 0) return ALDIC_OK;
  if (!u || !v) return fail(c, ALDIC_ERR_ARG, "missing array argument");
  CK(cudaSetDevice(c->device));
  const long long mn = (long long)m * n;
  const size_t bytes = (size_t)mn * sizeof(double);
  if (maxit <= 0) maxit = (int)std::min<long long>(8 * mn + 200, 20000);
  // u and v are both inputs and outputs: staged in, copied back
  Arg au{u, bytes, false, nullptr}, av{v, bytes, false, nullptr};
  c->arena.used = 0;
  c->back.clear();
  size_t need = 0;
  for (Arg* a : {&au, &av})
    if (!is_device_ptr(a->user)) need += bytes + 256;
  const size_t i2 = 2 * (((inpaint_scratch_bytes(mn) + 255) & ~(size_t)255) + 256);
  const size_t d2 = 2 * (((del4_scratch_bytes(mn) + 255) & ~(size_t)255) + 256);
  need += 4 * (bytes + 256) + 2 * ((size_t)mn * sizeof(float) + 256) + (size_t)mn + 256 + i2 + d2 + 128;
  int rc = arena_reserve(c, need);
  if (rc) return rc;
  for (Arg* a : {&au, &av}) {
    if (is_device_ptr(a->user)) {
      a->dev = const_cast<void*>(a->user);
    } else {
      a->dev = arena_take(c, a->bytes);
      CK(cudaMemcpyAsync(a->dev, a->user, a->bytes, cudaMemcpyHostToDevice, c->stream));
      c->back.push_back({const_cast<void*>(a->user), a->dev, a->bytes});
    }
  }
  double* du = (double*)au.dev;
  double* dv = (double*)av.dev;
  // the method-4 warm starts and the method-3 fills, written at the NaN entries only
  double* w4u = (double*)arena_take(c, bytes);
  double* w4v = (double*)arena_take(c, bytes);
  double* wfu = (double*)arena_take(c, bytes);
  double* wfv = (double*)arena_take(c, bytes);
  float* fu = (float*)arena_take(c, (size_t)mn * sizeof(float));
  float* fv = (float*)arena_take(c, (size_t)mn * sizeof(float));
  unsigned char* hole = (unsigned char*)arena_take(c, (size_t)mn);
  void* iscratch = arena_take(c, i2);
  void* dscratch = arena_take(c, d2);
  // status: [0..2] method 3 of u, [3..5] of v, [6] removed, [7..12] the method-4 solves,
  // [16] #NaN(u), [17] #NaN(v), [18] 0 (the hints' third term before the median test)
  int* status = (int*)arena_take(c, 128);
  CK(cudaMemsetAsync(status, 0, 128, c->stream));
  int* counts = status + 16;
  int l = launch_nan_count(du, dv, m, n, counts, c->stream);
  // inpaint_nans(., 3) of u and v, started from inpaint_nans(., 4); skipped without NaN
  l += launch_inpaint2(du, dv, w4u, w4v, m, n, iscratch, counts, status + 7, c->stream);
  l += launch_inpaint_del4(du, dv, w4u, w4v, wfu, wfv, m, n, maxit, dscratch, counts, status, c->stream);
  l += launch_median_fluct(du, dv, wfu, wfv, m, n, fu, fv, c->stream);
  // the removed count goes to counts[2]: the last fill runs when u, v or the removal has NaN
  l += launch_outlier_mark(fu, fv, m, n, (float)thr, du, dv, hole, counts + 2, c->stream);
  l += launch_inpaint2(du, dv, du, dv, m, n, iscratch, counts, status + 7, c->stream);
  l += launch_restore_holes(hole, m, n, du, dv, c->stream);
  if (info) {
    int st[19];
    CK(cudaMemcpyAsync(st, status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
    rc = finish(c, l);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    info[0] = st[18];
    info[1] = st[16];
    info[2] = std::max(st[1], st[4]);
    info[3] = (st[2] && st[5]) ? 1 : 0;
    return ALDIC_OK;
  }
  return finish(c, l);
}

namespace {

// Device layout of one mesh's tables: element table (8 n_el ints), node pointers (n + 1),
// node -> element entries (nadj), node kinds (n bytes); each part 256-byte aligned.
size_t sp2_bytes(int64_t n, int64_t n_el, size_t nadj) {
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  return up((size_t)n_el * 32) + up(((size_t)n + 1) * 4) + up(std::max<size_t>(nadj, 1) * 4) + up((size_t)n);
}

void sp2_parts(char* base, int64_t n, int64_t n_el, size_t nadj, int** E, int** ptr, int** adj,
               unsigned char** kind) {
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  *E = (int*)base;
  *ptr = (int*)(base + up((size_t)n_el * 32));
  *adj = (int*)((char*)*ptr + up(((size_t)n + 1) * 4));
  *kind = (unsigned char*)((char*)*adj + up(std::max<size_t>(nadj, 1) * 4));
}

// The mesh tables on the host from a caller's element table and dirichlet list (host or
// device pointers).
int sp2_tables(aldic_ctx* c, int64_t n, int64_t n_el, const int32_t* elements, int64_t n_dirichlet,
               const int32_t* dirichlet, std::vector<int32_t>& E, std::vector<int>& ptr, std::vector<int>& adj,
               std::vector<unsigned char>& kind) {
  if (n <= 0 || n_el <= 0)
    return fail(c, ALDIC_ERR_ARG, "empty mesh (%lld nodes, %lld elements)", (long long)n, (long long)n_el);
  if (n > (1LL << 28) || n_el > (1LL << 27)) return fail(c, ALDIC_ERR_ARG, "mesh too large");
  if (!elements || (n_dirichlet > 0 && !dirichlet)) return fail(c, ALDIC_ERR_ARG, "missing mesh array");
  if (n_dirichlet < 0) return fail(c, ALDIC_ERR_ARG, "n_dirichlet < 0");
  E.resize((size_t)n_el * 8);
  std::vector<int32_t> dir((size_t)std::max<int64_t>(n_dirichlet, 1));
  if (is_device_ptr(elements)) {
    CK(cudaMemcpy(E.data(), elements, E.size() * 4, cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(E.data(), elements, E.size() * 4);
  }
  if (n_dirichlet > 0) {
    if (is_device_ptr(dirichlet)) {
      CK(cudaMemcpy(dir.data(), dirichlet, (size_t)n_dirichlet * 4, cudaMemcpyDeviceToHost));
    } else {
      std::memcpy(dir.data(), dirichlet, (size_t)n_dirichlet * 4);
    }
  }
  char msg[160];
  if (subpb2_mesh_tables(n, n_el, E.data(), n_dirichlet, dir.data(), ptr, adj, kind, msg, sizeof(msg)))
    return fail(c, ALDIC_ERR_ARG, "%s", msg);
  return ALDIC_OK;
}

}  // namespace

int aldic_subpb2_set_mesh(aldic_ctx* c, int64_t n, int64_t n_el, const int32_t* elements, int64_t n_dirichlet,
                          const int32_t* dirichlet) {
  if (!c) return ALDIC_ERR_ARG;
  CK(cudaSetDevice(c->device));
  std::vector<int32_t> E;
  std::vector<int> ptr, adj;
  std::vector<unsigned char> kind;
  int rc = sp2_tables(c, n, n_el, elements, n_dirichlet, dirichlet, E, ptr, adj, kind);
  if (rc) return rc;
  const size_t bytes = sp2_bytes(n, n_el, adj.size());
  CK(cudaStreamSynchronize(c->stream));  // the previous tables may still be in use
  if (c->sp2_cap < bytes) {
    if (c->sp2) CK(cudaFree(c->sp2));
    c->sp2 = nullptr;
    c->sp2_cap = 0;
    CK(cudaMalloc(&c->sp2, bytes));
    c->sp2_cap = bytes;
  }
  int *dE, *dptr, *dadj;
  unsigned char* dkind;
  sp2_parts(c->sp2, n, n_el, adj.size(), &dE, &dptr, &dadj, &dkind);
  CK(cudaMemcpyAsync(dE, E.data(), E.size() * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(dptr, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice, c->stream));
  if (!adj.empty()) CK(cudaMemcpyAsync(dadj, adj.data(), adj.size() * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(dkind, kind.data(), kind.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->sp2_n = n;
  c->sp2_nel = n_el;
  c->sp2_nadj = adj.size();
  return ALDIC_OK;
}

int aldic_subpb2(aldic_ctx* c, int64_t n, const double* coords, int64_t n_el, const int32_t* elements,
                 int gauss_order, double beta, double mu, double alpha, const double* U, const double* F,
                 int64_t n_dirichlet, const int32_t* dirichlet, double tol, int maxit, double* Uhat,
                 int32_t* info) {
  if (!c) return ALDIC_ERR_ARG;
  if (info) info[0] = info[1] = 0;
  if (gauss_order < 2 || gauss_order > 5) return fail(c, ALDIC_ERR_ARG, "Gauss point order %d (2..5)", gauss_order);
  if (!(beta + alpha > 0.0) && !(mu > 0.0))
    return fail(c, ALDIC_ERR_ARG, "beta + alpha and mu are both 0: the system is singular");
  if (!coords || !U || !F || !Uhat) return fail(c, ALDIC_ERR_ARG, "missing array argument");
  if (!(tol > 0.0)) tol = 1e-12;
  if (maxit <= 0) maxit = (int)std::min<int64_t>(20 * n + 1000, 200000);
  CK(cudaSetDevice(c->device));
  const bool resident = elements == nullptr;
  std::vector<int32_t> E;
  std::vector<int> ptr, adj;
  std::vector<unsigned char> kind;
  if (resident) {  // the tables of aldic_subpb2_set_mesh
    if (!c->sp2 || c->sp2_n != n || c->sp2_nel != n_el)
      return fail(c, ALDIC_ERR_ARG, "no resident mesh of %lld nodes / %lld elements (aldic_subpb2_set_mesh)",
                  (long long)n, (long long)n_el);
    if (n_dirichlet != 0) return fail(c, ALDIC_ERR_ARG, "the resident mesh carries its dirichlet nodes");
  } else {
    int rc = sp2_tables(c, n, n_el, elements, n_dirichlet, dirichlet, E, ptr, adj, kind);
    if (rc) return rc;
  }
  // device buffers: inputs staged, the mesh tables (unless resident), K_e / b_e, the CG vectors
  const size_t nb = (size_t)subpb2_blocks(n);
  Arg ac{coords, (size_t)n * 16, false, nullptr}, au{U, (size_t)n * 16, false, nullptr},
      af{F, (size_t)n * 32, false, nullptr}, ao{Uhat, (size_t)n * 16, true, nullptr};
  c->arena.used = 0;
  c->back.clear();
  size_t need = 0;
  for (Arg* a : {&ac, &au, &af, &ao})
    if (!is_device_ptr(a->user)) need += ((a->bytes + 255) & ~size_t(255)) + 256;
  const size_t two_n = (size_t)n * 16;
  if (!resident) need += sp2_bytes(n, n_el, adj.size()) + 256;
  need += (size_t)n_el * (64 + 16) * 8 + 6 * two_n + (size_t)n * 8 + nb * 16 + subpb2_scalars_bytes() + 64 +
          16 * 256;
  int rc = arena_reserve(c, need);
  if (rc) return rc;
  for (Arg* a : {&ac, &au, &af, &ao}) {
    if (is_device_ptr(a->user)) {
      a->dev = const_cast<void*>(a->user);
    } else {
      a->dev = arena_take(c, a->bytes);
      if (a->output)
        c->back.push_back({const_cast<void*>(a->user), a->dev, a->bytes});
      else
        CK(cudaMemcpyAsync(a->dev, a->user, a->bytes, cudaMemcpyHostToDevice, c->stream));
    }
  }
  int *dE, *dptr, *dadj;
  unsigned char* dkind;
  if (resident) {
    sp2_parts(c->sp2, n, n_el, c->sp2_nadj, &dE, &dptr, &dadj, &dkind);
  } else {
    char* tb = (char*)arena_take(c, sp2_bytes(n, n_el, adj.size()));
    sp2_parts(tb, n, n_el, adj.size(), &dE, &dptr, &dadj, &dkind);
    // copied from pageable host vectors: each copy has completed when the call returns
    CK(cudaMemcpyAsync(dE, E.data(), E.size() * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dptr, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice, c->stream));
    if (!adj.empty()) CK(cudaMemcpyAsync(dadj, adj.data(), adj.size() * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dkind, kind.data(), kind.size(), cudaMemcpyHostToDevice, c->stream));
  }
  double* Ke = (double*)arena_take(c, (size_t)n_el * 64 * 8);
  double* be = (double*)arena_take(c, (size_t)n_el * 16 * 8);
  double* b = (double*)arena_take(c, two_n);
  double* r = (double*)arena_take(c, two_n);
  double* z = (double*)arena_take(c, two_n);
  double* p = (double*)arena_take(c, two_n);
  double* q = (double*)arena_take(c, two_n);
  double* D = (double*)arena_take(c, (size_t)n * 8);
  double* part = (double*)arena_take(c, nb * 16);
  Subpb2Scalars* sc = (Subpb2Scalars*)arena_take(c, subpb2_scalars_bytes() + 64);
  double* x = (double*)ao.dev;  // the solution builds in the output
  int l = launch_subpb2_setup((int)n_el, dE, (const double*)ac.dev, n, (const double*)au.dev, (const double*)af.dev,
                              gauss_order, beta, mu, alpha, dptr, dadj, dkind, Ke, be, b, D, x, r, z, p, part, sc,
                              c->stream);
  // batches of 16 iterations; the scalars are read back between batches (the kernels of a
  // batch that starts after convergence return at once)
  std::vector<unsigned char> host_sc(subpb2_scalars_bytes());
  int it = 0, done = 0, ok = 0;
  for (int launched = 0; launched < maxit;) {
    const int k = std::min(16, maxit - launched);
    l += launch_subpb2_iterations(k, (int)n_el, dE, n, dptr, dadj, Ke, dkind, D, x, r, z, p, q, part, tol * tol,
                                  maxit, sc, c->stream);
    launched += k;
    CK(cudaMemcpyAsync(host_sc.data(), sc, host_sc.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    subpb2_read_status(host_sc.data(), &it, &done, &ok);
    if (done) break;
  }
  if (info) {
    info[0] = it;
    info[1] = ok;
  }
  return finish(c, l);
}

int aldic_init_u0(aldic_ctx* c, int ny, int nx, const double* u, const double* v, int index, double* U0) {
  if (!c) return ALDIC_ERR_ARG;
  if (index != 0 && index != 1) return fail(c, ALDIC_ERR_ARG, "Init index %d (0 or 1)", index);
  if (ny < 0 || nx < 0) return fail(c, ALDIC_ERR_ARG, "grid size %d x %d", ny, nx);
  if ((long long)ny * nx > (1LL << 30)) return fail(c, ALDIC_ERR_ARG, "grid of %d x %d entries too large", ny, nx);
  if (ny == 0 || nx == 0) return ALDIC_OK;
  if (!u || !v || !U0) return fail(c, ALDIC_ERR_ARG, "missing array argument");
  CK(cudaSetDevice(c->device));
  const long long g = (long long)ny * nx;
  const size_t bytes = (size_t)g * sizeof(double);
  Arg au{u, bytes, false, nullptr}, av{v, bytes, false, nullptr}, ao{U0, 2 * bytes, true, nullptr};
  // the staged arrays, then the two working copies and the solver scratch
  c->arena.used = 0;
  c->back.clear();
  size_t need = 0;
  for (Arg* a : {&au, &av, &ao})
    if (!is_device_ptr(a->user)) need += ((a->bytes + 255) & ~size_t(255)) + 256;
  const size_t i2 = 2 * (((inpaint_scratch_bytes(g) + 255) & ~(size_t)255) + 256);
  need += 4 * (bytes + 256) + i2 + 512;
  int rc = arena_reserve(c, need);
  if (rc) return rc;
  for (Arg* a : {&au, &av, &ao}) {
    if (is_device_ptr(a->user)) {
      a->dev = const_cast<void*>(a->user);
    } else {
      a->dev = arena_take(c, a->bytes);
      if (a->output)
        c->back.push_back({const_cast<void*>(a->user), a->dev, a->bytes});
      else
        CK(cudaMemcpyAsync(a->dev, a->user, a->bytes, cudaMemcpyHostToDevice, c->stream));
    }
  }
  double* wu = (double*)arena_take(c, bytes);
  double* wv = (double*)arena_take(c, bytes);
  void* scratch = arena_take(c, i2);
  int* status = (int*)arena_take(c, 128);
  const double* du = (const double*)au.dev;
  const double* dv = (const double*)av.dev;
  int l = 0;
  if (index == 0) {  // the NaN entries solved into wu, wv; U0 takes u, v elsewhere
    CK(cudaMemsetAsync(status, 0, 128, c->stream));
    l += launch_nan_count(du, dv, ny, nx, status + 16, c->stream);
    l += launch_inpaint2(du, dv, wu, wv, ny, nx, scratch, status + 16, status, c->stream);
    l += launch_interleave_u0(du, dv, wu, wv, ny, nx, (double*)ao.dev, c->stream);
    return finish(c, l);
  }
  // index 1: working copies, then the three spring outlier passes, each on a copy of the
  // pass's input
  CK(cudaMemcpyAsync(wu, du, bytes, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(wv, dv, bytes, cudaMemcpyDeviceToDevice, c->stream));
  l += launch_inpaint2(wu, wv, wu, wv, ny, nx, scratch, nullptr, status, c->stream);
  double* tu = (double*)arena_take(c, bytes);
  double* tv = (double*)arena_take(c, bytes);
  for (int mode = 0; mode < 3; ++mode) {
    CK(cudaMemcpyAsync(tu, wu, bytes, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(tv, wv, bytes, cudaMemcpyDeviceToDevice, c->stream));
    l += launch_spring_pass(tu, tv, wu, wv, ny, nx, mode, c->stream);
    l += launch_inpaint2(wu, wv, wu, wv, ny, nx, scratch, nullptr, status, c->stream);
  }
  l += launch_interleave_u0(wu, wv, wu, wv, ny, nx, (double*)ao.dev, c->stream);
  return finish(c, l);
}

int aldic_undistort_points(aldic_ctx* c, int64_t n, const double* pts, const double* K, const double* radial,
                           int n_radial, const double* tangential, double* out) {
  if (!c) return ALDIC_ERR_ARG;
  if (n < 0) return fail(c, ALDIC_ERR_ARG, "n < 0");
  if (n_radial != 2 && n_radial != 3) return fail(c, ALDIC_ERR_ARG, "radial distortion needs 2 or 3 coefficients");
  if (n == 0) return ALDIC_OK;
  if (!pts || !K || !radial || !out) return fail(c, ALDIC_ERR_ARG, "missing array argument");
  CK(cudaSetDevice(c->device));
  // camera parameters (small, read on the host): K 3 x 3 column-major, (k1 k2 [k3]), (p1 p2)
  double k[9], rad[3] = {0.0, 0.0, 0.0}, tan2[2] = {0.0, 0.0};
  const double* srcs[3] = {K, radial, tangential};
  double* dsts[3] = {k, rad, tan2};
  const int cnts[3] = {9, n_radial, 2};
  for (int i = 0; i < 3; ++i) {
    if (!srcs[i]) continue;
    if (is_device_ptr(srcs[i])) {
      CK(cudaMemcpy(dsts[i], srcs[i], cnts[i] * 8, cudaMemcpyDeviceToHost));
    } else {
      std::memcpy(dsts[i], srcs[i], cnts[i] * 8);
    }
  }
  const double dist[5] = {rad[0], rad[1], rad[2], tan2[0], tan2[1]};
  Arg ap{pts, (size_t)n * 16, false, nullptr}, ao{out, (size_t)n * 16, true, nullptr};
  int rc = stage(c, {&ap, &ao});
  if (rc) return rc;
  return finish(c, launch_undistort_points(n, (const double*)ap.dev, k, dist, (double*)ao.dev, c->stream));
}

int aldic_triangulate(aldic_ctx* c, int64_t n, const double* pairs, const double* KL, const double* KR,
                      const double* R, const double* T, double* xyz, double* reproj_err) {
  if (!c) return ALDIC_ERR_ARG;
  if (n < 0) return fail(c, ALDIC_ERR_ARG, "n < 0");
  if (n == 0) return ALDIC_OK;
  if (!pairs || !KL || !KR || !R || !T || !xyz) return fail(c, ALDIC_ERR_ARG, "missing array argument");
  // camera matrices (small, always read on the host): MATLAB column-major 3x3 inputs
  double kl[9], kr[9], r[9], tt[3];
  const double* srcs[4] = {KL, KR, R, T};
  double* dsts[4] = {kl, kr, r, tt};
  const int cnts[4] = {9, 9, 9, 3};
  for (int i = 0; i < 4; ++i) {
    if (is_device_ptr(srcs[i])) {
      CK(cudaMemcpy(dsts[i], srcs[i], cnts[i] * 8, cudaMemcpyDeviceToHost));
    } else {
      std::memcpy(dsts[i], srcs[i], cnts[i] * 8);
    }
  }
  CamPair cams;  // PL (3x4 row-major) then PR
  double* P = cams.P;
  for (int row = 0; row < 3; ++row)
    for (int col = 0; col < 4; ++col) {
      // PL = KL [I | 0]
      P[row * 4 + col] = col < 3 ? kl[row + 3 * col] : 0.0;
      // PR = KR [R | T]
      double s = 0;
      for (int k = 0; k < 3; ++k) s += kr[row + 3 * k] * (col < 3 ? r[k + 3 * col] : tt[k]);
      P[12 + row * 4 + col] = s;
    }
  Arg ap{pairs, (size_t)n * 32, false, nullptr}, ax{xyz, (size_t)n * 24, true, nullptr};
  Arg ae{reproj_err, reproj_err ? (size_t)n * 8 : 0, true, nullptr};
  int rc = stage(c, {&ap, &ax, &ae});
  if (rc) return rc;
  return finish(c, launch_triangulate(n, (const double*)ap.dev, cams, (double*)ax.dev, (double*)ae.dev, c->stream));
}

int aldic_measure_fp32_peak(aldic_ctx* c, double* tflops) {
  if (!c || !tflops) return ALDIC_ERR_ARG;
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  c->arena.used = 0;
  int rc = arena_reserve(c, 4096);
  if (rc) return rc;
  float* out = (float*)arena_take(c, 64);
  const int threads = 256, blocks = sms * 8, iters = 2048;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  // scalar FFMA and packed FFMA2 loops; the peak is the faster of the two
  double best = 0.0;
  for (int packed = 0; packed < 2; ++packed) {
    launch_fp32_probe(blocks, threads, 64, out, packed != 0, c->stream);  // warm-up
    CK(cudaEventRecord(e0, c->stream));
    launch_fp32_probe(blocks, threads, iters, out, packed != 0, c->stream);
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    best = fmax(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->launches += 4;
  *tflops = best;
  return ALDIC_OK;
}

int aldic_set_iteration_cap(aldic_ctx* c, int cap) {
  if (!c) return ALDIC_ERR_ARG;
  if (cap < 1 || cap > 1000) return fail(c, ALDIC_ERR_ARG, "iteration cap %d outside 1..1000", cap);
  c->warp_cap = cap;
  return ALDIC_OK;
}

int aldic_set_option(aldic_ctx* c, int option, int value) {
  if (!c) return ALDIC_ERR_ARG;
  switch (option) {
    case ALDIC_OPT_ITERATION_CAP:
      return aldic_set_iteration_cap(c, value);
    case ALDIC_OPT_STAGING:
      if (value != 0 && value != 1) return fail(c, ALDIC_ERR_ARG, "staging must be 0 or 1, not %d", value);
      c->staging = value;
      return ALDIC_OK;
    case ALDIC_OPT_SLOW_WARPS:
      if (value != 2 && value != 4) return fail(c, ALDIC_ERR_ARG, "slow-pass warps must be 2 or 4, not %d", value);
      c->slow_nw = value;
      return ALDIC_OK;
    case ALDIC_OPT_SEARCH_IMPL:
      if (value < 0 || value > 2) return fail(c, ALDIC_ERR_ARG, "search implementation must be 0, 1 or 2");
      c->search_impl = value;
      return ALDIC_OK;
    case ALDIC_OPT_SEARCH_CHUNK:
      if (value != 0 && value != 16 && value != 24) return fail(c, ALDIC_ERR_ARG, "chunk must be 0, 16 or 24");
      c->search_chunk = value;
      return ALDIC_OK;
    case ALDIC_OPT_AUTOTUNE:
      if (value != 0 && value != 1) return fail(c, ALDIC_ERR_ARG, "autotune must be 0 or 1");
      c->autotune = value;
      return ALDIC_OK;
    case ALDIC_OPT_SLOW_FP64:
      if (value != 0 && value != 1) return fail(c, ALDIC_ERR_ARG, "slow_fp64 must be 0 or 1");
      c->slow_fp64 = value;
      return ALDIC_OK;
    case ALDIC_OPT_FP64_THREADS:
      if (value != 128 && value != 256 && value != 512)
        return fail(c, ALDIC_ERR_ARG, "FP64 threads must be 128, 256 or 512");
      c->fp64_threads = value;
      return ALDIC_OK;
    default:
      return fail(c, ALDIC_ERR_ARG, "unknown option %d", option);
  }
}

int aldic_get_option(aldic_ctx* c, int option, int* value) {
  if (!c || !value) return ALDIC_ERR_ARG;
  switch (option) {
    case ALDIC_OPT_ITERATION_CAP:
      *value = c->warp_cap;
      return ALDIC_OK;
    case ALDIC_OPT_STAGING:
      *value = c->staging;
      return ALDIC_OK;
    case ALDIC_OPT_SLOW_WARPS:
      *value = c->slow_nw;
      return ALDIC_OK;
    case ALDIC_OPT_SEARCH_IMPL:
      *value = c->search_impl;
      return ALDIC_OK;
    case ALDIC_OPT_SEARCH_CHUNK:
      *value = c->search_chunk;
      return ALDIC_OK;
    case ALDIC_OPT_AUTOTUNE:
      *value = c->autotune;
      return ALDIC_OK;
    case ALDIC_OPT_SLOW_FP64:
      *value = c->slow_fp64;
      return ALDIC_OK;
    case ALDIC_OPT_FP64_THREADS:
      *value = c->fp64_threads;
      return ALDIC_OK;
    case ALDIC_STAT_FP64_RESOLVES:
    case ALDIC_STAT_STAGING_TIMEOUT: {
      // counters the last aldic_local_icgn left in the context's queue block (waits for it)
      CK(cudaSetDevice(c->device));
      int q[16];
      CK(cudaMemcpyAsync(q, c->qcount, sizeof(q), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      *value = option == ALDIC_STAT_FP64_RESOLVES ? q[4] : q[8];
      return ALDIC_OK;
    }
    default:
      return fail(c, ALDIC_ERR_ARG, "unknown option %d", option);
  }
}

int aldic_tuning_report(aldic_ctx* c, char* buf, int64_t len) {
  if (!c || !buf || len < 3) return ALDIC_ERR_ARG;
  std::string r = "{";
  bool firstk = true;
  for (const auto& kv : c->tuned) {
    if (!firstk) r += ", ";
    firstk = false;
    r += "\"" + kv.first + "\": {\"choice\": " + kv.second.choice + ", \"ms\": {";
    bool f = true;
    for (const auto& m : kv.second.ms) {
      char t[96];
      std::snprintf(t, sizeof(t), "%s\"%s\": %.4f", f ? "" : ", ", m.first.c_str(), m.second);
      r += t;
      f = false;
    }
    r += "}}";
  }
  r += "}";
  if ((int64_t)r.size() + 1 > len) return fail(c, ALDIC_ERR_ARG, "report needs %zu bytes", r.size() + 1);
  std::memcpy(buf, r.c_str(), r.size() + 1);
  return ALDIC_OK;
}

int aldic_set_fp64_band(aldic_ctx* c, double band, double noise) {
  if (!c) return ALDIC_ERR_ARG;
  if (!(band >= 0.0) || !(band <= 1e300)) return fail(c, ALDIC_ERR_ARG, "band %g must be >= 0 and finite", band);
  if (!(noise >= 0.0) || !(noise <= 1e300)) return fail(c, ALDIC_ERR_ARG, "noise %g must be >= 0 and finite", noise);
  c->fp64_band = band;
  c->fp64_noise = noise;
  return ALDIC_OK;
}

int aldic_set_profiling(aldic_ctx* c, int on) {
  if (!c) return ALDIC_ERR_ARG;
  CK(cudaSetDevice(c->device));
  if (on && c->prof_ev.empty()) {
    c->prof_ev.resize(2 * 256);
    for (cudaEvent_t& e : c->prof_ev) CK(cudaEventCreate(&e));
  }
  c->prof = on != 0;
  return ALDIC_OK;
}

int aldic_profile_read(aldic_ctx* c, double* total_ms, int* launches) {
  if (!c || !total_ms || !launches) return ALDIC_ERR_ARG;
  CK(cudaSetDevice(c->device));
  double tot = 0.0;
  for (int k = 0; k < c->prof_n; ++k) {
    CK(cudaEventSynchronize(c->prof_ev[2 * k + 1]));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->prof_ev[2 * k], c->prof_ev[2 * k + 1]));
    tot += ms;
  }
  *total_ms = tot;
  *launches = c->prof_n;
  c->prof_n = 0;
  return ALDIC_OK;
}

}  // extern "C"
