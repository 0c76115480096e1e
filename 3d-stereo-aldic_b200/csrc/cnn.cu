// Proposal network of the learned initial guess: a small convolutional network that reads a
// 32 x 32 reference subset and the 64 x 64 deformed window around it and predicts the
// subset's displacement and displacement gradient, (u, v, du/dx, dv/dx, du/dy, dv/dy), the
// initial guess [F0 U0] of IC-GN in place of the FFT integer search.  No counterpart in the
// reference (its initial guess is the integer search, func/funIntegerSearch.m:132-180, which
// stays the fallback here).
//
// Architecture (NHWC BF16 activations, FP32 accumulation, ReLU after every layer but the last):
//   input 64 x 64 x 2 (channel 0: the normalised reference subset in the centre 32 x 32 of a
//   zero canvas; channel 1: the normalised deformed window)
//   conv 3x3 stride 2 pad 1:  2 -> 32 (32 x 32),  32 -> 32 (16 x 16),  32 -> 64 (8 x 8),
//                             64 -> 64 (4 x 4)
//   fully connected: 1024 -> 128 -> 6
// 197 254 trained parameters.  Every convolution, data gradient, weight gradient and fully
// connected layer is one tcgen05 GEMM (cnn_gemm.cu) over im2col rows; the rest are the small
// kernels below (im2col, col2im, transposes, ReLU gradient, loss, bias gradient, Adam, patch
// extraction).  Training: mean squared error on the scaled outputs (u / 8, v / 8, F x 20),
// Adam.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/aldic_b200.h"
#include "cnn.h"
#include "kernels.h"

namespace aldic {
namespace {

typedef __nv_bfloat16 bf16;

struct ConvL {
  int Hin, Win, Cin, Hout, Wout, Cout, K, Kp;
};
constexpr ConvL kConv[4] = {{64, 64, 2, 32, 32, 32, 18, 24},
                            {32, 32, 32, 16, 16, 32, 288, 288},
                            {16, 16, 32, 8, 8, 64, 288, 288},
                            {8, 8, 64, 4, 4, 64, 576, 576}};
constexpr int kFcIn = 1024, kFcHid = 128, kOut = 6, kOutP = 16;

// flat FP32 parameter layout: per conv layer W [Cout x Kp] then b [Cout]; FC1 W [128 x 1024],
// b [128]; FC2 W [16 x 128] (rows 6..15 zero), b [16] (entries 6..15 zero)
struct Layout {
  long long w[6], b[6], n;
  long long rows[6], cols[6];
  Layout() {
    long long o = 0;
    for (int l = 0; l < 6; ++l) {
      rows[l] = l < 4 ? kConv[l].Cout : (l == 4 ? kFcHid : kOutP);
      cols[l] = l < 4 ? kConv[l].Kp : (l == 4 ? kFcIn : kFcHid);
      w[l] = o;
      o += rows[l] * cols[l];
      b[l] = o;
      o += rows[l];
    }
    n = o;
  }
};
const Layout kL;

__device__ __forceinline__ long long ceil_div_ll(long long a, long long b) { return (a + b - 1) / b; }

// ------------------------------------------------------------------------- kernels
// im2col of a stride-2, pad-1, 3 x 3 convolution: row p = (b, oy, ox), column k = (ky, kx, ci),
// zero outside the input and in the K padding.
__global__ void im2col_kernel(const bf16* __restrict__ H, bf16* __restrict__ A, int batch, ConvL L) {
  const long long P = (long long)batch * L.Hout * L.Wout;
  const long long total = P * L.Kp;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long p = i / L.Kp;
    const int k = (int)(i % L.Kp);
    bf16 v = __float2bfloat16_rn(0.f);
    if (k < L.K) {
      const int tap = k / L.Cin, ci = k % L.Cin, ky = tap / 3, kx = tap % 3;
      const int ox = (int)(p % L.Wout), oy = (int)((p / L.Wout) % L.Hout);
      const long long b = p / ((long long)L.Wout * L.Hout);
      const int iy = 2 * oy - 1 + ky, ix = 2 * ox - 1 + kx;
      if (iy >= 0 && iy < L.Hin && ix >= 0 && ix < L.Win) v = H[((b * L.Hin + iy) * L.Win + ix) * L.Cin + ci];
    }
    A[i] = v;
  }
}

// col2im (gather form, no atomics): the gradient of input pixel (b, iy, ix, ci) sums the
// im2col gradient entries that read it.
__global__ void col2im_kernel(const float* __restrict__ dA, float* __restrict__ dH, int batch, ConvL L) {
  const long long total = (long long)batch * L.Hin * L.Win * L.Cin;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int ci = (int)(i % L.Cin);
    const int ix = (int)((i / L.Cin) % L.Win);
    const int iy = (int)((i / ((long long)L.Cin * L.Win)) % L.Hin);
    const long long b = i / ((long long)L.Cin * L.Win * L.Hin);
    float s = 0.f;
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
      const int ty = iy + 1 - ky;
      if (ty < 0 || (ty & 1) || (ty >> 1) >= L.Hout) continue;
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) {
        const int tx = ix + 1 - kx;
        if (tx < 0 || (tx & 1) || (tx >> 1) >= L.Wout) continue;
        const long long p = (b * L.Hout + (ty >> 1)) * L.Wout + (tx >> 1);
        s += dA[p * L.Kp + (ky * 3 + kx) * L.Cin + ci];
      }
    }
    dH[i] = s;
  }
}

// out[c, r] = in[r, c] (BF16, 32 x 32 tiles through shared memory)
__global__ void transpose_kernel(const bf16* __restrict__ in, bf16* __restrict__ out, long long R, long long Cn) {
  __shared__ bf16 t[32][33];
  const long long r0 = blockIdx.y * 32LL, c0 = blockIdx.x * 32LL;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const long long r = r0 + j, c = c0 + threadIdx.x;
    t[j][threadIdx.x] = (r < R && c < Cn) ? in[r * Cn + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const long long c = c0 + j, r = r0 + threadIdx.x;
    if (c < Cn && r < R) out[c * R + r] = t[threadIdx.x][j];
  }
}

// dZ = dH where the layer's output was positive (ReLU), as BF16
__global__ void relu_grad_kernel(const float* __restrict__ dH, const bf16* __restrict__ H, bf16* __restrict__ dZ,
                                 long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dZ[i] = __float2bfloat16_rn(__bfloat162float(H[i]) > 0.f ? dH[i] : 0.f);
}

// loss = mean over batch x 6 of (y - t)^2; dY = d loss / dy (BF16, the 6 outputs of 16 columns)
__global__ void mse_kernel(const float* __restrict__ Y, const float* __restrict__ T, int batch, bf16* __restrict__ dY,
                           float* __restrict__ loss) {
  __shared__ float red[256];
  float s = 0.f;
  const float scale = 2.f / (float)(batch * kOut);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch * kOutP; i += gridDim.x * blockDim.x) {
    const int b = i / kOutP, j = i % kOutP;
    float g = 0.f;
    if (j < kOut) {
      const float d = Y[(size_t)b * kOutP + j] - T[(size_t)b * kOut + j];
      s += d * d;
      g = scale * d;
    }
    dY[i] = __float2bfloat16_rn(g);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] / (float)(batch * kOut));
}

// db[c] += sum over rows of dZ[r, c] (each block sums a chunk of rows; one atomic per column)
__global__ void bias_grad_kernel(const bf16* __restrict__ dZ, long long R, int Cn, float* __restrict__ db) {
  const int c = threadIdx.x;
  if (c >= Cn) return;
  const long long per = ceil_div_ll(R, gridDim.x);
  const long long r0 = blockIdx.x * per, r1 = r0 + per < R ? r0 + per : R;
  float s = 0.f;
  for (long long r = r0; r < r1; ++r) s += __bfloat162float(dZ[r * Cn + c]);
  atomicAdd(db + c, s);
}

// Adam (Kingma & Ba 2015) on the flat FP32 parameters, refreshing their BF16 copies
__global__ void adam_kernel(float* __restrict__ w, bf16* __restrict__ wb, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, long long n, float lr, float b1, float b2,
                            float eps, float bc1, float bc2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ x, bf16* __restrict__ y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

// The network input of subset t: the reference subset (rows x0-16 .. x0+15, columns
// y0-16 .. y0+15, 1-based) in the centre of channel 0 and the deformed window (x0-32 ..
// x0+31, y0-32 .. y0+31) in channel 1, each normalised to zero mean and unit deviation over
// its own pixels (taps clamped to the image).  One block of 256 threads per subset.
__global__ void patch_kernel(FrameDev fr, const double* __restrict__ coords, long long n, bf16* __restrict__ X) {
  __shared__ double red[2][256];
  const long long t = blockIdx.x;
  if (t >= n) return;
  const int tid = threadIdx.x;
  const int x0 = (int)llround(coords[t]), y0 = (int)llround(coords[n + t]);
  auto at = [&](const float* img, int r1, int c1) {  // 1-based, clamped
    r1 = r1 < 1 ? 1 : (r1 > fr.M ? fr.M : r1);
    c1 = c1 < 1 ? 1 : (c1 > fr.N ? fr.N : c1);
    return img[(size_t)(r1 - 1) + (size_t)(c1 - 1) * fr.M];
  };
  double sr = 0, sr2 = 0, sd = 0, sd2 = 0;
  for (int p = tid; p < 4096; p += 256) {
    const int i = p >> 6, j = p & 63;  // canvas row, column
    const double d = at(fr.def, x0 - 32 + i, y0 - 32 + j);
    sd += d;
    sd2 += d * d;
    if (p < 1024) {
      const double r = at(fr.ref, x0 - 16 + (p >> 5), y0 - 16 + (p & 31));
      sr += r;
      sr2 += r * r;
    }
  }
  double st[4] = {sr, sr2, sd, sd2};
  double out[4];
  for (int k = 0; k < 4; ++k) {
    red[0][tid] = st[k];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if (tid < o) red[0][tid] += red[0][tid + o];
      __syncthreads();
    }
    out[k] = red[0][0];
    __syncthreads();
  }
  const double mr = out[0] / 1024.0, md = out[2] / 4096.0;
  const double ir = 1.0 / sqrt(fmax(out[1] / 1024.0 - mr * mr, 1e-12));
  const double id = 1.0 / sqrt(fmax(out[3] / 4096.0 - md * md, 1e-12));
  bf16* x = X + t * 64 * 64 * 2;
  for (int p = tid; p < 4096; p += 256) {
    const int i = p >> 6, j = p & 63;
    const bool in_ref = i >= 16 && i < 48 && j >= 16 && j < 48;
    const float r = in_ref ? (float)((at(fr.ref, x0 - 32 + i, y0 - 32 + j) - mr) * ir) : 0.f;
    const float d = (float)((at(fr.def, x0 - 32 + i, y0 - 32 + j) - md) * id);
    x[(size_t)p * 2] = __float2bfloat16_rn(r);
    x[(size_t)p * 2 + 1] = __float2bfloat16_rn(d);
  }
}

// Network outputs (scaled) -> IC-GN initial guess: U0 = (u, v), F0 = (du/dx, dv/dx, du/dy, dv/dy)
__global__ void unscale_kernel(const float* __restrict__ Y, long long n, double* __restrict__ U0, double* __restrict__ F0) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const float* y = Y + t * kOutP;
    U0[2 * t] = 8.0 * y[0];
    U0[2 * t + 1] = 8.0 * y[1];
    for (int k = 0; k < 4; ++k) F0[4 * t + k] = y[2 + k] / 20.0;
  }
}

inline unsigned blocks_for(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  return (unsigned)(b < 1 ? 1 : (b > 148 * 64 ? 148 * 64 : b));
}

}  // namespace

// ============================================================================ the network
struct ProposalNet {
  int device = 0, max_batch = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  std::string err;
  long long launches = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  bf16* wb = nullptr;
  bf16* wt[6] = {};  // transposed weights [cols x rows] for the data gradients
  int step_count = 0;
  // activations and their gradients (max_batch)
  bf16 *A[4] = {}, *At[4] = {}, *H[5] = {}, *Ht[5] = {}, *dZ[5] = {}, *dZt[5] = {}, *dY = nullptr, *dYt = nullptr;
  float *dAf = nullptr, *dHf = nullptr, *Y = nullptr, *loss = nullptr;
  bf16* Xbuf = nullptr;  // patch batch for predict
  int* errflag = nullptr;
};

}  // namespace aldic

using aldic::ProposalNet;
struct aldic_net : ProposalNet {};

namespace aldic {
namespace {

#define NK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      net->err = std::string(#call) + ": " + cudaGetErrorString(e_);              \
      return ALDIC_ERR_CUDA;                                                      \
    }                                                                             \
  } while (0)

long long P_of(int l, int batch) { return (long long)batch * kConv[l].Hout * kConv[l].Wout; }

int gemm(ProposalNet* net, const void* A, long long lda, const void* B, long long ldb, long long M, long long N,
         long long K, int mode, float* c32, bf16* c16, const float* bias, long long ldc, int splits) {
  GemmArgs ga;
  ga.A = A;
  ga.lda = lda;
  ga.B = B;
  ga.ldb = ldb;
  ga.M = M;
  ga.N = N;
  ga.K = K;
  ga.splits = splits;
  ga.epi.mode = mode;
  ga.epi.c32 = c32;
  ga.epi.c16 = c16;
  ga.epi.bias = bias;
  ga.epi.ldc = ldc;
  ga.epi.err = net->errflag;
  const int r = launch_umma_gemm(ga, net->stream);
  if (r < 0) {
    net->err = "GEMM operand layout not describable by a tensor map";
    return ALDIC_ERR_ARG;
  }
  net->launches += r;
  return ALDIC_OK;
}

void transpose(ProposalNet* net, const bf16* in, bf16* out, long long R, long long Cn) {
  const dim3 grid((unsigned)((Cn + 31) / 32), (unsigned)((R + 31) / 32));
  transpose_kernel<<<grid, dim3(32, 8), 0, net->stream>>>(in, out, R, Cn);
  ++net->launches;
}

// split-K count for a weight gradient: enough blocks to fill the SMs
int wsplit(long long M, long long N, long long K) {
  const long long tiles = ((M + 127) / 128) * ((N + 255) / 256);
  long long s = (2 * 148) / (tiles < 1 ? 1 : tiles);
  const long long kb = (K + 63) / 64;
  if (s > kb) s = kb;
  return (int)(s < 1 ? 1 : s);
}

int forward(ProposalNet* net, int batch, const bf16* X) {
  const bf16* in = X;
  for (int l = 0; l < 4; ++l) {
    const ConvL& L = kConv[l];
    const long long P = P_of(l, batch);
    im2col_kernel<<<blocks_for(P * L.Kp), 256, 0, net->stream>>>(in, net->A[l], batch, L);
    ++net->launches;
    int rc = gemm(net, net->A[l], L.Kp, net->wb + kL.w[l], L.Kp, P, L.Cout, L.Kp, kEpiBiasReluBf16, nullptr,
                  net->H[l], net->w + kL.b[l], L.Cout, 1);
    if (rc) return rc;
    in = net->H[l];
  }
  int rc = gemm(net, net->H[3], kFcIn, net->wb + kL.w[4], kFcIn, batch, kFcHid, kFcIn, kEpiBiasReluBf16, nullptr,
                net->H[4], net->w + kL.b[4], kFcHid, 1);
  if (rc) return rc;
  return gemm(net, net->H[4], kFcHid, net->wb + kL.w[5], kFcHid, batch, kOutP, kFcHid, kEpiStore, net->Y, nullptr,
              net->w + kL.b[5], kOutP, 1);
}

// gradients of the mean squared error into net->g (zeroed here)
int backward(ProposalNet* net, int batch, const float* T) {
  cudaStream_t st = net->stream;
  NK(cudaMemsetAsync(net->g, 0, sizeof(float) * kL.n, st));
  NK(cudaMemsetAsync(net->loss, 0, sizeof(float), st));
  mse_kernel<<<1, 256, 0, st>>>(net->Y, T, batch, net->dY, net->loss);
  ++net->launches;
  // transposed weights for the data gradients
  for (int l = 1; l < 6; ++l) transpose(net, net->wb + kL.w[l], net->wt[l], kL.rows[l], kL.cols[l]);
  // FC2: dW = dY^T H4, db = sum dY, dH4 = dY W
  transpose(net, net->dY, net->dYt, batch, kOutP);
  transpose(net, net->H[4], net->Ht[4], batch, kFcHid);
  int rc = gemm(net, net->dYt, batch, net->Ht[4], batch, kOutP, kFcHid, batch, kEpiAtomic, net->g + kL.w[5], nullptr,
                nullptr, kFcHid, wsplit(kOutP, kFcHid, batch));
  if (rc) return rc;
  bias_grad_kernel<<<64, kOutP, 0, st>>>(net->dY, batch, kOutP, net->g + kL.b[5]);
  rc = gemm(net, net->dY, kOutP, net->wt[5], kOutP, batch, kFcHid, kOutP, kEpiStore, net->dHf, nullptr, nullptr,
            kFcHid, 1);
  if (rc) return rc;
  relu_grad_kernel<<<blocks_for((long long)batch * kFcHid), 256, 0, st>>>(net->dHf, net->H[4], net->dZ[4],
                                                                         (long long)batch * kFcHid);
  // FC1: dW = dZ^T H3flat, db, dH3 = dZ W
  transpose(net, net->dZ[4], net->dZt[4], batch, kFcHid);
  transpose(net, net->H[3], net->Ht[3], batch, kFcIn);
  rc = gemm(net, net->dZt[4], batch, net->Ht[3], batch, kFcHid, kFcIn, batch, kEpiAtomic, net->g + kL.w[4], nullptr,
            nullptr, kFcIn, wsplit(kFcHid, kFcIn, batch));
  if (rc) return rc;
  bias_grad_kernel<<<64, kFcHid, 0, st>>>(net->dZ[4], batch, kFcHid, net->g + kL.b[4]);
  rc = gemm(net, net->dZ[4], kFcHid, net->wt[4], kFcHid, batch, kFcIn, kFcHid, kEpiStore, net->dHf, nullptr, nullptr,
            kFcIn, 1);
  if (rc) return rc;
  relu_grad_kernel<<<blocks_for((long long)batch * kFcIn), 256, 0, st>>>(net->dHf, net->H[3], net->dZ[3],
                                                                        (long long)batch * kFcIn);
  net->launches += 4;
  // conv layers 4 .. 1: dW = dZ^T A, db, dA = dZ W -> col2im -> ReLU gradient of the input
  for (int l = 3; l >= 0; --l) {
    const ConvL& L = kConv[l];
    const long long P = P_of(l, batch);
    transpose(net, net->dZ[l], net->dZt[l], P, L.Cout);
    transpose(net, net->A[l], net->At[l], P, L.Kp);
    rc = gemm(net, net->dZt[l], P, net->At[l], P, L.Cout, L.Kp, P, kEpiAtomic, net->g + kL.w[l], nullptr, nullptr,
              L.Kp, wsplit(L.Cout, L.Kp, P));
    if (rc) return rc;
    bias_grad_kernel<<<148, L.Cout, 0, st>>>(net->dZ[l], P, L.Cout, net->g + kL.b[l]);
    ++net->launches;
    if (l == 0) break;
    rc = gemm(net, net->dZ[l], L.Cout, net->wt[l], L.Cout, P, L.Kp, L.Cout, kEpiStore, net->dAf, nullptr, nullptr,
              L.Kp, 1);
    if (rc) return rc;
    const long long nin = (long long)batch * L.Hin * L.Win * L.Cin;
    col2im_kernel<<<blocks_for(nin), 256, 0, st>>>(net->dAf, net->dHf, batch, L);
    relu_grad_kernel<<<blocks_for(nin), 256, 0, st>>>(net->dHf, net->H[l - 1], net->dZ[l - 1], nin);
    net->launches += 2;
  }
  return ALDIC_OK;
}

int check_errflag(ProposalNet* net) {
  int e = 0;
  NK(cudaMemcpyAsync(&e, net->errflag, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
  NK(cudaStreamSynchronize(net->stream));
  if (e) {
    net->err = "a tensor-core GEMM wait timed out";
    return ALDIC_ERR_TIMEOUT;
  }
  return ALDIC_OK;
}

}  // namespace

int launch_net_patches(const FrameDev& fr, const double* coords, long long n, void* X, cudaStream_t st) {
  patch_kernel<<<(unsigned)n, 256, 0, st>>>(fr, coords, n, reinterpret_cast<bf16*>(X));
  return 1;
}

}  // namespace aldic

using namespace aldic;

extern "C" {

int64_t aldic_net_param_count(void) { return kL.n; }

int aldic_net_create(aldic_net** out, int device, int max_batch) {
  if (!out || max_batch < 8 || max_batch % 8 != 0 || max_batch > 65536) return ALDIC_ERR_ARG;
  *out = nullptr;
  aldic_net* net = new aldic_net();
  net->device = device;
  net->max_batch = max_batch;
  auto fail = [&](cudaError_t e) {
    aldic_net_destroy(net);
    (void)e;
    return ALDIC_ERR_CUDA;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&net->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(e);
  net->stream = net->own;
  const long long B = max_batch, n = kL.n;
  e = cudaMalloc(&net->w, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->g, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->m, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->v, n * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->wb, n * 2);
  for (int l = 0; l < 6 && e == cudaSuccess; ++l) e = cudaMalloc(&net->wt[l], kL.rows[l] * kL.cols[l] * 2);
  long long maxA = 0, maxH = 0;
  for (int l = 0; l < 4 && e == cudaSuccess; ++l) {
    const long long P = P_of(l, (int)B);
    maxA = std::max(maxA, P * kConv[l].Kp);
    maxH = std::max(maxH, (long long)B * kConv[l].Hin * kConv[l].Win * kConv[l].Cin);
    e = cudaMalloc(&net->A[l], P * kConv[l].Kp * 2);
    if (e == cudaSuccess) e = cudaMalloc(&net->At[l], P * kConv[l].Kp * 2);
    if (e == cudaSuccess) e = cudaMalloc(&net->H[l], P * kConv[l].Cout * 2);
    if (e == cudaSuccess) e = cudaMalloc(&net->Ht[l], P * kConv[l].Cout * 2);
    if (e == cudaSuccess) e = cudaMalloc(&net->dZ[l], P * kConv[l].Cout * 2);
    if (e == cudaSuccess) e = cudaMalloc(&net->dZt[l], P * kConv[l].Cout * 2);
  }
  if (e == cudaSuccess) e = cudaMalloc(&net->H[4], B * kFcHid * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->Ht[4], B * kFcHid * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->dZ[4], B * kFcHid * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->dZt[4], B * kFcHid * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->dY, B * kOutP * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->dYt, B * kOutP * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->Y, B * kOutP * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->dAf, maxA * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->dHf, std::max(maxH, B * kFcIn) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->loss, 4);
  if (e == cudaSuccess) e = cudaMalloc(&net->Xbuf, B * 64 * 64 * 2 * 2);
  if (e == cudaSuccess) e = cudaMalloc(&net->errflag, 4);
  if (e != cudaSuccess) return fail(e);
  cudaMemset(net->m, 0, n * 4);
  cudaMemset(net->v, 0, n * 4);
  cudaMemset(net->w, 0, n * 4);
  cudaMemset(net->wb, 0, n * 2);
  cudaMemset(net->errflag, 0, 4);
  *out = net;
  return ALDIC_OK;
}

void aldic_net_destroy(aldic_net* net) {
  if (!net) return;
  cudaSetDevice(net->device);
  if (net->stream) cudaStreamSynchronize(net->stream);
  void* bufs[] = {net->w,  net->g,  net->m,    net->v,    net->wb, net->dY, net->dYt,   net->Y,
                  net->dAf, net->dHf, net->loss, net->Xbuf, net->errflag};
  for (void* p : bufs)
    if (p) cudaFree(p);
  for (int l = 0; l < 6; ++l)
    if (net->wt[l]) cudaFree(net->wt[l]);
  for (int l = 0; l < 5; ++l) {
    if (l < 4) {
      if (net->A[l]) cudaFree(net->A[l]);
      if (net->At[l]) cudaFree(net->At[l]);
    }
    if (net->H[l]) cudaFree(net->H[l]);
    if (net->Ht[l]) cudaFree(net->Ht[l]);
    if (net->dZ[l]) cudaFree(net->dZ[l]);
    if (net->dZt[l]) cudaFree(net->dZt[l]);
  }
  if (net->own) cudaStreamDestroy(net->own);
  delete net;
}

const char* aldic_net_last_error(const aldic_net* net) { return net ? net->err.c_str() : "null network"; }

int aldic_net_set_stream(aldic_net* net, void* stream) {
  if (!net) return ALDIC_ERR_ARG;
  net->stream = stream ? static_cast<cudaStream_t>(stream) : net->own;
  return ALDIC_OK;
}

int64_t aldic_net_launch_count(const aldic_net* net) { return net ? net->launches : 0; }

int aldic_net_set_params(aldic_net* net, const float* params) {
  if (!net || !params) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  NK(cudaMemcpyAsync(net->w, params, sizeof(float) * kL.n, cudaMemcpyDefault, net->stream));
  to_bf16_kernel<<<blocks_for(kL.n), 256, 0, net->stream>>>(net->w, net->wb, kL.n);
  NK(cudaMemsetAsync(net->m, 0, sizeof(float) * kL.n, net->stream));
  NK(cudaMemsetAsync(net->v, 0, sizeof(float) * kL.n, net->stream));
  net->step_count = 0;
  ++net->launches;
  NK(cudaStreamSynchronize(net->stream));
  return ALDIC_OK;
}

int aldic_net_get_params(aldic_net* net, float* params) {
  if (!net || !params) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  NK(cudaMemcpyAsync(params, net->w, sizeof(float) * kL.n, cudaMemcpyDefault, net->stream));
  NK(cudaStreamSynchronize(net->stream));
  return ALDIC_OK;
}

int aldic_net_forward(aldic_net* net, int batch, const void* x, float* y) {
  if (!net || !x || !y || batch < 8 || batch % 8 != 0 || batch > net->max_batch) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  int rc = forward(net, batch, reinterpret_cast<const bf16*>(x));
  if (rc) return rc;
  NK(cudaMemcpy2DAsync(y, kOut * 4, net->Y, kOutP * 4, kOut * 4, batch, cudaMemcpyDefault, net->stream));
  NK(cudaGetLastError());
  return ALDIC_OK;
}

int aldic_net_gradients(aldic_net* net, int batch, const void* x, const float* t, float* grads, float* loss) {
  if (!net || !x || !t || batch < 8 || batch % 8 != 0 || batch > net->max_batch) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  int rc = forward(net, batch, reinterpret_cast<const bf16*>(x));
  if (!rc) rc = backward(net, batch, t);
  if (rc) return rc;
  if (grads) NK(cudaMemcpyAsync(grads, net->g, sizeof(float) * kL.n, cudaMemcpyDefault, net->stream));
  if (loss) NK(cudaMemcpyAsync(loss, net->loss, sizeof(float), cudaMemcpyDefault, net->stream));
  NK(cudaGetLastError());
  return check_errflag(net);
}

int aldic_net_train_step(aldic_net* net, int batch, const void* x, const float* t, float lr, float* loss) {
  if (!net || !x || !t || batch < 8 || batch % 8 != 0 || batch > net->max_batch || !(lr > 0)) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  int rc = forward(net, batch, reinterpret_cast<const bf16*>(x));
  if (!rc) rc = backward(net, batch, t);
  if (rc) return rc;
  net->step_count += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.f - std::pow(b1, (float)net->step_count), bc2 = 1.f - std::pow(b2, (float)net->step_count);
  adam_kernel<<<blocks_for(kL.n), 256, 0, net->stream>>>(net->w, net->wb, net->g, net->m, net->v, kL.n, lr, b1, b2,
                                                          1e-8f, bc1, bc2);
  ++net->launches;
  if (loss) {
    NK(cudaMemcpyAsync(loss, net->loss, sizeof(float), cudaMemcpyDefault, net->stream));
    NK(cudaStreamSynchronize(net->stream));
  }
  NK(cudaGetLastError());
  return ALDIC_OK;
}

int aldic_gemm_bf16(const void* A, int64_t lda, const void* B, int64_t ldb, int64_t M, int64_t N, int64_t K, float* C,
                    int64_t ldc, int splits, void* stream) {
  if (!A || !B || !C || M < 0 || N < 0 || K < 0 || lda < K || ldb < K || ldc < N || splits < 1) return ALDIC_ERR_ARG;
  if (M == 0 || N == 0 || K == 0) return ALDIC_OK;
  GemmArgs g;
  g.A = A;
  g.lda = lda;
  g.B = B;
  g.ldb = ldb;
  g.M = M;
  g.N = N;
  g.K = K;
  g.splits = splits;
  g.epi.mode = splits > 1 ? kEpiAtomic : kEpiStore;
  g.epi.c32 = C;
  g.epi.c16 = nullptr;
  g.epi.bias = nullptr;
  g.epi.ldc = ldc;
  static int* errflag = nullptr;  // the GEMM time-out flag of this entry (one per process)
  if (!errflag && cudaMalloc(&errflag, sizeof(int)) != cudaSuccess) return ALDIC_ERR_CUDA;
  g.epi.err = errflag;
  if (launch_umma_gemm(g, static_cast<cudaStream_t>(stream)) < 0) return ALDIC_ERR_ARG;
  return cudaGetLastError() == cudaSuccess ? ALDIC_OK : ALDIC_ERR_CUDA;
}

int aldic_net_status(aldic_net* net) {
  if (!net) return ALDIC_ERR_ARG;
  NK(cudaSetDevice(net->device));
  return check_errflag(net);
}

}  // extern "C"

namespace aldic {
// Predict the initial guesses of n subsets (coords device n x 2) on the frame fr, in batches of
// the network's max_batch; U0 (2n) and F0 (4n) device arrays.
int net_predict(aldic_net* net, const FrameDev& fr, const double* coords_dev, long long n, double* U0, double* F0) {
  NK(cudaSetDevice(net->device));
  const int B = net->max_batch;
  for (long long s = 0; s < n; s += B) {
    const long long nb = std::min<long long>(B, n - s);
    const int bpad = (int)((nb + 7) / 8 * 8);
    // the patch kernel reads x at coords[t] and y at coords[n + t]: the batch's slice is the
    // same arrays offset by s
    patch_kernel<<<(unsigned)nb, 256, 0, net->stream>>>(fr, coords_dev + s, n, net->Xbuf);
    ++net->launches;
    if (bpad > nb) NK(cudaMemsetAsync(net->Xbuf + nb * 64 * 64 * 2, 0, (size_t)(bpad - nb) * 64 * 64 * 2 * 2, net->stream));
    int rc = forward(net, bpad, net->Xbuf);
    if (rc) return rc;
    unscale_kernel<<<blocks_for(nb), 256, 0, net->stream>>>(net->Y, nb, U0 + 2 * s, F0 + 4 * s);
    ++net->launches;
  }
  NK(cudaGetLastError());
  return ALDIC_OK;
}
}  // namespace aldic
