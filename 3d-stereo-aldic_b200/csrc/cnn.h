// Internal interfaces of the proposal network (learned initial guess): the tcgen05 GEMM and
// its epilogues.  Not part of the public C ABI.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace aldic {

constexpr int kEpiStore = 0;         // c32[r, c] = acc (+ bias[c])
constexpr int kEpiAtomic = 1;        // c32[r, c] += acc (split-K partial sums)
constexpr int kEpiBiasReluBf16 = 2;  // c16[r, c] = bf16(max(acc + bias[c], 0))

struct GemmEpi {
  int mode;
  float* c32;
  __nv_bfloat16* c16;
  const float* bias;  // N entries or null
  long long ldc;      // row pitch of the output (elements)
  int* err;           // set (bit 0: a load or MMA wait timed out; bit 1: the epilogue's) on failure
};

// C[M x N] = A[M x K] * B[N x K]^T; A and B row-major BF16 with row pitches lda / ldb
// (elements, multiples of 8 so rows start on 16-byte boundaries), 16-byte aligned bases.
// Rows of A or B beyond M / N and columns beyond K read as zero.  splits > 1 divides K over
// that many blocks per tile (epilogue kEpiAtomic only).
struct GemmArgs {
  const void* A;
  long long lda;
  const void* B;
  long long ldb;
  long long M, N, K;
  int splits;
  GemmEpi epi;
};

int launch_umma_gemm(const GemmArgs& g, cudaStream_t st);

}  // namespace aldic
