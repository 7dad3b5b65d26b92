// Internal declarations of libtomo_nn (the learned warm start's kernels).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/tomo_nn.h"

namespace tomo_nn {

constexpr int NN_OK = TOMO_NN_OK;
constexpr int NN_EINVAL = TOMO_NN_EINVAL;
constexpr int NN_ECUDA = TOMO_NN_ECUDA;

enum GemmMode : int { GEMM_DENSE = 0, GEMM_CONV3X3 = 1 };

struct GemmArgs {
  int mode = GEMM_DENSE;
  const __nv_bfloat16 *A = nullptr;  // dense: A[m*lda + k]; conv: X[batch][H][W][Cin]
  int lda = 0;
  const __nv_bfloat16 *B = nullptr;  // B[n*ldb + k]
  int ldb = 0;
  int M = 0, N = 0, K = 0;
  int H = 0, W = 0, Cin = 0;         // conv mode
  float *Cf = nullptr;               // FP32 output (or partials with ksplit > 1) ...
  __nv_bfloat16 *Cb = nullptr;       // ... or BF16 output
  int ldc = 0;
  const float *bias = nullptr;
  int relu = 0;
  int ksplit = 1;
  unsigned *status = nullptr;        // bit 0 set if an MMA wait gave up
  int spins = 1 << 22;               // polls of a pipeline wait before it gives up
};


int gemm_launch(const GemmArgs &g, cudaStream_t s);

}  // namespace tomo_nn
