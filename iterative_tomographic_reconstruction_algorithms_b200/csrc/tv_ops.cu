// Finite-difference operators of the reference's ADMM-TV / CG solvers on the
// device (reference: algorithms/cg.py:62-71).
//
// G(m) = numpy.gradient(m): per axis (f[i+1] - f[i-1]) / 2 inside, one-sided
// differences f[1] - f[0] and f[n-1] - f[n-2] at the ends, in the input's
// float32 arithmetic.
//
// Gt(g) = g[1] . Gx + Gy . g[0] with Gx = gradient(I) along axis 0 and
// Gy = gradient(I) along axis 1 of identity matrices (cg.py:66-71): the
// reference forms these as dense matrices and multiplies (O(n^3)); each
// column of Gx and row of Gy has at most two non-zeros (+-1/2 inside, +-1 at
// the ends), so every output is the sum of at most two float64 products per
// term -- the same float64 numbers a stencil gives, computed here in O(n^2).
#include "tomo_internal.cuh"

namespace tomo {
namespace {

__global__ void grad2d_kernel(const float *__restrict__ m, int n0, int n1, float *__restrict__ g0,
                              float *__restrict__ g1) {
  const long long total = (long long)n0 * n1;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / n1), j = (int)(idx - (long long)i * n1);
    // axis 0
    float d0;
    if (n0 == 1) d0 = 0.0f;
    else if (i == 0) d0 = __fsub_rn(m[idx + n1], m[idx]);
    else if (i == n0 - 1) d0 = __fsub_rn(m[idx], m[idx - n1]);
    else d0 = __fdiv_rn(__fsub_rn(m[idx + n1], m[idx - n1]), 2.0f);
    // axis 1
    float d1;
    if (n1 == 1) d1 = 0.0f;
    else if (j == 0) d1 = __fsub_rn(m[idx + 1], m[idx]);
    else if (j == n1 - 1) d1 = __fsub_rn(m[idx], m[idx - 1]);
    else d1 = __fdiv_rn(__fsub_rn(m[idx + 1], m[idx - 1]), 2.0f);
    g0[idx] = d0;
    g1[idx] = d1;
  }
}

// Entry (k, j) of gradient(I_n) along axis 0 (the same numbers transposed
// for axis 1): +-1/2 at k = j -+ 1 inside, +-1 on the one-sided end rows.
__device__ __forceinline__ double dgrad(int k, int j, int n) {
  if (k == 0) return j == 1 ? 1.0 : (j == 0 ? -1.0 : 0.0);
  if (k == n - 1) return j == n - 1 ? 1.0 : (j == n - 2 ? -1.0 : 0.0);
  return j == k + 1 ? 0.5 : (j == k - 1 ? -0.5 : 0.0);
}

// out[i][j] = sum_k g1[i][k] Gx[k][j] + sum_k Gy[i][k] g0[k][j] with Gx[k][j] =
// dgrad(k, j, n1) and Gy[i][k] = dgrad(k, i, n0) (the gradient along axis 1 of
// the n0 x n0 identity is the transpose of the one along axis 0).
__global__ void grad2d_adjoint_kernel(const float *__restrict__ g0, const float *__restrict__ g1, int n0,
                                      int n1, double *__restrict__ out) {
  const long long total = (long long)n0 * n1;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(idx / n1), j = (int)(idx - (long long)i * n1);
    double a = 0.0, b = 0.0;
    // non-zeros of column j of Gx: rows k = j-1, j+1 (and the end rows 0, n1-1)
    for (int k = max(j - 1, 0); k <= min(j + 1, n1 - 1); ++k) {
      const double w = dgrad(k, j, n1);
      if (w != 0.0) a += (double)g1[(long long)i * n1 + k] * w;
    }
    for (int k = max(i - 1, 0); k <= min(i + 1, n0 - 1); ++k) {
      const double w = dgrad(k, i, n0);  // Gy[i][k]
      if (w != 0.0) b += w * (double)g0[(long long)k * n1 + j];
    }
    out[idx] = a + b;
  }
}

int grid_of(long long total) {
  const long long b = (total + 255) / 256;
  return (int)(b < 148 * 32 ? (b < 1 ? 1 : b) : 148 * 32);
}

}  // namespace
}  // namespace tomo

using namespace tomo;

extern "C" {

int tomo_grad2d(const float *d_m, int n0, int n1, float *d_g0, float *d_g1, void *stream) {
  if (!d_m || !d_g0 || !d_g1 || n0 < 1 || n1 < 1) return fail(TOMO_EINVAL, "grad2d: bad arguments");
  grad2d_kernel<<<grid_of((long long)n0 * n1), 256, 0, (cudaStream_t)stream>>>(d_m, n0, n1, d_g0, d_g1);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int tomo_grad2d_adjoint(const float *d_g0, const float *d_g1, int n0, int n1, double *d_out, void *stream) {
  if (!d_g0 || !d_g1 || !d_out || n0 < 2 || n1 < 2) return fail(TOMO_EINVAL, "grad2d adjoint: bad arguments");
  grad2d_adjoint_kernel<<<grid_of((long long)n0 * n1), 256, 0, (cudaStream_t)stream>>>(d_g0, d_g1, n0, n1, d_out);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // extern "C"
