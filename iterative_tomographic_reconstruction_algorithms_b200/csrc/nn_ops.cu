// libtomo_nn: the C ABI of include/tomo_nn.h and the small kernels around the
// tensor-core GEMM (nn_gemm.cu): weight preparation, the operand transposes of
// the weight gradient, its split-K reduction, ReLU backward and Adam.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "nn_internal.cuh"

namespace tomo_nn {
namespace {

__device__ unsigned g_status;  // bit 0: a tensor-core wait gave up
std::atomic<int> g_wait_spins{1 << 22};

unsigned *status_ptr() {
  static std::mutex mu;
  static unsigned *ptr[64] = {nullptr};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64) return nullptr;
  if (!ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_status) != cudaSuccess) return nullptr;
    ptr[dev] = (unsigned *)p;
  }
  return ptr[dev];
}

// out[(t*C + c)][p] = X[p shifted by tap t][c] (0 outside the image), for
// taps = 9 (3x3, pad 1) or 1 (plain transpose [P][C] -> [C][P]).  32x32 tiles
// through shared memory: reads run along channels, writes along pixels.
__global__ void im2col_t_kernel(const __nv_bfloat16 *__restrict__ X, int B, int H, int W, int C, int taps,
                                __nv_bfloat16 *__restrict__ out) {
  __shared__ __nv_bfloat16 tile[32][34];
  const long long P = (long long)B * H * W;
  const long long p0 = (long long)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32, t = blockIdx.z;
  const int dy = taps == 9 ? t / 3 - 1 : 0, dx = taps == 9 ? t % 3 - 1 : 0;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const long long p = p0 + i;
    const int c = c0 + threadIdx.x;
    __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
    if (p < P && c < C) {
      const int hw = H * W;
      const int b = (int)(p / hw), r = (int)(p - (long long)b * hw), y = r / W + dy, x = r % W + dx;
      if (y >= 0 && y < H && x >= 0 && x < W) v = X[(((long long)b * H + y) * W + x) * C + c];
    }
    tile[i][threadIdx.x] = v;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i;
    const long long p = p0 + threadIdx.x;
    if (c < C && p < P) out[((long long)t * C + c) * P + p] = tile[threadIdx.x][i];
  }
}

// dW[co][k] = sum_s part[s][k][co] (fixed order); part is [S][Kd][Cout].
__global__ void wgrad_reduce_kernel(const float *__restrict__ part, int S, int Kd, int Cout,
                                    float *__restrict__ dW) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)Kd * Cout) return;
  const int co = (int)(i / Kd), k = (int)(i - (long long)co * Kd);
  float acc = 0.0f;
  for (int s = 0; s < S; ++s) acc += part[((long long)s * Kd + k) * Cout + co];
  dW[(long long)co * Kd + k] = acc;
}

// db[c] = sum_p rows[c][p] (rows = dY transposed, [C][P]); one block per channel.
__global__ void row_sum_kernel(const __nv_bfloat16 *__restrict__ rows, long long P, float *__restrict__ db) {
  __shared__ float part[256];
  const __nv_bfloat16 *r = rows + (long long)blockIdx.x * P;
  float acc = 0.0f;
  for (long long p = threadIdx.x; p < P; p += blockDim.x) acc += __bfloat162float(r[p]);
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[blockIdx.x] = part[0];
}

__global__ void prepare_weights_kernel(const float *__restrict__ W, int Cout, int Cin, int taps,
                                       __nv_bfloat16 *__restrict__ Wb, __nv_bfloat16 *__restrict__ Wd) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)Cout * taps * Cin;
  if (i >= n) return;
  const int ci = (int)(i % Cin), t = (int)((i / Cin) % taps), co = (int)(i / ((long long)Cin * taps));
  const __nv_bfloat16 v = __float2bfloat16_rn(W[i]);
  Wb[i] = v;
  if (Wd) Wd[((long long)ci * taps + (taps - 1 - t)) * Cout + co] = v;
}

__global__ void relu_bwd_kernel(const __nv_bfloat16 *__restrict__ Y, __nv_bfloat16 *__restrict__ dY, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!(__bfloat162float(Y[i]) > 0.0f)) dY[i] = __float2bfloat16_rn(0.0f);
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

int wgrad_split(long long P, int M, int N) {
  const int bn = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
  const long long tiles = (long long)((M + 127) / 128) * ((N + bn - 1) / bn);
  long long s = std::max(1LL, 296 / tiles);
  s = std::min(s, std::max(1LL, P / 4096));
  return (int)std::min(s, 64LL);
}

}  // namespace
}  // namespace tomo_nn

using namespace tomo_nn;

extern "C" {

int tomo_nn_gemm(const void *A, int lda, const void *B, int ldb, int M, int N, int K, float *Cf, void *Cb,
                 int ldc, const float *bias, int relu, void *stream) {
  GemmArgs g;
  g.mode = GEMM_DENSE;
  g.A = (const __nv_bfloat16 *)A;
  g.lda = lda;
  g.B = (const __nv_bfloat16 *)B;
  g.ldb = ldb;
  g.M = M;
  g.N = N;
  g.K = K;
  g.Cf = Cf;
  g.Cb = (__nv_bfloat16 *)Cb;
  g.ldc = ldc;
  g.bias = bias;
  g.relu = relu;
  g.status = status_ptr();
  g.spins = g_wait_spins.load();
  return gemm_launch(g, (cudaStream_t)stream);
}

int tomo_nn_conv3x3(const void *X, int batch, int H, int W, int Cin, const void *Wt, int Cout, float *Yf,
                    void *Yb, const float *bias, int relu, void *stream) {
  if (batch < 1 || H < 1 || W < 1) return NN_EINVAL;
  GemmArgs g;
  g.mode = GEMM_CONV3X3;
  g.A = (const __nv_bfloat16 *)X;
  g.B = (const __nv_bfloat16 *)Wt;
  g.ldb = 9 * Cin;
  g.M = batch * H * W;
  g.N = Cout;
  g.K = 9 * Cin;
  g.H = H;
  g.W = W;
  g.Cin = Cin;
  g.Cf = Yf;
  g.Cb = (__nv_bfloat16 *)Yb;
  g.ldc = Cout;
  g.bias = bias;
  g.relu = relu;
  g.status = status_ptr();
  g.spins = g_wait_spins.load();
  return gemm_launch(g, (cudaStream_t)stream);
}

size_t tomo_nn_wgrad_workspace(int batch, int H, int W, int Cin, int Cout, int taps) {
  const long long P = (long long)batch * H * W;
  const int S = wgrad_split(P, taps * Cin, Cout);
  return align256(sizeof(__nv_bfloat16) * (size_t)taps * Cin * P) + align256(sizeof(__nv_bfloat16) * (size_t)Cout * P) +
         sizeof(float) * (size_t)S * taps * Cin * Cout;
}

int tomo_nn_wgrad(const void *X, const void *dY, int batch, int H, int W, int Cin, int Cout, int taps,
                  float *dW, float *db, void *work, size_t work_bytes, void *stream) {
  if ((taps != 9 && taps != 1) || Cin % 8 || Cout < 1 || batch < 1) return NN_EINVAL;
  const long long P = (long long)batch * H * W;
  if (P % 8) return NN_EINVAL;
  if (work_bytes < tomo_nn_wgrad_workspace(batch, H, W, Cin, Cout, taps)) return NN_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  const int Kd = taps * Cin, S = wgrad_split(P, Kd, Cout);
  char *w = (char *)work;
  __nv_bfloat16 *Xt = (__nv_bfloat16 *)w;
  __nv_bfloat16 *Yt = (__nv_bfloat16 *)(w + align256(sizeof(__nv_bfloat16) * (size_t)Kd * P));
  float *part = (float *)((char *)Yt + align256(sizeof(__nv_bfloat16) * (size_t)Cout * P));
  dim3 tb(32, 8);
  im2col_t_kernel<<<dim3((unsigned)((P + 31) / 32), (Cin + 31) / 32, taps), tb, 0, s>>>(
      (const __nv_bfloat16 *)X, batch, H, W, Cin, taps, Xt);
  im2col_t_kernel<<<dim3((unsigned)((P + 31) / 32), (Cout + 31) / 32, 1), tb, 0, s>>>(
      (const __nv_bfloat16 *)dY, batch, H, W, Cout, 1, Yt);
  if (cudaGetLastError() != cudaSuccess) return NN_ECUDA;
  // dW^T partials [S][Kd][Cout] = Xt . Yt^T over pixel slices
  GemmArgs g;
  g.mode = GEMM_DENSE;
  g.A = Xt;
  g.lda = (int)P;
  g.B = Yt;
  g.ldb = (int)P;
  g.M = Kd;
  g.N = Cout;
  g.K = (int)P;
  g.Cf = part;
  g.ldc = Cout;
  g.ksplit = S;
  g.status = status_ptr();
  g.spins = g_wait_spins.load();
  if (P > 0x7fffffffLL) return NN_EINVAL;
  int rc = gemm_launch(g, s);
  if (rc) return rc;
  const long long nout = (long long)Kd * Cout;
  wgrad_reduce_kernel<<<(unsigned)((nout + 255) / 256), 256, 0, s>>>(part, S, Kd, Cout, dW);
  if (db) row_sum_kernel<<<Cout, 256, 0, s>>>(Yt, P, db);
  return cudaGetLastError() == cudaSuccess ? NN_OK : NN_ECUDA;
}

int tomo_nn_prepare_weights(const float *W, int Cout, int Cin, int taps, void *Wb, void *Wd, void *stream) {
  const long long n = (long long)Cout * taps * Cin;
  if (n <= 0) return NN_EINVAL;
  prepare_weights_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      W, Cout, Cin, taps, (__nv_bfloat16 *)Wb, (__nv_bfloat16 *)Wd);
  return cudaGetLastError() == cudaSuccess ? NN_OK : NN_ECUDA;
}

int tomo_nn_relu_bwd(const void *Y, void *dY, size_t n, void *stream) {
  if (!n) return NN_OK;
  relu_bwd_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16 *)Y, (__nv_bfloat16 *)dY, n);
  return cudaGetLastError() == cudaSuccess ? NN_OK : NN_ECUDA;
}

int tomo_nn_adam(float *p, const float *g, float *m, float *v, size_t n, float lr, float beta1, float beta2,
                 float eps, int step, void *stream) {
  if (!n || step < 1) return NN_EINVAL;
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  adam_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, (cudaStream_t)stream>>>(
      p, g, m, v, n, lr, beta1, beta2, eps, c1, c2);
  return cudaGetLastError() == cudaSuccess ? NN_OK : NN_ECUDA;
}

int tomo_nn_set_wait_limit(int spins) {
  tomo_nn::g_wait_spins.store(spins < 0 ? (1 << 22) : spins);
  return NN_OK;
}

int tomo_nn_status(unsigned *flags) {
  unsigned *d = status_ptr();
  if (!d) return NN_ECUDA;
  unsigned h = 0;
  if (cudaDeviceSynchronize() != cudaSuccess) return NN_ECUDA;
  if (cudaMemcpy(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess) return NN_ECUDA;
  const unsigned zero = 0;
  if (cudaMemcpy(d, &zero, sizeof(unsigned), cudaMemcpyHostToDevice) != cudaSuccess) return NN_ECUDA;
  if (flags) *flags = h;
  return NN_OK;
}

}  // extern "C"
