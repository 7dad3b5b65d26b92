// On-chip throughput probes used as roofline denominators for the projector
// kernels, which gather from L1/shared memory and issue FP32 work rather than
// stream HBM.  Each probe saturates one resource on every SM and is timed with
// CUDA events at whatever clocks the GPU is running, so a bench run measures
// its own denominators.
#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr int kSmemWords = 8192;  // 32 KiB of float4
constexpr int kIters = 4096;

// Shared-memory load bandwidth: conflict-free 16-byte loads, 8 in flight.
__global__ void __launch_bounds__(512) smem_probe(float *out, int salt) {
  __shared__ float4 buf[kSmemWords / 4];
  for (int i = threadIdx.x; i < kSmemWords / 4; i += blockDim.x)
    buf[i] = make_float4(i + salt, i, i, i);
  __syncthreads();
  float4 acc[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) acc[u] = make_float4(0, 0, 0, 0);
  const int mask = kSmemWords / 4 - 1;
  int idx = threadIdx.x;
  for (int it = 0; it < kIters; it += 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      float4 v = buf[(idx + u * 512) & mask];
      acc[u].x += v.x; acc[u].y += v.y; acc[u].z += v.z; acc[u].w += v.w;
    }
    idx += 64;
  }
  float s = 0;
#pragma unroll
  for (int u = 0; u < 8; ++u) s += acc[u].x + acc[u].y + acc[u].z + acc[u].w;
  if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// L1 load bandwidth from a per-CTA 64 KiB window (L1-resident after the
// first pass), with every warp request one aligned, fully used block of
// memory: lane l of a warp reads word (base + l) for 4-byte loads (one 128-byte
// line per request) and float4 (base + l) for 16-byte loads (four lines).
// base steps by a multiple of the request size, so no request straddles lines.
template <typename T>
__global__ void __launch_bounds__(512) l1_probe(const T *__restrict__ src, float *out) {
  constexpr int kWin = 65536 / sizeof(T);  // window in elements
  const T *w = src + (size_t)(blockIdx.x % 8) * kWin;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int base = warp * 32 * 8;
  for (int it = 0; it < kIters; it += 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const T v = __ldg(w + ((base + u * 32 + lane) & (kWin - 1)));
      if constexpr (sizeof(T) == 16) acc[u] += v.x + v.y + v.z + v.w;
      else acc[u] += v;
    }
    base += 32 * 8 * 16 + 32;  // a multiple of 32 elements
  }
  float s = 0;
#pragma unroll
  for (int u = 0; u < 8; ++u) s += acc[u];
  if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// FP32 FMA rate: 8 independent dependency chains per thread.
__global__ void __launch_bounds__(512) fma_probe(float *out, float a, float b) {
  float x[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) x[u] = threadIdx.x * 1e-3f + u;
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int u = 0; u < 8; ++u) x[u] = fmaf(x[u], a, b);
  }
  float s = 0;
#pragma unroll
  for (int u = 0; u < 8; ++u) s += x[u];
  if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <typename F>
int time_launch(F launch, int reps, float *ms) {
  cudaEvent_t e0, e1;
  TOMO_CUDA(cudaEventCreate(&e0));
  TOMO_CUDA(cudaEventCreate(&e1));
  launch();  // warm-up
  TOMO_CUDA(cudaEventRecord(e0));
  for (int r = 0; r < reps; ++r) launch();
  TOMO_CUDA(cudaEventRecord(e1));
  TOMO_CUDA(cudaEventSynchronize(e1));
  TOMO_CUDA(cudaEventElapsedTime(ms, e0, e1));
  *ms /= reps;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return TOMO_OK;
}

}  // namespace
}  // namespace tomo

using namespace tomo;

extern "C" int tomo_measure_onchip_peaks2(double *smem_gbs, double *l1_4_gbs, double *l1_16_gbs,
                                          double *fp32_tflops) {
  int dev = 0, sms = 0;
  TOMO_CUDA(cudaGetDevice(&dev));
  TOMO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 4, threads = 512;
  float *out = nullptr, *src = nullptr;
  TOMO_CUDA(cudaMalloc(&out, sizeof(float) * blocks * threads));
  TOMO_CUDA(cudaMalloc(&src, 65536 * 8));
  TOMO_CUDA(cudaMemset(src, 0, 65536 * 8));
  float ms = 0;
  int rc = time_launch([&] { smem_probe<<<blocks, threads>>>(out, 1); }, 5, &ms);
  if (rc) return rc;
  if (smem_gbs) *smem_gbs = (double)blocks * threads * kIters * 16.0 / (ms * 1e-3) / 1e9;
  rc = time_launch([&] { l1_probe<float><<<blocks, threads>>>(src, out); }, 5, &ms);
  if (rc) return rc;
  if (l1_4_gbs) *l1_4_gbs = (double)blocks * threads * kIters * 4.0 / (ms * 1e-3) / 1e9;
  rc = time_launch([&] { l1_probe<float4><<<blocks, threads>>>((const float4 *)src, out); }, 5, &ms);
  if (rc) return rc;
  if (l1_16_gbs) *l1_16_gbs = (double)blocks * threads * kIters * 16.0 / (ms * 1e-3) / 1e9;
  rc = time_launch([&] { fma_probe<<<blocks, threads>>>(out, 0.999f, 0.001f); }, 5, &ms);
  if (rc) return rc;
  if (fp32_tflops) *fp32_tflops = (double)blocks * threads * kIters * 8 * 2.0 / (ms * 1e-3) / 1e12;
  TOMO_CUDA(cudaGetLastError());
  cudaFree(out);
  cudaFree(src);
  return TOMO_OK;
}

extern "C" int tomo_measure_onchip_peaks(double *smem_gbs, double *l1_gbs, double *fp32_tflops) {
  double l1_4 = 0.0, l1_16 = 0.0;
  int rc = tomo_measure_onchip_peaks2(smem_gbs, &l1_4, &l1_16, fp32_tflops);
  if (rc) return rc;
  if (l1_gbs) *l1_gbs = l1_4 > l1_16 ? l1_4 : l1_16;
  return TOMO_OK;
}
