// On-chip throughput probes used as roofline denominators for the projector
// kernels, which gather from L1/shared memory and issue FP32 work rather than
// stream HBM.  Each probe saturates one resource on every SM and is timed with
// CUDA events at whatever clocks the GPU is running, so a bench run measures
// its own denominators.
#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr int kIters = 4096;

// The loads of both probes are volatile inline PTX, so the compiler issues
// every one of them (a plain loop over a periodic address pattern can be
// folded, which once made a probe report nearly twice the bytes it moved).
// Addresses are a base plus a constant offset per unrolled load, and each
// load's value feeds one add, so the probes issue about two instructions per load and the
// memory pipe, not the schedulers, is the limit.
constexpr int kUnroll = 16;

// Shared-memory load bandwidth: 16-byte loads, a warp request = 512
// consecutive bytes (conflict-free), from a 32 KiB array.
__global__ void __launch_bounds__(512) smem_probe(float *out, int salt) {
  __shared__ __align__(16) float buf[8192];
  for (int i = threadIdx.x; i < 8192; i += blockDim.x) buf[i] = (float)(i + salt);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t base = (uint32_t)__cvta_generic_to_shared(buf) + lane * 16;
  uint32_t off = (warp * 3 * 512) & (32768 - 1) & ~(kUnroll * 512 - 1);
  float acc = 0.0f;
  for (int it = 0; it < kIters; it += kUnroll) {
    const uint32_t a = base + off;
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      float x, y, z, w;
      asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                   : "=f"(x), "=f"(y), "=f"(z), "=f"(w)
                   : "r"(a + u * 512));
      asm volatile("" ::"f"(y), "f"(z), "f"(w));  // the other lanes of the vector: no instruction
      acc += x;
    }
    off = (off + kUnroll * 512) & (32768 - 1);
  }
  if (acc == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

// L1 load bandwidth from a 32 KiB window that every CTA of an SM reads (so it
// stays in L1 after the first pass).  VEC = 1: 4-byte loads, a warp request =
// one 128-byte line; VEC = 4: 16-byte loads, four lines.  No request straddles
// a line.
template <int VEC>
__global__ void __launch_bounds__(512) l1_probe(const float *__restrict__ src, float *out) {
  constexpr int kReq = 32 * VEC * 4;  // bytes per warp request
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const char *base = (const char *)src + lane * VEC * 4;
  uint32_t off = (uint32_t)(warp * 3 * kReq) & (32768 - 1) & ~(uint32_t)(kUnroll * kReq - 1);
  float acc = 0.0f;
  for (int it = 0; it < kIters; it += kUnroll) {
    const char *p = base + off;
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      float x;
      if constexpr (VEC == 1) {
        asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(x) : "l"(p + u * kReq));
      } else {
        float y, z, w;
        asm volatile("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];"
                     : "=f"(x), "=f"(y), "=f"(z), "=f"(w)
                     : "l"(p + u * kReq));
        asm volatile("" ::"f"(y), "f"(z), "f"(w));  // the other lanes of the vector: no instruction
      }
      acc += x;
    }
    off = (off + kUnroll * kReq) & (32768 - 1);
  }
  if (acc == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
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
  TOMO_CUDA(cudaMalloc(&src, 32768));
  TOMO_CUDA(cudaMemset(src, 0, 32768));
  float ms = 0;
  int rc = time_launch([&] { smem_probe<<<blocks, threads>>>(out, 1); }, 5, &ms);
  if (rc) return rc;
  if (smem_gbs) *smem_gbs = (double)blocks * threads * kIters * 16.0 / (ms * 1e-3) / 1e9;
  rc = time_launch([&] { l1_probe<1><<<blocks, threads>>>(src, out); }, 5, &ms);
  if (rc) return rc;
  if (l1_4_gbs) *l1_4_gbs = (double)blocks * threads * kIters * 4.0 / (ms * 1e-3) / 1e9;
  rc = time_launch([&] { l1_probe<4><<<blocks, threads>>>(src, out); }, 5, &ms);
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
