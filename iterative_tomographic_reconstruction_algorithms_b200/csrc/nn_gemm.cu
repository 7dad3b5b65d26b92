// BF16 GEMM and 3x3 convolution on the 5th-generation tensor cores (sm_100a).
//
//   C[M][N] = A[M][K] . B[N][K]^T  (+ bias[N], ReLU), FP32 accumulation
//
// A and B are K-major BF16.  A is either a dense row-major matrix or the
// implicit im2col matrix of a 3x3, stride-1, zero-padded convolution over an
// NHWC BF16 input (row = output pixel, k = (tap, channel) with the channel
// fastest), so a convolution is one GEMM with M = pixels, N = output channels,
// K = 9 * input channels, and its input gradient is the same GEMM over the
// output gradient with the flipped, transposed weights.
//
// One CTA computes a 128 x BN tile with tcgen05.mma (cta_group::1, kind::f16,
// M = 128, N = BN, K = 16 per instruction) into a TMEM accumulator of BN
// FP32 columns.  Operands are staged in shared memory in the canonical
// K-major, non-swizzled layout the MMA's shared-memory descriptors describe
// (8-row x 16-byte core matrices; SBO = 128 B between row groups, LBO =
// rows x 16 B between K groups), by 16-byte cp.async copies (zero-filled
// outside the matrix), double-buffered: the copies of K block k+1 overlap
// the MMAs of block k.  One thread issues the MMAs and commits them to a
// per-stage mbarrier; every wait on it is bounded (the pipeline waits by a
// limit the caller may lower, tomo_nn_set_wait_limit), and a wait that gives
// up records an error in the status word, waits (with a long limit) for the
// last committed MMAs, frees the TMEM and returns without storing.  The epilogue reads TMEM with tcgen05.ld
// (warp w owns accumulator rows 32w..32w+31), applies bias and ReLU and
// stores FP32 or BF16.  With ksplit > 1 the K range is split over gridDim.z
// and each slice writes a partial FP32 tile, summed afterwards in a fixed
// order (nn_ops.cu), so results stay deterministic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "nn_internal.cuh"

namespace tomo_nn {
namespace {

constexpr int BM = 128, BK = 64, kThreads = 128;
// Drain limit: the wait for the last committed MMAs before the TMEM is freed
// keeps this long limit whatever the pipeline waits' limit (GemmArgs::spins).
constexpr int kDrainSpins = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
  const int n = valid ? 16 : 0;  // 0: zero-fill, nothing is read
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of the barrier: at most `spins` polls;
// false if it gave up (at once when spins is 0).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int spins) {
  for (int i = 0; i < spins; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle (version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: D F32, A and B BF16, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t instr_desc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
      "%13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Copies K block kb of the A and B tiles into one stage (canonical layout:
// element (row, k) of a tile with R rows at (k / 8) * R * 16 + row * 16 + (k % 8) * 2).
template <int BN>
__device__ __forceinline__ void load_stage(const GemmArgs &g, int m0, int n0, int kb, uint32_t sa, uint32_t sb) {
  const int tid = threadIdx.x;
  const int kc0 = kb * (BK / 8);  // first 8-element K chunk of the block
  for (int idx = tid; idx < BM * 8; idx += kThreads) {
    const int row = idx >> 3, c = idx & 7, kc = kc0 + c;
    const int m = m0 + row;
    const __nv_bfloat16 *src = g.A;
    bool ok = false;
    if (g.mode == GEMM_DENSE) {
      ok = m < g.M && kc * 8 < g.K;
      if (ok) src = g.A + (size_t)m * g.lda + kc * 8;
    } else {  // implicit im2col of a 3x3, pad-1 convolution over X[batch][H][W][Cin]
      const int cpt = g.Cin >> 3;  // chunks per tap
      const int tap = kc / cpt, cb = kc - tap * cpt;
      if (m < g.M && tap < 9) {
        const int hw = g.H * g.W, b = m / hw, r = m - b * hw, y = r / g.W, x = r - y * g.W;
        const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
        ok = yy >= 0 && yy < g.H && xx >= 0 && xx < g.W;
        if (ok) src = g.A + (((size_t)b * g.H + yy) * g.W + xx) * g.Cin + cb * 8;
      }
    }
    cp_async16(sa + c * (BM * 16) + row * 16, src, ok);
  }
  for (int idx = tid; idx < BN * 8; idx += kThreads) {
    const int row = idx >> 3, c = idx & 7, kc = kc0 + c;
    const int n = n0 + row;
    const bool ok = n < g.N && kc * 8 < g.K;
    cp_async16(sb + c * (BN * 16) + row * 16, ok ? (const void *)(g.B + (size_t)n * g.ldb + kc * 8) : (const void *)g.B,
               ok);
  }
}

template <int BN>
__global__ void __launch_bounds__(kThreads) gemm_tc_kernel(GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr int kStageA = BM * BK * 2, kStageB = BN * BK * 2;
  unsigned char *sA[2] = {smem, smem + kStageA + kStageB};
  unsigned char *sB[2] = {smem + kStageA, smem + 2 * kStageA + kStageB};
  uint64_t *bars = (uint64_t *)(smem + 2 * (kStageA + kStageB));
  uint32_t *tmem_slot = (uint32_t *)(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int nkb_all = (g.K + BK - 1) / BK;
  const int kb0 = (int)(((long long)nkb_all * blockIdx.z) / gridDim.z);
  const int kb1 = (int)(((long long)nkb_all * (blockIdx.z + 1)) / gridDim.z);
  const int nkb = kb1 - kb0;

  if (warp == 0) {  // TMEM accumulator: BN columns x 128 lanes of FP32
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    mbar_init(smem_u32(&bars[0]), 1);
    mbar_init(smem_u32(&bars[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = instr_desc(BN);
  bool ok = true;
  int last = -1;  // last K block whose MMAs were committed (block-uniform)

  if (nkb > 0) load_stage<BN>(g, m0, n0, kb0, smem_u32(sA[0]), smem_u32(sB[0]));
  cp_async_commit();
  for (int it = 0; it < nkb; ++it) {
    const int s = it & 1;
    if (it + 1 < nkb) {
      // the stage about to be refilled was read by the MMAs of block it-1
      if (it >= 1) {
        const bool w = mbar_wait(smem_u32(&bars[s ^ 1]), ((it - 1) >> 1) & 1, g.spins);
        ok = __syncthreads_and(w) != 0;  // block-uniform
        if (!ok) break;
      }
      load_stage<BN>(g, m0, n0, kb0 + it + 1, smem_u32(sA[s ^ 1]), smem_u32(sB[s ^ 1]));
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    fence_proxy_async();  // this thread's copies -> visible to the tensor-core (async) proxy
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sA[s]), b0 = smem_u32(sB[s]);
#pragma unroll
      for (int ks = 0; ks < BK / 16; ++ks) {
        const uint64_t da = smem_desc(a0 + ks * 2 * (BM * 16), BM * 16, 128);
        const uint64_t db = smem_desc(b0 + ks * 2 * (BN * 16), BN * 16, 128);
        mma_bf16(tmem, da, db, idesc, (it > 0 || ks > 0) ? 1u : 0u);
      }
      mma_commit(smem_u32(&bars[s]));
    }
    __syncwarp();
    last = it;
  }
  cp_async_wait<0>();
  // The last commit covers every MMA issued before it; it is also where the
  // error path (a pipeline wait that gave up, `last` = the block before it)
  // waits, with the long drain limit, before the TMEM is freed.  If even that
  // gives up, the TMEM is still freed: the status word says the output and the
  // kernel are not to be trusted.
  if (last >= 0) {
    const bool done = mbar_wait(smem_u32(&bars[last & 1]), (last >> 1) & 1, kDrainSpins);
    ok = __syncthreads_and(ok && done) != 0;
  }
  if (!ok && tid == 0 && g.status) atomicOr(g.status, 1);
  tc_fence_after();

  if (ok) {
    const int m = m0 + warp * 32 + lane;
    const size_t zoff = g.ksplit > 1 ? (size_t)blockIdx.z * g.M * g.ldc : 0;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      if (nkb > 0) {
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = 0.0f;
      }
      if (m < g.M) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int n = n0 + c0 + i;
          if (n < g.N) {
            float o = v[i];
            if (g.ksplit <= 1) {
              if (g.bias) o += g.bias[n];
              if (g.relu) o = fmaxf(o, 0.0f);
            }
            if (g.Cf) g.Cf[zoff + (size_t)m * g.ldc + n] = o;
            else g.Cb[(size_t)m * g.ldc + n] = __float2bfloat16_rn(o);
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(BN));
}

template <int BN>
int launch_bn(const GemmArgs &g, cudaStream_t s) {
  const size_t smem = 2 * (size_t)(BM * BK * 2 + BN * BK * 2) + 64;
  if (cudaFuncSetAttribute(gemm_tc_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return NN_ECUDA;
  dim3 grid((g.M + BM - 1) / BM, (g.N + BN - 1) / BN, g.ksplit > 1 ? g.ksplit : 1);
  gemm_tc_kernel<BN><<<grid, kThreads, smem, s>>>(g);
  return cudaGetLastError() == cudaSuccess ? NN_OK : NN_ECUDA;
}

}  // namespace

int gemm_launch(const GemmArgs &g, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0) return NN_EINVAL;
  if (g.K % 8 || (g.mode == GEMM_DENSE && g.lda % 8) || g.ldb % 8) return NN_EINVAL;
  if (g.mode == GEMM_CONV3X3 && (g.Cin % 8 || g.K != 9 * g.Cin || g.M % (g.H * g.W))) return NN_EINVAL;
  if ((g.Cf == nullptr) == (g.Cb == nullptr)) return NN_EINVAL;
  if (g.ksplit > 1 && !g.Cf) return NN_EINVAL;
  // 16-byte cp.async sources: base pointers must be 16-byte aligned
  if (((uintptr_t)g.A | (uintptr_t)g.B) & 15) return NN_EINVAL;
  if (g.N <= 32) return launch_bn<32>(g, s);
  if (g.N <= 64) return launch_bn<64>(g, s);
  if (g.N <= 128) return launch_bn<128>(g, s);
  return launch_bn<256>(g, s);
}

}  // namespace tomo_nn
