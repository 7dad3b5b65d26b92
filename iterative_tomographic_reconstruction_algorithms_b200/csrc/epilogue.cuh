// Solver arithmetic fused into the projector kernels.
//
// Forward epilogue (one thread owns one sinogram element e, acc = (A x)[e]):
//   NONE  out = acc
//   SIRT  out = R[e] * (b[e] - acc)                          art.py:212
//   MLEM  out = b[e] / (acc == 0 ? eps32 : acc)              sir.py:270-271
//   SPS   out = (acc - b[e]) * w[e]                          sir.py:438-442
// and, when requested, the squared data residual (acc - b[e])^2 summed per
// warp into a partial-sum slot (reduced in a fixed order afterwards, so the
// residual is deterministic).
//
// Adjoint epilogue (one thread owns one pixel p, acc = (A^T y)[p]):
//   NONE  out = acc
//   SIRT  out = x[p] + C[p] * acc                            art.py:212
//   MLEM  out = x[p] * (invd[p] * acc)                       sir.py:283
//   SPS   out = max(x[p] - acc / (den[p] + eps64), 0)        sir.py:535-540
// The SPS update is evaluated in double, as NumPy evaluates the reference's
// float32 / float64 expression; its clip to [0, max x] equals max(x, 0) unless
// every updated value is negative, which the fix-up kernel handles (the
// epilogue records the maximum and whether any value was >= 0).
// All elementwise arithmetic matches the reference's float32 rounding order.
#pragma once

#include <cuda_runtime.h>

namespace tomo {

enum EpiOp : int { EPI_NONE = 0, EPI_SIRT = 1, EPI_MLEM = 2, EPI_SPS = 3 };

// np.spacing(1) as the reference adds it: to a float32 array (MLEM, stored
// back as float32) or inside a float64 expression (SPS).
constexpr float kSpacing32 = 2.220446049250313e-16f;
constexpr double kSpacing64 = 2.220446049250313e-16;

struct FwdEpi {
  int op = EPI_NONE;
  const float *b = nullptr;  // measured sinogram, same layout as the output
  const float *w = nullptr;  // SIRT: R = 1/(A 1); SPS: w = exp(-b / max b)
  double *resid = nullptr;   // per-warp partial sums of (A x - b)^2, or null
};

struct AdjEpi {
  int op = EPI_NONE;
  const float *x = nullptr;    // current iterate (may alias the output)
  const float *aux = nullptr;  // SIRT: C = 1/(A^T 1); MLEM: 1/(A^T 1); SPS: den
  unsigned *sps_max = nullptr; // SPS: ordered-int maximum of the unclipped update
};

__device__ __forceinline__ unsigned float_to_ordered(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__device__ __forceinline__ size_t global_warp_slot() {
  const size_t block = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const unsigned tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  return block * ((blockDim.x * blockDim.y * blockDim.z) / 32) + tid / 32;
}

// The forward epilogue of sinogram element e; adds (acc - b[e])^2 to r2 when
// residuals are requested.
__device__ __forceinline__ float fwd_apply(const FwdEpi &ep, float acc, size_t e, double &r2) {
  if (ep.op == EPI_NONE) return acc;
  const float bv = __ldg(ep.b + e);
  float o;
  if (ep.op == EPI_SIRT) o = __fmul_rn(__ldg(ep.w + e), __fsub_rn(bv, acc));
  else if (ep.op == EPI_MLEM) o = __fdiv_rn(bv, acc == 0.0f ? kSpacing32 : acc);
  else o = __fmul_rn(__fsub_rn(acc, bv), __ldg(ep.w + e));
  if (ep.resid) {
    const double d = (double)acc - (double)bv;
    r2 += d * d;
  }
  return o;
}

// Warp sum of the lanes' r2 into partial-sum slot `slot` (every lane calls).
__device__ __forceinline__ void fwd_resid_commit(const FwdEpi &ep, double r2, size_t slot) {
  if (!ep.resid) return;
  for (int off = 16; off; off >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, off);
  if ((threadIdx.x & 31) == 0) ep.resid[slot] = r2;
}

// Every lane of the warp must call this (pass live = false for idle lanes).
__device__ __forceinline__ void fwd_store(const FwdEpi &ep, float acc, bool live, size_t e,
                                          float *out) {
  double r2 = 0.0;
  if (live) out[e] = fwd_apply(ep, acc, e, r2);
  fwd_resid_commit(ep, r2, global_warp_slot());
}

// Every lane of the warp must call this (pass live = false for idle lanes).
__device__ __forceinline__ void adj_store(const AdjEpi &ep, float acc, bool live, size_t p,
                                          float *out) {
  if (ep.op == EPI_SPS) {
    float f = -INFINITY;
    if (live) {
      f = (float)((double)ep.x[p] - (double)acc / ((double)__ldg(ep.aux + p) + kSpacing64));
      out[p] = fmaxf(f, 0.0f);
    }
    unsigned u = float_to_ordered(f);
    for (int off = 16; off; off >>= 1) u = max(u, __shfl_down_sync(0xffffffffu, u, off));
    if ((threadIdx.x & 31) == 0) atomicMax(ep.sps_max, u);  // max is order-independent
    return;
  }
  if (!live) return;
  float o = acc;
  if (ep.op == EPI_SIRT) o = __fadd_rn(ep.x[p], __fmul_rn(__ldg(ep.aux + p), acc));
  else if (ep.op == EPI_MLEM) o = __fmul_rn(ep.x[p], __fmul_rn(__ldg(ep.aux + p), acc));
  out[p] = o;
}

}  // namespace tomo
