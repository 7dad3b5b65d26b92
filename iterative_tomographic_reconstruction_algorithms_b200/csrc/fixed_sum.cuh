// Exact, order-independent sums of float products in 64-bit fixed point.
//
// Forward kernels that splat pixels into bins (B-spline, pixel-driven) add
// each product, as the reference rounds it, into shared-memory bins held as
// signed 64-bit integers in units of 2^-E.  Integer addition is associative,
// so the sums do not depend on the order in which threads add (the result is
// deterministic) and each bin is the exact sum of its products, rounded once
// to float at the end.  E is chosen per slice so that the largest possible
// bin, `bound` = (products reaching one bin) x max |factor| x max |image|,
// stays below 2^61; a product is scaled by 2^E in two exact float steps and
// rounded to the nearest unit (2^-E, far below float resolution of any bin
// that is not 2^-40 of the largest possible one).
#pragma once

#include <cuda_runtime.h>

namespace tomo {
namespace {

// Per slice z (blockIdx.y): out[z] = max |x| as the float's bits (non-negative
// floats order as their bit patterns).  out must be zeroed first.
__global__ void fixed_absmax_kernel(const float *__restrict__ x, size_t per_slice, unsigned *__restrict__ out) {
  const size_t z = blockIdx.y;
  unsigned m = 0u;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < per_slice; i += (size_t)gridDim.x * blockDim.x)
    m = max(m, __float_as_uint(fabsf(__ldg(x + z * per_slice + i))));
  for (int off = 16; off; off >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out + z, m);
}

struct FixedScale {
  int E;
  float s1, s2;  // 2^E = s1 * s2, each a normal float
};

__device__ __forceinline__ FixedScale fixed_scale(double bound) {
  FixedScale f{0, 1.0f, 1.0f};
  if (bound > 0.0) f.E = max(min(61 - (int)ceil(log2(bound)), 250), -126);
  const int e1 = min(f.E, 126);
  f.s1 = ldexpf(1.0f, e1);
  f.s2 = ldexpf(1.0f, f.E - e1);
  return f;
}

__device__ __forceinline__ unsigned long long fixed_of(float p, const FixedScale &f) {
  return (unsigned long long)__float2ll_rn(__fmul_rn(__fmul_rn(p, f.s1), f.s2));
}

// Adds v to the 64-bit shared-memory sum *a with 32-bit atomics: the low word
// first, then (high word of v + the carry out of the low word) to the high
// word, skipped when zero.  After all adds the pair holds the sum mod 2^64
// whatever the order (every carry is counted once).
__device__ __forceinline__ void fixed_add(unsigned long long *a, unsigned long long v) {
  unsigned *w = (unsigned *)a;  // little-endian: w[0] low, w[1] high
  const unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
  const unsigned old = atomicAdd(w, lo);
  const unsigned h = hi + ((unsigned)(old + lo) < old ? 1u : 0u);
  if (h) atomicAdd(w + 1, h);
}

__device__ __forceinline__ float fixed_to_float(unsigned long long a, const FixedScale &f) {
  return (float)ldexp((double)(long long)a, -f.E);
}

// floor(x) for |x| < 2^22 without the conversion pipe: x + 1.5 * 2^23 rounded
// down lies where floats are the integers, so it is 1.5 * 2^23 + floor(x)
// exactly; fl receives floor(x) as a float.
__device__ __forceinline__ int floor_i(float x, float &fl) {
  const float f = __fadd_rd(x, 12582912.0f);
  fl = __fsub_rn(f, 12582912.0f);
  return __float_as_int(f) - 0x4B400000;
}

}  // namespace
}  // namespace tomo
