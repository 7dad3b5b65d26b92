// Order-independent sums of float products in 64-bit fixed point.
//
// Kernels that splat values into bins (B-spline and pixel-driven forwards)
// add each product, as the reference rounds it, into shared-memory bins held
// as signed 64-bit integers in units of 2^-E.  Integer addition is
// associative, so the sums do not depend on the order in which threads add:
// the result is deterministic.  E is chosen per slice so that the largest
// possible bin, `bound` = (products reaching one bin) x max |factor| x
// max |finite value|, stays below 2^61.  A product is scaled by 2^E in two
// exact float steps and rounded to the nearest unit, so each product is off by
// at most 2^-(E+1) and a bin of k products by at most k 2^-(E+1) <= k bound
// 2^-62: far below float resolution for bins near the bound, but a bin much
// smaller than the bound (a cancelling sum) keeps only the bits above 2^-E.
// The integer sum is rounded to float once (fixed_to_float).
//
// inf and NaN have no integer: a product that is not finite sets a flag of its
// bin instead (nonfinite_flag), and a flagged bin takes the value the
// reference's float sum ends with (nonfinite_value): NaN if a NaN product or
// both infinities reached it, else the infinity that did.  The bound uses the
// finite values only (fixed_finite_absmax_kernel), so the finite bins keep
// their precision.
#pragma once

#include <cuda_runtime.h>

namespace tomo {
namespace {

// Per slice z (blockIdx.y): out[z] = max |x| over the finite x, as the float's
// bits (non-negative floats order as their bit patterns).  out must be zeroed
// first.
__global__ void fixed_finite_absmax_kernel(const float *__restrict__ x, size_t per_slice, unsigned *__restrict__ out) {
  const size_t z = blockIdx.y;
  unsigned m = 0u;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < per_slice; i += (size_t)gridDim.x * blockDim.x) {
    const unsigned b = __float_as_uint(fabsf(__ldg(x + z * per_slice + i)));
    if (b < 0x7f800000u) m = max(m, b);
  }
  for (int off = 16; off; off >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out + z, m);
}

// Flags of a non-finite product c: 1 +inf, 2 -inf, 4 NaN.
constexpr unsigned kFixPosInf = 1u, kFixNegInf = 2u, kFixNaN = 4u;

__device__ __forceinline__ unsigned nonfinite_flag(float c) {
  return c != c ? kFixNaN : (c > 0.0f ? kFixPosInf : kFixNegInf);
}

// The value of a bin with flags f != 0, as a float sum ends: NaN when a NaN
// product or both infinities reached it, else the infinity.
__device__ __forceinline__ float nonfinite_value(unsigned f) {
  if ((f & kFixNaN) || (f & (kFixPosInf | kFixNegInf)) == (kFixPosInf | kFixNegInf))
    return __int_as_float(0x7fffffff);
  return (f & kFixPosInf) ? __int_as_float(0x7f800000) : __int_as_float(0xff800000);
}

struct FixedScale {
  int E;
  float s1, s2;  // 2^E = s1 * s2, each a normal float
  float r1, r2;  // 2^-E = r1 * r2, each a normal float
};

__device__ __forceinline__ FixedScale fixed_scale(double bound) {
  FixedScale f{0, 1.0f, 1.0f, 1.0f, 1.0f};
  if (bound > 0.0) f.E = max(min(61 - (int)ceil(log2(bound)), 250), -126);
  const int e1 = min(f.E, 126);
  f.s1 = ldexpf(1.0f, e1);
  f.s2 = ldexpf(1.0f, f.E - e1);
  f.r1 = ldexpf(1.0f, -e1);
  f.r2 = ldexpf(1.0f, e1 - f.E);
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

// Adds the product p to the bin *a, or, when p is inf or NaN, sets its flag in
// the bin's flag word *fl (shared memory, zeroed with the bins).
__device__ __forceinline__ void fixed_add_product(unsigned long long *a, unsigned *fl, float p, const FixedScale &f) {
  if (__float_as_uint(fabsf(p)) < 0x7f800000u) fixed_add(a, fixed_of(p, f));
  else atomicOr(fl, nonfinite_flag(p));
}

// The integer rounded to float once (round to nearest even), then scaled by
// the two powers of two, which is exact unless the result is subnormal.
__device__ __forceinline__ float fixed_to_float(unsigned long long a, const FixedScale &f) {
  return __fmul_rn(__fmul_rn(__ll2float_rn((long long)a), f.r1), f.r2);
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
