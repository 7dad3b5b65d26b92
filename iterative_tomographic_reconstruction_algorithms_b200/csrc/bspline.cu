// Generalised (B-spline) Radon projector pair for sm_100a.
//
// Reference: common/operators/bspline_module/pymodule_genradon/gen_forwproj.c
// :22-78 and gen_backproj.c:22-74.  For every angle (degrees, converted as
// theta = (float)(deg * pi/180)), pixel (ky_i, kx_i) with kx = kx_i - n/2 and
// ky = n/2 - ky_i, the projection ps = cos*kx + sin*ky (compiled as
// fma(kx, cos, sin*ky)) feeds 2*ds+1 detector taps s = -ds..ds:
//   bin  yi = trunc((double)((float)s + ps) + n/2)         (C truncation),
//   lut  li = trunc((yi - n/2 - ps) * lut_step) + lut_size/2,
// skipped unless 0 <= yi < n and 0 <= li < lut_size - 1; the weight is
// lut[angle][li].  ds = (int)(support/2 + 0.5), lut_step = (lut_size/2) /
// (support/2).  The table itself is built on the host (bspline_functions.py).
//
// Forward = per (angle, block of bins) a pass over the band of pixels whose
// taps can reach the bins, summed in fixed point; adjoint = gather
// per pixel over angles and taps.  Output rows follow the angle order (no
// reversal).
#include <algorithm>
#include <cmath>

#include "fixed_sum.cuh"
#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr double kPi = 3.141592653589793;

struct BsConst {
  int n, na, lut_size, lut_half, lut_max, ds;
  float lut_step, fmid;
  double mid;
};

__device__ __forceinline__ int bs_bin(int s, float ps, double mid) {
  return (int)__dadd_rn((double)__fadd_rn((float)s, ps), mid);  // trunc toward zero
}


// Forward: a block owns kBsBins consecutive bins of one angle and slice.  Its
// warps walk the band of pixels whose taps can reach those bins (a line per
// warp, each pixel once) and add every tap's product lut * value, as the
// reference rounds it, into shared-memory bins summed in fixed point
// (fixed_sum.cuh): deterministic, each bin the sum of the reference's float
// products to within the fixed-point unit, rounded once.  At most 3 pixels per line and tap reach a bin
// (ps moves by at least 1/sqrt(2) per pixel), which bounds the sums.
constexpr int kBsBins = 128, kBsThreads = 256;


// LUT index trunc((yi - n/2 - ps) * lut_step) + lut_size/2 (gen_forwproj.c:61).
__device__ __forceinline__ int bs_lut(int yi, float ps, const BsConst &k) {
  const float y = __fsub_rn((float)yi, k.fmid);
  return (int)__fmul_rn(__fsub_rn(y, ps), k.lut_step) + k.lut_half;
}

// The same index with the truncation toward zero taken without the
// conversion pipe (the forward's inner loop is conversion-bound).
__device__ __forceinline__ int bs_lut_fast(int yi, float ps, const BsConst &k) {
  const float a = __fmul_rn(__fsub_rn(__fsub_rn((float)yi, k.fmid), ps), k.lut_step);
  float fl;
  const int t = floor_i(fabsf(a), fl);
  return (a < 0.0f ? -t : t) + k.lut_half;
}

// bs_bin for even n >= 4 without the conversion pipe: n/2 is an integer, so
// trunc((double)t + n/2) == floor(t) + n/2, except that t in (-n/2 - 1, -n/2)
// truncates to bin 0 and a tiny negative t may round up to n/2 in the double
// sum (t in (-1, 0) takes the double rule).  Odd n: the double rule.
__device__ __forceinline__ int bs_bin_fast(int s, float ps, const BsConst &k, bool even, int nh, float b0lo) {
  const float t = __fadd_rn((float)s, ps);
  if (even && !(t < 0.0f && t > -1.0f)) {
    float fl;
    int yi = floor_i(t, fl) + nh;
    if (yi == -1 && t > b0lo) yi = 0;
    return yi;
  }
  return bs_bin(s, ps, k.mid);
}


__global__ void __launch_bounds__(kBsThreads) bs_forward_kernel(
    const float *__restrict__ img, float *__restrict__ sino, const float2 *__restrict__ cs,
    const float *__restrict__ lut, const unsigned *__restrict__ vmax, float lutmax, BsConst k, FwdEpi ep) {
  extern __shared__ float slut[];  // this angle's lut row
  __shared__ unsigned long long acc[kBsBins];
  __shared__ unsigned flg[kBsBins];  // non-finite products per bin (fixed_sum.cuh)
  const int B0 = blockIdx.x * kBsBins, v = blockIdx.y;
  const size_t z = blockIdx.z;
  const int n = k.n;
  const float *L = lut + (size_t)v * k.lut_size;
  for (int i = threadIdx.x; i < k.lut_size; i += blockDim.x) slut[i] = __ldg(L + i);
  for (int i = threadIdx.x; i < kBsBins; i += blockDim.x) {
    acc[i] = 0ull;
    flg[i] = 0u;
  }
  // fixed-point unit: |bin| <= 3 n (2 ds + 1) max|lut| max|finite value|
  const float vm = __uint_as_float(vmax[z]);
  const FixedScale fs = fixed_scale(3.0 * n * (2.0 * k.ds + 1.0) * (double)lutmax * (double)vm);
  __syncthreads();
  const float C = cs[v].x, S = cs[v].y;
  const float *I = img + z * (size_t)n * n;
  const bool by_rows = fabsf(C) >= fabsf(S);  // along a row ps moves by C per pixel
  const int Bend = min(B0 + kBsBins, n);
  const float plo = (float)(B0 - k.ds - 2) - k.fmid, phi = (float)(Bend - 1 + k.ds + 2) - k.fmid;
  const bool even = (n & 1) == 0 && n >= 4;  // n = 2: the bin-0 boundary sits at 0, use the double rule
  const float b0lo = -k.fmid - 1.0f;
  const int nh = n / 2;
  // each warp takes every 8th line, its lanes the line's band of pixels
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int line = warp; line < n; line += kBsThreads / 32) {
    // by rows: ky fixed, ps = kx*C + S*ky; by columns: kx fixed, ps = ky*S + kx*C
    const float fixed = by_rows ? (float)(-line + k.mid) : (float)(line - k.mid);
    const float slope = by_rows ? C : S;
    const float base = by_rows ? S * fixed : C * fixed;
    float u0 = (plo - base) / slope, u1 = (phi - base) / slope;
    if (u0 > u1) { const float t = u0; u0 = u1; u1 = t; }
    int j0, j1;
    if (by_rows) {  // kx = kx_i - mid
      j0 = (int)floorf(u0 + k.fmid) - 1;
      j1 = (int)ceilf(u1 + k.fmid) + 1;
    } else {        // ky = mid - ky_i
      j0 = (int)floorf(k.fmid - u1) - 1;
      j1 = (int)ceilf(k.fmid - u0) + 1;
    }
    j0 = max(j0, 0);
    j1 = min(j1, n - 1);
    for (int j = j0 + lane; j <= j1; j += 32) {
      const int kyi = by_rows ? line : j, kxi = by_rows ? j : line;
      const float val = __ldg(I + (size_t)kyi * n + kxi);
      if (val == 0.0f) continue;  // adds exactly nothing
      const float ky = (float)(-kyi + k.mid), kx = (float)(kxi - k.mid);
      const float ps = __fmaf_rn(kx, C, __fmul_rn(S, ky));
      for (int s = -k.ds; s <= k.ds; ++s) {
        const int yi = bs_bin_fast(s, ps, k, even, nh, b0lo);
        if (yi < B0 || yi >= Bend) continue;
        const int li = bs_lut_fast(yi, ps, k);
        if (li >= k.lut_max || li < 0) continue;
        fixed_add_product(acc + (yi - B0), flg + (yi - B0), __fmul_rn(slut[li], val), fs);
      }
    }
  }
  __syncthreads();
  const int b = B0 + (int)threadIdx.x;
  const bool live = threadIdx.x < kBsBins && b < n;
  float out = 0.0f;
  if (live) out = flg[threadIdx.x] ? nonfinite_value(flg[threadIdx.x]) : fixed_to_float(acc[threadIdx.x], fs);
  fwd_store(ep, out, live, z * (size_t)k.na * n + (size_t)v * n + (live ? b : 0), sino);
}

constexpr int kBsChunk = 1024;

__global__ void __launch_bounds__(256) bs_adjoint_kernel(
    const float *__restrict__ sino, float *__restrict__ img, const float2 *__restrict__ cs,
    const float *__restrict__ lut, BsConst k, AdjEpi ep) {
  __shared__ float2 scs[kBsChunk];
  const int n = k.n;
  const int kxi = blockIdx.x * blockDim.x + threadIdx.x;
  const int kyi = blockIdx.y * blockDim.y + threadIdx.y;
  const size_t z = blockIdx.z;
  const bool live = kxi < n && kyi < n;
  const float *Sg = sino + z * (size_t)k.na * n;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
  const float ky = (float)(-kyi + k.mid), kx = (float)(kxi - k.mid);
  const bool even = (n & 1) == 0 && n >= 4;
  const int nh = n / 2;
  float acc = 0.0f;
  for (int v0 = 0; v0 < k.na; v0 += kBsChunk) {
    const int cnt = min(kBsChunk, k.na - v0);
    __syncthreads();
    for (int t = tid; t < cnt; t += nthr) scs[t] = cs[v0 + t];
    __syncthreads();
    if (!live) continue;
    for (int u = 0; u < cnt; ++u) {
      const int v = v0 + u;
      const float ps = __fmaf_rn(kx, scs[u].x, __fmul_rn(scs[u].y, ky));
      const float *row = Sg + (size_t)v * n;
      const float *L = lut + (size_t)v * k.lut_size;
      float fl;
      const int base = floor_i(ps, fl);
      const float frac = __fsub_rn(ps, fl);
      if (even && frac >= 0x1p-12f && frac <= 1.0f - 0x1p-12f) {
        // ps is at least 2^-12 from an integer, so fl(s + ps) never rounds
        // across one: every tap's bin is floor(ps) + s + n/2, with the
        // reference's truncation folding -1 onto bin 0 (t in (-n/2 - 1, -n/2))
        for (int s = -k.ds; s <= k.ds; ++s) {
          int yi = base + s + nh;
          if (yi == -1) yi = 0;
          if (yi >= n || yi < 0) continue;
          const int li = bs_lut(yi, ps, k);
          if (li >= k.lut_max || li < 0) continue;
          acc = fmaf(__ldg(row + yi), __ldg(L + li), acc);
        }
        continue;
      }
      for (int s = -k.ds; s <= k.ds; ++s) {
        const int yi = bs_bin(s, ps, k.mid);
        if (yi >= n || yi < 0) continue;
        const int li = bs_lut(yi, ps, k);
        if (li >= k.lut_max || li < 0) continue;
        acc = fmaf(__ldg(row + yi), __ldg(L + li), acc);
      }
    }
  }
  adj_store(ep, acc, live, z * (size_t)n * n + (size_t)(live ? kyi : 0) * n + (live ? kxi : 0), img);
}

BsConst make_const(const Plan &p) {
  BsConst k{};
  k.n = p.g.n;
  k.na = p.g.na;
  k.lut_size = p.g.lut_size;
  k.lut_half = p.g.lut_size / 2;
  k.lut_max = p.g.lut_size - 1;
  k.ds = (int)(0.5 * (double)p.g.support + 0.5);
  k.lut_step = (float)((p.g.lut_size * 0.5) / ((double)p.g.support * 0.5));
  k.mid = 0.5 * p.g.n;
  k.fmid = (float)k.mid;
  return k;
}

struct BsState {
  float lutmax = 0.0f;        // max |lut|
  unsigned *vmax = nullptr;   // per slice: max |image| as float bits
};

void bs_state_free(void *q) {
  auto *st = (BsState *)q;
  cudaFree(st->vmax);
  delete st;
}

}  // namespace

int bs_setup(Plan &p) {
  const int na = p.g.na;
  if (!p.g.lut || p.g.lut_size < 2)
    return fail(TOMO_EINVAL, "bspline: lut and lut_size >= 2 are required");
  if (!(p.g.support > 0.0f) || p.g.support > 64.0f)
    return fail(TOMO_EINVAL, "bspline: support must be in (0, 64]");
  std::vector<float2> tab(na);
  for (int v = 0; v < na; ++v) {
    const float theta = (float)((double)p.angles[v] * (kPi / 180.0));  // gen_forwproj.c:43
    float s, c;
    sincosf(theta, &s, &c);
    tab[v] = make_float2(c, s);
  }
  TOMO_CUDA(cudaMalloc(&p.d_angles, sizeof(float2) * (size_t)na));
  TOMO_CUDA(cudaMemcpy(p.d_angles, tab.data(), sizeof(float2) * (size_t)na, cudaMemcpyHostToDevice));
  const size_t lb = sizeof(float) * (size_t)na * p.g.lut_size;
  TOMO_CUDA(cudaMalloc(&p.d_aux, lb));
  TOMO_CUDA(cudaMemcpy(p.d_aux, p.g.lut, lb, cudaMemcpyHostToDevice));
  if (sizeof(float) * (size_t)p.g.lut_size > 200 * 1024)
    return fail(TOMO_EINVAL, "bspline: lut_size too large (one row must fit in shared memory)");
  auto *st = new BsState();
  p.ext = st;
  p.ext_free = bs_state_free;
  for (size_t i = 0; i < (size_t)na * p.g.lut_size; ++i) st->lutmax = std::max(st->lutmax, std::fabs(p.g.lut[i]));
  TOMO_CUDA(cudaMalloc(&st->vmax, sizeof(unsigned) * (size_t)std::max(1, p.g.nz)));
  if (sizeof(float) * (size_t)p.g.lut_size > 48 * 1024)
    TOMO_CUDA(cudaFuncSetAttribute(bs_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(float) * (size_t)p.g.lut_size)));
  // residual partials of the fused solvers: one per warp of the forward launch
  p.fwd_warps = (size_t)((p.g.n + kBsBins - 1) / kBsBins) * (kBsThreads / 32) * na * p.g.nz;
  p.g.lut = nullptr;
  return TOMO_OK;
}

int bs_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const BsConst k = make_const(p);
  BsState &st = *(BsState *)p.ext;
  const size_t per = (size_t)k.n * k.n;
  TOMO_CUDA(cudaMemsetAsync(st.vmax, 0, sizeof(unsigned) * p.g.nz, s));
  fixed_finite_absmax_kernel<<<dim3((unsigned)std::min<size_t>((per + 255) / 256, 1184), p.g.nz), 256, 0, s>>>(d_img, per,
                                                                                                   st.vmax);
  dim3 fg((k.n + kBsBins - 1) / kBsBins, k.na, p.g.nz);
  bs_forward_kernel<<<fg, kBsThreads, sizeof(float) * k.lut_size, s>>>(
      d_img, d_sino, (const float2 *)p.d_angles, (const float *)p.d_aux, st.vmax, st.lutmax, k, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int bs_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s, const AdjEpi &ep) {
  const BsConst k = make_const(p);
  dim3 ab(32, 8), ag((k.n + 31) / 32, (k.n + 7) / 8, p.g.nz);
  bs_adjoint_kernel<<<ag, ab, 0, s>>>(d_sino, d_img, (const float2 *)p.d_angles,
                                      (const float *)p.d_aux, k, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
