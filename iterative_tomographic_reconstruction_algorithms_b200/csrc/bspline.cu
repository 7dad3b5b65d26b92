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
// Forward = gather per (angle, bin) over the strip of pixels whose taps can
// reach the bin; adjoint = gather per pixel over angles and taps.  Output rows
// follow the angle order (no reversal).
#include <cmath>

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

__device__ __forceinline__ int bs_lut(int yi, float ps, const BsConst &k) {
  const float y = __fsub_rn((float)yi, k.fmid);
  return (int)__fmul_rn(__fsub_rn(y, ps), k.lut_step) + k.lut_half;
}

__global__ void __launch_bounds__(128) bs_forward_kernel(
    const float *__restrict__ img, float *__restrict__ sino, const float2 *__restrict__ cs,
    const float *__restrict__ lut, BsConst k, FwdEpi ep) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  const size_t z = blockIdx.z;
  const int n = k.n;
  const bool live = b < n;
  const float C = cs[v].x, S = cs[v].y;
  const float *I = img + z * (size_t)n * n;
  const float *L = lut + (size_t)v * k.lut_size;
  const bool by_rows = fabsf(C) >= fabsf(S);  // along a row ps moves by C per pixel
  // taps reach bin b when b <= ps + s + mid < b + 1 (b = 0 also takes (-1, 0))
  const float plo = (float)(b - k.ds - 2) - k.fmid, phi = (float)(b + k.ds + 2) - k.fmid;
  const bool even = (n & 1) == 0 && n >= 4;  // n = 2: the bin-0 boundary sits at 0, use the double rule
  const float bm = (float)b - k.fmid, fds = (float)k.ds;  // b - n/2 (exact for even n)
  const float b0lo = -k.fmid - 1.0f, b0hi = -k.fmid + 1.0f;
  float acc = 0.0f;
  for (int line = 0; line < (live ? n : 0); ++line) {
    // by rows: ky fixed, ps = kx*C + S*ky; by columns: kx fixed, ps = ky*S + kx*C
    const float fixed = by_rows ? (float)(-line + k.mid) : (float)(line - k.mid);
    const float slope = by_rows ? C : S;
    const float base = by_rows ? S * fixed : C * fixed;
    float u0 = (plo - base) / slope, u1 = (phi - base) / slope;
    if (u0 > u1) { float t = u0; u0 = u1; u1 = t; }
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
    for (int j = j0; j <= j1; ++j) {
      const int kyi = by_rows ? line : j, kxi = by_rows ? j : line;
      const float ky = (float)(-kyi + k.mid), kx = (float)(kxi - k.mid);
      const float ps = __fmaf_rn(kx, C, __fmul_rn(S, ky));
      // the tap that lands in bin b: s0 = b - floor(ps + n/2), or a neighbour
      // of it where the rounding of s + ps crosses an integer (or, for bin 0,
      // where truncation folds (-1, 0) onto 0); each is checked with the exact
      // bin rule, so the set of taps is the reference's
      if (even) {
        // n/2 is an integer: trunc((double)fl(s + ps) + n/2) == b reduces to
        // floor(fl(s + ps)) == b - n/2 for b >= 1 and to fl(s + ps) in
        // (-n/2 - 1, -n/2 + 1) for b = 0, exact in float (checked against the
        // double rule on CPU for n = 4..4096, including floats next to integers)
        const float s0 = __fsub_rn(bm, floorf(ps));
        const float slo = fmaxf(__fsub_rn(s0, b == 0 ? 2.0f : 1.0f), -fds), shi = fminf(__fadd_rn(s0, 1.0f), fds);
        if (slo > shi) continue;
        const float val = __ldg(I + (size_t)kyi * n + kxi);
        for (float sf = slo; sf <= shi; sf = __fadd_rn(sf, 1.0f)) {
          const float t = __fadd_rn(sf, ps);
          // (b = n/2: a tiny negative t rounds up to n/2 in the double sum)
          const bool hit = b == 0 ? (t > b0lo && t < b0hi)
                                  : (floorf(t) == bm ||
                                     (bm == 0.0f && t < 0.0f && (int)__dadd_rn((double)t, k.mid) == b));
          if (!hit) continue;
          const int li = bs_lut(b, ps, k);
          if (li >= k.lut_max || li < 0) continue;
          acc = fmaf(__ldg(L + li), val, acc);
        }
        continue;
      }
      const int s0 = b - (int)floor(__dadd_rn((double)ps, k.mid));
      const int slo = max(s0 - (b == 0 ? 2 : 1), -k.ds), shi = min(s0 + 1, k.ds);
      if (slo > shi) continue;
      const float val = __ldg(I + (size_t)kyi * n + kxi);
      for (int s = slo; s <= shi; ++s) {
        const int yi = bs_bin(s, ps, k.mid);
        if (yi != b) continue;
        const int li = bs_lut(yi, ps, k);
        if (li >= k.lut_max || li < 0) continue;
        acc = fmaf(__ldg(L + li), val, acc);
      }
    }
  }
  fwd_store(ep, acc, live, z * (size_t)k.na * n + (size_t)v * n + (live ? b : 0), sino);
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
  p.g.lut = nullptr;
  return TOMO_OK;
}

int bs_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const BsConst k = make_const(p);
  dim3 fb(128), fg((k.n + 127) / 128, k.na, p.g.nz);
  bs_forward_kernel<<<fg, fb, 0, s>>>(d_img, d_sino, (const float2 *)p.d_angles,
                                      (const float *)p.d_aux, k, ep);
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
