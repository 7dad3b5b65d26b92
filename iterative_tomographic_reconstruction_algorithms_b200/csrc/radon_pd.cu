// Pixel-driven projector pair (linear interpolation, method 1) for sm_100a.
//
// Reference: common/operators/radon_module/pymodule_radon_pixel_driven/
// radon_pd.c:20-90.  Every pixel (i, j) -- stored at image row n-1-i
// (:61) -- is represented by four sub-samples; the reference offsets x and y by
// the SAME delta[2k+1] (:42-43), so the four are (-1/4,-1/4) twice and
// (+1/4,+1/4) twice.  A sub-sample lands at T = nh - t, t = +-|x s - y c| with
// the sign rule of :46-55, and is split linearly between bins floor(T) and
// ceil(T) with weights |ceil(T) - T| and |T - floor(T)|; bin 0 never receives
// (:74,76) and an integral T gets weight 0 in both.  Output row v follows the
// (fftshifted) angle order of the input.
//
// Evaluation order of the compiled reference (-O3 -ffast-math, read from its
// x86-64 code), reproduced exactly: t = |fma(-c, y, x*s)|, the sign test uses
// (x*s) * (1/c), and the first weight is |(t + ceil(T)) - nh|.
//
// Forward = per (angle, block of bins) a pass over the band of pixels whose
// sub-samples land in the bins, summed in fixed point; adjoint =
// gather per pixel over angles.  The duplicate sub-samples are evaluated once
// with weight 2 * 1/4.
#include <algorithm>
#include <cmath>

#include "fixed_sum.cuh"
#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr double kPi = 3.141592653589793;
constexpr float kPdMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kPdMagicBits = 0x4B400000;  // its bit pattern

struct PdEval {
  float wl, wu;  // weights of bins l = floor(T), u = ceil(T)
  int l, u;      // -1 when the reference's bound test (0 < bin < n) fails
};

__device__ __forceinline__ PdEval pd_eval(float x, float y, const PdAngle &g, float fnh, int n) {
  const float xs = __fmul_rn(x, g.s);
  const float t = fabsf(__fmaf_rn(-g.c, y, xs));
  const float r = __fmul_rn(xs, g.rc);
  const bool keep = ((g.flags & 1) && y > r) || ((g.flags & 2) && y > r) || ((g.flags & 4) && y > 0.0f);
  const float ts = keep ? t : -t;
  const float T = __fsub_rn(fnh, ts);
  // floor and ceil of T without the conversion pipe: T + 1.5 * 2^23 rounded
  // down / up lies where floats are the integers (|T| < 2^22), so it is
  // 1.5 * 2^23 + floor(T) / ceil(T) exactly, and its bits give the integer
  const float fd = __fadd_rd(T, kPdMagic), fu = __fadd_ru(T, kPdMagic);
  const float lf = __fsub_rn(fd, kPdMagic), uf = __fsub_rn(fu, kPdMagic);
  PdEval e;
  e.wl = fabsf(__fsub_rn(__fadd_rn(ts, uf), fnh));
  e.wu = fabsf(__fsub_rn(T, lf));
  e.l = (lf >= 1.0f && lf < (float)n) ? __float_as_int(fd) - kPdMagicBits : -1;
  e.u = (uf >= 1.0f && uf < (float)n) ? __float_as_int(fu) - kPdMagicBits : -1;
  return e;
}

// Forward: a block owns kPdBins consecutive bins of one angle and slice; its
// warps walk the band of pixels whose sub-samples can land in (B0 - 1, Bend)
// (a line per warp, each pixel once, along the axis on which T moves fastest)
// and add 0.5 w value for every sub-sample and bin into shared-memory bins
// summed in fixed point (fixed_sum.cuh): deterministic, each bin the sum of
// its float products to within the fixed-point unit, rounded once.  Per line and sub-sample at
// most 3 pixels reach a bin (T moves by at least 1/sqrt(2) per pixel), so a
// bin is bounded by 2 (sub-samples) x 3 n x 0.5 x max|finite image value|;
// inf and NaN products flag their bins instead (fixed_sum.cuh).
constexpr int kPdBins = 128, kPdThreads = 256;

__global__ void __launch_bounds__(kPdThreads) pd_forward_kernel(
    const float *__restrict__ img, float *__restrict__ sino, const PdAngle *__restrict__ tab,
    int n, int nh, int na, const unsigned *__restrict__ vmax, FwdEpi ep) {
  __shared__ unsigned long long acc[kPdBins];
  __shared__ unsigned flg[kPdBins];  // non-finite products per bin (fixed_sum.cuh)
  const int B0 = blockIdx.x * kPdBins, v = blockIdx.y;
  const size_t z = blockIdx.z;
  for (int i = threadIdx.x; i < kPdBins; i += blockDim.x) {
    acc[i] = 0ull;
    flg[i] = 0u;
  }
  const FixedScale fs = fixed_scale(3.0 * n * (double)__uint_as_float(vmax[z]));
  __syncthreads();
  const PdAngle g = tab[v];
  const float *I = img + z * (size_t)n * n;
  const float fnh = (float)nh;
  const int Bend = min(B0 + kPdBins, n);
  // T ~ nh - sigma*((y0+d) c - (x0+d) s), sigma = sign(c)
  const float sg = g.c >= 0.0f ? 1.0f : -1.0f;
  const bool by_rows = fabsf(g.s) >= fabsf(g.c);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int line = warp; line < n; line += kPdThreads / 32) {
    const float o0 = (float)line - fnh + 0.5f;  // y0 (rows) or x0 (columns)
    float lo = 1e30f, hi = -1e30f;
    for (int e = 0; e < 2; ++e) {
      const float d = e ? 0.25f : -0.25f;
      for (int f = 0; f < 2; ++f) {
        const float T = (float)(f ? Bend : B0 - 1);
        float w;  // the other pixel-centre coordinate giving this T
        if (by_rows) w = (T - fnh + sg * ((o0 + d) * g.c)) / (sg * g.s) - d;
        else w = (fnh - T + sg * ((o0 + d) * g.s)) / (sg * g.c) - d;
        lo = fminf(lo, w);
        hi = fmaxf(hi, w);
      }
    }
    int j0 = (int)floorf(lo + fnh - 0.5f) - 1, j1 = (int)ceilf(hi + fnh - 0.5f) + 1;
    j0 = max(j0, 0);
    j1 = min(j1, n - 1);
    for (int j = j0 + lane; j <= j1; j += 32) {
      const int ii = by_rows ? line : j, jj = by_rows ? j : line;
      const float val = __ldg(I + (size_t)(n - 1 - ii) * n + jj);
      if (val == 0.0f) continue;  // adds exactly nothing
      const float x0 = (float)jj - fnh + 0.5f, y0 = (float)ii - fnh + 0.5f;
      for (int e = 0; e < 2; ++e) {
        const float d = e ? 0.25f : -0.25f;
        const PdEval q = pd_eval(__fadd_rn(x0, d), __fadd_rn(y0, d), g, fnh, n);
        if (q.l >= B0 && q.l < Bend) fixed_add_product(acc + (q.l - B0), flg + (q.l - B0), __fmul_rn(0.5f * q.wl, val), fs);
        if (q.u >= B0 && q.u < Bend) fixed_add_product(acc + (q.u - B0), flg + (q.u - B0), __fmul_rn(0.5f * q.wu, val), fs);
      }
    }
  }
  __syncthreads();
  const int b = B0 + (int)threadIdx.x;
  const bool live = threadIdx.x < kPdBins && b < n;
  float out = 0.0f;
  if (live) out = flg[threadIdx.x] ? nonfinite_value(flg[threadIdx.x]) : fixed_to_float(acc[threadIdx.x], fs);
  fwd_store(ep, out, live, z * (size_t)na * n + (size_t)v * n + (live ? b : 0), sino);
}

constexpr int kPdChunk = 1024;

// Adjoint: thread per output pixel (memory row R, column j); the reference's
// loop row is i = n-1-R.
__global__ void __launch_bounds__(256) pd_adjoint_kernel(
    const float *__restrict__ sino, float *__restrict__ img, const PdAngle *__restrict__ tab,
    int n, int nh, int na, AdjEpi ep) {
  __shared__ PdAngle stab[kPdChunk];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int R = blockIdx.y * blockDim.y + threadIdx.y;
  const size_t z = blockIdx.z;
  const bool live = R < n && j < n;
  const float *S = sino + z * (size_t)na * n;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
  const float fnh = (float)nh;
  const int i = n - 1 - R;
  const float x0 = (float)j - fnh + 0.5f, y0 = (float)i - fnh + 0.5f;
  float acc = 0.0f;
  for (int v0 = 0; v0 < na; v0 += kPdChunk) {
    const int cnt = min(kPdChunk, na - v0);
    __syncthreads();
    for (int t = tid; t < cnt; t += nthr) stab[t] = tab[v0 + t];
    __syncthreads();
    if (!live) continue;
    for (int u = 0; u < cnt; ++u) {
      const PdAngle g = stab[u];
      const float *row = S + (size_t)(v0 + u) * n;
      for (int e = 0; e < 2; ++e) {
        const float d = e ? 0.25f : -0.25f;
        const PdEval q = pd_eval(__fadd_rn(x0, d), __fadd_rn(y0, d), g, fnh, n);
        if (q.l >= 0) acc = fmaf(0.5f * q.wl, __ldg(row + q.l), acc);
        if (q.u >= 0) acc = fmaf(0.5f * q.wu, __ldg(row + q.u), acc);
      }
    }
  }
  adj_store(ep, acc, live, z * (size_t)n * n + (size_t)(live ? R : 0) * n + (live ? j : 0), img);
}

}  // namespace

int pd_setup(Plan &p) {
  const int na = p.g.na;
  std::vector<PdAngle> tab(na);
  for (int v = 0; v < na; ++v) {
    const float theta = p.angles[v];
    float s, c;
    sincosf(theta, &s, &c);
    PdAngle a{};
    a.s = s;
    a.c = c;
    a.rc = 1.0f / c;
    a.flags = ((double)theta < kPi / 2 ? 1 : 0) | ((double)theta > kPi / 2 ? 2 : 0) |
              (theta == 0.0f ? 4 : 0);
    tab[v] = a;
  }
  TOMO_CUDA(cudaMalloc(&p.d_angles, sizeof(PdAngle) * (size_t)na));
  TOMO_CUDA(cudaMemcpy(p.d_angles, tab.data(), sizeof(PdAngle) * (size_t)na, cudaMemcpyHostToDevice));
  // per-slice max |finite image value| of the forward's fixed-point sums
  TOMO_CUDA(cudaMalloc(&p.ext, sizeof(unsigned) * (size_t)std::max(1, p.g.nz)));
  p.ext_free = [](void *q) { cudaFree(q); };
  // residual partials of the fused solvers: one per warp of the forward launch
  p.fwd_warps = (size_t)((p.g.n + kPdBins - 1) / kPdBins) * (kPdThreads / 32) * na * p.g.nz;
  return TOMO_OK;
}

int pd_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz;
  unsigned *vmax = (unsigned *)p.ext;
  const size_t per = (size_t)n * n;
  TOMO_CUDA(cudaMemsetAsync(vmax, 0, sizeof(unsigned) * nz, s));
  fixed_finite_absmax_kernel<<<dim3((unsigned)std::min<size_t>((per + 255) / 256, 1184), nz), 256, 0, s>>>(d_img, per, vmax);
  dim3 fg((n + kPdBins - 1) / kPdBins, na, nz);
  pd_forward_kernel<<<fg, kPdThreads, 0, s>>>(d_img, d_sino, (const PdAngle *)p.d_angles, n, p.nh, na, vmax, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int pd_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s, const AdjEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz;
  dim3 ab(32, 8), ag((n + 31) / 32, (n + 7) / 8, nz);
  pd_adjoint_kernel<<<ag, ab, 0, s>>>(d_sino, d_img, (const PdAngle *)p.d_angles, n, p.nh, na, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
