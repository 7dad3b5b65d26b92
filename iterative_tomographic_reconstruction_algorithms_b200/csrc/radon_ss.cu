// Slant-stacking projector pair (linear interpolation) for sm_100a.
//
// Reference: common/operators/radon_module/pymodule_radon_slant_stacking/
// radon_ss.c:93-196 (method 1) with ray_limits :43-88.  For each angle and
// detector offset t in [-nh, nh) the reference steps along the major axis of
// the ray -- y when |sin| <= sqrt(1/2), else x -- over the integer range
// [round(lim_lo), round(lim_hi)) that ray_limits returns, interpolates the
// image linearly across the minor axis and weights by 1/|cos| or 1/|sin|.
// The output row is na - 1 - v.
//
// Evaluation order of the compiled reference (-O3 -ffast-math, read from its
// x86-64 code): minor coordinate f = fma(-m, s, t) * (1/c) (or fma(-m, c, t) *
// (1/s)), weights w = f - floor(f) and (floor(f) + 1) - f, limits
// fma(nh, s, t) / c etc. sorted.  The loop bounds are precomputed per (angle,
// t) on the host in that exact arithmetic (ss_setup) and shared by both
// kernels.
//
// Rays that miss the square [-nh, nh-1]^2 (possible only within about 1/nh
// radian of 180 degrees) make the reference index outside the image; here
// those rows are skipped.
#include <algorithm>
#include <cmath>

#include "fixed_sum.cuh"
#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr double kS45 = 0.70710678118654757;

__global__ void ss_transpose_kernel(const float *__restrict__ in, float *__restrict__ out, int n) {
  __shared__ float tile[32][33];
  const size_t stride = (size_t)n * n;
  const float *src = in + (size_t)blockIdx.z * stride;
  float *dst = out + (size_t)blockIdx.z * stride;
  int x = blockIdx.x * 32 + threadIdx.x;
  int y0 = blockIdx.y * 32;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    int y = y0 + dy;
    if (x < n && y < n) tile[dy][threadIdx.x] = src[(size_t)y * n + x];
  }
  __syncthreads();
  int ox = blockIdx.y * 32 + threadIdx.x;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    int oy = blockIdx.x * 32 + dy;
    if (ox < n && oy < n) dst[(size_t)oy * n + ox] = tile[threadIdx.x][dy];
  }
}

// Forward: one thread per (t, angle, slice).  For the steep branch the minor
// axis is x (row mm, columns q, q+1 of the image); otherwise the minor axis is
// y (rows q, q+1 of column mm), read from the transposed image so that
// neighbouring threads read neighbouring words.
__global__ void __launch_bounds__(128) ss_forward_kernel(
    const float *__restrict__ img, const float *__restrict__ imgT, float *__restrict__ sino,
    const SsAngle *__restrict__ tab, const int2 *__restrict__ lim, int n, int nh, int na, FwdEpi ep) {
  const int kt = blockIdx.x * blockDim.x + threadIdx.x;  // t + nh
  const int v = blockIdx.y;
  const size_t z = blockIdx.z;
  const bool live = kt < n;  // kt == 2nh (odd n) is never reached by a ray: stays 0
  const SsAngle g = tab[v];
  const int2 L = kt < 2 * nh ? lim[(size_t)v * (2 * nh) + kt] : make_int2(0, 0);
  const float ft = (float)(kt - nh);
  const float *M = (g.steep ? img : imgT) + z * (size_t)n * n;
  float acc = 0.0f;
  for (int m = L.x; m < L.y; ++m) {
    const int mm = m + nh;
    if (mm < 0 || mm > n - 1) continue;
    const float f = __fmul_rn(__fmaf_rn(-(float)m, g.a, ft), g.rb);
    float fl;
    const int q = floor_i(f, fl) + nh;
    const float w = __fsub_rn(f, fl), w1 = __fsub_rn(__fadd_rn(fl, 1.0f), f);
    const float *row = M + (size_t)mm * n;
    if (q >= 0 && q <= n - 1) acc = fmaf(g.wt * w1, __ldg(row + q), acc);
    if (q + 1 >= 0 && q + 1 <= n - 1) acc = fmaf(g.wt * w, __ldg(row + q + 1), acc);
  }
  fwd_store(ep, acc, live, z * (size_t)na * n + (size_t)g.out_row * n + (live ? kt : 0), sino);
}

// Adjoint: a thread holds 4 x 4 output pixels (rows R0..R0+3, columns
// C0..C0+3), all angles in order.  For an angle the pixels fall into 4
// groups of 4 along the minor axis (a row of the block for steep angles, a
// column otherwise); the rays that touch a pixel are those whose minor
// coordinate lands in [minor - 1, minor + 1) at the pixel's major coordinate,
// so a group's candidate rays are the integers t of one short interval (at
// most 7: |rb| >= 1), each checked once with the forward arithmetic and
// credited to the one or two pixels of the group it reaches.  Each pixel gets
// the credits of its rays in the order t ascending, angle after angle, as a
// thread per pixel would give them.
constexpr int kSsChunk = 512;
constexpr int kSsPix = 4;  // pixels per thread along each axis

// The credits of angle g to the group of pixels with major coordinate m and
// minor indices minor0 .. minor0 + 3 (a0 .. a3 the pixels at minor0 + 0 .. 3).
__device__ __forceinline__ void ss_adj_group(const SsAngle &g, float cb, int m, int minor0, int nh,
                                             const float *__restrict__ row, const int2 *__restrict__ lrow,
                                             float &a0, float &a1, float &a2, float &a3) {
  // f(t) = fma(-m, a, t) * rb ~ (t - m a) rb must land in [minor0 - nh - 1,
  // minor0 + 3 - nh + 1): t in [ta, tb] up to rounding (below 1e-3 here), so
  // the integers in [ta - 0.01, tb + 0.01] are the candidates
  const float ma = (float)m * g.a;
  const float lo = (float)(minor0 - nh - 1), hi = (float)(minor0 + kSsPix - nh);
  float ta = fmaf(lo, cb, ma), tb = fmaf(hi, cb, ma);
  if (ta > tb) {
    const float x = ta;
    ta = tb;
    tb = x;
  }
  float fl0, fl1;
  const int t0 = max(floor_i(ta - 0.01f, fl0) + 1, -nh), t1 = min(floor_i(tb + 0.01f, fl1), nh - 1);
  for (int t = t0; t <= t1; ++t) {
    const int2 L = __ldg(lrow + t + nh);
    if (m < L.x || m >= L.y) continue;
    const float f = __fmul_rn(__fmaf_rn(-(float)m, g.a, (float)t), g.rb);
    float fl;
    const int d = floor_i(f, fl) + nh - minor0;  // the ray's left pixel, relative to minor0
    if (d < -1 || d >= kSsPix) continue;
    const float y = __ldg(row + t + nh);
    const float c1 = __fmul_rn(g.wt, __fsub_rn(__fadd_rn(fl, 1.0f), f));  // to pixel d
    const float c0 = __fmul_rn(g.wt, __fsub_rn(f, fl));                     // to pixel d + 1
    if (d == 0) a0 = fmaf(c1, y, a0);
    if (d == -1) a0 = fmaf(c0, y, a0);
    if (d == 1) a1 = fmaf(c1, y, a1);
    if (d == 0) a1 = fmaf(c0, y, a1);
    if (d == 2) a2 = fmaf(c1, y, a2);
    if (d == 1) a2 = fmaf(c0, y, a2);
    if (d == 3) a3 = fmaf(c1, y, a3);
    if (d == 2) a3 = fmaf(c0, y, a3);
  }
}

__global__ void __launch_bounds__(256) ss_adjoint_kernel(
    const float *__restrict__ sino, float *__restrict__ img, const SsAngle *__restrict__ tab,
    const int2 *__restrict__ lim, int n, int nh, int na, AdjEpi ep) {
  __shared__ SsAngle stab[kSsChunk];
  __shared__ float cbs[kSsChunk];  // 1 / rb (cos or sin)
  const int C0 = (blockIdx.x * blockDim.x + threadIdx.x) * kSsPix;
  const int R0 = (blockIdx.y * blockDim.y + threadIdx.y) * kSsPix;
  const size_t z = blockIdx.z;
  const float *S = sino + z * (size_t)na * n;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
  const int nt = 2 * nh;
  float acc[kSsPix][kSsPix];
#pragma unroll
  for (int i = 0; i < kSsPix; ++i)
#pragma unroll
    for (int j = 0; j < kSsPix; ++j) acc[i][j] = 0.0f;
  for (int v0 = 0; v0 < na; v0 += kSsChunk) {
    const int cnt = min(kSsChunk, na - v0);
    __syncthreads();
    for (int t = tid; t < cnt; t += nthr) {
      stab[t] = tab[v0 + t];
      cbs[t] = 1.0f / tab[v0 + t].rb;
    }
    __syncthreads();
    if (R0 >= n || C0 >= n) continue;
    for (int u = 0; u < cnt; ++u) {
      const SsAngle g = stab[u];
      const float cb = cbs[u];
      const int v = v0 + u;
      const float *row = S + (size_t)g.out_row * n;
      const int2 *lrow = lim + (size_t)v * nt;
      if (g.steep) {  // major axis y: row R is m = R - nh, minor = column
#pragma unroll
        for (int i = 0; i < kSsPix; ++i)
          ss_adj_group(g, cb, R0 + i - nh, C0, nh, row, lrow, acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
      } else {  // major axis x: column C is m = C - nh, minor = row
#pragma unroll
        for (int j = 0; j < kSsPix; ++j)
          ss_adj_group(g, cb, C0 + j - nh, R0, nh, row, lrow, acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kSsPix; ++i)
#pragma unroll
    for (int j = 0; j < kSsPix; ++j) {
      const int R = R0 + i, C = C0 + j;
      const bool live = R < n && C < n;
      adj_store(ep, acc[i][j], live, z * (size_t)n * n + (live ? (size_t)R * n + C : 0), img);
    }
}

static void sort4(float *a) {
  for (int i = 1; i < 4; ++i)
    for (int j = i; j > 0 && a[j] < a[j - 1]; --j) std::swap(a[j], a[j - 1]);
}

}  // namespace

int ss_setup(Plan &p) {
  const int na = p.g.na, nh = p.nh, nt = 2 * nh;
  std::vector<SsAngle> tab(na);
  std::vector<int2> lim((size_t)na * nt);
  const float fnh = (float)nh, fnh1 = (float)(nh - 1);
  for (int v = 0; v < na; ++v) {
    float s, c;
    sincosf(p.angles[v], &s, &c);
    SsAngle a{};
    a.out_row = na - 1 - v;  // radon_ss.c:111
    a.steep = std::fabs((double)s) <= kS45 ? 1 : 0;
    // steep: f = fma(-y, s, t) * (1/c), weight 1/|c|; else f = fma(-x, c, t) * (1/s)
    a.a = a.steep ? s : c;
    a.rb = a.steep ? 1.0f / c : 1.0f / s;
    a.wt = (float)(1.0 / std::fabs((double)(a.steep ? c : s)));
    tab[v] = a;
    for (int kt = 0; kt < nt; ++kt) {
      const int t = kt - nh;
      const float ft = (float)t;
      float l0, l1, l2, l3;
      if (std::fabs((double)s) < 1e-5) {
        l0 = 0; l1 = 0; l2 = -fnh; l3 = fnh1;
      } else if (std::fabs((double)c) < 1e-5) {
        l0 = -fnh; l1 = fnh1; l2 = 0; l3 = 0;
      } else {
        float xa[4] = {std::fma(fnh, s, ft) / c, std::fma(-s, fnh1, ft) / c, -fnh, fnh1};
        float ya[4] = {std::fma(fnh, c, ft) / s, std::fma(-c, fnh1, ft) / s, -fnh, fnh1};
        sort4(xa);
        sort4(ya);
        l0 = xa[1]; l1 = xa[2]; l2 = ya[1]; l3 = ya[2];
      }
      const float lo = a.steep ? l2 : l0, hi = a.steep ? l3 : l1;
      lim[(size_t)v * nt + kt] = make_int2((int)std::round(lo), (int)std::round(hi));
    }
  }
  TOMO_CUDA(cudaMalloc(&p.d_angles, sizeof(SsAngle) * (size_t)na));
  TOMO_CUDA(cudaMemcpy(p.d_angles, tab.data(), sizeof(SsAngle) * (size_t)na, cudaMemcpyHostToDevice));
  TOMO_CUDA(cudaMalloc(&p.d_aux, sizeof(int2) * lim.size()));
  TOMO_CUDA(cudaMemcpy(p.d_aux, lim.data(), sizeof(int2) * lim.size(), cudaMemcpyHostToDevice));
  p.scratch_bytes = sizeof(float) * image_elems(p);
  TOMO_CUDA(cudaMalloc(&p.d_scratch, p.scratch_bytes));
  return TOMO_OK;
}

int ss_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz, nh = p.nh;
  dim3 tb(32, 8), tg((n + 31) / 32, (n + 31) / 32, nz);
  ss_transpose_kernel<<<tg, tb, 0, s>>>(d_img, p.d_scratch, n);
  dim3 fb(128), fg((n + 127) / 128, na, nz);
  ss_forward_kernel<<<fg, fb, 0, s>>>(d_img, p.d_scratch, d_sino, (const SsAngle *)p.d_angles,
                                      (const int2 *)p.d_aux, n, nh, na, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int ss_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s, const AdjEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz;
  dim3 ab(32, 8), ag((n + 32 * kSsPix - 1) / (32 * kSsPix), (n + 8 * kSsPix - 1) / (8 * kSsPix), nz);
  ss_adjoint_kernel<<<ag, ab, 0, s>>>(d_sino, d_img, (const SsAngle *)p.d_angles,
                                      (const int2 *)p.d_aux, n, p.nh, na, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
