// Ray-driven (Siddon) projector pair for sm_100a.
//
// Reference: common/operators/radon_module/pymodule_radon_ray_driven/
// radon_rd.c:15-71 (siddon) and :76-189 (radon_rd).  Each detector bin b is
// sampled by five sub-rays (sub-ray index i = 6b + 1 .. 6b + 5, offset t from
// |i/6 - nh| with the sign rules of :125-130).  A sub-ray enters the square
// [-nh, nh]^2 at p1 and leaves at p2 (:133-179).  The walk starts in pixel
// (round(p1x), round(p1y)) with alpha = 0 (the reference's `alpha` is
// uninitialised; its -O3 build behaves as 0), computes the next x and y
// crossing parameters in double precision, rounds them to float, steps across
// the smaller (both when equal), and credits (alpha - alpha_old) * |p2 - p1| / 5
// to the pixel it steps INTO (x index -> image row) if that pixel has row and
// column in [1, n-1]; it stops after the first step with alpha > 1.
//
// Forward: one thread per (bin, angle) replays its five walks exactly.
// Adjoint: one thread per pixel.  With X(a), Y(b) the a-th x and b-th y
// crossing of a walk, the walk visits the state with A x-steps and B y-steps
// iff X(A-1) < Y(B) and Y(B-1) < X(A); it enters it at max(X(A-1), Y(B-1)),
// coming from the state entered at the previous crossing, and credits it iff
// that previous alpha is <= 1.  That closed form is evaluated for the few
// sub-rays whose line crosses the pixel, giving the exact transpose of the
// forward without atomics.
#include <cmath>

#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr double kPi = 3.141592653589793;

struct SubRay {
  float p1x, p1y, ex, ey, incr;
  int ii0, jj0, dx, dy;
};

// Sub-ray offset (radon_rd.c:125-130), i/6 compiled as fma(i, 1/6, -nh) in double.
__device__ __forceinline__ float rd_offset(int i, int n, int nh, bool lt, bool gt) {
  float t = (float)fabs(__fma_rn((double)i, 1.0 / 6.0, -(double)nh));
  if (i >= 3 * n && lt) t = -t;
  if (i < 3 * n && gt) t = -t;
  return t;
}

// Entry/exit points (radon_rd.c:133-179) in the compiled order (K + t) * (1/c).
__device__ __forceinline__ SubRay rd_subray(float t, const RdAngle &g, int nh) {
  const float fnh = (float)nh;
  float p1x, p1y, p2x, p2y;
  if (g.lt) {
    const float y1 = __fmul_rn(__fadd_rn(g.mns, t), g.rc), x1 = __fmul_rn(__fsub_rn(g.mnc, t), g.rs);
    const float y2 = __fmul_rn(__fadd_rn(g.ns, t), g.rc), x2 = __fmul_rn(__fsub_rn(g.nc, t), g.rs);
    if (y1 >= -fnh && y1 <= fnh) { p1x = -fnh; p1y = y1; } else { p1x = x1; p1y = -fnh; }
    if (y2 >= -fnh && y2 <= fnh) { p2x = fnh; p2y = y2; } else { p2x = x2; p2y = fnh; }
  } else {
    const float y1 = __fmul_rn(__fsub_rn(g.ns, t), g.rc), x1 = __fmul_rn(__fadd_rn(g.mnc, t), g.rs);
    const float y2 = __fmul_rn(__fsub_rn(g.mns, t), g.rc), x2 = __fmul_rn(__fadd_rn(g.nc, t), g.rs);
    if (y1 >= -fnh && y1 <= fnh) { p1x = fnh; p1y = y1; } else { p1x = x1; p1y = -fnh; }
    if (y2 >= -fnh && y2 <= fnh) { p2x = -fnh; p2y = y2; } else { p2x = x2; p2y = fnh; }
  }
  SubRay r;
  r.p1x = p1x;
  r.p1y = p1y;
  r.ex = __fsub_rn(p2x, p1x);
  r.ey = __fsub_rn(p2y, p1y);
  r.incr = __fsqrt_rn(__fmaf_rn(r.ex, r.ex, __fmul_rn(r.ey, r.ey)));
  r.ii0 = (int)roundf(p1x);
  r.jj0 = (int)roundf(p1y);
  r.dx = p2x > p1x ? 1 : -1;
  r.dy = p2y > p1y ? 1 : -1;
  return r;
}

// Numerator of the crossing out of column/row state `idx`: (idx + d/2) - p,
// exact in double.
__device__ __forceinline__ double rd_num(int idx, int d, float p) {
  return __dsub_rn(__dadd_rn((double)idx, 0.5 * d), (double)p);
}

// alpha = the float of the double quotient num / e, as the reference computes
// it (one double division, rounded to float).  The product num * re, re the
// double reciprocal of e, is within 2^-51 (relative) of the correctly rounded
// quotient Q; if it rounds to the same float after moving it down and up by
// 2^-49 (relative), that float is Q's.  Otherwise (Q within a hair of a
// float rounding boundary, e == 0, overflow) the division is done.
__device__ __forceinline__ float rd_alpha_q(double num, float e, double re) {
  const double q = __dmul_rn(num, re);
  const double m = fabs(q) * 0x1p-49;
  const float lo = __double2float_rn(__dsub_rn(q, m)), hi = __double2float_rn(__dadd_rn(q, m));
  if (lo == hi) return lo;
  return __double2float_rn(__ddiv_rn(num, (double)e));
}

// alpha of the crossing out of column/row state `idx`
__device__ __forceinline__ float rd_alpha(int idx, int d, float p, float e, double re) {
  return rd_alpha_q(rd_num(idx, d, p), e, re);
}

__global__ void __launch_bounds__(128) rd_forward_kernel(
    const float *__restrict__ img, float *__restrict__ sino, const RdAngle *__restrict__ tab,
    int n, int nh, int na, FwdEpi ep) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  const size_t z = blockIdx.z;
  const bool live = b < n;
  const RdAngle g = tab[v];
  const float *I = img + z * (size_t)n * n;
  float acc = 0.0f;
  if (!live) {
  } else if (g.mode == 1) {  // |s| < 1e-7: bin n-1-i <- column i, i >= 1 (radon_rd.c:96-105)
    const int i = n - 1 - b;
    if (i >= 1)
      for (int j = 0; j < n; ++j) acc += __ldg(I + (size_t)j * n + i);
  } else if (g.mode == 2) {  // |c| < 1e-7: bin i <- row i (:108-117)
    for (int j = 0; j < n; ++j) acc += __ldg(I + (size_t)b * n + j);
  } else {
    const int guard = 4 * n + 16;
    for (int r = 1; r <= 5; ++r) {
      const int i = 6 * b + r;
      const SubRay s = rd_subray(rd_offset(i, n, nh, g.lt, g.gt), g, nh);
      int ii = s.ii0, jj = s.jj0;
      float alpha = 0.0f, alpha_old = 0.0f;
      const double rex = __drcp_rn((double)s.ex), rey = __drcp_rn((double)s.ey);
      const double ddx = (double)s.dx, ddy = (double)s.dy;
      // numerators of the next crossings, stepped exactly by +-1
      double nx = rd_num(ii, s.dx, s.p1x), ny = rd_num(jj, s.dy, s.p1y);
      float ax = rd_alpha_q(nx, s.ex, rex), ay = rd_alpha_q(ny, s.ey, rey);
      for (int it = 0; alpha <= 1.0f && it < guard; ++it) {
        if (ax < ay) {
          alpha = ax;
          ii += s.dx;
          nx = __dadd_rn(nx, ddx);
          ax = rd_alpha_q(nx, s.ex, rex);
        } else if (ax > ay) {
          alpha = ay;
          jj += s.dy;
          ny = __dadd_rn(ny, ddy);
          ay = rd_alpha_q(ny, s.ey, rey);
        } else if (ax == ay) {
          alpha = ay;
          ii += s.dx;
          jj += s.dy;
          nx = __dadd_rn(nx, ddx);
          ny = __dadd_rn(ny, ddy);
          ax = rd_alpha_q(nx, s.ex, rex);
          ay = rd_alpha_q(ny, s.ey, rey);
        } else {
          break;  // NaN crossing: the reference would never advance
        }
        const float l = __fmul_rn(__fsub_rn(alpha, alpha_old), s.incr);
        const int pi = ii + nh, pj = jj + nh;
        if (pi > 0 && pi < n && pj > 0 && pj < n)
          acc = fmaf(0.2f * l, __ldg(I + (size_t)pi * n + pj), acc);
        alpha_old = alpha;
      }
    }
  }
  fwd_store(ep, acc, live, z * (size_t)na * n + (size_t)v * n + (live ? b : 0), sino);
}

constexpr int kRdChunk = 256;

__global__ void __launch_bounds__(128) rd_adjoint_kernel(
    const float *__restrict__ sino, float *__restrict__ img, const RdAngle *__restrict__ tab,
    int n, int nh, int na, AdjEpi ep) {
  __shared__ RdAngle stab[kRdChunk];
  const int J = blockIdx.x * blockDim.x + threadIdx.x;  // column (walk y index jj + nh)
  const int I = blockIdx.y * blockDim.y + threadIdx.y;  // row    (walk x index ii + nh)
  const size_t z = blockIdx.z;
  const bool live = I < n && J < n;
  const float *S = sino + z * (size_t)na * n;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
  const int iiP = I - nh, jjP = J - nh;
  const bool interior = I > 0 && J > 0;
  const float NEG = -INFINITY;
  float acc = 0.0f;
  for (int v0 = 0; v0 < na; v0 += kRdChunk) {
    const int cnt = min(kRdChunk, na - v0);
    __syncthreads();
    for (int t = tid; t < cnt; t += nthr) stab[t] = tab[v0 + t];
    __syncthreads();
    if (!live) continue;
    for (int u = 0; u < cnt; ++u) {
      const RdAngle g = stab[u];
      const float *row = S + (size_t)(v0 + u) * n;
      if (g.mode == 1) {
        if (J >= 1) acc += __ldg(row + n - 1 - J);
        continue;
      }
      if (g.mode == 2) {
        acc += __ldg(row + I);
        continue;
      }
      if (!interior) continue;
      // offset of the line through the pixel centre: y c - x s = t (lt) or x s - y c = t
      const float tP = g.lt ? (float)jjP * g.c - (float)iiP * g.s : (float)iiP * g.s - (float)jjP * g.c;
      const float half = 0.5f * (fabsf(g.c) + fabsf(g.s)) + 0.05f;
      // sub-ray index i from t: lt: t = nh - i/6; gt: t = i/6 - nh (even n)
      float ia, ib;
      if (g.lt) { ia = 6.0f * ((float)nh - (tP + half)); ib = 6.0f * ((float)nh - (tP - half)); }
      else      { ia = 6.0f * ((tP - half) + (float)nh); ib = 6.0f * ((tP + half) + (float)nh); }
      int i0 = max((int)floorf(ia) - 1, 1), i1 = min((int)ceilf(ib) + 1, 6 * n - 1);
      // odd n: sub-rays with i in [6 nh, 3n) carry the mirrored offset (radon_rd.c:127-130)
      const bool odd = (n & 1) != 0;
      const int extra0 = 6 * nh, extra1 = 3 * n - 1;
      for (int pass = 0; pass < (odd ? 2 : 1); ++pass) {
        const int a0 = pass == 0 ? i0 : extra0, a1 = pass == 0 ? i1 : extra1;
        for (int i = a0; i <= a1; ++i) {
          if (i % 6 == 0) continue;
          if (pass == 1 && i >= i0 && i <= i1) continue;
          const SubRay s = rd_subray(rd_offset(i, n, nh, g.lt, g.gt), g, nh);
          const int A = (iiP - s.ii0) * s.dx, B = (jjP - s.jj0) * s.dy;
          if (A < 0 || B < 0 || (A == 0 && B == 0)) continue;
          const double rex = __drcp_rn((double)s.ex), rey = __drcp_rn((double)s.ey);
          const float XA = rd_alpha(s.ii0 + A * s.dx, s.dx, s.p1x, s.ex, rex);
          const float YB = rd_alpha(s.jj0 + B * s.dy, s.dy, s.p1y, s.ey, rey);
          const float XA1 = A >= 1 ? rd_alpha(s.ii0 + (A - 1) * s.dx, s.dx, s.p1x, s.ex, rex) : NEG;
          const float YB1 = B >= 1 ? rd_alpha(s.jj0 + (B - 1) * s.dy, s.dy, s.p1y, s.ey, rey) : NEG;
          if (!(XA1 < YB && YB1 < XA)) continue;  // state (A, B) never visited
          float ain, aprev;
          if (XA1 > YB1) {  // entered by an x step from (A-1, B)
            ain = XA1;
            const float XA2 = A >= 2 ? rd_alpha(s.ii0 + (A - 2) * s.dx, s.dx, s.p1x, s.ex, rex) : 0.0f;
            aprev = fmaxf(XA2, B >= 1 ? YB1 : 0.0f);
          } else if (YB1 > XA1) {  // y step from (A, B-1)
            ain = YB1;
            const float YB2 = B >= 2 ? rd_alpha(s.jj0 + (B - 2) * s.dy, s.dy, s.p1y, s.ey, rey) : 0.0f;
            aprev = fmaxf(A >= 1 ? XA1 : 0.0f, YB2);
          } else {  // diagonal step from (A-1, B-1)
            ain = XA1;
            const float XA2 = A >= 2 ? rd_alpha(s.ii0 + (A - 2) * s.dx, s.dx, s.p1x, s.ex, rex) : 0.0f;
            const float YB2 = B >= 2 ? rd_alpha(s.jj0 + (B - 2) * s.dy, s.dy, s.p1y, s.ey, rey) : 0.0f;
            aprev = fmaxf(XA2, YB2);
          }
          if (!(aprev <= 1.0f)) continue;  // the walk had already stopped
          const float l = __fmul_rn(__fsub_rn(ain, aprev), s.incr);
          acc = fmaf(0.2f * l, __ldg(row + i / 6), acc);
        }
      }
    }
  }
  adj_store(ep, acc, live, z * (size_t)n * n + (size_t)(live ? I : 0) * n + (live ? J : 0), img);
}

}  // namespace

int rd_setup(Plan &p) {
  const int na = p.g.na, nh = p.nh;
  std::vector<RdAngle> tab(na);
  const float fnh = (float)nh;
  for (int v = 0; v < na; ++v) {
    const float theta = p.angles[v];
    float s, c;
    sincosf(theta, &s, &c);
    RdAngle a{};
    a.s = s;
    a.c = c;
    a.mode = std::fabs((double)s) < 1e-7 ? 1 : (std::fabs((double)c) < 1e-7 ? 2 : 0);
    a.lt = (double)theta < kPi / 2;
    a.gt = (double)theta > kPi / 2;
    a.rc = 1.0f / c;
    a.rs = 1.0f / s;
    a.ns = fnh * s;
    a.nc = fnh * c;
    a.mns = -fnh * s;
    a.mnc = -fnh * c;
    tab[v] = a;
  }
  TOMO_CUDA(cudaMalloc(&p.d_angles, sizeof(RdAngle) * (size_t)na));
  TOMO_CUDA(cudaMemcpy(p.d_angles, tab.data(), sizeof(RdAngle) * (size_t)na, cudaMemcpyHostToDevice));
  return TOMO_OK;
}

int rd_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz;
  dim3 fb(128), fg((n + 127) / 128, na, nz);
  rd_forward_kernel<<<fg, fb, 0, s>>>(d_img, d_sino, (const RdAngle *)p.d_angles, n, p.nh, na, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int rd_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s, const AdjEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz;
  dim3 ab(32, 4), ag((n + 31) / 32, (n + 3) / 4, nz);
  rd_adjoint_kernel<<<ag, ab, 0, s>>>(d_sino, d_img, (const RdAngle *)p.d_angles, n, p.nh, na, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
