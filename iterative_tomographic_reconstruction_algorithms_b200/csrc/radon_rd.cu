// Ray-driven (Siddon) projector pair for sm_100a.
//
// Reference: common/operators/radon_module/pymodule_radon_ray_driven/
// radon_rd.c:15-71 (siddon) and :76-189 (radon_rd).  Each detector bin b is
// sampled by five sub-rays (sub-ray index i = 6b + 1 .. 6b + 5, offset t from
// |i/6 - nh| with the sign rules of :125-130).  A sub-ray enters the square
// [-nh, nh]^2 at p1 and leaves at p2 (:133-179).  The walk starts in pixel
// (round(p1x), round(p1y)) with alpha = 0 (the reference's `alpha` is
// uninitialised; its -O3 build behaves as 0), computes the next x and y
// crossing parameters as double quotients rounded to float, steps across the
// smaller (both when equal), and credits (alpha - alpha_old) * |p2 - p1| / 5
// to the pixel it steps INTO (x index -> image row) if that pixel has row and
// column in [1, n-1]; it stops after the first step with alpha > 1.
//
// Both directions run the same walks (rd_walk_loop), one thread per (bin, angle,
// slice) replaying its bin's five sub-rays (the adjoint, on grids too small to
// fill the GPU, one thread per sub-ray):
//   forward  gathers 0.2 l x[pixel] into the bin, in walk order;
//   adjoint  scatters 0.2 l y[bin] into a 64-bit fixed-point image with
//            integer reductions (order-independent sums, so deterministic, of
//            credits rounded to the fixed-point unit), rounded to float once,
//            through the solver epilogue, at the end.
//            Non-finite credits (inf or NaN in y, or 0 * inf) cannot be held
//            as integers: they set per-pixel flags instead, and a flagged
//            pixel becomes what the reference's float sum gives (+inf, -inf,
//            or NaN when it met NaN or both infinities).
// The lanes of a warp are neighbouring bins, so at each step they sit side by
// side across the ray.  For angles whose rays run along image columns
// (|s| > |c|) that is down a column: those angles read a transposed copy of
// the image (forward) and scatter into a transposed fixed-point image
// (adjoint), so neighbouring lanes touch neighbouring words.  Both copies are
// framed (rows and columns -1 .. n+1, zero or ignored outside [1, n-1]^2), so
// that the walks whose end points lie within nh + 1/4 of the centre -- all of
// them but for rounding -- run without a range test (rd_walk_framed).
// The walk's arithmetic is float only: the crossing parameters reproduce the
// reference's double quotients exactly (rd_alpha_mf), with a double division
// only for quotients within 2^-38 of a float rounding boundary.
#include <algorithm>
#include <cmath>

#include "fixed_sum.cuh"
#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr double kPi = 3.141592653589793;

// Sub-ray offset |i/6 - nh| (radon_rd.c:125-126) read from a table made on the
// host in the reference's double arithmetic, with the signs of :127-130.
__device__ __forceinline__ float rd_offset_tab(const float *__restrict__ toff, int i, int n, bool lt, bool gt) {
  float t = __ldg(toff + i);
  if (i >= 3 * n && lt) t = -t;
  if (i < 3 * n && gt) t = -t;
  return t;
}

// (int)roundf(x) (halves away from zero) for |x| < 2^22: floor(|x| + 0.5) is
// the floor of the round-down sum (the integer below is a float), and a
// round-down add of 1.5 * 2^23 puts that floor in the low mantissa bits.
__device__ __forceinline__ int rd_round_i(float x) {
  const float f = __fadd_rd(__fadd_rd(fabsf(x), 0.5f), 12582912.0f);
  const int k = __float_as_int(f) - 0x4B400000;
  return x < 0.0f ? -k : k;
}

// Entry point, extents, start pixel and step directions of a sub-ray at
// offset t (radon_rd.c:133-179 and :21-36); the walk computes its length.
struct RdGeom {
  float p1x, p1y, p2x, p2y, ex, ey;
  int ii0, jj0, dx, dy;
};

__device__ __forceinline__ RdGeom rd_geom(float t, const RdAngle &g, int nh) {
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
  RdGeom r;
  r.p1x = p1x;
  r.p1y = p1y;
  r.p2x = p2x;
  r.p2y = p2y;
  r.ex = __fsub_rn(p2x, p1x);
  r.ey = __fsub_rn(p2y, p1y);
  r.ii0 = rd_round_i(p1x);
  r.jj0 = rd_round_i(p1y);
  r.dx = p2x > p1x ? 1 : -1;
  r.dy = p2y > p1y ? 1 : -1;
  return r;
}

// Geometry of sub-ray i of angle v, out of line: the angle's table entry is
// read here, so the walks' callers do not hold it across the walks.
__device__ __noinline__ RdGeom rd_geom_of(const RdAngle *__restrict__ tab, int v, const float *__restrict__ toff,
                                          int i, int n, int nh) {
  const RdAngle g = tab[v];
  return rd_geom(rd_offset_tab(toff, i, n, g.lt, g.gt), g, nh);
}

// The double division of rd_alpha_mf, out of line: rarely taken, and its
// double registers stay out of the walk loops.
__device__ __noinline__ float rd_alpha_div(float h, float l, float e) {
  return __double2float_rn(__ddiv_rn(__dadd_rn((double)h, (double)l), (double)e));
}

// alpha of a crossing, for a sub-ray that enters at p with extent e,
// r = RN(1/e): the float of the correctly rounded double quotient
// ((double)a - p) / e that the reference computes (radon_rd.c:41-42), a the
// crossing's half-integer coordinate, in float arithmetic.  The numerator is
// given as m - f with p = P + f, P = rint(p), |f| <= 1/2 (exact), and
// m = a - P, a half-integer (exact), which the walk steps by +-1.
//
// a - p = m - f = h + l exactly (Fast2Sum, valid since |m| >= 1/2 >= |f|).
// q1 = RN(h r); the remainder h + l - q1 e (one FMA, then + l) times r gives
// q2, and q1 + q2 is within 2^-44 |x| of the exact quotient x (r and q1 are
// within 2^-23 of exact, the remainder is 2^-23 |h| small).  With
// d = 2^-38 |q1|, RN(q1 + RN(q2 - d)) and RN(q1 + RN(q2 + d)) round points
// below and above every value within 2^-44 |x| of q1 + q2 (the inner roundings
// move them by 2^-47 at most).  Rounding to nearest is monotone, so when both
// give the same float s, x and the double nearest x (2^-53 |x| from it) round
// to s too.  Otherwise (x within about 2^-38 of a float rounding boundary, or
// e zero) divide in double.
__device__ __forceinline__ float rd_alpha_mf(float m, float f, float e, float r) {
  const float h = __fsub_rn(m, f);
  const float l = __fsub_rn(-f, __fsub_rn(h, m));
  const float q1 = __fmul_rn(h, r);
  const float rho = __fadd_rn(__fmaf_rn(-q1, e, h), l);
  const float q2 = __fmul_rn(rho, r);
  const float d = __fmul_rn(fabsf(q1), 0x1p-38f);
  const float lo = __fadd_rn(q1, __fsub_rn(q2, d)), hi = __fadd_rn(q1, __fadd_rn(q2, d));
  if (lo == hi) return lo;
  return rd_alpha_div(h, l, e);
}

// One sub-ray's walk (radon_rd.c:39-70): visit(ok, off, l) for every step,
// ok when the pixel stepped into has image row pi and column pj in [1, n-1]
// (the reference credits only those), off = (pi + pad) sA + (pj + pad) sB its
// offset in the image the caller reads or writes (sA = row stride, sB = 1
// row-major; sA = 1, sB = row stride transposed), l the length credited.
//
// Two forms.  Checked (Safe): ok as above, and the walk stops after 4n + 16
// steps: a zero or tiny extent makes that axis' alphas infinite or NaN, on
// which the reference never ends.  Unchecked (Safe false), for walks with
// |1/e| <= 2^64 on both axes, where each step raises the stepped axis' next
// alpha by about 1/|e| (far above the float spacing of alphas <= 1) and no
// alpha is inf or NaN, so a walk ends after at most |ex| + |ey| + 4 steps;
// visit gets ok = true for every step:
// the caller's image then has a frame, rows and columns -1 .. n+1 at
// pad = 1, holding zeros (reads) or ignored sums (writes) outside
// [1, n-1]^2.  They are used for walks whose end points all lie within
// nh + 1/4 of the centre: such a walk stays in rows and columns -1 .. n+1.
// (x steps, dx = 1: x step j >= 1 happens only if the alpha of x step j - 1
// was <= 1, i.e. its crossing c <= p1x + ex (1 + 2^-21) <= p2x + 2^-5, so
// c <= nh - 1/2 and the pixel stepped into, c + 3/2, is <= nh + 1; step 0
// goes to round(p1x) + 1 <= nh + 1; and round(p1x) >= -nh.  The same for
// dx = -1 and for y.)
template <bool Safe, class Visit>
__device__ __forceinline__ void rd_walk_loop(const RdGeom &s, int n, int nh, int sA, int sB, int pad, float rx,
                                             float ry, Visit &visit) {
  const float incr = __fsqrt_rn(__fmaf_rn(s.ex, s.ex, __fmul_rn(s.ey, s.ey)));
  const float hx = s.dx > 0 ? 0.5f : -0.5f, hy = s.dy > 0 ? 0.5f : -0.5f;
  const float fdx = hx + hx, fdy = hy + hy;
  const float Px = rintf(s.p1x), Py = rintf(s.p1y);
  const float fx = __fsub_rn(s.p1x, Px), fy = __fsub_rn(s.p1y, Py);
  // numerators of the next x and y crossings, m - f, m stepped exactly by +-1
  float mx = __fsub_rn(__fadd_rn((float)s.ii0, hx), Px), my = __fsub_rn(__fadd_rn((float)s.jj0, hy), Py);
  float ax = rd_alpha_mf(mx, fx, s.ex, rx), ay = rd_alpha_mf(my, fy, s.ey, ry);
  // the current pixel's row is pi = mx + Px - hx + nh (its next x crossing is
  // at pi - nh + hx), so pi - n/2 = mx + kx; pi in [1, n-1] iff
  // |pi - n/2| <= n/2 - 1.  All of it exact in float.
  const float half = 0.5f * (float)n, lim = half - 1.0f;
  const float kx = __fsub_rn(__fadd_rn(__fsub_rn(Px, hx), (float)nh), half);
  const float ky = __fsub_rn(__fadd_rn(__fsub_rn(Py, hy), (float)nh), half);
  int off = (s.ii0 + nh + pad) * sA + (s.jj0 + nh + pad) * sB;
  const int ox = s.dx * sA, oy = s.dy * sB;
  float alpha = 0.0f, alpha_old = 0.0f;
  for (int it = Safe ? 4 * n + 16 : 1; alpha <= 1.0f && it > 0; it -= Safe ? 1 : 0) {
    // x step if ax < ay, y step if ax > ay, both if equal (radon_rd.c:45-58);
    // a NaN crossing would never advance the reference: stop.  Written
    // without branches on the step kind, so the lanes of a warp stay together:
    // one new crossing parameter (two on a diagonal step).
    const bool sx = ax <= ay, sy = ay <= ax;
    if (Safe && !(sx || sy)) break;
    alpha = sx ? ax : ay;
    mx = sx ? __fadd_rn(mx, fdx) : mx;
    my = sy ? __fadd_rn(my, fdy) : my;
    off += (sx ? ox : 0) + (sy ? oy : 0);
    const float a1 = rd_alpha_mf(sx ? mx : my, sx ? fx : fy, sx ? s.ex : s.ey, sx ? rx : ry);
    ax = sx ? a1 : ax;
    ay = sx ? ay : a1;
    if (sx && sy) ay = rd_alpha_mf(my, fy, s.ey, ry);
    const float l = __fmul_rn(__fsub_rn(alpha, alpha_old), incr);
    visit(!Safe || (fabsf(__fadd_rn(mx, kx)) <= lim && fabsf(__fadd_rn(my, ky)) <= lim), off, l);
    alpha_old = alpha;
  }
}

// Whether a walk may run unchecked on a framed image (above): its end points
// within nh + 1/4 of the centre and |1/e| <= 2^64 on both axes.  Walks that
// fail it are few: an end point is on the square's edge up to the rounding of
// the reference's entry / exit arithmetic.
__device__ __forceinline__ bool rd_walk_framed(const RdGeom &s, int nh, float rx, float ry) {
  const float reach = fmaxf(fmaxf(fabsf(s.p1x), fabsf(s.p1y)), fmaxf(fabsf(s.p2x), fabsf(s.p2y)));
  return reach <= (float)nh + 0.25f && fabsf(rx) <= 0x1p64f && fabsf(ry) <= 0x1p64f;
}

// The forward's credits along walks: acc += 0.2 l x[pixel] in walk order,
// each credit added one step after its load is issued, so the load is in
// flight during the next step; a step outside [1, n-1]^2 adds 0 * 0 (checked
// walks) or w * 0 from the frame (acc is never -0, so that leaves it
// unchanged).
struct RdGather {
  const float *P;
  float acc, w, xv;
  __device__ __forceinline__ void operator()(bool ok, int off, float l) {
    const float x = ok ? __ldg(P + off) : 0.0f;
    acc = fmaf(w, xv, acc);
    w = ok ? 0.2f * l : 0.0f;
    xv = x;
  }
};

// The adjoint's credits: fixed_of(0.2 l y) with ys = y 2^E (scaling by a power
// of two commutes with the rounding of the product).
// The add is a fire-and-forget reduction (red.global.add.u64: no result comes
// back), which measured 17 % faster than atomicAdd here.
struct RdScatter {
  unsigned long long *P;
  float ys;
  __device__ __forceinline__ void operator()(bool ok, int off, float l) {
    if (ok) {
      const unsigned long long q = (unsigned long long)__float2ll_rn(__fmul_rn(0.2f * l, ys));
      asm volatile("red.global.add.u64 [%0], %1;" ::"l"(P + off), "l"(q) : "memory");
    }
  }
};

// Checked walks out of line, state passed by value: rarely taken, and kept
// out of the register budget of the unchecked loop.
__device__ __noinline__ RdGather rd_walk_safe(RdGeom s, int n, int nh, int sA, int sB, int pad, float rx, float ry,
                                              RdGather v) {
  rd_walk_loop<true>(s, n, nh, sA, sB, pad, rx, ry, v);
  return v;
}

__device__ __noinline__ void rd_walk_safe(RdGeom s, int n, int nh, int sA, int sB, int pad, float rx, float ry,
                                          RdScatter v) {
  rd_walk_loop<true>(s, n, nh, sA, sB, pad, rx, ry, v);
}

// Framed copies of slice blockIdx.z for the forward's walks: Q (row-major)
// and QT (transposed), (n + 3)^2 each, Q[(pi + 1)(n + 3) + pj + 1] = x[pi][pj]
// for pi, pj in [1, n-1] and 0 elsewhere (pi, pj in -1 .. n+1); a 32 x 32
// tile of the framed grid per block (blockDim 32 x 8).
__global__ void rd_frame_kernel(const float *__restrict__ in, float *__restrict__ Q, float *__restrict__ QT, int n) {
  __shared__ float tile[32][33];
  const int m = n + 3;
  const float *src = in + (size_t)blockIdx.z * n * n;
  float *q = Q + (size_t)blockIdx.z * m * m, *qt = QT + (size_t)blockIdx.z * m * m;
  const int C0 = blockIdx.x * 32, R0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int R = R0 + k, C = C0 + threadIdx.x, pi = R - 1, pj = C - 1;
    const bool in_img = pi >= 1 && pi <= n - 1 && pj >= 1 && pj <= n - 1;
    const float v = in_img ? src[(size_t)pi * n + pj] : 0.0f;
    tile[k][threadIdx.x] = v;
    if (R < m && C < m) q[(size_t)R * m + C] = v;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int R = C0 + k, C = R0 + threadIdx.x;  // QT[R][C] = Q[C][R]
    if (R < m && C < m) qt[(size_t)R * m + C] = tile[threadIdx.x][k];
  }
}

// Forward over slices z0 + blockIdx.z; Q and QT hold the chunk's slices
// framed (rd_frame_kernel).  A block is kBins bins of kFwdAngles consecutive
// angles (threadIdx.y): the walks of neighbouring angles cover nearly the same
// pixels at nearly the same time, so its warps share L1 lines.  kBins = 128,
// or 32 for grids of at most a few blocks per SM, where 512-thread blocks
// leave some SMs with one more block than others (at 256 x 256, 304 angles:
// 152 blocks on 148 SMs, two resident per SM).  A row of the sinogram has
// ceil(n / 128) * 4 warps in both layouts (dead lanes included), and warp
// b / 32 of row (z, v) writes residual slot (z na + v) * that + b / 32.
constexpr int kFwdAngles = 4;

template <int kBins>
__global__ void __launch_bounds__(kBins * kFwdAngles, 1024 / (kBins * kFwdAngles)) rd_forward_kernel(
    const float *__restrict__ img, const float *__restrict__ Q, const float *__restrict__ QT,
    float *__restrict__ sino, const RdAngle *__restrict__ tab, const float *__restrict__ toff, int n, int nh, int na,
    int z0, FwdEpi ep) {
  const int b = blockIdx.x * kBins + threadIdx.x;
  const int v = blockIdx.y * kFwdAngles + threadIdx.y;
  if (v >= na) return;  // whole warps
  const size_t z = (size_t)z0 + blockIdx.z;
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
    const int m = n + 3;
    const bool tr = g.tr != 0;
    const float *P = (tr ? QT : Q) + (size_t)blockIdx.z * m * m;
    const int sA = tr ? 1 : m, sB = tr ? m : 1;
    RdGather gat{P, 0.0f, 0.0f, 0.0f};
    for (int r = 1; r <= 5; ++r) {
      const RdGeom s = rd_geom_of(tab, v, toff, 6 * b + r, n, nh);
      const float rx = __frcp_rn(s.ex), ry = __frcp_rn(s.ey);
      if (rd_walk_framed(s, nh, rx, ry))
        rd_walk_loop<false>(s, n, nh, sA, sB, 1, rx, ry, gat);
      else
        gat = rd_walk_safe(s, n, nh, sA, sB, 1, rx, ry, gat);
    }
    acc = fmaf(gat.w, gat.xv, gat.acc);
  }
  // store through the epilogue; residual slot as in one launch over all slices
  const size_t e = (z * na + v) * (size_t)n + (live ? b : 0);
  double r2 = 0.0;
  if (live) sino[e] = fwd_apply(ep, acc, e, r2);
  fwd_resid_commit(ep, r2, (z * na + v) * (gridDim.x * (kBins / 32)) + b / 32);
}

// Flag bytes of non-finite credits (nonfinite_flag: 1 +inf, 2 -inf, 4 NaN),
// byte p of the chunk's flag array for pixel p (four pixels to a 32-bit word).
__device__ __forceinline__ void rd_flag(unsigned *flags, size_t p, float c) {
  atomicOr(flags + (p >> 2), nonfinite_flag(c) << (8u * (unsigned)(p & 3)));
}

// The adjoint scatter of a bin whose value y is inf or NaN: the same walks
// (and row / column sums), flags instead of sums, in the natural pixel layout.
// Out of line: rarely taken, and kept out of the register budget of the walk.
__device__ __noinline__ void rd_scatter_nonfinite(float y, const RdAngle *__restrict__ gp, int b, int n, int nh,
                                                  const float *__restrict__ toff, unsigned *Fl) {
  const RdAngle g = *gp;
  if (g.mode == 1) {
    const int i = n - 1 - b;
    if (i >= 1)
      for (int j = 0; j < n; ++j) rd_flag(Fl, (size_t)j * n + i, y);
  } else if (g.mode == 2) {
    for (int j = 0; j < n; ++j) rd_flag(Fl, (size_t)b * n + j, y);
  } else {
    for (int r = 1; r <= 5; ++r) {
      const RdGeom s = rd_geom(rd_offset_tab(toff, 6 * b + r, n, g.lt, g.gt), g, nh);
      auto flag = [&](bool ok, int off, float l) {
        if (ok) rd_flag(Fl, (size_t)off, __fmul_rn(0.2f * l, y));
      };
      rd_walk_loop<true>(s, n, nh, n, 1, 0, __frcp_rn(s.ex), __frcp_rn(s.ey), flag);
    }
  }
}

// Fixed-point scale of slice z's adjoint: per angle a pixel receives at most
// 11 credits 0.2 l |y| with l <= sqrt(2) (the segment in one pixel), or one
// credit |y| (row and column sums), below 4 max|y|; the bound holds for each of
// the two fixed-point images and for their sum.
__device__ __forceinline__ FixedScale rd_adj_scale(const unsigned *smax, int na) {
  return fixed_scale(4.0 * (double)na * (double)__uint_as_float(*smax));
}

// Adjoint scatter: slice blockIdx.z of the chunk.  Walk credits go to the
// framed fixed-point images F (row-major) and FT (transposed, for angles with
// |s| > |c|), (n + 3)^2 each, pixel (pi, pj) at (pi + 1)(n + 3) + pj + 1; the
// frame and row / column 0 collect credits the reference does not make, which
// the finalize ignores.  The row / column-sum angles add their one credit per
// pixel to per-column (cols) and per-row (rows) sums instead.
// kSplit: one thread per sub-ray (thread t walks sub-ray t % 5 + 1 of bin
// t / 5) instead of one per bin walking all five, for grids too small to fill
// the GPU; the sums are order-independent, so both give the same bits.  The
// bin's first thread alone makes its row / column sum and non-finite flags.
template <bool kSplit>
__global__ void __launch_bounds__(128) rd_scatter_kernel(
    const float *__restrict__ sino, unsigned long long *__restrict__ accf, unsigned long long *__restrict__ accT,
    unsigned long long *__restrict__ lines, unsigned *__restrict__ flags, const RdAngle *__restrict__ tab,
    const float *__restrict__ toff, int n, int nh, int na, const unsigned *__restrict__ smax) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = kSplit ? t / 5 : t;
  const int r0 = kSplit ? t - 5 * b + 1 : 1, r1 = kSplit ? r0 : 5;
  const int v = blockIdx.y;
  const size_t z = blockIdx.z;
  if (b >= n) return;
  const float y = __ldg(sino + (z * na + v) * (size_t)n + b);
  if (y == 0.0f) return;
  const RdAngle g = tab[v];
  if (!(fabsf(y) <= 3.4028235e38f)) {  // inf or NaN
    if (r0 == 1) rd_scatter_nonfinite(y, tab + v, b, n, nh, toff, flags + z * (((size_t)n * n + 3) / 4));
    return;
  }
  if (g.mode != 0 && r0 != 1) return;
  const FixedScale fs = rd_adj_scale(smax + z, na);
  const int m = n + 3;
  unsigned long long *cols = lines + z * 2 * (size_t)n, *rows = cols + n;
  if (g.mode == 1) {  // column n-1-b, every row (transpose of radon_rd.c:96-105)
    const int i = n - 1 - b;
    if (i >= 1) atomicAdd(cols + i, fixed_of(y, fs));
    return;
  }
  if (g.mode == 2) {  // row b, every column (:108-117)
    atomicAdd(rows + b, fixed_of(y, fs));
    return;
  }
  const bool tr = g.tr != 0;
  unsigned long long *P = (tr ? accT : accf) + z * (size_t)m * m;
  const int sA = tr ? 1 : m, sB = tr ? m : 1;
  RdScatter add{P, __fmul_rn(__fmul_rn(y, fs.s1), fs.s2)};
  for (int r = r0; r <= r1; ++r) {
    const RdGeom s = rd_geom_of(tab, v, toff, 6 * b + r, n, nh);
    const float rx = __frcp_rn(s.ex), ry = __frcp_rn(s.ey);
    if (rd_walk_framed(s, nh, rx, ry))
      rd_walk_loop<false>(s, n, nh, sA, sB, 1, rx, ry, add);
    else
      rd_walk_safe(s, n, nh, sA, sB, 1, rx, ry, add);
  }
}

// Walk credits of pixels in [1, n-1]^2 (F + FT transposed) plus the row and
// column sums -> float through the adjoint epilogue, a 32 x 32 tile per block
// (blockDim 32 x 8); slice blockIdx.z of the chunk is slice z0 + it.
__global__ void rd_finalize_kernel(const unsigned long long *__restrict__ accf,
                                   const unsigned long long *__restrict__ accT,
                                   const unsigned long long *__restrict__ lines, const unsigned *__restrict__ flags,
                                   float *__restrict__ img, int n, int z0, int na, const unsigned *__restrict__ smax,
                                   AdjEpi ep) {
  __shared__ unsigned long long tile[32][33];
  const size_t zl = blockIdx.z, per = (size_t)n * n;
  const int m = n + 3;
  const unsigned long long *F = accf + zl * (size_t)m * m, *FT = accT + zl * (size_t)m * m;
  const unsigned long long *cols = lines + zl * 2 * (size_t)n, *rows = cols + n;
  const int R0 = blockIdx.y * 32, C0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y)  // tile[c][r] = FT at pixel (R0 + r, C0 + c)
    if (C0 + k < n && R0 + threadIdx.x < n)
      tile[k][threadIdx.x] = FT[(size_t)(C0 + k + 1) * m + R0 + threadIdx.x + 1];
  __syncthreads();
  const FixedScale fs = rd_adj_scale(smax + zl, na);
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int R = R0 + k, C = C0 + threadIdx.x;
    const bool live = R < n && C < n;
    float val = 0.0f;
    if (live) {
      const size_t p = (size_t)R * n + C;
      const unsigned f = (flags[zl * ((per + 3) / 4) + (p >> 2)] >> (8u * (unsigned)(p & 3))) & 0xffu;
      unsigned long long q = cols[C] + rows[R];
      if (R >= 1 && C >= 1) q += F[(size_t)(R + 1) * m + C + 1] + tile[threadIdx.x][k];
      val = f == 0u ? fixed_to_float(q, fs) : nonfinite_value(f);
    }
    adj_store(ep, val, live, ((size_t)z0 + zl) * per + (live ? (size_t)R * n + C : 0), img);
  }
}

// slices per chunk: the adjoint's two framed fixed-point images, row and
// column sums and flag bytes (the forward's framed images use the same space)
// of at most 512 MiB, and no more than a grid dimension holds
size_t rd_flag_words(const Plan &p) { return ((size_t)p.g.n * p.g.n + 3) / 4; }

size_t rd_framed(const Plan &p) { return (size_t)(p.g.n + 3) * (p.g.n + 3); }

int rd_chunk(const Plan &p) {
  const size_t per = 16 * rd_framed(p) + 16 * (size_t)p.g.n + 4 * rd_flag_words(p);
  const size_t cap = std::min<size_t>(((size_t)512 << 20) / per, 65535);
  return (int)std::max<size_t>(1, std::min<size_t>((size_t)p.g.nz, cap));
}

}  // namespace

int rd_setup(Plan &p) {
  const int na = p.g.na, nh = p.nh, n = p.g.n;
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
    a.tr = std::fabs((double)s) > std::fabs((double)c) ? 1 : 0;
    a.rc = 1.0f / c;
    a.rs = 1.0f / s;
    a.ns = fnh * s;
    a.nc = fnh * c;
    a.mns = -fnh * s;
    a.mnc = -fnh * c;
    tab[v] = a;
  }
  // |i/6 - nh| per sub-ray index, i/6 compiled as fma(i, 1/6, -nh) in double
  std::vector<float> toff((size_t)6 * n);
  for (int i = 0; i < 6 * n; ++i) toff[i] = (float)std::fabs(std::fma((double)i, 1.0 / 6.0, -(double)nh));
  TOMO_CUDA(cudaMalloc(&p.d_angles, sizeof(RdAngle) * (size_t)na));
  TOMO_CUDA(cudaMemcpy(p.d_angles, tab.data(), sizeof(RdAngle) * (size_t)na, cudaMemcpyHostToDevice));
  TOMO_CUDA(cudaMalloc(&p.d_aux, sizeof(float) * toff.size()));
  TOMO_CUDA(cudaMemcpy(p.d_aux, toff.data(), sizeof(float) * toff.size(), cudaMemcpyHostToDevice));
  // scratch: a chunk of framed fixed-point images, of transposed ones, of row
  // and column sums and of flag bytes (the forward's framed images in the
  // same space), then max |y| per slice
  p.scratch_bytes = (16 * rd_framed(p) + 16 * (size_t)n + 4 * rd_flag_words(p)) * rd_chunk(p) +
                    sizeof(unsigned) * (size_t)p.g.nz;
  TOMO_CUDA(cudaMalloc(&p.d_scratch, p.scratch_bytes));
  return TOMO_OK;
}

int rd_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz, chunk = rd_chunk(p), m = n + 3;
  float *Q = p.d_scratch, *QT = Q + (size_t)chunk * rd_framed(p);
  for (int z0 = 0; z0 < nz; z0 += chunk) {
    const int zc = std::min(chunk, nz - z0);
    rd_frame_kernel<<<dim3((m + 31) / 32, (m + 31) / 32, zc), dim3(32, 8), 0, s>>>(d_img + (size_t)z0 * n * n, Q,
                                                                                     QT, n);
    const int rows = (na + kFwdAngles - 1) / kFwdAngles, w128 = (n + 127) / 128;
    // 128-bin blocks once there are 8 or more per SM, else 32-bin ones
    if ((size_t)w128 * rows * zc >= (size_t)148 * 8)
      rd_forward_kernel<128><<<dim3(w128, rows, zc), dim3(128, kFwdAngles), 0, s>>>(
          d_img, Q, QT, d_sino, (const RdAngle *)p.d_angles, (const float *)p.d_aux, n, p.nh, na, z0, ep);
    else
      rd_forward_kernel<32><<<dim3(4 * w128, rows, zc), dim3(32, kFwdAngles), 0, s>>>(
          d_img, Q, QT, d_sino, (const RdAngle *)p.d_angles, (const float *)p.d_aux, n, p.nh, na, z0, ep);
  }
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int rd_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s, const AdjEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz, chunk = rd_chunk(p);
  const size_t per_sino = (size_t)na * n;
  const size_t per_fr = rd_framed(p);
  unsigned long long *accf = reinterpret_cast<unsigned long long *>(p.d_scratch);
  unsigned long long *accT = accf + (size_t)chunk * per_fr;
  unsigned long long *lines = accT + (size_t)chunk * per_fr;
  const size_t fw = rd_flag_words(p);
  unsigned *flags = reinterpret_cast<unsigned *>(lines + (size_t)chunk * 2 * n);
  unsigned *smax = flags + (size_t)chunk * fw;
  TOMO_CUDA(cudaMemsetAsync(smax, 0, sizeof(unsigned) * (size_t)nz, s));
  for (int z0 = 0; z0 < nz; z0 += chunk) {
    const int zc = std::min(chunk, nz - z0);
    fixed_finite_absmax_kernel<<<dim3(64, zc), 256, 0, s>>>(d_sino + (size_t)z0 * per_sino, per_sino, smax + z0);
    TOMO_CUDA(cudaMemsetAsync(accf, 0, sizeof(unsigned long long) * zc * per_fr, s));
    TOMO_CUDA(cudaMemsetAsync(accT, 0, sizeof(unsigned long long) * zc * per_fr, s));
    TOMO_CUDA(cudaMemsetAsync(lines, 0, sizeof(unsigned long long) * zc * 2 * (size_t)n, s));
    TOMO_CUDA(cudaMemsetAsync(flags, 0, sizeof(unsigned) * zc * fw, s));
    // one thread per bin when that fills the GPU (148 SMs x 1024 threads at
    // the kernel's 64 registers), else one per sub-ray
    if ((size_t)n * na * zc >= (size_t)148 * 1024)
      rd_scatter_kernel<false><<<dim3((n + 127) / 128, na, zc), 128, 0, s>>>(
          d_sino + (size_t)z0 * per_sino, accf, accT, lines, flags, (const RdAngle *)p.d_angles,
          (const float *)p.d_aux, n, p.nh, na, smax + z0);
    else
      rd_scatter_kernel<true><<<dim3((5 * n + 127) / 128, na, zc), 128, 0, s>>>(
          d_sino + (size_t)z0 * per_sino, accf, accT, lines, flags, (const RdAngle *)p.d_angles,
          (const float *)p.d_aux, n, p.nh, na, smax + z0);
    rd_finalize_kernel<<<dim3((n + 31) / 32, (n + 31) / 32, zc), dim3(32, 8), 0, s>>>(
        accf, accT, lines, flags, d_img, n, z0, na, smax + z0, ep);
  }
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
