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
// Both directions run the same walks (rd_walk), one thread per (bin, angle,
// slice) replaying its bin's five sub-rays:
//   forward  gathers 0.2 l x[pixel] into the bin, in walk order;
//   adjoint  scatters 0.2 l y[bin] into a 64-bit fixed-point image with
//            integer atomics (order-independent sums, so deterministic, of
//            credits rounded to the fixed-point unit), rounded to float once, through the solver epilogue, at the end.
//            Non-finite credits (inf or NaN in y, or 0 * inf) cannot be held
//            as integers: they set per-pixel flags instead, and a flagged
//            pixel becomes what the reference's float sum gives (+inf, -inf,
//            or NaN when it met NaN or both infinities).
// The lanes of a warp are neighbouring bins, so at each step they sit side by
// side across the ray.  For angles whose rays run along image columns
// (|s| > |c|) that is down a column: those angles read a transposed copy of
// the image (forward) and scatter into a transposed fixed-point image
// (adjoint), so neighbouring lanes touch neighbouring words.
// The walk's arithmetic is float only: the crossing parameters reproduce the
// reference's double quotients exactly (rd_alpha_ff), with a double division
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
  float p1x, p1y, ex, ey;
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
  r.ex = __fsub_rn(p2x, p1x);
  r.ey = __fsub_rn(p2y, p1y);
  r.ii0 = rd_round_i(p1x);
  r.jj0 = rd_round_i(p1y);
  r.dx = p2x > p1x ? 1 : -1;
  r.dy = p2y > p1y ? 1 : -1;
  return r;
}

// The double division of rd_alpha_ff, out of line: rarely taken, and its
// double registers stay out of the walk loops.
__device__ __noinline__ float rd_alpha_div(float h, float l, float e) {
  return __double2float_rn(__ddiv_rn(__dadd_rn((double)h, (double)l), (double)e));
}

// alpha of the crossing at the half-integer coordinate a, for a sub-ray that
// enters at p with extent e, r = RN(1/e): the float of the correctly rounded
// double quotient ((double)a - p) / e that the reference computes
// (radon_rd.c:41-42), in float arithmetic.
//
// a - p = h + l exactly (Knuth's TwoSum).  q1 = RN(h r); the remainder
// h + l - q1 e (one FMA, then + l) times r gives q2, and q1 + q2 is within
// 2^-44 |x| of the exact quotient x (r and q1 are within 2^-23 of exact, the
// remainder is 2^-23 |h| small).  With d = 2^-38 |q1|, RN(q1 + RN(q2 - d))
// and RN(q1 + RN(q2 + d)) round points below and above every value within
// 2^-44 |x| of q1 + q2 (the inner roundings move them by 2^-47 at most).
// Rounding to nearest is monotone, so when both give the same float s, x and
// the double nearest x (2^-53 |x| from it) round to s too.  Otherwise (x within
// about 2^-38 of a float rounding boundary, or e zero) divide in double.
__device__ __forceinline__ float rd_alpha_ff(float a, float p, float e, float r) {
  const float h = __fsub_rn(a, p);
  const float bb = __fsub_rn(h, a);
  const float l = __fadd_rn(__fsub_rn(a, __fsub_rn(h, bb)), __fsub_rn(-p, bb));
  const float q1 = __fmul_rn(h, r);
  const float rho = __fadd_rn(__fmaf_rn(-q1, e, h), l);
  const float q2 = __fmul_rn(rho, r);
  const float d = __fmul_rn(fabsf(q1), 0x1p-38f);
  const float lo = __fadd_rn(q1, __fsub_rn(q2, d)), hi = __fadd_rn(q1, __fadd_rn(q2, d));
  if (lo == hi) return lo;
  return rd_alpha_div(h, l, e);
}

// One sub-ray's walk (radon_rd.c:39-70): visit(pi, pj, l) for every credited
// step, (pi, pj) the image row and column stepped into, l the length credited.
template <class Visit>
__device__ __forceinline__ void rd_walk(const RdGeom &s, int n, int nh, Visit visit) {
  const float incr = __fsqrt_rn(__fmaf_rn(s.ex, s.ex, __fmul_rn(s.ey, s.ey)));
  const float hx = s.dx > 0 ? 0.5f : -0.5f, hy = s.dy > 0 ? 0.5f : -0.5f;
  const float fdx = hx + hx, fdy = hy + hy;
  const float rx = __frcp_rn(s.ex), ry = __frcp_rn(s.ey);
  int ii = s.ii0, jj = s.jj0;
  // coordinates of the next x and y crossings, stepped exactly by +-1
  float cx = __fadd_rn((float)s.ii0, hx), cy = __fadd_rn((float)s.jj0, hy);
  float ax = rd_alpha_ff(cx, s.p1x, s.ex, rx), ay = rd_alpha_ff(cy, s.p1y, s.ey, ry);
  float alpha = 0.0f, alpha_old = 0.0f;
  const int guard = 4 * n + 16;  // a walk crosses at most 2n + 2 lines
  for (int it = 0; alpha <= 1.0f && it < guard; ++it) {
    // x step if ax < ay, y step if ax > ay, both if equal (radon_rd.c:45-58);
    // a NaN crossing would never advance the reference: stop.  Written
    // without branches on the step kind, so the lanes of a warp stay together:
    // one new crossing parameter (two on a diagonal step).
    const bool sx = ax <= ay, sy = ay <= ax;
    if (!(sx || sy)) break;
    alpha = sx ? ax : ay;
    ii += sx ? s.dx : 0;
    jj += sy ? s.dy : 0;
    cx = sx ? __fadd_rn(cx, fdx) : cx;
    cy = sy ? __fadd_rn(cy, fdy) : cy;
    const float a1 = rd_alpha_ff(sx ? cx : cy, sx ? s.p1x : s.p1y, sx ? s.ex : s.ey, sx ? rx : ry);
    ax = sx ? a1 : ax;
    ay = sx ? ay : a1;
    if (sx && sy) ay = rd_alpha_ff(cy, s.p1y, s.ey, ry);
    const float l = __fmul_rn(__fsub_rn(alpha, alpha_old), incr);
    const int pi = ii + nh, pj = jj + nh;
    if ((unsigned)(pi - 1) < (unsigned)(n - 1) && (unsigned)(pj - 1) < (unsigned)(n - 1)) visit(pi, pj, l);
    alpha_old = alpha;
  }
}

__global__ void rd_transpose_kernel(const float *__restrict__ in, float *__restrict__ out, int n) {
  __shared__ float tile[32][33];
  const size_t stride = (size_t)n * n;
  const float *src = in + (size_t)blockIdx.z * stride;
  float *dst = out + (size_t)blockIdx.z * stride;
  const int x = blockIdx.x * 32 + threadIdx.x, y0 = blockIdx.y * 32;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y)
    if (x < n && y0 + dy < n) tile[dy][threadIdx.x] = src[(size_t)(y0 + dy) * n + x];
  __syncthreads();
  const int ox = blockIdx.y * 32 + threadIdx.x;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int oy = blockIdx.x * 32 + dy;
    if (ox < n && oy < n) dst[(size_t)oy * n + ox] = tile[threadIdx.x][dy];
  }
}

// Forward over slices z0 + blockIdx.z; imgT holds the chunk's slices transposed.
__global__ void __launch_bounds__(128) rd_forward_kernel(
    const float *__restrict__ img, const float *__restrict__ imgT, float *__restrict__ sino,
    const RdAngle *__restrict__ tab, const float *__restrict__ toff, int n, int nh, int na, int z0, FwdEpi ep) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  const size_t z = (size_t)z0 + blockIdx.z;
  const bool live = b < n;
  const RdAngle g = tab[v];
  const float *I = img + z * (size_t)n * n, *IT = imgT + (size_t)blockIdx.z * n * n;
  float acc = 0.0f;
  if (!live) {
  } else if (g.mode == 1) {  // |s| < 1e-7: bin n-1-i <- column i, i >= 1 (radon_rd.c:96-105)
    const int i = n - 1 - b;
    if (i >= 1)
      for (int j = 0; j < n; ++j) acc += __ldg(I + (size_t)j * n + i);
  } else if (g.mode == 2) {  // |c| < 1e-7: bin i <- row i (:108-117), read down the transposed image
    for (int j = 0; j < n; ++j) acc += __ldg(IT + (size_t)j * n + b);
  } else {
    const bool tr = g.tr != 0;
    const float *P = tr ? IT : I;
    for (int r = 1; r <= 5; ++r) {
      const RdGeom s = rd_geom(rd_offset_tab(toff, 6 * b + r, n, g.lt, g.gt), g, nh);
      rd_walk(s, n, nh, [&](int pi, int pj, float l) {
        acc = fmaf(0.2f * l, __ldg(P + (tr ? (size_t)pj * n + pi : (size_t)pi * n + pj)), acc);
      });
    }
  }
  // store through the epilogue; residual slot as in one launch over all slices
  const size_t e = (z * na + v) * (size_t)n + (live ? b : 0);
  double r2 = 0.0;
  if (live) sino[e] = fwd_apply(ep, acc, e, r2);
  fwd_resid_commit(ep, r2, ((z * gridDim.y + v) * gridDim.x + blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32);
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
      rd_walk(s, n, nh, [&](int pi, int pj, float l) { rd_flag(Fl, (size_t)pi * n + pj, __fmul_rn(0.2f * l, y)); });
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

// Adjoint scatter: slice blockIdx.z of the chunk; accf its fixed-point image,
// accT the transposed one that angles with |s| > |c| add into.
__global__ void __launch_bounds__(128) rd_scatter_kernel(
    const float *__restrict__ sino, unsigned long long *__restrict__ accf, unsigned long long *__restrict__ accT,
    unsigned *__restrict__ flags, const RdAngle *__restrict__ tab, const float *__restrict__ toff, int n, int nh,
    int na, const unsigned *__restrict__ smax) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  const size_t z = blockIdx.z;
  if (b >= n) return;
  const float y = __ldg(sino + (z * na + v) * (size_t)n + b);
  if (y == 0.0f) return;
  const RdAngle g = tab[v];
  if (!(fabsf(y) <= 3.4028235e38f)) {  // inf or NaN
    rd_scatter_nonfinite(y, tab + v, b, n, nh, toff, flags + z * (((size_t)n * n + 3) / 4));
    return;
  }
  const FixedScale fs = rd_adj_scale(smax + z, na);
  unsigned long long *F = accf + z * (size_t)n * n, *FT = accT + z * (size_t)n * n;
  if (g.mode == 1) {  // column n-1-b, every row (transpose of radon_rd.c:96-105)
    const int i = n - 1 - b;
    if (i >= 1) {
      const unsigned long long q = fixed_of(y, fs);
      for (int j = 0; j < n; ++j) atomicAdd(F + (size_t)j * n + i, q);
    }
    return;
  }
  if (g.mode == 2) {  // row b, every column (:108-117), down the transposed image
    const unsigned long long q = fixed_of(y, fs);
    for (int j = 0; j < n; ++j) atomicAdd(FT + (size_t)j * n + b, q);
    return;
  }
  const bool tr = g.tr != 0;
  unsigned long long *P = tr ? FT : F;
  // y 2^E: scaling by a power of two commutes with the rounding of the
  // product, so each credit is fixed_of(0.2 l y) with one multiply fewer
  const float ys = __fmul_rn(__fmul_rn(y, fs.s1), fs.s2);
  for (int r = 1; r <= 5; ++r) {
    const RdGeom s = rd_geom(rd_offset_tab(toff, 6 * b + r, n, g.lt, g.gt), g, nh);
    rd_walk(s, n, nh, [&](int pi, int pj, float l) {
      atomicAdd(P + (tr ? (size_t)pj * n + pi : (size_t)pi * n + pj),
                (unsigned long long)__float2ll_rn(__fmul_rn(0.2f * l, ys)));
    });
  }
}

// accf + accT transposed -> float through the adjoint epilogue, a 32 x 32 tile
// per block (blockDim 32 x 8); slice blockIdx.z of the chunk is slice z0 + it.
__global__ void rd_finalize_kernel(const unsigned long long *__restrict__ accf,
                                   const unsigned long long *__restrict__ accT, const unsigned *__restrict__ flags,
                                   float *__restrict__ img, int n, int z0, int na, const unsigned *__restrict__ smax,
                                   AdjEpi ep) {
  __shared__ unsigned long long tile[32][33];
  const size_t zl = blockIdx.z, per = (size_t)n * n;
  const unsigned long long *F = accf + zl * per, *FT = accT + zl * per;
  const int R0 = blockIdx.y * 32, C0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y)  // tile[c][r] = accT[(C0 + c) n + R0 + r]
    if (C0 + k < n && R0 + threadIdx.x < n) tile[k][threadIdx.x] = FT[(size_t)(C0 + k) * n + R0 + threadIdx.x];
  __syncthreads();
  const FixedScale fs = rd_adj_scale(smax + zl, na);
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int R = R0 + k, C = C0 + threadIdx.x;
    const bool live = R < n && C < n;
    float val = 0.0f;
    if (live) {
      const size_t p = (size_t)R * n + C;
      const unsigned f = (flags[zl * ((per + 3) / 4) + (p >> 2)] >> (8u * (unsigned)(p & 3))) & 0xffu;
      val = f == 0u ? fixed_to_float(F[p] + tile[threadIdx.x][k], fs) : nonfinite_value(f);
    }
    adj_store(ep, val, live, ((size_t)z0 + zl) * per + (live ? (size_t)R * n + C : 0), img);
  }
}

// slices per chunk: the adjoint's two fixed-point images and flag bytes (the
// forward's transposed image uses the same space) of at most 512 MiB, and no
// more than a grid dimension holds
size_t rd_flag_words(const Plan &p) { return ((size_t)p.g.n * p.g.n + 3) / 4; }

int rd_chunk(const Plan &p) {
  const size_t per = (size_t)16 * p.g.n * p.g.n + 4 * rd_flag_words(p);
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
  // scratch: a chunk of fixed-point images, of transposed ones and of flag
  // bytes (the forward's transposed images in the same space), then max |y|
  // per slice
  p.scratch_bytes = ((size_t)16 * n * n + 4 * rd_flag_words(p)) * rd_chunk(p) + sizeof(unsigned) * (size_t)p.g.nz;
  TOMO_CUDA(cudaMalloc(&p.d_scratch, p.scratch_bytes));
  return TOMO_OK;
}

int rd_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz, chunk = rd_chunk(p);
  float *imgT = p.d_scratch;
  for (int z0 = 0; z0 < nz; z0 += chunk) {
    const int zc = std::min(chunk, nz - z0);
    rd_transpose_kernel<<<dim3((n + 31) / 32, (n + 31) / 32, zc), dim3(32, 8), 0, s>>>(
        d_img + (size_t)z0 * n * n, imgT, n);
    rd_forward_kernel<<<dim3((n + 127) / 128, na, zc), 128, 0, s>>>(
        d_img, imgT, d_sino, (const RdAngle *)p.d_angles, (const float *)p.d_aux, n, p.nh, na, z0, ep);
  }
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int rd_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s, const AdjEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz, chunk = rd_chunk(p);
  const size_t per_img = (size_t)n * n, per_sino = (size_t)na * n;
  unsigned long long *accf = reinterpret_cast<unsigned long long *>(p.d_scratch);
  unsigned long long *accT = accf + (size_t)chunk * per_img;
  const size_t fw = rd_flag_words(p);
  unsigned *flags = reinterpret_cast<unsigned *>(accT + (size_t)chunk * per_img);
  unsigned *smax = flags + (size_t)chunk * fw;
  TOMO_CUDA(cudaMemsetAsync(smax, 0, sizeof(unsigned) * (size_t)nz, s));
  for (int z0 = 0; z0 < nz; z0 += chunk) {
    const int zc = std::min(chunk, nz - z0);
    fixed_finite_absmax_kernel<<<dim3(64, zc), 256, 0, s>>>(d_sino + (size_t)z0 * per_sino, per_sino, smax + z0);
    TOMO_CUDA(cudaMemsetAsync(accf, 0, sizeof(unsigned long long) * zc * per_img, s));
    TOMO_CUDA(cudaMemsetAsync(accT, 0, sizeof(unsigned long long) * zc * per_img, s));
    TOMO_CUDA(cudaMemsetAsync(flags, 0, sizeof(unsigned) * zc * fw, s));
    rd_scatter_kernel<<<dim3((n + 127) / 128, na, zc), 128, 0, s>>>(
        d_sino + (size_t)z0 * per_sino, accf, accT, flags, (const RdAngle *)p.d_angles, (const float *)p.d_aux, n,
        p.nh, na, smax + z0);
    rd_finalize_kernel<<<dim3((n + 31) / 32, (n + 31) / 32, zc), dim3(32, 8), 0, s>>>(
        accf, accT, flags, d_img, n, z0, na, smax + z0, ep);
  }
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
