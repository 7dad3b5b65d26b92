// Gridding (Fourier-slice) projector pair for sm_100a.
//
// Reference: common/operators/gridrec_module/pymodule_gridrec_v4/
// gridrec_v4_forwproj.c:59-442, gridrec_v4_backproj.c:64-511, filters.c:143-296.
//
// Forward (gridrec_v4_forwproj.c):
//   H[iu][iv] = deapod[j][k] * image[npix-1-(k-padleft)][j-padleft] inside the
//     padded square, iu = (j + pdim/2) mod pdim (:213-248);
//   H <- unnormalised 2-D FFT, sign +1 (:256-259)                 [cuFFT]
//   per angle and frequency w < pdim/2: the polar sample at
//     U = w cos + pdim/2, V = w sin + pdim/2 gathers H (and its mirror
//     H[pdim-iu][pdim-iv]) over the window [ceil(U-h), floor(U+h)] x [..V..]
//     with weights lut(|U-iu| s) lut(|V-iv| s) (:271-380), times the centring
//     phase filter (:188-205, 363-379); lconv is fixed at 2*7/pi (:159);
//   1-D FFT of each polar row, sign -1 (:390); the real part of the centre
//     npix samples, times 1/pdim, is the projection (:397-398).   [hand-written]
// Adjoint (gridrec_v4_backproj.c): edge-padded projection (:262-292), 1-D FFT
//   (:301), filter and centring phase (:312-344), window scatter into H and its
//   mirror (:389-409) -- here a deterministic GATHER over the polar samples
//   whose window contains each Cartesian point --, 2-D FFT (:427), deapodise,
//   crop and flip (:440-491).  lconv is param[6] here (:124,180-183).
//
// Float evaluation follows the compiled reference (-O3 -ffast-math): angles via
// double sincos of deg*(pi/180); U = fma(cos, w, pdim/2); window bounds by float
// ceil/floor; lut argument |V - iv| * tblspcg; convolv_lin as
// fma((1 - x) + floor x, lut[i], (x - floor x) * lut[i+1]); nearest as
// lut[(int)(x + 0.49999997f)]; complex products as the compiler fused them.
// The reference stores the window's lower bound in an unsigned long, so a
// negative bound (samples near the grid edge at angles near 180 degrees)
// turns its loop into a no-op: such samples contribute nothing, here too.
//
// Matched adjoint (grid_mode 1): the exact transpose of the forward above,
// so that <A x, y> = <x, A^T y>.  The forward is y = Re(P x) with P complex-
// linear, hence A^T y = Re(P^H y): the projection zero-padded (the adjoint of
// the crop) and scaled by 1/pdim; its 1-D DFT with sign +1 (for a real row,
// the conjugate of the sign -1 transform); per polar sample the values the
// forward's two gathers took, f_w rho[pdim - w] for the window and
// conj(f_w) rho[w] for its mirror (f the forward's centring filter); the
// forward's window (lconv 2*7/pi, same LUT, same skip rules) gathered back into
// H; the 2-D DFT with sign -1; the forward's deapodisation, crop and flip.
//
// Only the 2-D transform uses cuFFT; the per-projection 1-D transforms are a
// mixed-radix Stockham FFT in shared memory (radix 4/2/3/5/7 and generic odd
// primes; Govindaraju et al., SC'08 formulation).
#include <cufft.h>
#include <cstring>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>
#include <vector>

#include "tomo_internal.cuh"

namespace tomo {

struct GridState {
  int pdim = 0, pdim_h = 0, padleft = 0, padright = 0;
  int interp = 0, radon_degree = 0, ltbl = 0, lut_len = 0;
  float h_f = 0, tbl_f = 0;  // forward: lconv/2 and table spacing
  float h_b = 0, tbl_b = 0;  // adjoint
  float inv_pdim = 0;        // float(1.0/pdim)
  bool matched = false;      // grid_mode 1: the adjoint is the forward's exact transpose
  int nfac = 0;
  int fac[32] = {0};
  float *lut = nullptr, *deapod = nullptr;
  float2 *sc = nullptr;       // per angle (sin, cos)
  float2 *filt_f = nullptr;   // forward centring filter [pdim/2]
  float2 *filt_b = nullptr;   // adjoint filter [pdim/2]
  float2 *tw = nullptr;       // exp(-2 pi i t / pdim), t < pdim
  float2 *sorted = nullptr;   // adjoint gather: (polar angle, angle index as float bits), sorted
  float4 *sc4 = nullptr;      // adjoint gather: per angle (sin, cos, 1/cos, 1/sin)
  float2 *H = nullptr;        // [nz][pdim][pdim]
  float2 *rows = nullptr;     // [nz][na][pdim]
  float4 *cd = nullptr;       // [nz][na][pdim/2]: Cdata1, Cdata2
  cufftHandle fft2 = 0;
  bool have_fft = false;
};

namespace {

constexpr double kPi = 3.141592653589793;
constexpr int kFftThreads = 256;
constexpr int kMaxWin = 8;

struct FftConst {
  int n, nfac;
  int fac[32];
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-place (ping-pong) Stockham FFT of one row in shared memory, sign -1.
// Returns the buffer holding the result.
__device__ float2 *stockham(float2 *a, float2 *b, const FftConst &c, const float2 *__restrict__ tw) {
  const int N = c.n;
  int Ns = 1;
  for (int s = 0; s < c.nfac; ++s) {
    const int R = c.fac[s];
    const int NR = N / R, span = N / (Ns * R);
    for (int j = threadIdx.x; j < NR; j += blockDim.x) {
      const int jm = j % Ns;
      float2 v[16];
      float2 out[16];
      if (R <= 16) {
        for (int r = 0; r < R; ++r) {
          float2 x = a[j + r * NR];
          if (r) x = cmul(x, __ldg(tw + ((long long)r * jm * span) % N));
          v[r] = x;
        }
        if (R == 2) {
          out[0] = make_float2(v[0].x + v[1].x, v[0].y + v[1].y);
          out[1] = make_float2(v[0].x - v[1].x, v[0].y - v[1].y);
        } else if (R == 4) {
          const float2 s0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
          const float2 d0 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
          const float2 s1 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
          const float2 d1 = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
          out[0] = make_float2(s0.x + s1.x, s0.y + s1.y);
          out[2] = make_float2(s0.x - s1.x, s0.y - s1.y);
          out[1] = make_float2(d0.x + d1.y, d0.y - d1.x);  // d0 - i d1
          out[3] = make_float2(d0.x - d1.y, d0.y + d1.x);  // d0 + i d1
        } else {
          for (int k = 0; k < R; ++k) {
            float2 acc = v[0];
            for (int q = 1; q < R; ++q) {
              const float2 w = __ldg(tw + ((long long)(N / R) * ((q * k) % R)) % N);
              const float2 t = cmul(v[q], w);
              acc.x += t.x;
              acc.y += t.y;
            }
            out[k] = acc;
          }
        }
        const int base = (j / Ns) * Ns * R + jm;
        for (int r = 0; r < R; ++r) b[base + r * Ns] = out[r];
      } else {  // large prime radix: generic DFT straight from the input
        const int base = (j / Ns) * Ns * R + jm;
        for (int k = 0; k < R; ++k) {
          float2 acc = make_float2(0, 0);
          for (int q = 0; q < R; ++q) {
            float2 x = a[j + q * NR];
            if (q) x = cmul(x, __ldg(tw + ((long long)q * jm * span) % N));
            const float2 w = __ldg(tw + ((long long)(N / R) * ((q * k) % R)) % N);
            const float2 t = cmul(x, w);
            acc.x += t.x;
            acc.y += t.y;
          }
          b[base + k * Ns] = acc;
        }
      }
    }
    __syncthreads();
    float2 *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

__device__ __forceinline__ float lut_eval(const float *__restrict__ lut, float x, int interp) {
  if (interp == 0) return __ldg(lut + (int)__fadd_rn(x, 0.49999997f));  // convolv_nn, x >= 0
  const float fl = floorf(x);
  const int i = (int)fl;
  const float w0 = __fadd_rn(__fsub_rn(1.0f, x), fl), d = __fsub_rn(x, fl);
  return __fmaf_rn(w0, __ldg(lut + i), __fmul_rn(d, __ldg(lut + i + 1)));  // convolv_lin
}

// Forward step 1: deapodised, transposed and flipped image into the quadrant-
// swapped Fourier grid (gridrec_v4_forwproj.c:213-248).
__global__ void grid_fill_kernel(const float *__restrict__ img, float2 *__restrict__ H,
                                 const float *__restrict__ deapod, int pdim, int pdim_h, int padleft,
                                 int npix) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const size_t z = blockIdx.z;
  if (j >= pdim || k >= pdim) return;
  const int iu = j < pdim_h ? j + (pdim - pdim_h) : j - pdim_h;
  const int iv = k < pdim_h ? k + (pdim - pdim_h) : k - pdim_h;
  float v = 0.0f;
  if (j >= padleft && j < padleft + npix && k >= padleft && k < padleft + npix)
    v = __fmul_rn(__ldg(deapod + (size_t)j * pdim + k),
                  __ldg(img + z * (size_t)npix * npix + (size_t)(npix - 1 - (k - padleft)) * npix + (j - padleft)));
  H[z * (size_t)pdim * pdim + (size_t)iu * pdim + iv] = make_float2(v, 0.0f);
}

// Forward step 3: one thread per polar sample (frequency w, angle n, slice).
__global__ void __launch_bounds__(128) grid_polar_kernel(
    const float2 *__restrict__ H, float2 *__restrict__ rows, const float2 *__restrict__ sc,
    const float2 *__restrict__ filt, const float *__restrict__ lut, int pdim, int pdim_h, int na,
    float h, float tbl, int interp) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = blockIdx.y;
  const size_t z = blockIdx.z;
  if (w >= pdim_h) return;
  const float2 ang = sc[n];
  const float SIN = ang.x, COS = ang.y, fph = (float)pdim_h;
  const float U = __fmaf_rn(COS, (float)w, fph), V = __fmaf_rn(SIN, (float)w, fph);
  const float cu = ceilf(__fsub_rn(U, h)), fu = floorf(__fadd_rn(h, U));
  const float cv = ceilf(__fsub_rn(V, h)), fv = floorf(__fadd_rn(V, h));
  float2 c1 = make_float2(0, 0), c2 = make_float2(0, 0);
  if (cu >= 0.0f && cv >= 0.0f) {
    const int iul = (int)cu, ivl = (int)cv;
    const int iuh = min((int)fu, pdim - 1), ivh = min((int)fv, pdim - 1);
    const float2 *Hz = H + z * (size_t)pdim * pdim;
    float work[kMaxWin];
    for (int iv = ivl, q = 0; iv <= ivh && q < kMaxWin; ++iv, ++q)
      work[q] = lut_eval(lut, __fmul_rn(fabsf(__fsub_rn(V, (float)iv)), tbl), interp);
    for (int iu = iul; iu <= iuh; ++iu) {
      const float rt = lut_eval(lut, __fmul_rn(fabsf(__fsub_rn(U, (float)iu)), tbl), interp);
      for (int iv = ivl, q = 0; iv <= ivh && q < kMaxWin; ++iv, ++q) {
        const float conv = __fmul_rn(rt, work[q]);
        const float2 h1 = Hz[(size_t)iu * pdim + iv];
        c1.x = __fmaf_rn(h1.x, conv, c1.x);
        c1.y = __fmaf_rn(h1.y, conv, c1.y);
        if (iu != 0 && iv != 0 && w != 0) {
          const float2 h2 = Hz[(size_t)(pdim - iu) * pdim + (pdim - iv)];
          c2.x = __fmaf_rn(h2.x, conv, c2.x);
          c2.y = __fmaf_rn(h2.y, conv, c2.y);
        }
      }
    }
  }
  const float2 f = filt[w];
  const float cr = f.x, ci = -f.y;
  float2 *row = rows + (z * na + n) * (size_t)pdim;
  const float2 o1 = make_float2(__fmaf_rn(cr, c1.x, -__fmul_rn(ci, c1.y)),
                                __fmaf_rn(c1.y, cr, __fmul_rn(ci, c1.x)));
  if (w != 0) {
    row[pdim - w] = o1;
    row[w] = make_float2(__fmaf_rn(cr, c2.x, -__fmul_rn(f.y, c2.y)),
                         __fmaf_rn(cr, c2.y, __fmul_rn(f.y, c2.x)));
  } else {
    row[0] = o1;
    row[pdim_h] = make_float2(0, 0);
  }
}

// Forward step 4: FFT each polar row; projection = Re(out[padleft + k]) / pdim.
__global__ void __launch_bounds__(kFftThreads) grid_fft_fwd_kernel(
    const float2 *__restrict__ rows, float *__restrict__ sino, const float2 *__restrict__ tw,
    FftConst c, int na, int npix, int padleft, float inv_pdim, FwdEpi ep) {
  extern __shared__ float2 sm[];
  float2 *a = sm, *b = sm + c.n;
  const size_t row = blockIdx.x;  // z * na + n
  const float2 *src = rows + row * c.n;
  for (int i = threadIdx.x; i < c.n; i += blockDim.x) a[i] = src[i];
  __syncthreads();
  const float2 *o = stockham(a, b, c, tw);
  double r2 = 0.0;
  for (int k = threadIdx.x; k < npix; k += blockDim.x) {
    const float acc = __fmul_rn(inv_pdim, o[padleft + k].x);
    const size_t e = row * npix + k;
    float out = acc;
    if (ep.op != EPI_NONE) {
      const float bv = __ldg(ep.b + e);
      if (ep.op == EPI_SIRT) out = __fmul_rn(__ldg(ep.w + e), __fsub_rn(bv, acc));
      else if (ep.op == EPI_MLEM) out = __fdiv_rn(bv, acc == 0.0f ? kSpacing32 : acc);
      else out = __fmul_rn(__fsub_rn(acc, bv), __ldg(ep.w + e));
      const double d = (double)acc - (double)bv;
      r2 += d * d;
    }
    sino[e] = out;
  }
  if (ep.resid) {
    for (int off = 16; off; off >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, off);
    if ((threadIdx.x & 31) == 0) ep.resid[row * (kFftThreads / 32) + threadIdx.x / 32] = r2;
  }
}

// Adjoint step 1: edge-padded projection -> FFT -> filtered half spectrum,
// Cdata1 (from bin pdim-j) and Cdata2 (from bin j), gridrec_v4_backproj.c:262-344.
__global__ void __launch_bounds__(kFftThreads) grid_fft_adj_kernel(
    const float *__restrict__ sino, float4 *__restrict__ cd, const float2 *__restrict__ tw,
    const float2 *__restrict__ filt, FftConst c, int npix, int padleft, int pdim_h,
    int radon_degree, float tmp2) {
  extern __shared__ float2 sm[];
  float2 *a = sm, *b = sm + c.n;
  const size_t row = blockIdx.x;
  const float *src = sino + row * npix;
  const int padright = padleft + npix;
  for (int i = threadIdx.x; i < c.n; i += blockDim.x) {
    float v;
    if (i < padleft) v = radon_degree ? 0.0f : src[0];
    else if (i < padright) v = src[i - padleft];
    else v = radon_degree ? 0.0f : src[npix - 1];
    a[i] = make_float2(v, 0.0f);
  }
  __syncthreads();
  const float2 *o = stockham(a, b, c, tw);
  float4 *dst = cd + row * pdim_h;
  for (int j = threadIdx.x; j < pdim_h; j += blockDim.x) {
    const float2 f = filt[j];
    const float2 t2 = make_float2(__fmul_rn(tmp2, o[j].x), __fmul_rn(tmp2, o[j].y));
    float4 r;
    if (j != 0) {
      const float2 t3 = make_float2(__fmul_rn(tmp2, o[c.n - j].x), __fmul_rn(tmp2, o[c.n - j].y));
      r.x = __fmaf_rn(f.x, t3.x, -__fmul_rn(f.y, t3.y));
      r.y = __fmaf_rn(f.x, t3.y, __fmul_rn(f.y, t3.x));
      const float ci = -f.y;
      r.z = __fmaf_rn(f.x, t2.x, -__fmul_rn(ci, t2.y));
      r.w = __fmaf_rn(f.x, t2.y, __fmul_rn(ci, t2.x));
    } else {
      r.x = __fmul_rn(f.x, t2.x);
      r.y = __fmul_rn(f.x, t2.y);
      r.z = 0.0f;
      r.w = 0.0f;
    }
    dst[j] = r;
  }
}

// Matched adjoint step 1: rho = the projection zero-padded to pdim and scaled
// by 1/pdim, o = its sign -1 DFT; rho^ = conj(o) is the sign +1 DFT, and by
// the Hermitian symmetry of a real row conj(o[pdim - w]) = o[w].  cd[w] =
// {f_w rho^[pdim - w] (window), conj(f_w) rho^[w] (mirror, w != 0)}.
__global__ void __launch_bounds__(kFftThreads) grid_fft_adj_matched_kernel(
    const float *__restrict__ sino, float4 *__restrict__ cd, const float2 *__restrict__ tw,
    const float2 *__restrict__ filt, FftConst c, int npix, int padleft, int pdim_h, float scale) {
  extern __shared__ float2 sm[];
  float2 *a = sm, *b = sm + c.n;
  const size_t row = blockIdx.x;
  const float *src = sino + row * npix;
  for (int i = threadIdx.x; i < c.n; i += blockDim.x) {
    const int k = i - padleft;
    a[i] = make_float2(k >= 0 && k < npix ? __fmul_rn(scale, src[k]) : 0.0f, 0.0f);
  }
  __syncthreads();
  const float2 *o = stockham(a, b, c, tw);
  float4 *dst = cd + row * pdim_h;
  for (int w = threadIdx.x; w < pdim_h; w += blockDim.x) {
    const float2 f = filt[w], d = o[w];                       // rho^[pdim - w] = o[w]
    float4 r;
    r.x = __fmaf_rn(f.x, d.x, -__fmul_rn(f.y, d.y));
    r.y = __fmaf_rn(f.x, d.y, __fmul_rn(f.y, d.x));
    if (w != 0) {
      const float2 m = o[c.n - w];                            // rho^[w] = o[pdim - w]
      r.z = __fmaf_rn(f.x, m.x, __fmul_rn(f.y, m.y));        // conj(f) m
      r.w = __fmaf_rn(f.x, m.y, -__fmul_rn(f.y, m.x));
    } else {
      r.z = 0.0f;
      r.w = 0.0f;
    }
    dst[w] = r;
  }
}

// floor(x) for 0 <= x < 2^23 without the conversion pipe: x + 2^23 rounded
// down is 2^23 + floor(x) exactly (unit spacing in [2^23, 2^24)).
__device__ __forceinline__ float floor_small(float x, int &i) {
  const float t = __fadd_rd(x, 8388608.0f);
  i = __float_as_int(t) - 0x4B000000;
  return __fsub_rn(t, 8388608.0f);
}

// lut_eval with the floor / truncation on the FMA pipe (x >= 0, same values).
__device__ __forceinline__ float lut_eval_fast(const float *__restrict__ lut, float x, int interp) {
  int i;
  if (interp == 0) {
    floor_small(__fadd_rn(x, 0.49999997f), i);
    return __ldg(lut + i);
  }
  const float fl = floor_small(x, i);
  const float w0 = __fadd_rn(__fsub_rn(1.0f, x), fl), d = __fsub_rn(x, fl);
  return __fmaf_rn(w0, __ldg(lut + i), __fmul_rn(d, __ldg(lut + i + 1)));
}

// Adjoint step 2: every Cartesian point gathers the polar samples whose
// window contains it (directly, or through the mirror H[pdim-iu][pdim-iv]).
//
// The reference's window of sample (U, V) is [ceil(U-h), min(floor(U+h),
// pdim-1)] x [..V..], and the sample is skipped when ceil(U-h) < 0 or
// ceil(V-h) < 0.  For an integer t, ceil(a) <= t <=> a <= t, t <= floor(b) <=>
// t <= b and ceil(a) < 0 <=> a <= -1, so membership is decided by float
// compares of the same rounded a = U - h, b = U + h.  Per angle only the w
// with COS w and SIN w within h (+1 of margin, far above the rounding of U,
// V and of the reciprocals) of the target's offsets are visited.
//
// Angles are visited in polar-angle order from the start of the target's
// angular window (all angles when the target is within reach of the
// centre), w ascending; a lane handles every STRIDE-th angle of that order.
constexpr int kGatherCentre = 48;  // half-size of the central box of the adjoint gather

struct GatherArgs {
  const float4 *cd;       // [nz][na][pdim_h] direct (x, y) and mirror (z, w) values
  float2 *H;              // [nz][pdim][pdim]
  const float4 *sc4;      // per angle (sin, cos, 1/cos, 1/sin)
  const float2 *sorted;   // (polar angle, angle index as float bits), ascending
  const float *lut;
  int pdim, pdim_h, na, interp, centre;  // centre: half-size of the box done by warps
  float h, tbl;
};

template <int STRIDE>
__device__ __forceinline__ void gather_point(const GatherArgs &A, int IU, int IV, size_t z, int lane, float &hr,
                                             float &hi) {
  const float4 *cdz = A.cd + z * (size_t)A.na * A.pdim_h;
  const int pdim = A.pdim, pdim_h = A.pdim_h, na = A.na;
  const float h = A.h, fph = (float)pdim_h;
  const float reach = h * 1.41421356f + 1.0f;
  for (int mirror = 0; mirror < 2; ++mirror) {
    // the window point the sample must contain, and its offset from the centre
    const int tu = mirror ? pdim - IU : IU, tv = mirror ? pdim - IV : IV;
    if (mirror && (IU == 0 || IV == 0)) continue;  // targets pdim - 0 are outside the grid
    const float ftu = (float)tu, ftv = (float)tv;
    const float du = (float)(tu - pdim_h), dv = (float)(tv - pdim_h);
    const float rho = sqrtf(du * du + dv * dv);
    const bool windowed = rho > reach + 1.0f;
    int a0 = 0;
    float phi = 0.0f, dmax = 0.0f;
    if (windowed) {
      phi = atan2f(dv, du);
      if (phi < 0.0f) phi += 6.2831853f;
      dmax = asinf(fminf(1.0f, reach / rho)) + 1e-3f;
      // first sorted angle >= phi - dmax (with wrap-around)
      float lo = phi - dmax;
      if (lo < 0.0f) lo += 6.2831853f;
      int l = 0, r = na;
      while (l < r) {
        const int m = (l + r) >> 1;
        if (A.sorted[m].x < lo) l = m + 1;
        else r = m;
      }
      a0 = l;
    }
    const float wbase = mirror ? 1.0f : 0.0f;
    // the in-window angles are a prefix of the cyclic order from a0
    for (int t = lane; t < na; t += STRIDE) {
      int si = a0 + t;
      if (si >= na) si -= na;
      const float2 e = A.sorted[si];
      if (windowed) {
        // Stop once past the window.  The test is looser than the window by
        // far more than the float rounding of lo = phi - dmax and of e.x - phi:
        // the search starts at the first angle >= lo, which the exact test
        // could judge just outside and so end the scan before the window.
        // Which samples count is decided below, per sample, whatever this.
        float dphi = fabsf(e.x - phi);
        dphi = fminf(dphi, 6.2831853f - dphi);
        if (dphi > dmax + 1e-5f) break;  // left the window
      }
      const int n = __float_as_int(e.y);
      const float4 ang = A.sc4[n];  // SIN, COS, 1/COS, 1/SIN
      const float SIN = ang.x, COS = ang.y;
      const float tt = du * COS + dv * SIN;  // along-ray position of the target
      float lo = tt - reach, hi2 = tt + reach;
      if (fabsf(COS) >= 1e-2f) {
        const float a = (du - h) * ang.z, b = (du + h) * ang.z;
        lo = fmaxf(lo, fminf(a, b) - 1.0f);
        hi2 = fminf(hi2, fmaxf(a, b) + 1.0f);
      }
      if (fabsf(SIN) >= 1e-2f) {
        const float a = (dv - h) * ang.w, b = (dv + h) * ang.w;
        lo = fmaxf(lo, fminf(a, b) - 1.0f);
        hi2 = fminf(hi2, fmaxf(a, b) + 1.0f);
      }
      lo = fmaxf(ceilf(lo), wbase);
      hi2 = fminf(floorf(hi2), (float)(pdim_h - 1));
      if (lo > hi2) continue;
      int w = (int)lo;
      for (float wf = lo; wf <= hi2; wf += 1.0f, ++w) {
        const float U = __fmaf_rn(COS, wf, fph), V = __fmaf_rn(SIN, wf, fph);
        const float ua = __fsub_rn(U, h), va = __fsub_rn(V, h);
        if (ua <= -1.0f || va <= -1.0f) continue;  // the reference skips this sample entirely
        if (ua > ftu || __fadd_rn(h, U) < ftu || va > ftv || __fadd_rn(V, h) < ftv) continue;
        const float rt = lut_eval_fast(A.lut, __fmul_rn(fabsf(__fsub_rn(U, ftu)), A.tbl), A.interp);
        const float wk = lut_eval_fast(A.lut, __fmul_rn(fabsf(__fsub_rn(V, ftv)), A.tbl), A.interp);
        const float conv = __fmul_rn(rt, wk);
        const float4 c = cdz[(size_t)n * pdim_h + w];
        if (!mirror) {
          hr = __fmaf_rn(conv, c.x, hr);
          hi = __fmaf_rn(conv, c.y, hi);
        } else if (tu != 0 && tv != 0 && w != 0) {
          hr = __fmaf_rn(conv, c.z, hr);
          hi = __fmaf_rn(conv, c.w, hi);
        }
      }
    }
  }
}

// One thread per Cartesian point outside the central box.
__global__ void __launch_bounds__(128) grid_gather_kernel(GatherArgs A) {
  const int IV = blockIdx.x * blockDim.x + threadIdx.x;
  const int IU = blockIdx.y;
  const size_t z = blockIdx.z;
  if (IV >= A.pdim) return;
  if (abs(IU - A.pdim_h) <= A.centre && abs(IV - A.pdim_h) <= A.centre) return;  // grid_gather_centre_kernel
  float hr = 0.0f, hi = 0.0f;
  gather_point<1>(A, IU, IV, z, 0, hr, hi);
  A.H[z * (size_t)A.pdim * A.pdim + (size_t)IU * A.pdim + IV] = make_float2(hr, hi);
}

// One warp per point of the central box, where every angle's first samples
// overlap and a point gathers thousands of them: lanes take every 32nd angle
// and the partial sums are combined by a fixed butterfly (deterministic).
__global__ void __launch_bounds__(128) grid_gather_centre_kernel(GatherArgs A) {
  const int side = 2 * A.centre + 1;
  const int p = blockIdx.x * 4 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  const size_t z = blockIdx.y;
  if (p >= side * side) return;  // warp-uniform
  const int IU = A.pdim_h - A.centre + p / side, IV = A.pdim_h - A.centre + p % side;
  float hr = 0.0f, hi = 0.0f;
  gather_point<32>(A, IU, IV, z, lane, hr, hi);
  for (int off = 16; off; off >>= 1) {
    hr = __fadd_rn(hr, __shfl_xor_sync(0xffffffffu, hr, off));
    hi = __fadd_rn(hi, __shfl_xor_sync(0xffffffffu, hi, off));
  }
  if (lane == 0) A.H[z * (size_t)A.pdim * A.pdim + (size_t)IU * A.pdim + IV] = make_float2(hr, hi);
}

// Adjoint step 4: deapodise, crop and flip (gridrec_v4_backproj.c:440-491).
__global__ void __launch_bounds__(256) grid_extract_kernel(const float2 *__restrict__ H,
                                                           float *__restrict__ img,
                                                           const float *__restrict__ deapod, int pdim,
                                                           int pdim_h, int padleft, int npix, AdjEpi ep) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;  // image column
  const int r = blockIdx.y * blockDim.y + threadIdx.y;  // image row
  const size_t z = blockIdx.z;
  const bool live = r < npix && c < npix;
  float v = 0.0f;
  if (live) {
    const int j = c + padleft, k = padleft + npix - 1 - r;
    const int iu = j < pdim_h ? j + (pdim - pdim_h) : j - pdim_h;
    const int iv = k < pdim_h ? k + (pdim - pdim_h) : k - pdim_h;
    v = __fmul_rn(__ldg(deapod + (size_t)j * pdim + k), H[z * (size_t)pdim * pdim + (size_t)iu * pdim + iv].x);
  }
  adj_store(ep, v, live, z * (size_t)npix * npix + (size_t)(live ? r : 0) * npix + (live ? c : 0), img);
}

// ---- host helpers ----
std::vector<int> factorize(int n) {
  std::vector<int> f;
  while (n % 4 == 0) { f.push_back(4); n /= 4; }
  while (n % 2 == 0) { f.push_back(2); n /= 2; }
  for (int p = 3; n > 1; p += 2)
    while (n % p == 0) { f.push_back(p); n /= p; }
  return f;
}

// filters.c:17-38 ramp kernel, its unnormalised FFT magnitude (double here)
std::vector<float> ramp_magnitude(int N) {
  std::vector<double> re(N), mag(N, 0.0);
  const int sizeH = (int)(N * 0.5);
  for (int i = 0; i < N; ++i) {
    const int c = i - (sizeH - 1);
    if (c == 0) re[i] = 0.25;
    else if (c % 2 == 0) re[i] = 0.0;
    else re[i] = -1.0 / (kPi * kPi * c * c);
    re[i] = (double)(float)re[i];
  }
  std::vector<float> out(N, 0.0f);
  for (int k = 0; k < N / 2; ++k) {
    double sr = 0, si = 0;
    for (int i = 0; i < N; ++i) {
      const double a = -2.0 * kPi * (double)(((long long)i * k) % N) / N;
      sr += re[i] * std::cos(a);
      si += re[i] * std::sin(a);
    }
    out[k] = (float)std::sqrt((double)(float)sr * (float)sr + (double)(float)si * (float)si);
  }
  return out;
}

float filter_add(int type, float x, float fm) {
  switch (type) {
    case 2: {  // shepp_logan
      const float ffm = (float)(x / (2. * fm));
      if (x == 0) return 1.0f;
      if (x < fm) return (float)(std::sin(kPi * ffm) / (kPi * ffm));
      return 0.0f;
    }
    case 3: {  // hanning
      const float ffm = x / fm;
      return std::fabs(x) <= fm ? (float)(0.5 * (1.0 + std::cos(kPi * ffm))) : 0.0f;
    }
    case 4: {  // hamming
      const float ffm = x / fm;
      return std::fabs(x) <= fm ? (float)(0.54 + 0.46 * std::cos(kPi * ffm)) : 0.0f;
    }
    case 5: {  // lanczos
      const float ffm = x / fm;
      if (x == 0) return 1.0f;
      if (x < fm) return (float)(std::sin(kPi * ffm) / (kPi * ffm));
      return 0.0f;
    }
    case 6: {  // parzen
      const float ffm = std::fabs(x) / fm;
      if (std::fabs(x) <= fm / 2.) return (float)(1 - 6 * ffm * ffm * (1 - ffm));
      if (std::fabs(x) > fm / 2. && std::fabs(x) <= fm) return (float)(2 * (1 - ffm) * (1 - ffm) * (1 - ffm));
      return 0.0f;
    }
  }
  return 1.0f;
}

// calc_filter (filters.c:143-277) for flag_filter == 0; pairs (filter[2k], filter[2k+1]).
std::vector<float2> calc_filter(int nang, int N, float center, int type, int radon_degree) {
  std::vector<float> ramp;
  if (type && radon_degree == 0) ramp = ramp_magnitude(N);
  const float fw = 1.0f, fm = 0.5f;
  const float rtmp1 = (float)(2 * kPi * center / N);
  const float norm = (float)(kPi / N / nang);
  std::vector<float2> f(N / 2);
  for (int j = 0, k = 0; j < N; j += 2, ++k) {
    const float x = (float)k * rtmp1;
    float rtmp2;
    if (radon_degree == 0) {
      if (type && type != 1) rtmp2 = (1 - fw + fw * filter_add(type, (float)k / N, fm) * ramp[k]) * norm * N;
      else if (type == 1) rtmp2 = (1 - fw + fw * ramp[k]) * norm * N;
      else rtmp2 = 1.0f;
    } else {
      if (type && type != 1) rtmp2 = (1 - fw + fw * filter_add(type, (float)k / N, fm)) * norm * N;
      else if (type == 1) rtmp2 = norm * N;
      else rtmp2 = 1.0f;
    }
    float a = (float)(rtmp2 * std::cos((double)x)), b = (float)(-rtmp2 * std::sin((double)x));
    if (radon_degree) {
      if (type) {
        if (j > 0) {
          const float t = a;
          a = (float)(b * (-1) / (2.f * kPi));
          b = (float)(t / (2.f * kPi));
        } else {
          a = b = 0.0f;
        }
      } else {
        if (j > 0) {
          const float t = a;
          a = (float)(b * (-2 * kPi * k) / (1.0 * N));
          b = (float)(t * (2 * kPi * k) / (1.0 * N));
        } else {
          a = b = 0.0f;
        }
      }
    }
    f[k] = make_float2(a, b);
  }
  return f;
}

}  // namespace

static void grid_free(void *ext) {
  auto *g = (GridState *)ext;
  if (!g) return;
  cudaFree(g->lut);
  cudaFree(g->deapod);
  cudaFree(g->sc);
  cudaFree(g->filt_f);
  cudaFree(g->filt_b);
  cudaFree(g->tw);
  cudaFree(g->sorted);
  cudaFree(g->sc4);
  cudaFree(g->H);
  cudaFree(g->rows);
  cudaFree(g->cd);
  if (g->have_fft) cufftDestroy(g->fft2);
  delete g;
}

int grid_setup(Plan &p) {
  const tomo_geom &G = p.g;
  if (!G.grid_param || !G.grid_lut || !G.grid_deapod || G.grid_lut_len < 8)
    return fail(TOMO_EINVAL, "grid: param[8], lut and deapod are required");
  const float *prm = G.grid_param;
  const int npix = G.n, na = G.na, nz = G.nz;
  auto *g = new GridState();
  p.ext = g;
  p.ext_free = grid_free;
  const float ctr_in = prm[0], oversampl = prm[3];
  const int type_filter = (int)prm[1], flag_filter = (int)prm[2];
  g->interp = (int)prm[4];
  g->ltbl = (int)prm[5];
  const float lconv_b = prm[6];
  g->radon_degree = (int)prm[7];
  g->lut_len = G.grid_lut_len;
  if (flag_filter != 0) return fail(TOMO_EINVAL, "grid: only the built-in filter (param[2] == 0) is provided");
  if (G.grid_mode != 0 && G.grid_mode != 1)
    return fail(TOMO_EINVAL, "grid: grid_mode must be 0 (the reference's arithmetic) or 1 (matched adjoint)");
  g->matched = G.grid_mode == 1;
  if (g->ltbl + 2 > g->lut_len) return fail(TOMO_EINVAL, "grid: param[5] exceeds the lut length");
  // pdim: gridrec_v4_forwproj.c:128-130
  int pdim = (int)(std::pow(2, (int)std::ceil(std::log10((double)npix) / std::log10(2.0))) * oversampl);
  while (pdim % 4 != 0) pdim++;
  if (pdim < npix || pdim > 8192) return fail(TOMO_EINVAL, "grid: the Fourier grid must have 4..8192 points per axis");
  g->pdim = pdim;
  g->pdim_h = (int)(0.5 * pdim);
  g->padleft = (int)((pdim - npix) * 0.5);
  g->padright = g->padleft + npix;
  // forward constants (lconv fixed, tblspcg via the folded reciprocal)
  const float lconv_f = (float)(2 * 7.0 * 1.0 / kPi);
  g->h_f = lconv_f * 0.5f;
  g->tbl_f = (float)(2 * (unsigned long)g->ltbl) * (1.0f / lconv_f);
  // adjoint constants
  if (!(lconv_b > 0.0f) || (int)lconv_b + 1 > kMaxWin)
    return fail(TOMO_EINVAL, "grid: kernel width param[6] must be in (0, 7)");
  g->h_b = lconv_b * 0.5f;
  g->tbl_b = (float)(2 * g->ltbl) / lconv_b;
  g->inv_pdim = 1.0f / (float)pdim;
  std::vector<int> f = factorize(pdim);
  if ((int)f.size() > 32) return fail(TOMO_EINVAL, "grid: too many FFT factors");
  g->nfac = (int)f.size();
  for (int i = 0; i < g->nfac; ++i) g->fac[i] = f[i];
  // per-angle sin/cos (double sincos of deg * pi/180, as compiled)
  std::vector<float2> sc(na);
  std::vector<float4> sc4(na);
  std::vector<std::pair<float, int>> order(na);
  for (int n = 0; n < na; ++n) {
    const double t = (double)p.angles[n] * 0.017453292519943295;
    const float s = (float)std::sin(t), c = (float)std::cos(t);
    sc[n] = make_float2(s, c);
    sc4[n] = make_float4(s, c, c != 0.0f ? 1.0f / c : 0.0f, s != 0.0f ? 1.0f / s : 0.0f);
    float phi = std::atan2(s, c);
    if (phi < 0) phi += 6.2831853f;
    order[n] = {phi, n};
  }
  std::sort(order.begin(), order.end());
  std::vector<float2> sorted(na);
  for (int n = 0; n < na; ++n) {
    float idx;
    std::memcpy(&idx, &order[n].second, sizeof(int));
    sorted[n] = make_float2(order[n].first, idx);
  }
  // forward centring filter (gridrec_v4_forwproj.c:182-205)
  float ctr_f = (float)(npix * 0.5);
  if (pdim != npix) ctr_f += (float)g->padleft;
  const float tmp = (float)(2 * kPi * ctr_f / pdim);
  std::vector<float2> ff(g->pdim_h);
  for (int k = 0; k < g->pdim_h; ++k) {
    const float x = (float)k * tmp;
    float a = (float)(1.0f * 1.0f * std::cos((double)x)), b = (float)(1.0f * 1.0f * std::sin((double)x));
    if (g->radon_degree) {
      const float t1 = a;
      a = (float)(b * (2 * kPi * k) / (1.0 * pdim));
      b = (float)(t1 * (-2 * kPi * k) / (1.0 * pdim));
    }
    ff[k] = make_float2(a, b);
  }
  // adjoint filter (gridrec_v4_backproj.c:191-206, filters.c:143-277)
  float ctr_b = ctr_in;
  if (ctr_b == 0) ctr_b = (float)(npix * 0.5);
  if (pdim != npix) ctr_b += (float)g->padleft;
  std::vector<float2> fb = calc_filter(na, pdim, ctr_b, type_filter, g->radon_degree);
  // twiddles exp(-2 pi i t / pdim)
  std::vector<float2> tw(pdim);
  for (int t = 0; t < pdim; ++t)
    tw[t] = make_float2((float)std::cos(-2 * kPi * t / pdim), (float)std::sin(-2 * kPi * t / pdim));
  auto up = [&](void **dst, const void *src, size_t bytes) -> int {
    TOMO_CUDA(cudaMalloc(dst, bytes));
    TOMO_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return TOMO_OK;
  };
  int rc;
  if ((rc = up((void **)&g->lut, G.grid_lut, sizeof(float) * g->lut_len))) return rc;
  if ((rc = up((void **)&g->deapod, G.grid_deapod, sizeof(float) * (size_t)pdim * pdim))) return rc;
  if ((rc = up((void **)&g->sc, sc.data(), sizeof(float2) * na))) return rc;
  if ((rc = up((void **)&g->sorted, sorted.data(), sizeof(float2) * na))) return rc;
  if ((rc = up((void **)&g->sc4, sc4.data(), sizeof(float4) * na))) return rc;
  if ((rc = up((void **)&g->filt_f, ff.data(), sizeof(float2) * ff.size()))) return rc;
  if ((rc = up((void **)&g->filt_b, fb.data(), sizeof(float2) * fb.size()))) return rc;
  if ((rc = up((void **)&g->tw, tw.data(), sizeof(float2) * tw.size()))) return rc;
  TOMO_CUDA(cudaMalloc(&g->H, sizeof(float2) * (size_t)nz * pdim * pdim));
  TOMO_CUDA(cudaMalloc(&g->rows, sizeof(float2) * (size_t)nz * na * pdim));
  TOMO_CUDA(cudaMalloc(&g->cd, sizeof(float4) * (size_t)nz * na * g->pdim_h));
  int dims[2] = {pdim, pdim};
  if (cufftPlanMany(&g->fft2, 2, dims, nullptr, 1, pdim * pdim, nullptr, 1, pdim * pdim, CUFFT_C2C, nz) !=
      CUFFT_SUCCESS)
    return fail(TOMO_ECUDA, "grid: cufftPlanMany failed");
  g->have_fft = true;
  const int smem = (int)(2 * sizeof(float2) * pdim);
  TOMO_CUDA(cudaFuncSetAttribute(grid_fft_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  TOMO_CUDA(cudaFuncSetAttribute(grid_fft_adj_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  TOMO_CUDA(cudaFuncSetAttribute(grid_fft_adj_matched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  p.fwd_warps = (size_t)nz * na * (kFftThreads / 32);
  return TOMO_OK;
}

static FftConst fft_const(const GridState &g) {
  FftConst c{};
  c.n = g.pdim;
  c.nfac = g.nfac;
  for (int i = 0; i < g.nfac; ++i) c.fac[i] = g.fac[i];
  return c;
}

int grid_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  GridState &g = *(GridState *)p.ext;
  const int npix = p.g.n, na = p.g.na, nz = p.g.nz, pdim = g.pdim;
  dim3 fb(32, 8), fg((pdim + 31) / 32, (pdim + 7) / 8, nz);
  grid_fill_kernel<<<fg, fb, 0, s>>>(d_img, g.H, g.deapod, pdim, g.pdim_h, g.padleft, npix);
  if (cufftSetStream(g.fft2, s) != CUFFT_SUCCESS ||
      cufftExecC2C(g.fft2, (cufftComplex *)g.H, (cufftComplex *)g.H, CUFFT_INVERSE) != CUFFT_SUCCESS)
    return fail(TOMO_ECUDA, "grid: 2-D FFT failed");
  dim3 pb(128), pg((g.pdim_h + 127) / 128, na, nz);
  grid_polar_kernel<<<pg, pb, 0, s>>>(g.H, g.rows, g.sc, g.filt_f, g.lut, pdim, g.pdim_h, na, g.h_f,
                                      g.tbl_f, g.interp);
  const int smem = (int)(2 * sizeof(float2) * pdim);
  grid_fft_fwd_kernel<<<na * nz, kFftThreads, smem, s>>>(g.rows, d_sino, g.tw, fft_const(g), na, npix,
                                                         g.padleft, g.inv_pdim, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int grid_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s, const AdjEpi &ep) {
  GridState &g = *(GridState *)p.ext;
  const int npix = p.g.n, na = p.g.na, nz = p.g.nz, pdim = g.pdim;
  const int smem = (int)(2 * sizeof(float2) * pdim);
  if (g.matched)
    grid_fft_adj_matched_kernel<<<na * nz, kFftThreads, smem, s>>>(d_sino, g.cd, g.tw, g.filt_f, fft_const(g),
                                                                   npix, g.padleft, g.pdim_h, g.inv_pdim);
  else
    grid_fft_adj_kernel<<<na * nz, kFftThreads, smem, s>>>(d_sino, g.cd, g.tw, g.filt_b, fft_const(g), npix,
                                                           g.padleft, g.pdim_h, g.radon_degree,
                                                           (float)(1.0 / pdim));
  GatherArgs ga{g.cd, g.H, g.sc4, g.sorted, g.lut, pdim, g.pdim_h, na, g.interp, 0,
                g.matched ? g.h_f : g.h_b, g.matched ? g.tbl_f : g.tbl_b};
  ga.centre = std::min(kGatherCentre, g.pdim_h - 1);
  const int side = 2 * ga.centre + 1;
  grid_gather_centre_kernel<<<dim3((side * side + 3) / 4, nz), 128, 0, s>>>(ga);
  dim3 gb(128), gg((pdim + 127) / 128, pdim, nz);
  grid_gather_kernel<<<gg, gb, 0, s>>>(ga);
  if (cufftSetStream(g.fft2, s) != CUFFT_SUCCESS ||
      cufftExecC2C(g.fft2, (cufftComplex *)g.H, (cufftComplex *)g.H, g.matched ? CUFFT_FORWARD : CUFFT_INVERSE) !=
          CUFFT_SUCCESS)
    return fail(TOMO_ECUDA, "grid: 2-D FFT failed");
  dim3 eb(32, 8), eg((npix + 31) / 32, (npix + 7) / 8, nz);
  grid_extract_kernel<<<eg, eb, 0, s>>>(g.H, d_img, g.deapod, pdim, g.pdim_h, g.padleft, npix, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
