// Distance-driven projector pair for sm_100a.
//
// Reference: common/operators/radon_module/pymodule_radon_distance_driven/
// radon_dd.c:54-285.  For every angle and every image line (a row when
// theta > pi/2, a column when 0 < theta < pi/2) the reference projects the
// n+1 pixel boundaries P_j = (j - nh) - q and the n+1 detector boundaries
// D_m = (m - nh) * r onto one axis, sorts them together (radon_dd.c:117) and
// walks the merged list (:125-189), crediting every gap between consecutive
// boundaries -- an overlap of pixel k with detector m -- with weight
// |gap| * value.  Two properties of that walk are kept here:
//   * the first gap after a label change is outside one of the two ranges and
//     is not credited; gaps are credited only once both ranges have started;
//   * the walk stops at the first boundary whose index is n (:176-177), so the
//     LAST overlap piece of each line (the gap ending at min(P_n, D_n)) is
//     never credited.
// Rather than sorting, the kernels enumerate the overlaps in closed form.
// Every boundary is the same float the compiled reference computes:
// q = ((i - nh) + 0.5) * k, P = x - q, D = x * r (x = j - nh, k = c*r,
// r = 1/s or 1/c; radon_dd.c:101-115 and 196-207 under -O3 -ffast-math).
//
// Forward: the overlap-weighted sum of a line over [D_m, D_m+1] is
// F(D_m+1) - F(D_m), F the running integral of the line, held as a double
// prefix sum per image row and column.  One thread per (detector, angle,
// slice) evaluates F once per line at its lower boundary and takes the upper
// one from the neighbouring lane, whatever the detector width.  (The pixel
// widths of the reference are P_j+1 - P_j in float, i.e. 1 to within an ulp of
// P; the prefix sum takes them as 1, a difference of ~5e-8 relative L2.)
// Adjoint: one thread per 2x2 pixel tile walks the angles; per angle and line
// a segment of two pixels overlaps at most three detectors, whose boundaries
// and values the two pixels share.  Both read zero-guarded copies of their
// input (scratch owned by the plan), so the inner loops carry no bounds tests;
// the exact dropped-piece rule only matters for the last pixel of a line or
// the last detector and is evaluated on a separate path there.  No atomics:
// each output element is owned by one thread, so results are deterministic.
// The projection arithmetic of the solvers (epilogue.cuh) is applied where the
// result is stored.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "epilogue.cuh"
#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr double kPi = 3.141592653589793;
constexpr int kPadL = 4;  // zero guard on each side of an image line copy

__device__ __forceinline__ float pix_bound(int j, int nh, float q) {
  return __fsub_rn((float)(j - nh), q);
}
__device__ __forceinline__ float det_bound(int m, int nh, float r) {
  return __fmul_rn((float)(m - nh), r);
}

// ---------------------------------------------------------------------------
// v1 kernels: plain transpose + forward.  Kept for the allocation-free entry
// point (dd_noalloc.cu), whose static scratch holds one transposed image.
// ---------------------------------------------------------------------------
__global__ void transpose_kernel(const float *__restrict__ in, float *__restrict__ out, int n,
                                 size_t stride) {
  __shared__ float tile[32][33];
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

__global__ void __launch_bounds__(128) dd_forward_kernel(
    const float *__restrict__ img, const float *__restrict__ imgT, float *__restrict__ sino,
    const DdAngle *__restrict__ tab, int n, int nh, int na) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  const size_t z = blockIdx.z;
  if (m >= n) return;
  const DdAngle g = tab[v];
  const float *I = img + z * (size_t)n * n;
  const float *IT = imgT + z * (size_t)n * n;
  float acc = 0.0f;
  if (g.mode == DD_ROWSUM) {
    for (int j = 0; j < n; ++j) acc += IT[(size_t)j * n + m];
  } else if (g.mode == DD_COLSUM) {
    for (int j = 0; j < n; ++j) acc += I[(size_t)j * n + m];
  } else if (g.mode == DD_ROWS || g.mode == DD_COLS) {
    const float *L = g.mode == DD_ROWS ? I : IT;
    const float r = g.r, k = g.k;
    const float Dlo = det_bound(m, nh, r), Dhi = det_bound(m + 1, nh, r);
    const float Dn = det_bound(n, nh, r);
    int i0 = 0, i1 = n - 1;
    if (k != 0.0f) {
      double qa = -(double)nh - (double)Dhi, qb = (double)(n - nh) - (double)Dlo;
      double ya = qa / (double)k, yb = qb / (double)k;
      double ylo = fmin(ya, yb), yhi = fmax(ya, yb);
      double flo = floor(ylo + nh - 0.5) - 1.0, fhi = ceil(yhi + nh - 0.5) + 1.0;
      i0 = flo < 0.0 ? 0 : (flo > (double)(n - 1) ? n : (int)flo);
      i1 = fhi > (double)(n - 1) ? n - 1 : (fhi < 0.0 ? -1 : (int)fhi);
    }
    for (int i = i0; i <= i1; ++i) {
      const float q = __fmul_rn(__fadd_rn((float)(i - nh), 0.5f), k);
      const float Pn = pix_bound(n, nh, q);
      const bool lastIsPixel = Pn <= Dn;
      const float *row = L + (size_t)i * n;
      int kk = (int)floorf(Dlo + q + (float)nh) - 1;
      kk = kk < 0 ? 0 : (kk > n - 1 ? n - 1 : kk);
      float Pk = pix_bound(kk, nh, q);
      while (kk > 0 && Pk > Dlo) {
        --kk;
        Pk = pix_bound(kk, nh, q);
      }
      for (; kk < n && Pk < Dhi; ++kk) {
        const float Pk1 = pix_bound(kk + 1, nh, q);
        const float lo = fmaxf(Pk, Dlo), hi = fminf(Pk1, Dhi);
        if (hi > lo) {
          const bool drop = lastIsPixel ? (kk == n - 1 && Pn <= Dhi) : (m == n - 1 && Pk1 > Dn);
          if (!drop) acc = fmaf(__fsub_rn(hi, lo), __ldg(row + kk), acc);
        }
        Pk = Pk1;
      }
    }
  }
  sino[z * (size_t)na * n + (size_t)g.out_row * n + m] = acc;
}

// ---------------------------------------------------------------------------
// Exact single-line / single-pixel contributions (used on the edge paths).
// ---------------------------------------------------------------------------
// Detector m, line with offset q: every overlap piece, minus the dropped one.
__device__ float dd_fwd_line_exact(const float *row, int m, float q, float r, float Dlo, float Dhi,
                                   float Dn, int n, int nh) {
  const float Pn = pix_bound(n, nh, q);
  const bool lastIsPixel = Pn <= Dn;
  int kk = (int)floorf(Dlo + q + (float)nh) - 1;
  kk = kk < 0 ? 0 : (kk > n - 1 ? n - 1 : kk);
  float Pk = pix_bound(kk, nh, q);
  while (kk > 0 && Pk > Dlo) {
    --kk;
    Pk = pix_bound(kk, nh, q);
  }
  float acc = 0.0f;
  for (; kk < n && Pk < Dhi; ++kk) {
    const float Pk1 = pix_bound(kk + 1, nh, q);
    const float lo = fmaxf(Pk, Dlo), hi = fminf(Pk1, Dhi);
    if (hi > lo) {
      const bool drop = lastIsPixel ? (kk == n - 1 && Pn <= Dhi) : (m == n - 1 && Pk1 > Dn);
      if (!drop) acc = fmaf(__fsub_rn(hi, lo), __ldg(row + kk), acc);
    }
    Pk = Pk1;
  }
  return acc;
}

// Pixel kk of a line with offset q: every overlap piece with detectors
// 0..n-1, minus the line's dropped piece.  srow[m] is the detector value.
__device__ float dd_adj_pixel_exact(const float *srow, int kk, float q, float r, int n, int nh) {
  const float Pk = pix_bound(kk, nh, q), Pk1 = pix_bound(kk + 1, nh, q);
  const float Pn = pix_bound(n, nh, q), Dn = det_bound(n, nh, r);
  const bool lastIsPixel = Pn <= Dn;
  int m = (int)floorf(Pk / r + (float)nh);
  m = m < 0 ? 0 : (m > n - 1 ? n - 1 : m);
  float Dm = det_bound(m, nh, r);
  while (m > 0 && Dm > Pk) {
    --m;
    Dm = det_bound(m, nh, r);
  }
  float Dm1 = det_bound(m + 1, nh, r);
  while (m < n - 1 && Dm1 <= Pk) {
    ++m;
    Dm = Dm1;
    Dm1 = det_bound(m + 1, nh, r);
  }
  float acc = 0.0f;
  for (; m < n && Dm < Pk1; ++m) {
    const float lo = fmaxf(Pk, Dm), hi = fminf(Pk1, Dm1);
    if (hi > lo) {
      const bool drop = lastIsPixel ? (kk == n - 1 && Pn <= Dm1) : (m == n - 1 && Pk1 > Dn);
      if (!drop) acc = fmaf(__fsub_rn(hi, lo), __ldg(srow + m), acc);
    }
    Dm = Dm1;
    Dm1 = det_bound(m + 2, nh, r);
  }
  return acc;
}

// ---------------------------------------------------------------------------
// v2: zero-guarded copies and lean inner loops.
// ---------------------------------------------------------------------------
// Lr[z][i][kPadL + k] = img[z][i][k], Lc[z][i][kPadL + k] = img[z][k][i];
// guard words are zero.  Stride wl = n + 2*kPadL.
__global__ void dd_pad_image_kernel(const float *__restrict__ img, float *__restrict__ Lr,
                                    float *__restrict__ Lc, int n, int wl) {
  __shared__ float tile[32][33];
  const size_t z = blockIdx.z;
  const float *src = img + z * (size_t)n * n;
  float *dr = Lr + z * (size_t)n * wl, *dc = Lc + z * (size_t)n * wl;
  const int x = blockIdx.x * 32 + threadIdx.x, y0 = blockIdx.y * 32;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int y = y0 + dy;
    float v = 0.0f;
    if (x < n && y < n) v = src[(size_t)y * n + x];
    tile[dy][threadIdx.x] = v;
    if (y < n && x < n) dr[(size_t)y * wl + kPadL + x] = v;
  }
  __syncthreads();
  const int ox = blockIdx.y * 32 + threadIdx.x;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int oy = blockIdx.x * 32 + dy;
    if (ox < n && oy < n) dc[(size_t)oy * wl + kPadL + ox] = tile[threadIdx.x][dy];
  }
  // guards: the blocks of the first column of tiles zero both ends of their rows
  if (blockIdx.x == 0) {
    for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
      const int y = y0 + dy;
      if (y < n && threadIdx.x < 2 * kPadL) {
        const int col = threadIdx.x < kPadL ? threadIdx.x : n + threadIdx.x;
        dr[(size_t)y * wl + col] = 0.0f;
        dc[(size_t)y * wl + col] = 0.0f;
      }
    }
  }
}

// Sp[z][v][pads + m] = sino[z][na-1-v... the row of angle v][m]; guards zero.
__global__ void dd_pad_sino_kernel(const float *__restrict__ sino, float *__restrict__ Sp,
                                   const DdAngle *__restrict__ tab, int n, int na, int w, int pads) {
  const int v = blockIdx.y;
  const size_t z = blockIdx.z;
  const float *src = sino + z * (size_t)na * n + (size_t)tab[v].out_row * n;
  float *dst = Sp + z * (size_t)na * w + (size_t)v * w;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < w; c += gridDim.x * blockDim.x) {
    const int m = c - pads;
    dst[c] = (m >= 0 && m < n) ? src[m] : 0.0f;
  }
}

// Line prefix sums in double, interleaved with the line values:
// SL[line][kk] = {S(kk), L[kk]} for kk in [-1, n], S(kk) = sum_{j < kk} L[j],
// with the guards SL[-1] = {0, 0} and SL[n] = {S(n), 0}.  The integral of a
// line from its start to a boundary D inside pixel kk is then
// F(D) = S(kk) + (D - P_kk) L[kk] for every kk in [-1, n] (pixel widths 1).
// One block per line; passes of 256 values, each a fixed-order block scan,
// so the sums are deterministic.
constexpr int kScanThreads = 256;
__global__ void __launch_bounds__(kScanThreads) dd_prefix_kernel(const float *__restrict__ L,
                                                                 double2 *__restrict__ SL, int n, int wl,
                                                                 int wsl) {
  __shared__ double wsum[kScanThreads / 32];
  __shared__ double carry_s;
  const size_t line = blockIdx.x;
  const float *src = L + line * wl + kPadL;
  double2 *dst = SL + line * wsl + 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double carry = 0.0;
  for (int base = 0; base < n; base += kScanThreads) {
    const int k = base + tid;
    const float vf = k < n ? src[k] : 0.0f;
    double x = (double)vf;  // inclusive warp scan
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    double before = carry;  // carry + totals of the earlier warps, in warp order
    for (int w = 0; w < warp; ++w) before += wsum[w];
    if (k < n) dst[k] = make_double2(before + (x - (double)vf), (double)vf);
    if (tid == kScanThreads - 1) carry_s = before + x;
    __syncthreads();
    carry = carry_s;
  }
  if (tid == 0) {
    dst[-1] = make_double2(0.0, 0.0);
    dst[n] = make_double2(carry, 0.0);
  }
}

// Lines i of [0, n) with q_i = ((i - nh) + 0.5) k inside [qlo, qhi], widened
// by one line on each side; [ia, ib] is empty when ia > ib.
__device__ __forceinline__ void dd_line_range(double qlo, double qhi, double k, int n, int nh, int &ia,
                                              int &ib) {
  if (k == 0.0) {
    const bool all = qlo <= 0.0 && 0.0 <= qhi;
    ia = all ? 0 : n;
    ib = all ? n - 1 : -1;
    return;
  }
  const double ya = qlo / k, yb = qhi / k;
  const double flo = floor(fmin(ya, yb) + nh - 0.5) - 1.0, fhi = ceil(fmax(ya, yb) + nh - 0.5) + 1.0;
  ia = flo < 0.0 ? 0 : (flo > (double)(n - 1) ? n : (int)flo);
  ib = fhi > (double)(n - 1) ? n - 1 : (fhi < 0.0 ? -1 : (int)fhi);
}

// Forward.  A warp owns 31 consecutive detectors (lane 31 only supplies the
// upper boundary of lane 30).  Lane j accumulates T_j = sum over lines of
// F(D_j) at its lower boundary, and detector m = T_m+1 - T_m: one integral
// evaluation per line and detector, whatever the detector's width.  The lines
// on which the dropped last piece of the line can belong to one of the warp's
// detectors (P_n within the warp's detector span, or beyond D_n for the warp
// holding detector n-1) form one contiguous band; there every lane walks the
// pieces exactly instead.
constexpr int kFwdDet = 31;
constexpr int kFwdWarps = 4;
__global__ void __launch_bounds__(32 * kFwdWarps) dd_forward_v4_kernel(
    const float *__restrict__ Lr, const float *__restrict__ Lc, const double2 *__restrict__ SLr,
    const double2 *__restrict__ SLc, float *__restrict__ sino, const DdAngle *__restrict__ tab, int n,
    int nh, int na, int wl, int wsl, FwdEpi ep) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int mA = (blockIdx.x * kFwdWarps + warp) * kFwdDet;
  const int m = mA + lane;
  const int v = blockIdx.y;
  const size_t z = blockIdx.z;
  const bool live = lane < kFwdDet && m < n;
  const DdAngle g = tab[v];
  float acc = 0.0f;
  const float *Rz = Lr + z * (size_t)n * wl + kPadL, *Cz = Lc + z * (size_t)n * wl + kPadL;
  if (g.mode == DD_ROWSUM) {
    if (live)
      for (int j = 0; j < n; ++j) acc += __ldg(Cz + (size_t)j * wl + m);
  } else if (g.mode == DD_COLSUM) {
    if (live)
      for (int j = 0; j < n; ++j) acc += __ldg(Rz + (size_t)j * wl + m);
  } else if ((g.mode == DD_ROWS || g.mode == DD_COLS) && mA < n) {
    const float *L = g.mode == DD_ROWS ? Rz : Cz;
    const double2 *SL = (g.mode == DD_ROWS ? SLr : SLc) + z * (size_t)n * wsl + 1;
    const float r = g.r, k = g.k;
    const float Dlo = det_bound(m, nh, r), Dhi = det_bound(m + 1, nh, r);
    const float Dn = det_bound(n, nh, r);
    const int mB = min(mA + kFwdDet - 1, n - 1);
    const double DA = (double)det_bound(mA, nh, r), DB = (double)det_bound(mB + 1, nh, r);
    const double kd = (double)k, PN = (double)(n - nh);
    int i0, i1, j0, j1;
    dd_line_range(-(double)nh - DB, PN - DA, kd, n, nh, i0, i1);
    const double margin = 2.0 + 1e-6 * (fabs(DA) + fabs(DB) + (double)n * (1.0 + fabs(kd)));
    const double BL = DA - margin, BH = mB == n - 1 ? 1e30 : DB + margin;
    dd_line_range(PN - BH, PN - BL, kd, n, nh, j0, j1);
    j0 = max(j0, i0);
    j1 = min(j1, i1);
    if (j0 > j1) {  // no band: all lines are fast
      j0 = i1 + 1;
      j1 = i1;
    }
    const float lo_nh = __fadd_rn(Dlo, (float)nh);
    double T = 0.0, X = 0.0;
    for (int seg = 0; seg < 2; ++seg) {
      const int ia = seg == 0 ? i0 : j1 + 1, ib = seg == 0 ? j0 : i1 + 1;
      float y = (float)(ia - nh) + 0.5f;
      const double2 *sl = SL + (size_t)ia * wsl;
#pragma unroll 4
      for (int i = ia; i < ib; ++i) {
        const float q = __fmul_rn(y, k);
        const int kk = min(max(__float2int_rd(__fadd_rn(lo_nh, q)), -1), n);
        const float Pk = __fsub_rn((float)(kk - nh), q);
        const double2 e = __ldg(sl + kk);
        T = fma((double)__fsub_rn(Dlo, Pk), e.y, T + e.x);
        y = __fadd_rn(y, 1.0f);
        sl += wsl;
      }
    }
    if (live) {
      float y = (float)(j0 - nh) + 0.5f;
      for (int i = j0; i <= j1; ++i, y = __fadd_rn(y, 1.0f))
        X += (double)dd_fwd_line_exact(L + (size_t)i * wl, m, __fmul_rn(y, k), r, Dlo, Dhi, Dn, n, nh);
    }
    const double Tup = __shfl_down_sync(0xffffffffu, T, 1);
    acc = (float)((Tup - T) + X);
  }
  fwd_store(ep, acc, live, z * (size_t)na * n + (size_t)g.out_row * n + (live ? m : 0), sino);
}

constexpr int kAdjChunk = 1024;

// One line segment of two pixels [P0, P1], [P1, P2] (the line's offset q is
// applied); adds their weights times the detector values into a0, a1.  Exact
// unless the segment touches the last pixel or detector, where the caller
// takes dd_adj_pixel_exact instead.
__device__ __forceinline__ void dd_adj_segment(float P0, float P1, float P2, const float4 e,
                                               const float *__restrict__ S, float nhp, int pads, int n,
                                               float &a0, float &a1, bool &edge) {
  const float r = e.x;
  int mp = (int)floorf(fmaf(P0, e.z, nhp));
  float fm = __fsub_rn((float)mp, nhp);
  float Dm = __fmul_rn(fm, r);
  if (Dm > P0) {
    --mp;
    fm = __fsub_rn(fm, 1.0f);
    Dm = __fmul_rn(fm, r);
  }
  float D1 = __fmul_rn(__fadd_rn(fm, 1.0f), r);
  if (D1 <= P0) {
    ++mp;
    fm = __fadd_rn(fm, 1.0f);
    D1 = __fmul_rn(__fadd_rn(fm, 1.0f), r);
  }
  edge = (unsigned)(mp - pads - (n - 3)) <= 2u;  // the segment meets detector n-1
  const float D2 = __fmul_rn(__fadd_rn(fm, 2.0f), r);
  const float *sp = S + __float_as_int(e.w) + mp;
  const float v0 = __ldg(sp), v1 = __ldg(sp + 1), v2 = __ldg(sp + 2);
  const float t0 = fminf(D1, P1);
  a0 = fmaf(__fsub_rn(t0, P0), v0, a0);
  a0 = fmaf(__fsub_rn(P1, t0), v1, a0);
  const bool c = P1 >= D1;
  const float Da = c ? D2 : D1, va = c ? v1 : v0, vb = c ? v2 : v1;
  const float t1 = fminf(Da, P2);
  a1 = fmaf(__fsub_rn(t1, P1), va, a1);
  a1 = fmaf(__fsub_rn(P2, t1), vb, a1);
}

// Adjoint: one thread per 2x2 pixel tile (rows a0, a0+1; columns b0, b0+1).
// For a ROWS angle the tile is two row segments of two pixels, for a COLS
// angle two column segments; each segment shares its boundary and detector
// arithmetic between its two pixels.
__global__ void __launch_bounds__(256) dd_adjoint_v3_kernel(
    const float *__restrict__ Sp, float *__restrict__ img, const float4 *__restrict__ tabR, int nR,
    const float4 *__restrict__ tabC, int nC, const int2 *__restrict__ tabS, int nS, int n, int nh,
    int na, int w, int pads, AdjEpi ep) {
  __shared__ float4 st[kAdjChunk];
  const int b0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int a0 = 2 * (blockIdx.y * blockDim.y + threadIdx.y);
  const size_t z = blockIdx.z;
  const bool any = a0 < n && b0 < n;
  const float *S = Sp + z * (size_t)na * w;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
  const float nhp = (float)(nh + pads);
  float acc[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // [row - a0][col - b0]
  for (int pass = 0; pass < 2; ++pass) {
    const float4 *tab = pass == 0 ? tabR : tabC;
    const int cnt_all = pass == 0 ? nR : nC;
    // ROWS: lines are rows a0, a0+1 and the segment is columns b0, b0+1; COLS: transposed
    const int l0 = pass == 0 ? a0 : b0, k0 = pass == 0 ? b0 : a0;
    const float y0 = (float)(l0 - nh) + 0.5f, y1 = __fadd_rn(y0, 1.0f);
    const float x0 = (float)(k0 - nh), x1 = __fadd_rn(x0, 1.0f), x2 = __fadd_rn(x0, 2.0f);
    const bool edge_pixel = k0 + 1 >= n - 1;
    for (int v0 = 0; v0 < cnt_all; v0 += kAdjChunk) {
      const int cnt = min(kAdjChunk, cnt_all - v0);
      __syncthreads();
      for (int t = tid; t < cnt; t += nthr) st[t] = tab[v0 + t];
      __syncthreads();
      if (!any) continue;
      for (int u = 0; u < cnt; ++u) {
        const float4 e = st[u];
        for (int li = 0; li < 2; ++li) {
          if (l0 + li >= n) break;  // odd n: the tile's second line is outside the image
          const float q = __fmul_rn(li ? y1 : y0, e.y);
          const float P0 = __fsub_rn(x0, q), P1 = __fsub_rn(x1, q), P2 = __fsub_rn(x2, q);
          float s0 = 0.0f, s1 = 0.0f;
          bool edge;
          dd_adj_segment(P0, P1, P2, e, S, nhp, pads, n, s0, s1, edge);
          if (edge || edge_pixel) {
            const float *srow = S + __float_as_int(e.w) + pads;
            s0 = dd_adj_pixel_exact(srow, k0, q, e.x, n, nh);
            s1 = k0 + 1 < n ? dd_adj_pixel_exact(srow, k0 + 1, q, e.x, n, nh) : 0.0f;
          }
          if (pass == 0) {
            acc[li][0] += s0;
            acc[li][1] += s1;
          } else {
            acc[0][li] += s0;
            acc[1][li] += s1;
          }
        }
      }
    }
  }
  if (any) {
    for (int t = 0; t < nS; ++t) {  // row / column sums (|sin| or |cos| < 1e-7)
      const int2 e = __ldg(tabS + t);
      const float *srow = S + e.y + pads;
      for (int dr = 0; dr < 2; ++dr)
        for (int dc = 0; dc < 2; ++dc) acc[dr][dc] += __ldg(srow + (e.x == DD_ROWSUM ? a0 + dr : b0 + dc));
    }
  }
  for (int dr = 0; dr < 2; ++dr)
    for (int dc = 0; dc < 2; ++dc) {
      const int a = a0 + dr, b = b0 + dc;
      const bool live = a < n && b < n;
      adj_store(ep, acc[dr][dc], live, z * (size_t)n * n + (size_t)(live ? a : 0) * n + (live ? b : 0), img);
    }
}

}  // namespace

int dd_build_table(const float *angles, int na, DdAngle *tab) {
  for (int v = 0; v < na; ++v) {
    const float theta = angles[v];
    float s, c;
    sincosf(theta, &s, &c);
    DdAngle a{};
    a.out_row = na - 1 - v;  // radon_dd.c:79,181,273
    if (std::fabs((double)s) < 1e-7) {
      a.mode = DD_ROWSUM;
    } else if (std::fabs((double)c) < 1e-7) {
      a.mode = DD_COLSUM;
    } else if ((double)theta > kPi / 2) {
      if (!(s > 0.0f))
        return fail(TOMO_EINVAL, "dd: angle " + std::to_string(theta) +
                                     " rad is outside [-pi/2, pi], where the reference merge is undefined");
      a.mode = DD_ROWS;
      a.r = 1.0f / s;
      a.k = c * a.r;
    } else if ((double)theta < kPi / 2 && theta != 0.0f) {
      if (!(c > 0.0f))
        return fail(TOMO_EINVAL, "dd: angle " + std::to_string(theta) +
                                     " rad is outside [-pi/2, pi], where the reference merge is undefined");
      a.mode = DD_COLS;
      a.r = 1.0f / c;
      a.k = s * a.r;
    } else {
      a.mode = DD_NONE;
    }
    tab[v] = a;
  }
  return TOMO_OK;
}

int dd_forward_launch(const float *d_img, float *d_scratch, float *d_sino, const DdAngle *d_tab,
                      int n, int na, int nz, cudaStream_t s) {
  const int nh = (int)(n * 0.5);
  const size_t stride = (size_t)n * n;
  dim3 tb(32, 8), tg((n + 31) / 32, (n + 31) / 32, nz);
  transpose_kernel<<<tg, tb, 0, s>>>(d_img, d_scratch, n, stride);
  dim3 fb(128), fg((n + 127) / 128, na, nz);
  dd_forward_kernel<<<fg, fb, 0, s>>>(d_img, d_scratch, d_sino, d_tab, n, nh, na);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

// Plan layout: d_angles = DdAngle[na] (angle order); d_aux = adjoint tables
// (float4 ROWS[nR], float4 COLS[nC], int2 SUMS[nS]); d_scratch = Lr | Lc | Sp.
int dd_setup(Plan &p) {
  const int na = p.g.na, n = p.g.n, nh = p.nh, nz = p.g.nz;
  std::vector<DdAngle> tab(na);
  int rc = dd_build_table(p.angles.data(), na, tab.data());
  if (rc) return rc;
  p.dd_pads = (int)std::ceil((nh + 1) * (std::sqrt(2.0) - 1.0)) + 4;
  p.dd_w = ((n + 2 * p.dd_pads) + 3) / 4 * 4;
  p.dd_wl = n + 2 * kPadL;
  std::vector<float4> rows, cols;
  std::vector<int2> sums;
  for (int v = 0; v < na; ++v) {
    const DdAngle &a = tab[v];
    const int off = v * p.dd_w;
    if (a.mode == DD_ROWS || a.mode == DD_COLS) {
      // z = 1/r (= sin or cos): the detector index of a boundary P is about P/r + nh
      float s, c;
      sincosf(p.angles[v], &s, &c);
      float4 e = make_float4(a.r, a.k, a.mode == DD_ROWS ? s : c, 0.0f);
      std::memcpy(&e.w, &off, sizeof(int));
      (a.mode == DD_ROWS ? rows : cols).push_back(e);
    } else if (a.mode == DD_ROWSUM || a.mode == DD_COLSUM) {
      sums.push_back(make_int2(a.mode, off));
    }
  }
  p.dd_nR = (int)rows.size();
  p.dd_nC = (int)cols.size();
  p.dd_nS = (int)sums.size();
  TOMO_CUDA(cudaMalloc(&p.d_angles, sizeof(DdAngle) * (size_t)na));
  TOMO_CUDA(cudaMemcpy(p.d_angles, tab.data(), sizeof(DdAngle) * (size_t)na, cudaMemcpyHostToDevice));
  const size_t aux_bytes = sizeof(float4) * (rows.size() + cols.size()) + sizeof(int2) * (sums.size() + 1);
  TOMO_CUDA(cudaMalloc(&p.d_aux, aux_bytes));
  char *aux = (char *)p.d_aux;
  if (!rows.empty())
    TOMO_CUDA(cudaMemcpy(aux, rows.data(), sizeof(float4) * rows.size(), cudaMemcpyHostToDevice));
  if (!cols.empty())
    TOMO_CUDA(cudaMemcpy(aux + sizeof(float4) * rows.size(), cols.data(), sizeof(float4) * cols.size(),
                         cudaMemcpyHostToDevice));
  if (!sums.empty())
    TOMO_CUDA(cudaMemcpy(aux + sizeof(float4) * (rows.size() + cols.size()), sums.data(),
                         sizeof(int2) * sums.size(), cudaMemcpyHostToDevice));
  const size_t lines = 2 * (size_t)nz * n * p.dd_wl, sp = (size_t)nz * na * p.dd_w;
  const size_t nsum = 2 * (size_t)nz * n * (n + 2);  // double2
  p.scratch_bytes = (sizeof(float) * (lines + sp) + 255) / 256 * 256 + sizeof(double2) * nsum;
  // residual partials: one per warp of the forward grid (dd_forward)
  const int per_block = kFwdDet * kFwdWarps;
  p.fwd_warps = (size_t)((n + per_block - 1) / per_block) * kFwdWarps * na * nz;
  TOMO_CUDA(cudaMalloc(&p.d_scratch, p.scratch_bytes));
  return TOMO_OK;
}

// scratch layout: Lr | Lc (floats, nz*n*wl each) | Sp (floats) | SLr | SLc (double2, nz*n*(n+2) each)
static double2 *dd_sums(Plan &p) {
  const size_t fl = 2 * (size_t)p.g.nz * p.g.n * p.dd_wl + (size_t)p.g.nz * p.g.na * p.dd_w;
  const size_t off = (fl * sizeof(float) + 255) / 256 * 256;
  return (double2 *)((char *)p.d_scratch + off);
}

int dd_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz, wsl = n + 2;
  float *Lr = p.d_scratch, *Lc = p.d_scratch + (size_t)nz * n * p.dd_wl;
  double2 *SLr = dd_sums(p), *SLc = SLr + (size_t)nz * n * wsl;
  dim3 tb(32, 8), tg((n + 31) / 32, (n + 31) / 32, nz);
  dd_pad_image_kernel<<<tg, tb, 0, s>>>(d_img, Lr, Lc, n, p.dd_wl);
  dd_prefix_kernel<<<nz * n, kScanThreads, 0, s>>>(Lr, SLr, n, p.dd_wl, wsl);
  dd_prefix_kernel<<<nz * n, kScanThreads, 0, s>>>(Lc, SLc, n, p.dd_wl, wsl);
  const int per_block = kFwdDet * kFwdWarps;
  dim3 fb(32 * kFwdWarps), fg((n + per_block - 1) / per_block, na, nz);
  dd_forward_v4_kernel<<<fg, fb, 0, s>>>(Lr, Lc, SLr, SLc, d_sino, (const DdAngle *)p.d_angles, n, p.nh, na,
                                         p.dd_wl, wsl, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int dd_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s, const AdjEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz;
  float *Sp = p.d_scratch + 2 * (size_t)nz * n * p.dd_wl;
  dim3 pb(256), pg((p.dd_w + 255) / 256, na, nz);
  dd_pad_sino_kernel<<<pg, pb, 0, s>>>(d_sino, Sp, (const DdAngle *)p.d_angles, n, na, p.dd_w,
                                       p.dd_pads);
  const float4 *tR = (const float4 *)p.d_aux, *tC = tR + p.dd_nR;
  const int2 *tS = (const int2 *)(tC + p.dd_nC);
  dim3 ab(32, 8), ag((n + 63) / 64, (n + 15) / 16, nz);
  dd_adjoint_v3_kernel<<<ag, ab, 0, s>>>(Sp, d_img, tR, p.dd_nR, tC, p.dd_nC, tS, p.dd_nS, n, p.nh,
                                         na, p.dd_w, p.dd_pads, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
