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
//   * gaps are credited only inside both ranges ([P_0, P_n] and [D_0, D_n]);
//   * the walk stops at the first boundary whose index is n (:176-177), so the
//     LAST overlap piece of each line (the gap ending at min(P_n, D_n)) is
//     never credited.
// Every boundary is the same float the compiled reference computes:
// q = ((i - nh) + 0.5) * k, P = x - q, D = x * r (x = j - nh, k = c*r,
// r = 1/s or 1/c; radon_dd.c:101-115 and 196-207 under -O3 -ffast-math).
//
// Rather than sorting, the overlaps are enumerated in closed form:
//   forward  detector m of a line = F(D_m+1) - F(D_m), F the running integral
//            of the line's pixel values, kept per image row and column as a
//            double prefix sum (the integral-image form of distance-driven
//            projection: Basu & De Man, "Branchless distance driven projection
//            and backprojection", SPIE 6065, 2006).  One table read per
//            detector and line, however wide the detector (r = 1/|s| can be
//            large).  The prefix sums take pixel widths as 1; the
//            reference's are P_j+1 - P_j in float, which is 1 exactly except
//            for pixels straddling a binade of P (|P| = 2^e), whose width
//            differs by a rounding of q: those are added per line, and the
//            dropped last piece of every line is subtracted, by a kernel of
//            their own (dd_fwd_corr_kernel) into a float row per angle that
//            the forward adds where it stores.  Angles whose coordinates
//            reach 2^22 walk the pieces instead (dd_fwd_exact).
//   adjoint  a pixel is at most one detector wide (r >= 1), so it overlaps the
//            detector holding its left boundary and possibly the next: two
//            float gaps, as the reference forms them, from one 8-byte table
//            entry {S_a, S_a+1} per angle and the boundary D_a+1 recomputed.
// The dropped last piece is subtracted where it falls (dd_dropped_piece):
// forward in dd_fwd_corr_kernel, adjoint in the pixel loop.
//
// Work is described by a table of instances (one per slice, or per geometry
// of an uneven batch) and consumed by persistent kernels: each warp takes the
// next work item (forward: 127 detectors of one angle; adjoint: a 16x8 pixel
// tile over all angles) from a device counter, finds its instance by binary
// search and runs it.  Every output element is owned by one lane and its sum
// order is fixed, so results do not depend on scheduling and are
// deterministic.  Warps per block and the fetch mode are chosen per plan by timing the
// candidates (dd_autotune).  The projection arithmetic of the solvers
// (epilogue.cuh) is applied where the result is stored.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "epilogue.cuh"
#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr double kPi = 3.141592653589793;

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
// Instances
// ---------------------------------------------------------------------------
constexpr int kGrpDet = 127;              // detectors per forward item (128 boundaries, 4 per lane)
#ifndef FWD_UNROLL
#define FWD_UNROLL 2
#endif
constexpr int kFwdUnroll = FWD_UNROLL;  // image lines per unrolled step of the forward
constexpr int kTileW = 32, kTileH = 16;   // pixels per adjoint item (4x4 per lane, 8x4 lanes)
constexpr int kScanThreads = 256;
constexpr int kColWarps = 4, kColRows = 16;
// Adding 1.5 * 2^23 rounds a float of magnitude < 2^22 to an integer held in
// the low mantissa bits: int = bits - kMagicBits.
constexpr float kMagic = 12582912.0f;
constexpr int kMagicBits = 0x4B400000;

struct DdInst {
  long long img, sino;   // offsets (floats) of the image / sinogram in the packed arrays
  long long sl;          // offset (double2) of the row prefix lines; column lines follow
  long long as;          // offset (double2) of the sinogram prefix rows [na][w2]
  long long xs;          // offset (double2) of the forward's corrections, float [na][n], or the adjoint's dropped-piece image [n][n]
  long long f0, a0;      // first forward / adjoint work item
  long long r0, c0, s0;  // first row-prefix / column-prefix / sinogram-prefix block
  const DdAngle *ang;    // [na] per-angle geometry, angle order
  const float4 *tab;     // adjoint lines: ROWS angles then COLS angles {r, k, z, v*w2 (int bits)}
  const int2 *tabS;      // adjoint sums: {mode, v*w2}
  const int *fperm;      // forward angle order: the nRf angles on row lines first, then those on columns
  int n, nh, na, pads, w2, nR, nC, nS, ngrp, tx, ty, nRf;
};

// Index of the instance whose range [key, next key) holds item (keys ascend).
__device__ __forceinline__ int find_inst(const DdInst *__restrict__ inst, int ninst, long long item,
                                         long long DdInst::*key) {
  int lo = 0, hi = ninst - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (inst[mid].*key <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// The piece of a line that the reference never credits: the last gap of its
// boundary walk, ending at min(P_n, D_n) (radon_dd.c:176-177).  If P_n <= D_n
// it is the overlap of pixel n-1 with the detector m holding P_n
// (D_m < P_n <= D_m+1); otherwise the overlap of detector n-1 with the pixel k
// holding D_n (P_k < D_n < P_k+1; if D_n falls on a pixel boundary no piece
// is lost).  Returns false when nothing is lost, including lines that do not
// meet the detector range.
struct DdDrop {
  int pix, det;
  float gap;
};
__device__ __noinline__ bool dd_dropped_piece(float q, float r, int n, int nh, DdDrop &d) {
  const float Pn = pix_bound(n, nh, q), Dn = det_bound(n, nh, r);
  if (Pn <= Dn) {
    int m = min(max(__float2int_rd(__fdiv_rn(Pn, r)) + nh, -1), n - 1);
    for (int it = 0; it < 8 && m >= 0 && !(det_bound(m, nh, r) < Pn); ++it) --m;
    for (int it = 0; it < 8 && m < n - 1 && !(Pn <= det_bound(m + 1, nh, r)); ++it) ++m;
    if (m < 0) return false;
    d.pix = n - 1;
    d.det = m;
    d.gap = __fsub_rn(Pn, fmaxf(pix_bound(n - 1, nh, q), det_bound(m, nh, r)));
    return true;
  }
  int k = min(max(__float2int_rd(__fadd_rn(__fadd_rn(Dn, q), (float)nh)), -1), n - 1);
  for (int it = 0; it < 8 && k >= 0 && !(pix_bound(k, nh, q) < Dn); ++it) --k;
  for (int it = 0; it < 8 && k < n - 1 && !(Dn <= pix_bound(k + 1, nh, q)); ++it) ++k;
  if (k < 0 || Dn == pix_bound(k + 1, nh, q)) return false;
  d.pix = k;
  d.det = n - 1;
  d.gap = __fsub_rn(Dn, fmaxf(det_bound(n - 1, nh, r), pix_bound(k, nh, q)));
  return true;
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

// ---------------------------------------------------------------------------
// Pre-passes: prefix sums of the image lines and of the sinogram rows
// ---------------------------------------------------------------------------
// Inclusive scan of x over the block (kScanThreads threads), added to carry;
// returns carry + sum of the values before this thread's and updates carry to
// carry + block total.  Fixed order, so the result is deterministic.
__device__ __forceinline__ double block_exclusive_scan(double x, double &carry, double *wsum,
                                                       double *carry_s) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double x0 = x;
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  double before = carry;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  if (tid == kScanThreads - 1) *carry_s = before + x;
  __syncthreads();
  carry = *carry_s;
  return before + (x - x0);
}

// Row lines: work[sl + line*(n+2) + 1 + kk] = {S(kk), L[kk]}, kk in [-1, n],
// S(kk) = sum_{j<kk} L[j], L the image row; guards {0, 0} and {S(n), 0}.
__global__ void __launch_bounds__(kScanThreads) dd_row_prefix_kernel(const DdInst *__restrict__ inst,
                                                                     int ninst, const float *__restrict__ img,
                                                                     double2 *__restrict__ work) {
  __shared__ double wsum[kScanThreads / 32];
  __shared__ double carry_s;
  const long long b = blockIdx.x;
  const DdInst &I = inst[find_inst(inst, ninst, b, &DdInst::r0)];
  const int n = I.n, line = (int)(b - I.r0);
  const float *src = img + I.img + (size_t)line * n;
  double2 *dst = work + I.sl + (size_t)line * (n + 2) + 1;
  double carry = 0.0;
  for (int base = 0; base < n; base += kScanThreads) {
    const int k = base + threadIdx.x;
    const float v = k < n ? __ldg(src + k) : 0.0f;
    const double ex = block_exclusive_scan((double)v, carry, wsum, &carry_s);
    if (k < n) dst[k] = make_double2(ex, (double)v);
  }
  if (threadIdx.x == 0) {
    dst[-1] = make_double2(0.0, 0.0);
    dst[n] = make_double2(carry, 0.0);
  }
}

// Column lines (line c = image column c), 32 columns per block: each warp
// sums a quarter of the rows, then rescans its rows 16 at a time through
// shared memory so that each column line is written contiguously.
__global__ void __launch_bounds__(32 * kColWarps) dd_col_prefix_kernel(const DdInst *__restrict__ inst,
                                                                       int ninst, const float *__restrict__ img,
                                                                       double2 *__restrict__ work) {
  __shared__ double tot[kColWarps][32];
  __shared__ double2 tile[kColWarps][kColRows][33];
  const long long b = blockIdx.x;
  const DdInst &I = inst[find_inst(inst, ninst, b, &DdInst::c0)];
  const int n = I.n, c0 = (int)(b - I.c0) * 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int col = c0 + lane;
  const float *im = img + I.img;
  double2 *SLc = work + I.sl + (size_t)n * (n + 2) + 1;
  const int ch = (n + kColWarps - 1) / kColWarps;
  const int r0 = min(w * ch, n), r1 = min(r0 + ch, n);
  double t = 0.0;
  if (col < n)
    for (int r = r0; r < r1; ++r) t += (double)__ldg(im + (size_t)r * n + col);
  tot[w][lane] = t;
  __syncthreads();
  double run = 0.0, total = 0.0;
  for (int u = 0; u < kColWarps; ++u) {
    if (u < w) run += tot[u][lane];
    total += tot[u][lane];
  }
  for (int rb = r0; rb < r1; rb += kColRows) {
    for (int rr = 0; rr < kColRows; ++rr) {
      const int r = rb + rr;
      const float v = (col < n && r < r1) ? __ldg(im + (size_t)r * n + col) : 0.0f;
      tile[w][rr][lane] = make_double2(run, (double)v);
      run += (double)v;
    }
    __syncwarp();
    for (int cc2 = 0; cc2 < 16; ++cc2) {
      const int cc = 2 * cc2 + (lane >> 4), rr = lane & 15;
      const int cg = c0 + cc, r = rb + rr;
      if (cg < n && r < r1) SLc[(size_t)cg * (n + 2) + r] = tile[w][rr][cc];
    }
    __syncwarp();
  }
  if (w == 0 && col < n) {
    SLc[(size_t)col * (n + 2) - 1] = make_double2(0.0, 0.0);
    SLc[(size_t)col * (n + 2) + n] = make_double2(total, 0.0);
  }
}

// Sinogram rows, one block per angle v: entry e = m + pads (m in
// [-pads, n + pads)) holds {S_m, S_m+1}, the values (0 outside [0, n)) of the
// two detectors a pixel starting in detector m can overlap.  (The boundary
// D_m+1 between them is recomputed from m where it is needed.)
__global__ void __launch_bounds__(kScanThreads) dd_sino_expand_kernel(const DdInst *__restrict__ inst,
                                                                      int ninst, const float *__restrict__ sino,
                                                                      double2 *__restrict__ work) {
  const long long b = blockIdx.x;
  const DdInst &I = inst[find_inst(inst, ninst, b, &DdInst::s0)];
  const int v = (int)(b - I.s0), n = I.n, nh = I.nh, pads = I.pads, w2 = I.w2;
  const DdAngle g = I.ang[v];
  const float *src = sino + I.sino + (size_t)g.out_row * n;
  float2 *dst = (float2 *)(work + I.as) + (size_t)v * w2;
  (void)nh;
  for (int e = threadIdx.x; e < w2; e += blockDim.x) {
    const int m = e - pads;
    const float s0 = (m >= 0 && m < n) ? __ldg(src + m) : 0.0f;
    const float s1 = (m + 1 >= 0 && m + 1 < n) ? __ldg(src + m + 1) : 0.0f;
    dst[e] = make_float2(s0, s1);
  }
}

// ---------------------------------------------------------------------------
// Forward: a warp item is 127 detectors of one angle; lane l holds the lower
// boundaries of detectors B0 + 32 j + l (j = 0..3), and T_j = sum over lines of
// F(boundary).  The dropped pieces and the binade corrections come from
// dd_fwd_corr_kernel's row; keeping them out of this loop leaves it 64
// registers (with them inline: 76, and 24 instead of 32 warps per SM).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dd_fwd_lines(int ia, int ib, const double2 *__restrict__ SL, int ws, float k,
                                             int n, int nh, const float (&Dlo)[4], const float (&lo_nh)[4],
                                             double (&T)[4]) {
  float y = (float)(ia - nh) + 0.5f;
  const double2 *sl = SL + (size_t)ia * ws;
  const float nlim = (float)n + 0.25f, cmn = kMagic + (float)nh;
#pragma unroll kFwdUnroll
  for (int i = ia; i < ib; ++i) {
    const float q = __fmul_rn(y, k);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      // kk = floor(D + nh + q) clamped to [-1, n], as a float and an int:
      // t + 1.5 * 2^23 rounded down lies where floats are the integers, so
      // f = 1.5 * 2^23 + floor(t) exactly, and its bits give kk
      const float t = fminf(fmaxf(__fadd_rn(lo_nh[j], q), -0.5f), nlim);
      const float f = __fadd_rd(t, kMagic);
      const int kk = __float_as_int(f) - kMagicBits;
      // P_kk = (kk - nh) - q, with kk - nh = f - (1.5 * 2^23 + nh) exactly
      const float Pk = __fsub_rn(__fsub_rn(f, cmn), q);
      const double2 e = __ldg(sl + kk);
      T[j] = fma((double)__fsub_rn(Dlo[j], Pk), e.y, T[j] + e.x);
    }
    y = __fadd_rn(y, 1.0f);
    sl += ws;
  }
}

// Boundary index of the main loop: kk = floor(D + nh + q) clamped to [-1, n],
// computed exactly as dd_fwd_lines does (lo_nh = D + nh in float).
__device__ __forceinline__ int dd_fwd_kk(float lo_nh, float q, float nlim) {
  const float t = fminf(fmaxf(__fadd_rn(lo_nh, q), -0.5f), nlim);
  return __float_as_int(__fadd_rd(t, kMagic)) - kMagicBits;
}

// Pixel widths that are not 1.  P_j = RN(x_j - q) with x_j integral: while
// |P| < 2^23 (float spacing <= 1/2) all P_j of one binade are x_j minus the
// same rounding of q, so P_j+1 - P_j = 1 exactly; a pixel whose boundaries
// lie in different binades has width 1 + delta, delta the difference of two
// roundings of q: up to 2^(e-23) at |P| ~ 2^e, i.e. 1/16 pixel at 2^19, which
// near-axis angles reach (q = y k with |k| up to 1/|cos|).  dd_fwd_lines
// integrates unit widths, so on each line the detector m whose boundary
// indices bracket such a pixel j (kk_m <= j < kk_m+1, the loop's own kk) is
// short by delta * L_j.  This adds those amounts for the detectors [B0, mEnd)
// to X[m - B0] (a row of the angle's corrections in global memory, zeroed by
// the caller); only lane 0 writes, crossing after crossing, so the sums are
// deterministic.  A crossing is taken at P = +-2^e, e >= 0, each
// pixel at the smallest one it straddles; below |P| = 1 deltas are < 2^-23.
// Lanes take the lines of one crossing in turn; the four sums per crossing
// (the detector holding the crossing and its neighbours) are reduced over the
// warp in a fixed order, so the result is deterministic.
// One crossing, c = 2 e + (B < 0), B = +-2^e: false if no detector of the
// angle can get a correction from it; otherwise mc (the detector holding B)
// and, in every lane, the warp's sums for detectors mc-1 .. mc+2 (a fixed
// butterfly, so deterministic).
constexpr int kNumCrossings = 46;  // e = 0 .. 22, both signs

__device__ __forceinline__ bool dd_fwd_crossing(const float *__restrict__ V, int si, int sj, float k, float r, int n,
                                                int nh, int c, int lane, int &mc, double (&a)[4]) {
  const int e = c >> 1, sg = c & 1;
  const float DA = det_bound(0, nh, r), DB = det_bound(n, nh, r);
  const float nlim = (float)n + 0.25f, fnh = (float)nh;
  const float B = sg ? -ldexpf(1.0f, e) : ldexpf(1.0f, e);
  if (!(B >= DA - 3.0f && B <= DB + 3.0f)) return false;
  // detector holding B: D_mc <= B < D_mc+1
  mc = (int)floor((double)B / (double)r) + nh;
  for (int it = 0; it < 4 && det_bound(mc, nh, r) > B; ++it) --mc;
  for (int it = 0; it < 4 && det_bound(mc + 1, nh, r) <= B; ++it) ++mc;
  // lines on which the crossing lies within [P_0, P_n]: q in [-nh - B - 2, n - nh - B + 2]
  int ia, ib;
  dd_line_range(-(double)nh - B - 2.0, (double)(n - nh) - B + 2.0, (double)k, n, nh, ia, ib);
  // and on which delta can be nonzero: a float q with |q| >= 2^e is a
  // multiple of both binades' spacings (2^(e-24), 2^(e-23)), so then both
  // roundings are exact and the width is 1: only |y k| < 2^e matters
  const double ymax = ldexp(1.0, e) * (1.0 + 1e-6) / fabs((double)k) + 1.0;
  if (ymax < (double)n) {
    ia = max(ia, (int)floor((double)nh - 0.5 - ymax));
    ib = min(ib, (int)ceil((double)nh - 0.5 + ymax));
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) a[t] = 0.0;
#pragma unroll 1
  for (int i = ia + lane; i <= ib; i += 32) {
    const float q = __fmul_rn(__fadd_rn((float)(i - nh), 0.5f), k);
    int j = (int)floor((double)B + (double)q) + nh - 1;
    // j with P_j < B <= P_j+1 (B > 0) or P_j <= B < P_j+1 (B < 0)
    if (!sg) {
      for (int it = 0; it < 4 && pix_bound(j, nh, q) >= B; ++it) --j;
      for (int it = 0; it < 4 && pix_bound(j + 1, nh, q) < B; ++it) ++j;
    } else {
      for (int it = 0; it < 4 && pix_bound(j, nh, q) > B; ++it) --j;
      for (int it = 0; it < 4 && pix_bound(j + 1, nh, q) <= B; ++it) ++j;
    }
    if (j < 0 || j >= n) continue;
    const float Pj = pix_bound(j, nh, q), Pj1 = pix_bound(j + 1, nh, q);
    const bool at = sg ? (Pj <= B && B < Pj1 && (e == 0 || Pj1 <= 0.5f * B))
                       : (Pj < B && B <= Pj1 && (e == 0 || Pj >= 0.5f * B));
    if (!at) continue;
    const float delta = __fsub_rn(__fsub_rn(Pj1, Pj), 1.0f);
    if (delta == 0.0f) continue;
    // the detector m with kk_m <= j < kk_m+1, among mc-1 .. mc+2
    int m = mc;
    for (int it = 0; it < 4; ++it) {
      if (dd_fwd_kk(__fadd_rn(det_bound(m, nh, r), fnh), q, nlim) > j) --m;
      else if (dd_fwd_kk(__fadd_rn(det_bound(m + 1, nh, r), fnh), q, nlim) <= j) ++m;
      else break;
    }
    const double amt = (double)delta * (double)__ldg(V + (size_t)i * si + (size_t)j * sj);
#pragma unroll
    for (int t = 0; t < 4; ++t)
      if (m == mc - 1 + t) a[t] += amt;
  }
#pragma unroll
  for (int t = 0; t < 4; ++t)
    for (int o = 16; o; o >>= 1) a[t] += __shfl_xor_sync(0xffffffffu, a[t], o);
  return true;
}

// An item of an angle whose pixel coordinates reach |P| >= 2^22 (|cos| or
// |sin| ~ 1e-4, q up to nh / |cos|): there the float spacing of P is 1 or more,
// widths are 0 or 2, and neither the unit-width integral nor its binade
// corrections hold.  Each lane walks, for each of its detectors and each line
// meeting it, the overlap pieces of the detector with the line's pixels, from
// the same float boundaries as the reference, the dropped last piece skipped
// (radon_dd.c:125-189), summed in double.
__device__ __forceinline__ void dd_fwd_exact(const double2 *__restrict__ SL, int ws, float k, float r, int n, int nh,
                                          int B0, int mEnd, int lane, double (&T)[4]) {
  const float Dn = det_bound(n, nh, r);
#pragma unroll 1
  for (int t = 0; t < 4; ++t) {
    const int m = B0 + 32 * t + lane;
    if (32 * t + lane >= kGrpDet || m >= mEnd) continue;
    const float Dlo = det_bound(m, nh, r), Dhi = det_bound(m + 1, nh, r);
    int i0, i1;
    dd_line_range(-(double)nh - (double)Dhi, (double)(n - nh) - (double)Dlo, (double)k, n, nh, i0, i1);
    double acc = 0.0;
    for (int i = i0; i <= i1; ++i) {
      const float q = __fmul_rn(__fadd_rn((float)(i - nh), 0.5f), k);
      const float Pn = pix_bound(n, nh, q);
      const bool lastIsPixel = Pn <= Dn;
      const double2 *row = SL + (size_t)i * ws;
      int kk = (int)floor((double)Dlo + (double)q + (double)nh) - 1;
      kk = kk < 0 ? 0 : (kk > n - 1 ? n - 1 : kk);
      float Pk = pix_bound(kk, nh, q);
      while (kk > 0 && Pk > Dlo) Pk = pix_bound(--kk, nh, q);
      for (; kk < n && Pk < Dhi; ++kk) {
        const float Pk1 = pix_bound(kk + 1, nh, q);
        const float lo = fmaxf(Pk, Dlo), hi = fminf(Pk1, Dhi);
        if (hi > lo) {
          const bool drop = lastIsPixel ? (kk == n - 1 && Pn <= Dhi) : (m == n - 1 && Pk1 > Dn);
          if (!drop) acc += (double)__fsub_rn(hi, lo) * __ldg(&row[kk].y);
        }
        Pk = Pk1;
      }
    }
    T[t] = acc;
  }
}

// The binade corrections and the dropped pieces of every angle into the float
// rows X[v][m] that the forward adds where it stores: one block per angle of
// every instance, its warps taking the crossings in turn (dd_fwd_crossing);
// the crossings' sums are added into the row in crossing order through shared
// memory, then each line's dropped piece in line order, so the result is
// deterministic.  A launch of its own, so that the forward's register budget
// is that of its main loop.
__device__ __forceinline__ bool dd_wide(float k, int nh) {
  return fabsf(k) * (float)(nh + 1) + (float)(nh + 2) >= 4194304.0f;
}

constexpr int kCorrWarps = 8, kCorrRow = 4096;  // rows longer than kCorrRow are added in global memory
constexpr int kDropChunk = 1024;                 // lines whose dropped pieces are staged at a time

__global__ void __launch_bounds__(32 * kCorrWarps) dd_fwd_corr_kernel(const DdInst *__restrict__ inst, int ninst,
                                                                      const float *__restrict__ img,
                                                                      double2 *__restrict__ work) {
  __shared__ double sums[kNumCrossings][4];
  __shared__ int smc[kNumCrossings];
  __shared__ float row[kCorrRow];
  __shared__ int ddet[kDropChunk];
  __shared__ double damt[kDropChunk];
  const long long b = blockIdx.x;
  const DdInst &I = inst[find_inst(inst, ninst, b, &DdInst::s0)];
  const int v = (int)(b - I.s0), n = I.n, nh = I.nh;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float *X = reinterpret_cast<float *>(work + I.xs) + (size_t)v * n;
  const DdAngle g = I.ang[v];
  const bool lines = (g.mode == DD_ROWS || g.mode == DD_COLS) && !dd_wide(g.k, nh);
  // pixel j of line i (an image row, or a column) read from the image itself:
  // 17 MB that stay in L2, where the prefix tables' values (134 MB) would not
  const float *V = img + I.img;
  const int si = g.mode == DD_ROWS ? n : 1, sj = g.mode == DD_ROWS ? 1 : n;
  for (int c = warp; c < kNumCrossings; c += kCorrWarps) {
    int mc = 0;
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    const bool used = lines && dd_fwd_crossing(V, si, sj, g.k, g.r, n, nh, c, lane, mc, a);
    if (lane == 0) {
      smc[c] = used ? mc : INT_MIN;
#pragma unroll
      for (int t = 0; t < 4; ++t) sums[c][t] = a[t];
    }
  }
  const bool in_smem = n <= kCorrRow;
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    if (in_smem) row[m] = 0.0f;
    else X[m] = 0.0f;
  }
  __syncthreads();
  float *R = in_smem ? row : X;
  if (threadIdx.x == 0) {
    for (int c = 0; c < kNumCrossings; ++c) {
      if (smc[c] == INT_MIN) continue;
      for (int t = 0; t < 4; ++t) {
        const int m = smc[c] - 1 + t;
        if (m >= 0 && m < n) R[m] += (float)sums[c][t];
      }
    }
  }
  // The piece of every line the reference never credits (dd_dropped_piece),
  // subtracted from its detector, line after line by one thread.
  if (lines) {
    for (int i0 = 0; i0 < n; i0 += kDropChunk) {
      __syncthreads();
      for (int t = threadIdx.x; t < kDropChunk && i0 + t < n; t += blockDim.x) {
        const int i = i0 + t;
        const float q = __fmul_rn(__fadd_rn((float)(i - nh), 0.5f), g.k);
        DdDrop d;
        int det = -1;
        double amt = 0.0;
        if (dd_dropped_piece(q, g.r, n, nh, d)) {
          det = d.det;
          amt = (double)d.gap * (double)__ldg(V + (size_t)i * si + (size_t)d.pix * sj);
        }
        ddet[t] = det;
        damt[t] = amt;
      }
      __syncthreads();
      // warp 0, 32 lines at a time: the lanes with the same detector form a
      // group whose lowest lane subtracts the group's pieces summed in line
      // order; different groups touch different detectors, and the batches
      // go in line order
      if (warp == 0)
        for (int t0 = 0; t0 < kDropChunk && i0 + t0 < n; t0 += 32) {
          const int t = t0 + lane;
          const int det = i0 + t < n ? ddet[t] : -1;
          const unsigned grp = __match_any_sync(0xffffffffu, det);
          if (det >= 0 && lane == __ffs(grp) - 1) {
            double sum = 0.0;
            for (unsigned mk = grp; mk; mk &= mk - 1) sum += damt[t0 + __ffs(mk) - 1];
            R[det] = __double2float_rn((double)R[det] - sum);
          }
          __syncwarp();
        }
    }
  }
  __syncthreads();
  if (in_smem)
    for (int m = threadIdx.x; m < n; m += blockDim.x) X[m] = row[m];
}

__device__ __forceinline__ void dd_fwd_item(const DdInst &I, int v, int grp, int lane,
                                            const double2 *__restrict__ work, float *__restrict__ sino,
                                            const FwdEpi &ep, long long slot) {
  const DdAngle g = I.ang[v];
  const int n = I.n, nh = I.nh, ws = n + 2;
  const int B0 = grp * kGrpDet;
  const double2 *SLr = work + I.sl + 1, *SLc = SLr + (size_t)n * ws;
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  if (g.mode == DD_ROWSUM || g.mode == DD_COLSUM) {
    // detector m <- total of image row m (ROWSUM) or column m (COLSUM)
    const double2 *SL = g.mode == DD_ROWSUM ? SLr : SLc;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int m = B0 + 32 * j + lane;
      if (32 * j + lane < kGrpDet && m < n) acc[j] = (float)__ldg(&SL[(size_t)m * ws + n].x);
    }
  } else if (g.mode == DD_ROWS || g.mode == DD_COLS) {
    const double2 *SL = g.mode == DD_ROWS ? SLr : SLc;
    const float r = g.r, k = g.k;
    float Dlo[4], lo_nh[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      Dlo[j] = det_bound(B0 + 32 * j + lane, nh, r);
      lo_nh[j] = __fadd_rn(Dlo[j], (float)nh);
    }
    const int mEnd = min(B0 + kGrpDet, n);
    const double DA = (double)det_bound(B0, nh, r), DB = (double)det_bound(mEnd, nh, r);
    const double kd = (double)k, PN = (double)(n - nh);
    int i0, i1;
    dd_line_range(-(double)nh - DB, PN - DA, kd, n, nh, i0, i1);
    if (dd_wide(k, nh)) {
      // |P| reaches 2^22: pieces walked exactly (rare near-axis angles)
      double T[4] = {0.0, 0.0, 0.0, 0.0};
      dd_fwd_exact(SL, ws, k, r, n, nh, B0, mEnd, lane, T);
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[j] = (float)T[j];
    } else {
      double T[4] = {0.0, 0.0, 0.0, 0.0};
      dd_fwd_lines(i0, i1 + 1, SL, ws, k, n, nh, Dlo, lo_nh, T);
      // the upper boundary of detector B0 + 32 j + l is lane l+1's j-th, or lane 0's (j+1)-th
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double a = __shfl_down_sync(0xffffffffu, T[j], 1);
        const double b = __shfl_sync(0xffffffffu, j < 3 ? T[j < 3 ? j + 1 : 3] : 0.0, 0);
        const double up = lane < 31 ? a : b;
        const int m = B0 + 32 * j + lane;
        const float x = (32 * j + lane < kGrpDet && m < n)
                            ? __ldg(reinterpret_cast<const float *>(work + I.xs) + (size_t)v * n + m)
                            : 0.0f;
        acc[j] = (float)((up - T[j]) + (double)x);
      }
    }
  }
  double r2 = 0.0;
  const size_t row = (size_t)I.sino + (size_t)g.out_row * n;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int m = B0 + 32 * j + lane;
    if (32 * j + lane < kGrpDet && m < n) sino[row + m] = fwd_apply(ep, acc[j], row + m, r2);
  }
  fwd_resid_commit(ep, r2, (size_t)slot);
}

// Work fetch.  BLOCK: a block takes W consecutive items at a time (for the
// forward, consecutive angles of one detector group, whose warps read nearly
// the same prefix lines, which then hit in L1); otherwise each warp takes one
// item.  The autotuner picks the mode; results do not depend on it.
template <bool BLOCK>
__device__ __forceinline__ long long fetch_item(unsigned long long *ctr, int W, long long *slot) {
  if (BLOCK) {
    if (threadIdx.x == 0) *slot = (long long)atomicAdd(ctr, (unsigned long long)W);
    __syncthreads();
    const long long b = *slot;
    __syncthreads();
    return b + (threadIdx.x >> 5);
  }
  unsigned long long it = 0;
  if ((threadIdx.x & 31) == 0) it = atomicAdd(ctr, 1ull);
  return (long long)__shfl_sync(0xffffffffu, it, 0);
}

// Detector groups are taken centre first: central groups meet the most lines,
// so the long items run first and the short ones fill the tail.
__device__ __forceinline__ int centre_out(int gi, int ngrp) {
  const int c = (ngrp - 1) >> 1;
  return (gi & 1) ? c + ((gi + 1) >> 1) : c - (gi >> 1);
}

template <int W, bool BLOCK>
__global__ void __launch_bounds__(32 * W) dd_fwd_kernel(const DdInst *__restrict__ inst, int ninst,
                                                         long long nitems, unsigned long long *__restrict__ ctr,
                                                         const double2 *__restrict__ work,
                                                         float *__restrict__ sino, FwdEpi ep) {
  __shared__ long long base_s;
  const int lane = threadIdx.x & 31;
  for (;;) {
    const long long item = fetch_item<BLOCK>(ctr, W, &base_s);
    if (item - (BLOCK ? (threadIdx.x >> 5) : 0) >= nitems) break;  // block-uniform under BLOCK
    if (item < nitems) {
      const DdInst &I = inst[find_inst(inst, ninst, item, &DdInst::f0)];
      // items run all angles on row lines (every detector group) before those on
      // column lines, so that the warps in flight read one of the two prefix
      // tables at a time (each about half of L2 at 2048^2)
      const int local = (int)(item - I.f0), nRg = I.nRf * I.ngrp;
      int gi, v;
      if (local < nRg) {
        gi = local / I.nRf;
        v = __ldg(I.fperm + local % I.nRf);
      } else {
        const int l2 = local - nRg, nCf = I.na - I.nRf;
        gi = l2 / nCf;
        v = __ldg(I.fperm + I.nRf + l2 % nCf);
      }
      dd_fwd_item(I, v, centre_out(gi, I.ngrp), lane, work, sino, ep, item);
    }
  }
}

// ---------------------------------------------------------------------------
// Adjoint: a warp item is a 32x16 pixel tile; lane l holds the 4x4 pixels at
// rows a0..a0+3 and columns b0..b0+3.  Per angle and line each pixel [P0, P1]
// overlaps the detector a holding P0 and possibly a+1 (detectors are at least
// one pixel wide): (min(D_a+1, P1) - P0) S_a + (P1 - min(D_a+1, P1)) S_a+1,
// the reference's two gaps, both accumulated by FMA.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dd_adj_pixel(float P0, float P1, float z, float r, float cm, float cm1,
                                             const float2 *__restrict__ rowm, float &acc) {
  // f = cm + floor(P0 z) exactly: rounded down in [2^23, 2^24), where floats
  // are the integers; a = floor(P0 z + nh) is f's bits minus kMagicBits (rowm
  // is the row base minus kMagicBits entries)
  const float f = __fmaf_rd(P0, z, cm);
  const float2 t = __ldg(rowm + __float_as_int(f));  // {S_a, S_a+1}
  // D_a+1 = (a + 1 - nh) r, with a + 1 - nh = f - (kMagic + nh - 1) exactly
  const float D1 = __fmul_rn(__fsub_rn(f, cm1), r);
  const float m = fminf(D1, P1);
  acc = __fmaf_rn(__fsub_rn(m, P0), t.x, acc);
  acc = __fmaf_rn(__fsub_rn(P1, m), t.y, acc);
}

template <bool COLS>
__device__ __forceinline__ void dd_adj_pass(const float4 *__restrict__ tab, int cnt,
                                            const float2 *__restrict__ AS, int a0, int b0, int n, int nh,
                                            float (&acc)[4][4]) {
  const int l0 = COLS ? b0 : a0, k0 = COLS ? a0 : b0;
  const float y0 = (float)(l0 - nh) + 0.5f;
  float x[5];
#pragma unroll
  for (int j = 0; j < 5; ++j) x[j] = (float)(k0 - nh + j);
  const float cm = kMagic + (float)nh, cm1 = cm - 1.0f;
#pragma unroll 1
  for (int u = 0; u < cnt; ++u) {
    const float4 e = __ldg(tab + u);
    const float r = e.x, k = e.y, z = e.z;
    const float2 *rowm = AS + __float_as_int(e.w) - kMagicBits;
#pragma unroll
    for (int li = 0; li < 4; ++li) {
      const float q = __fmul_rn(__fadd_rn(y0, (float)li), k);
      float P[5];
#pragma unroll
      for (int j = 0; j < 5; ++j) P[j] = __fsub_rn(x[j], q);
#pragma unroll
      for (int j = 0; j < 4; ++j) dd_adj_pixel(P[j], P[j + 1], z, r, cm, cm1, rowm, COLS ? acc[j][li] : acc[li][j]);
    }
  }
}

// The adjoint's dropped pieces (the last piece of each line and angle that
// the reference never credits, dd_dropped_piece), as an image C that the
// adjoint adds where it stores: a warp per line (an image row for the angles
// on rows, a column for those on columns), 32 angles at a time; the lanes
// whose pieces fall on the same pixel form a group whose lowest lane
// subtracts their sum, taken in angle order, from C.  The row launch zeroes
// its lines first and runs before the column launch, so every pixel gets its
// pieces in one fixed order.  Out of the adjoint's main loop, which then holds
// 64 registers (with the pieces inline: 80, and 24 instead of 32 warps per SM).
template <bool COLS>
__global__ void __launch_bounds__(32) dd_adj_drop_kernel(const DdInst *__restrict__ inst, int ninst,
                                                         double2 *__restrict__ work) {
  __shared__ double samt[32];
  const long long b = blockIdx.x;
  const DdInst &I = inst[find_inst(inst, ninst, b, &DdInst::r0)];
  const int l = (int)(b - I.r0), n = I.n, nh = I.nh, lane = threadIdx.x;
  float *C = reinterpret_cast<float *>(work + I.xs);
  const size_t si = COLS ? 1 : (size_t)n, sp = COLS ? (size_t)n : 1;  // pixel p of line l: C[l si + p sp]
  if (!COLS)
    for (int p = lane; p < n; p += 32) C[(size_t)l * n + p] = 0.0f;
  __syncwarp();
  const float4 *tab = I.tab + (COLS ? I.nR : 0);
  const int cnt = COLS ? I.nC : I.nR;
  const float2 *AS = (const float2 *)(work + I.as) + I.pads;
  const float y = __fadd_rn((float)(l - nh), 0.5f);
  for (int u0 = 0; u0 < cnt; u0 += 32) {
    const int u = u0 + lane;
    int pix = -1;
    float amt = 0.0f;
    if (u < cnt) {
      const float4 e = __ldg(tab + u);
      DdDrop d;
      if (dd_dropped_piece(__fmul_rn(y, e.y), e.x, n, nh, d)) {
        pix = d.pix;
        amt = __fmul_rn(d.gap, __ldg(&(AS + __float_as_int(e.w))[d.det].x));
      }
    }
    samt[lane] = (double)amt;
    __syncwarp();
    const unsigned grp = __match_any_sync(0xffffffffu, pix);
    if (pix >= 0 && lane == __ffs(grp) - 1) {
      double sum = 0.0;
      for (unsigned mk = grp; mk; mk &= mk - 1) sum += samt[__ffs(mk) - 1];
      float *c = C + (size_t)l * si + (size_t)pix * sp;
      *c = __double2float_rn((double)*c - sum);
    }
    __syncwarp();
  }
}

// One item = one 32x16 tile, worked on by 4 warps: warp `quarter` sums the
// angles [quarter T / 4, (quarter + 1) T / 4) of the ROWS-then-COLS order (T =
// nR + nC), and the tile's first warp adds the quarters in order, then the
// row / column sums, then stores.  The split never depends on the launch
// shape, so every shape gives the same bits.
template <int TB>
__global__ void __launch_bounds__(128 * TB) dd_adj_kernel(const DdInst *__restrict__ inst, int ninst,
                                                           long long nitems, unsigned long long *__restrict__ ctr,
                                                           const double2 *__restrict__ work,
                                                           float *__restrict__ img, AdjEpi ep) {
  __shared__ long long base_s;
  __shared__ float part[TB][3][16][32];  // quarters 1..3 of each tile
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tile = warp >> 2, quarter = warp & 3;
  for (;;) {
    if (threadIdx.x == 0) base_s = (long long)atomicAdd(ctr, (unsigned long long)TB);
    __syncthreads();
    const long long first = base_s;
    __syncthreads();
    if (first >= nitems) break;  // block-uniform
    const long long item = first + tile;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
    const DdInst *Ip = nullptr;
    int a0 = 0, b0 = 0;
    bool inside = false;
    if (item < nitems) {
      Ip = &inst[find_inst(inst, ninst, item, &DdInst::a0)];
      const DdInst &I = *Ip;
      const int local = (int)(item - I.a0);
      b0 = (local % I.tx) * kTileW + 4 * (lane & 7);
      a0 = (local / I.tx) * kTileH + 4 * (lane >> 3);
      // lanes whose block starts outside the image (n not a multiple of 4)
      // only take part in the epilogue's warp reductions
      inside = a0 < I.n && b0 < I.n;
      if (inside) {
        const int T = I.nR + I.nC;
        const int u0 = (int)((long long)T * quarter / 4), u1 = (int)((long long)T * (quarter + 1) / 4);
        const float2 *AS = (const float2 *)(work + I.as) + I.pads;
        const int r0 = min(u0, I.nR), r1 = min(u1, I.nR);
        if (r1 > r0) dd_adj_pass<false>(I.tab + r0, r1 - r0, AS, a0, b0, I.n, I.nh, acc);
        const int c0 = max(u0, I.nR), c1 = max(u1, I.nR);
        if (c1 > c0) dd_adj_pass<true>(I.tab + c0, c1 - c0, AS, a0, b0, I.n, I.nh, acc);
      }
    }
    if (quarter > 0) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) part[tile][quarter - 1][4 * i + j][lane] = acc[i][j];
    }
    __syncthreads();
    if (quarter == 0 && Ip) {
      const DdInst &I = *Ip;
      const int n = I.n;
#pragma unroll
      for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] += part[tile][q][4 * i + j][lane];
      const float2 *AS = (const float2 *)(work + I.as) + I.pads;
      for (int t = 0; inside && t < I.nS; ++t) {  // row / column sums (|sin| or |cos| < 1e-7)
        const int2 e = __ldg(I.tabS + t);
        const float2 *row = AS + e.y;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] += __ldg(&row[e.x == DD_ROWSUM ? a0 + i : b0 + j].x);
      }
      // the dropped pieces (dd_adj_drop_kernel)
      const float *Cimg = reinterpret_cast<const float *>(work + I.xs);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int a = a0 + i, b = b0 + j;
          const bool live = inside && a < n && b < n;
          if (live) acc[i][j] += __ldg(Cimg + (size_t)a * n + b);
          adj_store(ep, acc[i][j], live, (size_t)I.img + (size_t)(live ? a : 0) * n + (live ? b : 0), img);
        }
    }
    __syncthreads();  // part[] is rewritten by the next item
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

namespace {

// Per-plan state: the instance table, the geometry tables of every distinct
// geometry, the persistent kernels' work counters and the tuned launch shape.
struct DdState {
  std::vector<DdInst> inst;  // scheduling order (largest work first)
  DdInst *d_inst = nullptr;
  void *d_tables = nullptr;
  unsigned long long *d_ctr = nullptr;  // [0] forward items, [1] adjoint items
  long long fwd_items = 0, adj_items = 0, row_blocks = 0, col_blocks = 0, sino_blocks = 0;
  double updates = 0.0;  // pixel x angle updates per application
  int wf = 1, wa = 1;    // launch shape (kDdCfg index) of the forward / adjoint kernels
  int grid_f = 0, grid_a = 0;
  std::vector<size_t> img_off, sino_off;  // packed offsets in the caller's order (count + 1)
  std::string tuning;
};

void dd_state_free(void *q) {
  auto *S = (DdState *)q;
  if (S->d_inst) cudaFree(S->d_inst);
  if (S->d_tables) cudaFree(S->d_tables);
  if (S->d_ctr) cudaFree(S->d_ctr);
  delete S;
}

using FwdFn = void (*)(const DdInst *, int, long long, unsigned long long *, const double2 *, float *,
                      FwdEpi);
using AdjFn = void (*)(const DdInst *, int, long long, unsigned long long *, const double2 *, float *,
                      AdjEpi);
// Launch shapes the autotuner chooses from.  Forward: warps per block x
// fetch mode.  Adjoint: tiles per block (4 warps each).
struct DdCfg {
  int W;
  bool block;
  FwdFn fwd;
};
const DdCfg kDdCfg[] = {
    {2, false, dd_fwd_kernel<2, false>}, {4, false, dd_fwd_kernel<4, false>}, {8, false, dd_fwd_kernel<8, false>},
    {2, true, dd_fwd_kernel<2, true>},   {4, true, dd_fwd_kernel<4, true>},   {8, true, dd_fwd_kernel<8, true>},
};
constexpr int kNumCfg = (int)(sizeof(kDdCfg) / sizeof(kDdCfg[0]));
struct AdjCfg {
  int TB;
  AdjFn adj;
};
const AdjCfg kAdjCfg[] = {{1, dd_adj_kernel<1>}, {2, dd_adj_kernel<2>}, {4, dd_adj_kernel<4>}};
constexpr int kNumAdj = (int)(sizeof(kAdjCfg) / sizeof(kAdjCfg[0]));
int num_cfg(bool fwd) { return fwd ? kNumCfg : kNumAdj; }
std::string cfg_name(int c, bool fwd = true) {
  if (!fwd) return "t" + std::to_string(kAdjCfg[c].TB);
  return "w" + std::to_string(kDdCfg[c].W) + (kDdCfg[c].block ? "b" : "w");
}
int cfg_threads(int c, bool fwd) { return fwd ? 32 * kDdCfg[c].W : 128 * kAdjCfg[c].TB; }

// Persistent grid: as many blocks as fit on the device at once.
int dd_grid(int c, bool fwd, int *grid) {
  int dev = 0, sms = 0, nb = 0;
  TOMO_CUDA(cudaGetDevice(&dev));
  TOMO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const void *k = fwd ? (const void *)kDdCfg[c].fwd : (const void *)kAdjCfg[c].adj;
  TOMO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, cfg_threads(c, fwd), 0));
  *grid = std::max(1, nb) * sms;
  return TOMO_OK;
}

int dd_launch_fwd(const DdState &S, int c, int grid, const double2 *work, float *sino, cudaStream_t s,
                  const FwdEpi &ep) {
  TOMO_CUDA(cudaMemsetAsync(S.d_ctr, 0, sizeof(unsigned long long), s));
  kDdCfg[c].fwd<<<grid, 32 * kDdCfg[c].W, 0, s>>>(S.d_inst, (int)S.inst.size(), S.fwd_items, S.d_ctr, work,
                                                    sino, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int dd_launch_adj(const DdState &S, int c, int grid, const double2 *work, float *img, cudaStream_t s,
                  const AdjEpi &ep) {
  TOMO_CUDA(cudaMemsetAsync(S.d_ctr + 1, 0, sizeof(unsigned long long), s));
  kAdjCfg[c].adj<<<grid, cfg_threads(c, false), 0, s>>>(S.d_inst, (int)S.inst.size(), S.adj_items,
                                                         S.d_ctr + 1, work, img, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

// Tuned shapes, shared by plans of the same workload within the process.
std::mutex g_tune_mu;
std::map<std::tuple<long long, long long, int, int, int>, std::pair<int, int>> g_tuned;

constexpr double kTuneMinUpdates = 5e7;  // below this the default shape is used untimed

// Chooses the launch shape (warps per block and fetch mode, kDdCfg) of the
// forward and adjoint kernels by timing each candidate on the plan's own
// scratch: the scratch is zeroed, the forward reads its prefix-line area and
// writes into its sinogram-row area, the adjoint the reverse, so no caller
// buffer is touched.  The choice does not change any result (each output is
// owned by one lane whatever the shape), only the time.
int dd_autotune(Plan &p, DdState &S) {
  const auto key = std::make_tuple(S.fwd_items, S.adj_items, (int)S.inst.size(), S.inst[0].n, S.inst[0].na);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      S.wf = it->second.first;
      S.wa = it->second.second;
      S.tuning = "cached";
    }
  }
  if (S.tuning.empty() && S.updates >= kTuneMinUpdates) {
    cudaStream_t st;
    TOMO_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double2 *work = (double2 *)p.d_scratch;
    int rc = TOMO_OK;
    if (cudaMemsetAsync(p.d_scratch, 0, p.scratch_bytes, st) != cudaSuccess) rc = TOMO_ECUDA;
    // the sinogram-row area (after all prefix lines) holds the packed sinograms,
    // the prefix-line area the packed images
    float *fwd_out = (float *)(work + S.inst[0].as);
    float *adj_out = (float *)work;
    std::string log;
    for (int dir = 0; dir < 2 && rc == TOMO_OK; ++dir) {
      float best = 1e30f;
      log += dir == 0 ? "fwd" : "; adj";
      for (int c = 0; c < num_cfg(dir == 0) && rc == TOMO_OK; ++c) {
        int grid = 0;
        if ((rc = dd_grid(c, dir == 0, &grid))) break;
        float ms = 0.0f;
        for (int rep = 0; rep < 3 && rc == TOMO_OK; ++rep) {
          cudaEventRecord(e0, st);
          rc = dir == 0 ? dd_launch_fwd(S, c, grid, work, fwd_out, st, FwdEpi())
                        : dd_launch_adj(S, c, grid, work, adj_out, st, AdjEpi());
          cudaEventRecord(e1, st);
          cudaEventSynchronize(e1);
          float t = 0.0f;
          cudaEventElapsedTime(&t, e0, e1);
          if (rep) ms += t;
        }
        char buf[48];
        std::snprintf(buf, sizeof(buf), " %s=%.3fms", cfg_name(c, dir == 0).c_str(), ms / 2);
        log += buf;
        if (ms < best) {
          best = ms;
          (dir == 0 ? S.wf : S.wa) = c;
        }
      }
    }
    cudaError_t err = cudaStreamSynchronize(st);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    if (rc) return rc;
    if (err != cudaSuccess) return cuda_fail(err, "dd autotune");
    S.tuning = "timed:" + log.substr(0);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = std::make_pair(S.wf, S.wa);
  }
  if (S.tuning.empty()) S.tuning = "default (small workload)";
  int rc = dd_grid(S.wf, true, &S.grid_f);
  if (!rc) rc = dd_grid(S.wa, false, &S.grid_a);
  S.tuning = "fwd " + cfg_name(S.wf) + ", adj " + cfg_name(S.wa, false) +
             " (forward w<warps/block> + b: block fetch, w: warp fetch; adjoint t<tiles/block>)" +
             ", grids " + std::to_string(S.grid_f) + "/" + std::to_string(S.grid_a) + " (" + S.tuning + ")";
  return rc;
}

// One geometry of a plan or batch: n, angles and the number of slices.
struct DdGeo {
  int n, na, nz;
  const float *angles;
};

// Builds the instance table, the device tables and the scratch of a plan
// whose geometries are geo[0..count) (in the caller's packed order).
int dd_build(Plan &p, const DdGeo *geo, int count) {
  auto *S = new DdState();
  p.ext = S;
  p.ext_free = dd_state_free;
  // host tables per geometry, packed into one device buffer
  struct GeoTabs {
    size_t ang, tab, tabS, fperm;
    int nR, nC, nS, pads, w2, nRf;
  };
  std::vector<GeoTabs> gt(count);
  std::vector<char> blob;
  auto put = [&blob](const void *src, size_t bytes) {
    const size_t off = (blob.size() + 15) / 16 * 16;
    blob.resize(off + bytes);
    if (bytes) std::memcpy(blob.data() + off, src, bytes);
    return off;
  };
  for (int gi = 0; gi < count; ++gi) {
    const DdGeo &G = geo[gi];
    const int n = G.n, na = G.na, nh = (int)(n * 0.5);
    std::vector<DdAngle> tab(na);
    int rc = dd_build_table(G.angles, na, tab.data());
    if (rc) return rc;
    GeoTabs &t = gt[gi];
    // detector boundaries of every pixel boundary of the image (and of a
    // 4-pixel tile margin beyond it) lie within pads entries of [0, n)
    t.pads = (int)std::ceil((nh + 1) * (std::sqrt(2.0) - 1.0)) + 12;
    t.w2 = n + 2 * t.pads;
    if ((double)na * t.w2 >= 2147483647.0) return fail(TOMO_EINVAL, "dd: nang * (npix + pads) too large");
    std::vector<float4> rows, cols;
    std::vector<int2> sums;
    for (int v = 0; v < na; ++v) {
      const DdAngle &a = tab[v];
      const int off = v * t.w2;
      if (a.mode == DD_ROWS || a.mode == DD_COLS) {
        // z = 1/r (the sine or cosine): the detector of a boundary P is about P z + nh
        float s, c;
        sincosf(G.angles[v], &s, &c);
        float4 e = make_float4(a.r, a.k, a.mode == DD_ROWS ? s : c, 0.0f);
        std::memcpy(&e.w, &off, sizeof(int));
        (a.mode == DD_ROWS ? rows : cols).push_back(e);
      } else if (a.mode == DD_ROWSUM || a.mode == DD_COLSUM) {
        sums.push_back(make_int2(a.mode, off));
      }
    }
    t.nR = (int)rows.size();
    t.nC = (int)cols.size();
    t.nS = (int)sums.size();
    // forward order: angles on row lines (ROWS, ROWSUM) first, each group in angle order
    std::vector<int> fperm;
    for (int pass = 0; pass < 2; ++pass)
      for (int v = 0; v < na; ++v) {
        const bool on_rows = tab[v].mode == DD_ROWS || tab[v].mode == DD_ROWSUM;
        if (on_rows == (pass == 0)) fperm.push_back(v);
      }
    t.nRf = 0;
    for (int v = 0; v < na; ++v) t.nRf += (tab[v].mode == DD_ROWS || tab[v].mode == DD_ROWSUM) ? 1 : 0;
    t.fperm = put(fperm.data(), sizeof(int) * na);
    rows.insert(rows.end(), cols.begin(), cols.end());
    t.ang = put(tab.data(), sizeof(DdAngle) * na);
    t.tab = put(rows.data(), sizeof(float4) * rows.size());
    t.tabS = put(sums.data(), sizeof(int2) * sums.size());
  }
  TOMO_CUDA(cudaMalloc(&S->d_tables, std::max<size_t>(blob.size(), 16)));
  TOMO_CUDA(cudaMemcpy(S->d_tables, blob.data(), blob.size(), cudaMemcpyHostToDevice));
  const char *tb = (const char *)S->d_tables;
  // instances in the caller's order, with packed offsets
  std::vector<DdInst> inst;
  std::vector<double> cost;
  size_t io = 0, so = 0;
  S->img_off.push_back(0);
  S->sino_off.push_back(0);
  for (int gi = 0; gi < count; ++gi) {
    const DdGeo &G = geo[gi];
    const GeoTabs &t = gt[gi];
    for (int z = 0; z < G.nz; ++z) {
      DdInst I{};
      I.n = G.n;
      I.nh = (int)(G.n * 0.5);
      I.na = G.na;
      I.pads = t.pads;
      I.w2 = t.w2;
      I.nR = t.nR;
      I.nC = t.nC;
      I.nS = t.nS;
      I.ngrp = (G.n + kGrpDet - 1) / kGrpDet;
      I.tx = (G.n + kTileW - 1) / kTileW;
      I.ty = (G.n + kTileH - 1) / kTileH;
      I.ang = (const DdAngle *)(tb + t.ang);
      I.tab = (const float4 *)(tb + t.tab);
      I.tabS = (const int2 *)(tb + t.tabS);
      I.fperm = (const int *)(tb + t.fperm);
      I.nRf = t.nRf;
      I.img = (long long)io;
      I.sino = (long long)so;
      io += (size_t)G.n * G.n;
      so += (size_t)G.na * G.n;
      S->img_off.push_back(io);
      S->sino_off.push_back(so);
      inst.push_back(I);
      cost.push_back((double)G.n * G.n * G.na);
      S->updates += (double)G.n * G.n * G.na;
    }
  }
  // scheduling order: largest work first, caller's order among equals
  std::vector<int> order(inst.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&cost](int a, int b) { return cost[a] > cost[b]; });
  // scratch: every instance's prefix lines, then every instance's sinogram rows
  size_t work = 0;
  for (int idx : order) work += 2 * (size_t)inst[idx].n * (inst[idx].n + 2);
  size_t sl_at = 0, as_at = work;
  for (int idx : order) work += (size_t)inst[idx].na * inst[idx].w2;
  // float rows, 4 to a double2: the forward's corrections [na][n] or, in an
  // adjoint, the dropped-piece image [n][n] (never both at once)
  size_t xs_at = work;
  for (int idx : order) work += ((size_t)std::max(inst[idx].na, inst[idx].n) * inst[idx].n + 3) / 4;
  for (int idx : order) {
    DdInst I = inst[idx];
    I.sl = (long long)sl_at;
    sl_at += 2 * (size_t)I.n * (I.n + 2);
    I.as = (long long)as_at;
    as_at += (size_t)I.na * I.w2;
    I.xs = (long long)xs_at;
    xs_at += ((size_t)std::max(I.na, I.n) * I.n + 3) / 4;
    I.f0 = S->fwd_items;
    S->fwd_items += (long long)I.na * I.ngrp;
    I.a0 = S->adj_items;
    S->adj_items += (long long)I.tx * I.ty;
    I.r0 = S->row_blocks;
    S->row_blocks += I.n;
    I.c0 = S->col_blocks;
    S->col_blocks += (I.n + 31) / 32;
    I.s0 = S->sino_blocks;
    S->sino_blocks += I.na;
    S->inst.push_back(I);
  }
  if (S->row_blocks > 2147483647LL || S->sino_blocks > 2147483647LL)
    return fail(TOMO_EINVAL, "dd: batch too large for one launch");
  TOMO_CUDA(cudaMalloc(&S->d_inst, sizeof(DdInst) * S->inst.size()));
  TOMO_CUDA(cudaMemcpy(S->d_inst, S->inst.data(), sizeof(DdInst) * S->inst.size(), cudaMemcpyHostToDevice));
  TOMO_CUDA(cudaMalloc(&S->d_ctr, 2 * sizeof(unsigned long long)));
  p.scratch_bytes = sizeof(double2) * work;
  TOMO_CUDA(cudaMalloc(&p.d_scratch, p.scratch_bytes));
  p.fwd_warps = (size_t)S->fwd_items;  // one residual partial per forward item
  p.img_total = io;
  p.sino_total = so;
  return dd_autotune(p, *S);
}

}  // namespace

int dd_setup(Plan &p) {
  DdGeo G{p.g.n, p.g.na, p.g.nz, p.angles.data()};
  return dd_build(p, &G, 1);
}

int dd_setup_batch(Plan &p, const tomo_geom *geoms, int count) {
  std::vector<DdGeo> geo(count);
  for (int i = 0; i < count; ++i) geo[i] = DdGeo{geoms[i].n, geoms[i].na, geoms[i].nz, geoms[i].angles};
  return dd_build(p, geo.data(), count);
}

int dd_layout(const Plan &p, int *instances, size_t *img_off, size_t *sino_off, size_t cap) {
  const DdState &S = *(const DdState *)p.ext;
  const size_t ni = S.img_off.size() - 1;
  if (instances) *instances = (int)ni;
  if (img_off || sino_off) {
    if (cap < ni + 1) return fail(TOMO_EINVAL, "layout: arrays need instances + 1 entries");
    for (size_t i = 0; i <= ni; ++i) {
      if (img_off) img_off[i] = S.img_off[i];
      if (sino_off) sino_off[i] = S.sino_off[i];
    }
  }
  return TOMO_OK;
}

const std::string &dd_tuning(const Plan &p) { return ((const DdState *)p.ext)->tuning; }

int dd_set_tuning(Plan &p, const char *fwd, const char *adj) {
  DdState &S = *(DdState *)p.ext;
  int wf = S.wf, wa = S.wa;
  for (int dir = 0; dir < 2; ++dir) {
    const char *name = dir == 0 ? fwd : adj;
    if (!name) continue;
    int found = -1;
    for (int c = 0; c < num_cfg(dir == 0); ++c)
      if (cfg_name(c, dir == 0) == name) found = c;
    if (found < 0) return fail(TOMO_EINVAL, std::string("set_tuning: unknown ") + (dir ? "adjoint" : "forward") +
                                                " shape '" + name + "'");
    (dir == 0 ? wf : wa) = found;
  }
  int rc = dd_grid(wf, true, &S.grid_f);
  if (!rc) rc = dd_grid(wa, false, &S.grid_a);
  if (rc) return rc;
  S.wf = wf;
  S.wa = wa;
  S.tuning = "fwd " + cfg_name(wf) + ", adj " + cfg_name(wa, false) + " (set by the caller)";
  return TOMO_OK;
}

int dd_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const DdState &S = *(const DdState *)p.ext;
  double2 *work = (double2 *)p.d_scratch;
  const int ni = (int)S.inst.size();
  dd_row_prefix_kernel<<<(unsigned)S.row_blocks, kScanThreads, 0, s>>>(S.d_inst, ni, d_img, work);
  dd_col_prefix_kernel<<<(unsigned)S.col_blocks, 32 * kColWarps, 0, s>>>(S.d_inst, ni, d_img, work);
  dd_fwd_corr_kernel<<<(unsigned)S.sino_blocks, 32 * kCorrWarps, 0, s>>>(S.d_inst, ni, d_img, work);
  TOMO_CUDA(cudaGetLastError());
  return dd_launch_fwd(S, S.wf, S.grid_f, work, d_sino, s, ep);
}

int dd_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s, const AdjEpi &ep) {
  const DdState &S = *(const DdState *)p.ext;
  double2 *work = (double2 *)p.d_scratch;
  const int ni = (int)S.inst.size();
  dd_sino_expand_kernel<<<(unsigned)S.sino_blocks, kScanThreads, 0, s>>>(S.d_inst, ni, d_sino, work);
  dd_adj_drop_kernel<false><<<(unsigned)S.row_blocks, 32, 0, s>>>(S.d_inst, ni, work);
  dd_adj_drop_kernel<true><<<(unsigned)S.row_blocks, 32, 0, s>>>(S.d_inst, ni, work);
  TOMO_CUDA(cudaGetLastError());
  return dd_launch_adj(S, S.wa, S.grid_a, work, d_img, s, ep);
}

}  // namespace tomo
