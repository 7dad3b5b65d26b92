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
// Forward: one thread per (detector, angle, slice) walks the image lines that
// overlap its detector and the pixels of each line inside [D_m, D_m+1].
// Adjoint: one thread per pixel walks the angles and the (at most two)
// detectors its interval overlaps.  Both read zero-guarded copies of their
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

__global__ void __launch_bounds__(128) dd_forward_v2_kernel(
    const float *__restrict__ Lr, const float *__restrict__ Lc, float *__restrict__ sino,
    const DdAngle *__restrict__ tab, int n, int nh, int na, int wl, FwdEpi ep) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  const size_t z = blockIdx.z;
  const bool live = m < n;
  const DdAngle g = tab[v];
  float acc = 0.0f;
  if (live) {
    const float *Rz = Lr + z * (size_t)n * wl + kPadL, *Cz = Lc + z * (size_t)n * wl + kPadL;
    if (g.mode == DD_ROWSUM) {  // detector m <- image row m = Lc[j][m]
      for (int j = 0; j < n; ++j) acc += __ldg(Cz + (size_t)j * wl + m);
    } else if (g.mode == DD_COLSUM) {  // detector m <- image column m = Lr[j][m]
      for (int j = 0; j < n; ++j) acc += __ldg(Rz + (size_t)j * wl + m);
    } else if (g.mode == DD_ROWS || g.mode == DD_COLS) {
      const float *L = g.mode == DD_ROWS ? Rz : Cz;
      const float r = g.r, k = g.k;
      const float Dlo = det_bound(m, nh, r), Dhi = det_bound(m + 1, nh, r);
      const float Dn = det_bound(n, nh, r);
      int i0 = 0, i1 = n - 1;
      if (k != 0.0f) {
        const double qa = -(double)nh - (double)Dhi, qb = (double)(n - nh) - (double)Dlo;
        const double ya = qa / (double)k, yb = qb / (double)k;
        const double flo = floor(fmin(ya, yb) + nh - 0.5) - 1.0, fhi = ceil(fmax(ya, yb) + nh - 0.5) + 1.0;
        i0 = flo < 0.0 ? 0 : (flo > (double)(n - 1) ? n : (int)flo);
        i1 = fhi > (double)(n - 1) ? n - 1 : (fhi < 0.0 ? -1 : (int)fhi);
      }
      const float fnh = (float)nh;
      const float lo_nh = Dlo + fnh, hi_nh = Dhi + fnh;
      float y = (float)(i0 - nh) + 0.5f;
      for (int i = i0; i <= i1; ++i, y += 1.0f) {
        const float q = __fmul_rn(y, k);
        const float *row = L + (size_t)i * wl;
        const int kk1 = (int)floorf(hi_nh + q);
        if (kk1 >= n - 2 || m == n - 1) {  // the line's dropped piece may be ours
          acc += dd_fwd_line_exact(row, m, q, r, Dlo, Dhi, Dn, n, nh);
          continue;
        }
        int kk = max((int)floorf(lo_nh + q), -1);
        float P = pix_bound(kk, nh, q);
        if (P > Dlo && kk > -1) {  // rounding put the estimate one pixel too far
          --kk;
          P = pix_bound(kk, nh, q);
        }
        for (; P < Dhi && kk <= n; ++kk) {
          const float P1 = pix_bound(kk + 1, nh, q);
          const float w = fmaxf(__fsub_rn(fminf(P1, Dhi), fmaxf(P, Dlo)), 0.0f);
          acc = fmaf(w, __ldg(row + kk), acc);  // row[-1], row[n]: zero guards
          P = P1;
        }
      }
    }
  }
  fwd_store(ep, acc, live, z * (size_t)na * n + (size_t)g.out_row * n + (live ? m : 0), sino);
}

constexpr int kAdjChunk = 1024;

// Adjoint tables: lines = rows (ROWS) or columns (COLS); entry = {r, k, rinv, row offset}.
__global__ void __launch_bounds__(256) dd_adjoint_v2_kernel(
    const float *__restrict__ Sp, float *__restrict__ img, const float4 *__restrict__ tabR, int nR,
    const float4 *__restrict__ tabC, int nC, const int2 *__restrict__ tabS, int nS, int n, int nh,
    int na, int w, int pads, AdjEpi ep) {
  __shared__ float4 st[kAdjChunk];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y * blockDim.y + threadIdx.y;
  const size_t z = blockIdx.z;
  const bool live = a < n && b < n;
  const float *S = Sp + z * (size_t)na * w;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
  const float nhp = (float)(nh + pads);
  float acc = 0.0f;
  for (int pass = 0; pass < 2; ++pass) {
    const float4 *tab = pass == 0 ? tabR : tabC;
    const int cnt_all = pass == 0 ? nR : nC;
    // ROWS: the pixel is kk = b of line a; COLS: kk = a of line b
    const int line = pass == 0 ? a : b, kk = pass == 0 ? b : a;
    const float y = (float)(line - nh) + 0.5f;
    const float xk = (float)(kk - nh), xk1 = (float)(kk + 1 - nh);
    const bool edge_pixel = kk == n - 1;
    for (int v0 = 0; v0 < cnt_all; v0 += kAdjChunk) {
      const int cnt = min(kAdjChunk, cnt_all - v0);
      __syncthreads();
      for (int t = tid; t < cnt; t += nthr) st[t] = tab[v0 + t];
      __syncthreads();
      if (!live) continue;
#pragma unroll 2
      for (int u = 0; u < cnt; ++u) {
        const float4 e = st[u];
        const float r = e.x, k = e.y;
        const int off = __float_as_int(e.w);
        const float q = __fmul_rn(y, k);
        const float Pk = __fsub_rn(xk, q), Pk1 = __fsub_rn(xk1, q);
        int mp = (int)floorf(fmaf(Pk, e.z, nhp));
        float fm = __fsub_rn((float)mp, nhp);  // m - nh, exact
        float Dm = __fmul_rn(fm, r);
        if (Dm > Pk) {
          --mp;
          fm = __fsub_rn(fm, 1.0f);
          Dm = __fmul_rn(fm, r);
        }
        const float Dm1 = __fmul_rn(__fadd_rn(fm, 1.0f), r);
        const float *srow = S + off;
        if (edge_pixel || mp - pads >= n - 2) {
          acc += dd_adj_pixel_exact(srow + pads, kk, q, r, n, nh);
        } else {
          const float w1 = fmaxf(__fsub_rn(fminf(Pk1, Dm1), fmaxf(Pk, Dm)), 0.0f);
          const float w2 = fmaxf(__fsub_rn(Pk1, fmaxf(Dm1, Pk)), 0.0f);
          acc = fmaf(w1, __ldg(srow + mp), acc);
          acc = fmaf(w2, __ldg(srow + mp + 1), acc);
        }
      }
    }
  }
  if (live) {
    for (int t = 0; t < nS; ++t) {  // row / column sums (|sin| or |cos| < 1e-7)
      const int2 e = __ldg(tabS + t);
      acc += __ldg(S + e.y + pads + (e.x == DD_ROWSUM ? a : b));
    }
  }
  adj_store(ep, acc, live, z * (size_t)n * n + (size_t)(live ? a : 0) * n + (live ? b : 0), img);
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
  p.scratch_bytes = sizeof(float) * (lines + sp);
  TOMO_CUDA(cudaMalloc(&p.d_scratch, p.scratch_bytes));
  return TOMO_OK;
}

int dd_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s, const FwdEpi &ep) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz;
  float *Lr = p.d_scratch, *Lc = p.d_scratch + (size_t)nz * n * p.dd_wl;
  dim3 tb(32, 8), tg((n + 31) / 32, (n + 31) / 32, nz);
  dd_pad_image_kernel<<<tg, tb, 0, s>>>(d_img, Lr, Lc, n, p.dd_wl);
  dim3 fb(128), fg((n + 127) / 128, na, nz);
  dd_forward_v2_kernel<<<fg, fb, 0, s>>>(Lr, Lc, d_sino, (const DdAngle *)p.d_angles, n, p.nh, na,
                                         p.dd_wl, ep);
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
  dim3 ab(32, 8), ag((n + 31) / 32, (n + 7) / 8, nz);
  dd_adjoint_v2_kernel<<<ag, ab, 0, s>>>(Sp, d_img, tR, p.dd_nR, tC, p.dd_nC, tS, p.dd_nS, n, p.nh,
                                         na, p.dd_w, p.dd_pads, ep);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
