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
// Rather than sorting, the kernels below enumerate the overlaps in closed
// form: the forward is a gather per detector bin (over the lines and the
// pixels that overlap it), the adjoint a gather per pixel (over the angles and
// the one or two detectors it overlaps).  Every boundary is the same float the
// compiled reference computes: q = ((i - nh) + 0.5) * k, P = x - q, D = x * r
// (x = j - nh, k = c*r, r = 1/s or 1/c; radon_dd.c:101-115 and 196-207 under
// -O3 -ffast-math).  No atomics: each output element is owned by one thread,
// so results are deterministic.
#include <cmath>
#include <cstdio>
#include <cstring>

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

// 32x32 tiled transpose: out[c][r] = in[r][c] for each slice.
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

// Forward: one thread per (detector m, angle v, slice z).
//   img  : [nz][n][n] image, row-major
//   imgT : [nz][n][n] its transpose (lines of the COLS branch are contiguous)
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
    // detector m <- sum_j image[m][j]  (image[m][j] == IT[j][m]: coalesced)
    for (int j = 0; j < n; ++j) acc += IT[(size_t)j * n + m];
  } else if (g.mode == DD_COLSUM) {
    for (int j = 0; j < n; ++j) acc += I[(size_t)j * n + m];
  } else if (g.mode == DD_ROWS || g.mode == DD_COLS) {
    const float *L = g.mode == DD_ROWS ? I : IT;  // line i = L[i][*]
    const float r = g.r, k = g.k;
    const float Dlo = det_bound(m, nh, r), Dhi = det_bound(m + 1, nh, r);
    const float Dn = det_bound(n, nh, r);
    // Lines whose pixel span [P_0, P_n] meets [Dlo, Dhi]: q in (-nh - Dhi, n - nh - Dlo).
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
      const bool lastIsPixel = Pn <= Dn;  // the dropped piece ends at P_n
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

// Adjoint: one thread per output pixel (row a, column b), looping over all
// angles in order; the angle table is staged in shared memory in chunks.
constexpr int kAdjChunk = 1024;

__global__ void __launch_bounds__(256) dd_adjoint_kernel(
    const float *__restrict__ sino, float *__restrict__ img, const DdAngle *__restrict__ tab,
    int n, int nh, int na) {
  __shared__ DdAngle stab[kAdjChunk];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y * blockDim.y + threadIdx.y;
  const size_t z = blockIdx.z;
  const bool live = a < n && b < n;
  const float *S = sino + z * (size_t)na * n;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nthr = blockDim.x * blockDim.y;
  float acc = 0.0f;
  for (int v0 = 0; v0 < na; v0 += kAdjChunk) {
    const int cnt = min(kAdjChunk, na - v0);
    __syncthreads();
    for (int t = tid; t < cnt; t += nthr) stab[t] = tab[v0 + t];
    __syncthreads();
    if (!live) continue;
    for (int t = 0; t < cnt; ++t) {
      const DdAngle g = stab[t];
      const float *row = S + (size_t)g.out_row * n;
      if (g.mode == DD_ROWSUM) {
        acc += __ldg(row + a);
      } else if (g.mode == DD_COLSUM) {
        acc += __ldg(row + b);
      } else if (g.mode == DD_ROWS || g.mode == DD_COLS) {
        const int line = g.mode == DD_ROWS ? a : b;
        const int kk = g.mode == DD_ROWS ? b : a;
        const float r = g.r;
        const float q = __fmul_rn(__fadd_rn((float)(line - nh), 0.5f), g.k);
        const float Pk = pix_bound(kk, nh, q), Pk1 = pix_bound(kk + 1, nh, q);
        const float Pn = pix_bound(n, nh, q), Dn = det_bound(n, nh, r);
        const bool lastIsPixel = Pn <= Dn;
        int m = (int)floorf(__fdividef(Pk, r) + (float)nh);
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
        for (; m < n && Dm < Pk1; ++m) {
          const float lo = fmaxf(Pk, Dm), hi = fminf(Pk1, Dm1);
          if (hi > lo) {
            const bool drop = lastIsPixel ? (kk == n - 1 && Pn <= Dm1) : (m == n - 1 && Pk1 > Dn);
            if (!drop) acc = fmaf(__fsub_rn(hi, lo), __ldg(row + m), acc);
          }
          Dm = Dm1;
          Dm1 = det_bound(m + 2, nh, r);
        }
      }
    }
  }
  if (live) img[z * (size_t)n * n + (size_t)a * n + b] = acc;
}

}  // namespace

int dd_setup(Plan &p) {
  const int na = p.g.na;
  std::vector<DdAngle> tab(na);
  for (int v = 0; v < na; ++v) {
    const float theta = p.angles[v];
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
  TOMO_CUDA(cudaMalloc(&p.d_angles, sizeof(DdAngle) * (size_t)na));
  TOMO_CUDA(cudaMemcpy(p.d_angles, tab.data(), sizeof(DdAngle) * (size_t)na, cudaMemcpyHostToDevice));
  // scratch: transposed image for the COLS/ROWSUM lines of the forward
  p.scratch_bytes = sizeof(float) * image_elems(p);
  TOMO_CUDA(cudaMalloc(&p.d_scratch, p.scratch_bytes));
  return TOMO_OK;
}

int dd_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz;
  const size_t stride = (size_t)n * n;
  dim3 tb(32, 8), tg((n + 31) / 32, (n + 31) / 32, nz);
  transpose_kernel<<<tg, tb, 0, s>>>(d_img, p.d_scratch, n, stride);
  dim3 fb(128), fg((n + 127) / 128, na, nz);
  dd_forward_kernel<<<fg, fb, 0, s>>>(d_img, p.d_scratch, d_sino, (const DdAngle *)p.d_angles, n,
                                      p.nh, na);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

// Per-angle table for a plan-less caller: same arithmetic as dd_setup.
int dd_build_table(const float *angles, int na, DdAngle *tab) {
  for (int v = 0; v < na; ++v) {
    const float theta = angles[v];
    float s, c;
    sincosf(theta, &s, &c);
    DdAngle a{};
    a.out_row = na - 1 - v;
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

// Forward launch with caller-provided scratch (>= nz*n*n floats) and device table.
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

int dd_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s) {
  const int n = p.g.n, na = p.g.na, nz = p.g.nz;
  dim3 ab(32, 8), ag((n + 31) / 32, (n + 7) / 8, nz);
  dd_adjoint_kernel<<<ag, ab, 0, s>>>(d_sino, d_img, (const DdAngle *)p.d_angles, n, p.nh, na);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // namespace tomo
