/*
 * tomo_oracle.c -- FP64 CPU oracle for the Radon-family projector pairs.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the project's own restatement of the
 * reference kernels, written to check the CUDA path; it is never linked into
 * the product library.  Each function follows one reference C function and
 * keeps its float32 geometry, bin/branch decisions and output permutations,
 * but accumulates in double and writes double outputs, so that the distance
 * between the reference (float accumulation) and this oracle is pure
 * accumulation error.
 *
 * Argument convention (all functions): `in` is the image [n*n] when oper==0
 * (forward) and the sinogram [na*n] when oper==1 (adjoint); `out` (double)
 * is overwritten with the other one.  `ang` holds the angles exactly as the
 * reference C function receives them (after its Cython shim).
 *
 * Float evaluation of the geometry: the reference is built with
 * -O3 -ffast-math on an FMA-capable x86-64 target.  Under those flags GCC
 * (13.3) evaluates the reference expressions in a specific way, read from the
 * x86-64 assembly of the reference sources compiled in this tree:
 *   - sin/cos of a float angle become glibc sincosf() (float in, float out);
 *   - divisions by a loop-invariant s or c become products with 1.0f/s, 1.0f/c;
 *   - several a*b+c patterns are contracted into one fused multiply-add.
 * This file writes each of those evaluations out explicitly (it is itself
 * compiled with -ffp-contract=off), so its bin and branch decisions are the
 * compiled reference's.  The same evaluation order is what the CUDA kernels
 * reproduce.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.141592653589793

/* Per-angle sine and cosine exactly as the compiled reference gets them. */
static inline void orc_sincos(float theta, float *s, float *c) {
  sincosf(theta, s, c);
}

/* ---------------------------------------------------------------------- */
/* pixel-driven pair: radon_pd.c:20-90 (method 1 = linear interpolation)   */
/* ---------------------------------------------------------------------- */
/* Sub-sample offsets: radon_pd.c:12-15,42-43 use delta[2k+1] for BOTH x and y,
 * i.e. offsets (-1/4,-1/4) twice and (+1/4,+1/4) twice. */
static const float orc_pd_off[4] = {-0.25f, -0.25f, 0.25f, 0.25f};

void orc_pd(const float *in, int n, const float *ang, int na, int oper,
            double *out) {
  int nh = (int)(n * 0.5);
  float fnh = (float)nh;
  size_t nout = oper == 0 ? (size_t)na * n : (size_t)n * n;
  memset(out, 0, nout * sizeof(double));
  for (int v = 0; v < na; ++v) {
    float theta = ang[v], s, c;
    orc_sincos(theta, &s, &c);
    float rc = 1.0f / c;
    int lt = (double)theta < ORC_PI / 2, gt = (double)theta > ORC_PI / 2;
    for (int i = 0; i < n; ++i) {
      for (int j = 0; j < n; ++j) {
        float x0 = (float)j - fnh + 0.5f, y0 = (float)i - fnh + 0.5f;
        size_t pix = (size_t)(n - 1 - i) * n + j; /* row flip, radon_pd.c:61 */
        for (int k = 0; k < 4; ++k) {
          float x = x0 + orc_pd_off[k], y = y0 + orc_pd_off[k];
          float xs = x * s;
          float t = fabsf(fmaf(-c, y, xs)); /* |x*s - y*c|, :44 */
          float r = xs * rc;                /* x*s/c, :46-48 */
          int keep = (lt && y > r) || (gt && y > r) || (theta == 0.0f && y > 0.0f);
          if (!keep) t = -t; /* :46-55 */
          float T = fnh - t; /* :67 */
          float lf = floorf(T), uf = ceilf(T);
          int l = (int)round((double)lf - 0.5), u = (int)round((double)uf - 0.5);
          double wl = 0.25 * (double)fabsf((t + uf) - fnh); /* |uf - T| */
          double wu = 0.25 * (double)fabsf(T - lf);
          if (l > 0 && l < n) {
            if (oper == 0) out[(size_t)v * n + l] += wl * in[pix];
            else out[pix] += wl * in[(size_t)v * n + l];
          }
          if (u > 0 && u < n) {
            if (oper == 0) out[(size_t)v * n + u] += wu * in[pix];
            else out[pix] += wu * in[(size_t)v * n + u];
          }
        }
      }
    }
  }
}

/* ---------------------------------------------------------------------- */
/* ray-driven (Siddon) pair: radon_rd.c:15-71 (siddon), :76-189            */
/* ---------------------------------------------------------------------- */
/* One sub-ray walk.  The reference leaves `alpha` uninitialised
 * (radon_rd.c:17,40); its -O3 build behaves as alpha = 0, which is what the
 * loop below does.  Each step's length is credited to the pixel the walk
 * steps INTO (radon_rd.c:44-64), and the walk runs until alpha > 1. */
static void orc_siddon(const float *in, double *out, int n, const float p1[2],
                       const float p2[2], size_t index, int oper) {
  int nh = (int)(n * 0.5);
  float ex = p2[0] - p1[0], ey = p2[1] - p1[1];
  float incr = sqrtf(fmaf(ex, ex, ey * ey));
  int ii = (int)roundf(p1[0]);
  int jj = (int)roundf(p1[1]);
  float dx = p2[0] > p1[0] ? 1.0f : -1.0f;
  float dy = p2[1] > p1[1] ? 1.0f : -1.0f;
  float alpha = 0.0f, alpha_old = 0.0f;
  int guard = 0;
  while (alpha <= 1.0f) {
    float ay = (float)(((double)jj + 0.5 * dy - (double)p1[1]) / (double)ey);
    float ax = (float)(((double)ii + 0.5 * dx - (double)p1[0]) / (double)ex);
    if (ax < ay) {
      alpha = ax;
      ii = (int)((float)ii + dx);
    } else if (ax > ay) {
      alpha = ay;
      jj = (int)((float)jj + dy);
    } else if (ax == ay) {
      alpha = ay;
      ii = (int)((float)ii + dx);
      jj = (int)((float)jj + dy);
    }
    float l = (alpha - alpha_old) * incr;
    int i = ii + nh, j = jj + nh;
    if (i > 0 && i < n && j > 0 && j < n) {
      if (oper == 0) out[index] += 0.2 * (double)l * in[(size_t)i * n + j];
      else out[(size_t)i * n + j] += 0.2 * (double)l * in[index];
    }
    alpha_old = alpha;
    if (++guard > 8 * n + 64) break; /* NaN alphas would never advance */
  }
}

/* Entry (p1) and exit (p2) points of sub-ray offset t on the square
 * [-nh, nh]^2, radon_rd.c:133-179, in the compiled evaluation order:
 * (K + t) * (1/c) with K = (+-nh)*s a float product. */
void orc_rd_endpoints(float theta, float s, float c, int nh, float t,
                      float p1[2], float p2[2]) {
  float fnh = (float)nh, rc = 1.0f / c, rs = 1.0f / s;
  float ns = fnh * s, nc = fnh * c; /* nh*s, nh*c */
  float mns = -fnh * s, mnc = -fnh * c;
  if ((double)theta < ORC_PI / 2) {
    float y1 = (mns + t) * rc, x1 = (mnc - t) * rs;
    float y2 = (ns + t) * rc, x2 = (nc - t) * rs;
    if (y1 >= -fnh && y1 <= fnh) { p1[0] = -fnh; p1[1] = y1; }
    else { p1[0] = x1; p1[1] = -fnh; }
    if (y2 >= -fnh && y2 <= fnh) { p2[0] = fnh; p2[1] = y2; }
    else { p2[0] = x2; p2[1] = fnh; }
  } else {
    float y1 = (ns - t) * rc, x1 = (mnc + t) * rs;
    float y2 = (mns - t) * rc, x2 = (nc + t) * rs;
    if (y1 >= -fnh && y1 <= fnh) { p1[0] = fnh; p1[1] = y1; }
    else { p1[0] = x1; p1[1] = -fnh; }
    if (y2 >= -fnh && y2 <= fnh) { p2[0] = -fnh; p2[1] = y2; }
    else { p2[0] = x2; p2[1] = fnh; }
  }
}

/* Sub-ray offset of sub-ray i (i % 6 != 0), radon_rd.c:125-130; i/6.0 is
 * evaluated as fma(i, 1/6, -nh) in double. */
float orc_rd_offset(int i, int n, float theta) {
  int nh = (int)(n * 0.5);
  float t = (float)fabs(fma((double)i, 1.0 / 6.0, -(double)nh));
  if (i >= 3 * n && (double)theta < ORC_PI / 2) t = -t;
  if (i < 3 * n && (double)theta > ORC_PI / 2) t = -t;
  return t;
}

void orc_rd(const float *in, int n, const float *ang, int na, int oper,
            double *out) {
  int nh = (int)(n * 0.5);
  size_t nout = oper == 0 ? (size_t)na * n : (size_t)n * n;
  memset(out, 0, nout * sizeof(double));
  for (int v = 0; v < na; ++v) {
    float theta = ang[v], s, c;
    orc_sincos(theta, &s, &c);
    if (fabs((double)s) < 1e-7) { /* radon_rd.c:96-105 */
      for (int i = 1; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          if (oper == 0) out[(size_t)v * n + n - 1 - i] += in[(size_t)j * n + i];
          else out[(size_t)j * n + i] += in[(size_t)v * n + n - 1 - i];
        }
      continue;
    }
    if (fabs((double)c) < 1e-7) { /* radon_rd.c:108-117 */
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          if (oper == 0) out[(size_t)v * n + i] += in[(size_t)i * n + j];
          else out[(size_t)i * n + j] += in[(size_t)v * n + i];
        }
      continue;
    }
    for (int i = 1; i < 6 * n; ++i) {
      if (i % 6 == 0) continue;
      size_t index = (size_t)v * n + (size_t)(i / 6); /* :121,184-185 */
      float p1[2], p2[2];
      orc_rd_endpoints(theta, s, c, nh, orc_rd_offset(i, n, theta), p1, p2);
      orc_siddon(in, out, n, p1, p2, index, oper);
    }
  }
}

/* ---------------------------------------------------------------------- */
/* distance-driven pair: radon_dd.c:54-285                                 */
/* ---------------------------------------------------------------------- */
/* Walk the merged, increasing pixel boundaries P[0..n] and detector
 * boundaries D[0..n] of one image line (the reference sorts them together,
 * radon_dd.c:117, then labels each gap, :125-189).  Restated rule: a gap
 * between consecutive boundaries is an overlap piece of (last pixel boundary
 * index seen, last detector boundary index seen) once both ranges have
 * started; the walk stops, without crediting the gap, at the first boundary
 * whose index is n (:176-177).  Ties put the pixel boundary first. */
static void dd_line(const float *P, const float *D, int n, const float *img,
                    size_t img_stride, const float *sino_row, double *out_img,
                    double *out_sino, int oper) {
  int a = 0, b = 0; /* next P, next D */
  int ip = -1, id = -1;
  float prev = 0.0f;
  for (int t = 0; t < 2 * n + 2; ++t) {
    int lab, idx;
    float val;
    if (b > n || (a <= n && P[a] <= D[b])) {
      lab = 0; idx = a; val = P[a]; ++a;
    } else {
      lab = 1; idx = b; val = D[b]; ++b;
    }
    if (t > 0) {
      if (idx == n) break;
      if (ip >= 0 && id >= 0) {
        float w = fabsf(val - prev);
        if (oper == 0) out_sino[id] += (double)w * img[(size_t)ip * img_stride];
        else out_img[(size_t)ip * img_stride] += (double)w * sino_row[id];
      }
    }
    if (lab == 0) ip = idx; else id = idx;
    prev = val;
  }
}

void orc_dd(const float *in, int n, const float *ang, int na, int oper,
            double *out) {
  int nh = (int)(n * 0.5);
  size_t nout = oper == 0 ? (size_t)na * n : (size_t)n * n;
  memset(out, 0, nout * sizeof(double));
  float *P = malloc(sizeof(float) * (n + 1));
  float *D = malloc(sizeof(float) * (n + 1));
  for (int v = 0; v < na; ++v) {
    float theta = ang[v], s, c;
    orc_sincos(theta, &s, &c);
    size_t row = (size_t)(na - 1 - v) * n; /* output row reversal, :79,181 */
    if (fabs((double)s) < 1e-7) { /* :75-84 row sums */
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          if (oper == 0) out[row + i] += in[(size_t)i * n + j];
          else out[(size_t)i * n + j] += in[row + i];
        }
    } else if (fabs((double)c) < 1e-7) { /* :87-96 column sums */
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          if (oper == 0) out[row + i] += in[(size_t)j * n + i];
          else out[(size_t)j * n + i] += in[row + i];
        }
    } else if ((double)theta > ORC_PI / 2) { /* :99-190, lines = image rows */
      float r = 1.0f / s, k = c * r; /* x/s -> x*r, y*c/s -> y*(c*r) */
      for (int i = 0; i < n; ++i) {
        float q = ((float)(i - nh) + 0.5f) * k;
        for (int j = 0; j <= n; ++j) {
          float x = (float)(j - nh);
          P[j] = x - q;
          D[j] = x * r;
        }
        if (oper == 0) dd_line(P, D, n, in + (size_t)i * n, 1, NULL, NULL, out + row, 0);
        else dd_line(P, D, n, NULL, 1, in + row, out + (size_t)i * n, NULL, 1);
      }
    } else if ((double)theta < ORC_PI / 2 && theta != 0.0f) { /* :194-283, lines = columns */
      float r = 1.0f / c, k = s * r;
      for (int i = 0; i < n; ++i) {
        float q = ((float)(i - nh) + 0.5f) * k;
        for (int j = 0; j <= n; ++j) {
          float y = (float)(j - nh);
          P[j] = y - q;
          D[j] = y * r;
        }
        if (oper == 0) dd_line(P, D, n, in + i, (size_t)n, NULL, NULL, out + row, 0);
        else dd_line(P, D, n, NULL, (size_t)n, in + row, out + i, NULL, 1);
      }
    }
  }
  free(P);
  free(D);
}

/* ---------------------------------------------------------------------- */
/* slant-stacking pair: radon_ss.c:43-88 (ray_limits), :93-196 (method 1)  */
/* ---------------------------------------------------------------------- */
static void sort4(float *a) {
  for (int i = 1; i < 4; ++i)
    for (int j = i; j > 0 && a[j] < a[j - 1]; --j) {
      float t = a[j]; a[j] = a[j - 1]; a[j - 1] = t;
    }
}

/* Limits of a ray in the square [-nh, nh-1]^2: for each axis the middle two
 * of {entry, exit, -nh, nh-1} (radon_ss.c:70-87); compiled as
 * fma(nh, s, t) / c etc. */
void orc_ss_limits(float lim[4], int t, float s, float c, int n) {
  int nh = (int)(n * 0.5);
  float fnh = (float)nh, fnh1 = (float)(nh - 1), ft = (float)t;
  if (fabs((double)s) < 1e-5) {
    lim[0] = 0; lim[1] = 0; lim[2] = -fnh; lim[3] = fnh1;
  } else if (fabs((double)c) < 1e-5) {
    lim[0] = -fnh; lim[1] = fnh1; lim[2] = 0; lim[3] = 0;
  } else {
    float x1 = fmaf(fnh, s, ft) / c, x2 = fmaf(-s, fnh1, ft) / c;
    float y1 = fmaf(fnh, c, ft) / s, y2 = fmaf(-c, fnh1, ft) / s;
    float a[4] = {x1, x2, -fnh, fnh1};
    sort4(a);
    float b[4] = {y1, y2, -fnh, fnh1};
    sort4(b);
    lim[0] = a[1]; lim[1] = a[2]; lim[2] = b[1]; lim[3] = b[2];
  }
}

void orc_ss(const float *in, int n, const float *ang, int na, int oper,
            double *out) {
  int nh = (int)(n * 0.5);
  size_t nout = oper == 0 ? (size_t)na * n : (size_t)n * n;
  memset(out, 0, nout * sizeof(double));
  for (int v = 0; v < na; ++v) {
    float theta = ang[v], s, c;
    orc_sincos(theta, &s, &c);
    float rs = 1.0f / s, rc = 1.0f / c;
    double ws = 1.0 / fabs((double)s), wc = 1.0 / fabs((double)c);
    size_t srow = (size_t)(na - 1 - v) * n; /* radon_ss.c:111 */
    for (int t = -nh; t < nh; ++t) {
      size_t sidx = srow + (size_t)(t + nh);
      float lim[4];
      orc_ss_limits(lim, t, s, c, n);
      float ft = (float)t;
      int steep = fabs((double)s) <= 0.70710678118654757;
      int a0 = (int)roundf(steep ? lim[2] : lim[0]);
      int a1 = (int)roundf(steep ? lim[3] : lim[1]);
      for (int m = a0; m < a1; ++m) {
        /* steep: m is y, interpolate x (:120-154); else m is x (:158-192) */
        float f = steep ? fmaf(-(float)m, s, ft) * rc : fmaf(-(float)m, c, ft) * rs;
        float fl = floorf(f);
        float w = f - fl, w1 = (fl + 1.0f) - f;
        int q = (int)fl + nh, mm = m + nh;
        double wt = steep ? wc : ws;
        if (mm < 0 || mm > n - 1) continue; /* rays that miss the square */
        for (int tap = 0; tap < 2; ++tap) {
          int qq = q + tap;
          if (qq < 0 || qq > n - 1) continue;
          size_t p = steep ? (size_t)mm * n + qq : (size_t)qq * n + mm;
          double wgt = wt * (double)(tap ? w : w1);
          if (oper == 0) out[sidx] += wgt * in[p];
          else out[p] += wgt * in[sidx];
        }
      }
    }
  }
}

/* ---------------------------------------------------------------------- */
/* B-spline (generalised Radon) pair: gen_forwproj.c:22-78, gen_backproj.c */
/* ---------------------------------------------------------------------- */
void orc_bspline(const float *in, int n, const float *ang_deg, int na,
                 const float *lut, int lut_size, float support, int oper,
                 double *out) {
  float lut_step = (float)((lut_size * 0.5) / ((double)support * 0.5));
  int lut_max = lut_size - 1, lut_half = lut_size / 2;
  double mid = 0.5 * n; /* half_pixel = 0: middle_left == middle_right */
  int ds = (int)(0.5 * support + 0.5);
  size_t nout = oper == 0 ? (size_t)na * n : (size_t)n * n;
  memset(out, 0, nout * sizeof(double));
  for (int v = 0; v < na; ++v) {
    float theta = (float)((double)ang_deg[v] * (ORC_PI / 180.0)), S, C;
    orc_sincos(theta, &S, &C);
    for (int ky_i = 0; ky_i < n; ++ky_i) {
      float ky = (float)(-ky_i + mid);
      float sky = S * ky;
      for (int kx_i = 0; kx_i < n; ++kx_i) {
        float kx = (float)(kx_i - mid);
        float ps = fmaf(kx, C, sky); /* COS*kx + SIN*ky */
        size_t pix = (size_t)ky_i * n + kx_i;
        for (int sft = -ds; sft <= ds; ++sft) {
          int yi = (int)((double)((float)sft + ps) + mid);
          if (yi >= n || yi < 0) continue;
          float y = (float)((double)yi - mid);
          int li = (int)((y - ps) * lut_step) + lut_half;
          if (li >= lut_max || li < 0) continue;
          double w = lut[(size_t)v * lut_size + li];
          if (oper == 0) out[(size_t)v * n + yi] += w * in[pix];
          else out[pix] += w * in[(size_t)v * n + yi];
        }
      }
    }
  }
}
