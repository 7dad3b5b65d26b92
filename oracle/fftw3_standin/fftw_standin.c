/*
 * Double-precision mixed-radix DFT behind the FFTW3 API subset declared in
 * fftw3.h.  TEST INFRASTRUCTURE ONLY (oracle side): it lets the reference's
 * gridding C code compile and run here, and it is the FFT of the project's
 * own CPU oracle for the gridding pair.
 *
 * Algorithm: recursive decimation in time.  n = p * m with p the smallest
 * prime factor; the p interleaved sub-sequences are transformed recursively
 * (length m) and combined with twiddles exp(sign*2*pi*i*r*k/n).  Prime
 * lengths fall through to a direct O(p^2) DFT, so every n >= 1 works.
 */
#include "fftw3.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

struct fftwf_plan_s {
  int n0, n1; /* n1 == 0 for a 1-D plan */
  int sign;
  fftwf_complex *in, *out;
};

void *fftwf_malloc(size_t n) { return malloc(n ? n : 1); }
void fftwf_free(void *p) { free(p); }

static void dft_rec(const double complex *x, size_t xs, double complex *y,
                    int n, int sign, double complex *tmp) {
  if (n == 1) {
    y[0] = x[0];
    return;
  }
  int p = 0;
  for (int f = 2; f * f <= n; ++f)
    if (n % f == 0) {
      p = f;
      break;
    }
  if (p == 0) { /* prime: direct DFT */
    for (int k = 0; k < n; ++k) {
      double complex acc = 0;
      for (int j = 0; j < n; ++j) {
        long long jk = ((long long)j * k) % n;
        double a = sign * 2.0 * M_PI * (double)jk / (double)n;
        acc += x[j * xs] * (cos(a) + I * sin(a));
      }
      y[k] = acc;
    }
    return;
  }
  int m = n / p;
  /* sub-transform r lands in y[r*m .. r*m+m-1] */
  for (int r = 0; r < p; ++r)
    dft_rec(x + r * xs, xs * p, y + r * m, m, sign, tmp + n);
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) {
      int kk = k + q * m;
      double complex acc = 0;
      for (int r = 0; r < p; ++r) {
        long long e = ((long long)r * kk) % n;
        double a = sign * 2.0 * M_PI * (double)e / (double)n;
        acc += y[r * m + k] * (cos(a) + I * sin(a));
      }
      tmp[kk] = acc;
    }
  }
  memcpy(y, tmp, sizeof(double complex) * n);
}

static void dft_line(double complex *line, int n, int sign,
                     double complex *work) {
  /* work needs room for the output copy plus the recursion scratch */
  double complex *y = work;
  double complex *scratch = work + n;
  dft_rec(line, 1, y, n, sign, scratch);
  memcpy(line, y, sizeof(double complex) * n);
}

static size_t scratch_len(int n) {
  /* output copy + one level of tmp per recursion depth (< 64 levels) */
  return (size_t)n * 66 + 16;
}

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags) {
  (void)flags;
  fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
  p->n0 = n;
  p->n1 = 0;
  p->sign = sign;
  p->in = in;
  p->out = out;
  return p;
}

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in,
                             fftwf_complex *out, int sign, unsigned flags) {
  (void)flags;
  fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
  p->n0 = n0;
  p->n1 = n1;
  p->sign = sign;
  p->in = in;
  p->out = out;
  return p;
}

void fftwf_execute(const fftwf_plan p) {
  if (!p) return;
  if (p->n1 == 0) {
    int n = p->n0;
    double complex *buf = malloc(sizeof(double complex) * n);
    double complex *work = malloc(sizeof(double complex) * scratch_len(n));
    for (int i = 0; i < n; ++i) buf[i] = p->in[i][0] + I * p->in[i][1];
    dft_line(buf, n, p->sign, work);
    for (int i = 0; i < n; ++i) {
      p->out[i][0] = (float)creal(buf[i]);
      p->out[i][1] = (float)cimag(buf[i]);
    }
    free(work);
    free(buf);
    return;
  }
  int n0 = p->n0, n1 = p->n1;
  size_t tot = (size_t)n0 * n1;
  double complex *buf = malloc(sizeof(double complex) * tot);
  int nmax = n0 > n1 ? n0 : n1;
  double complex *line = malloc(sizeof(double complex) * nmax);
  double complex *work = malloc(sizeof(double complex) * scratch_len(nmax));
  for (size_t i = 0; i < tot; ++i) buf[i] = p->in[i][0] + I * p->in[i][1];
  for (int r = 0; r < n0; ++r) dft_line(buf + (size_t)r * n1, n1, p->sign, work);
  for (int c = 0; c < n1; ++c) {
    for (int r = 0; r < n0; ++r) line[r] = buf[(size_t)r * n1 + c];
    dft_line(line, n0, p->sign, work);
    for (int r = 0; r < n0; ++r) buf[(size_t)r * n1 + c] = line[r];
  }
  for (size_t i = 0; i < tot; ++i) {
    p->out[i][0] = (float)creal(buf[i]);
    p->out[i][1] = (float)cimag(buf[i]);
  }
  free(work);
  free(line);
  free(buf);
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }
int fftwf_import_wisdom_from_file(FILE *f) {
  (void)f;
  return 0;
}
void fftwf_export_wisdom_to_file(FILE *f) { (void)f; }
