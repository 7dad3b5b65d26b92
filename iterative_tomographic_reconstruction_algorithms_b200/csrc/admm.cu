// ADMM and conjugate-gradient solvers on a projector plan, device resident.
//
// References (algorithms/): plain CG cg.py:83-185 (as admm.py:245-288 calls
// it); Lasso-L1 admm.py:291-457 with cg.py:189-253; Lasso-TV admm.py:470-640
// with cg.py:256-320; G / Gt cg.py:62-71; hard_thres utils.py:214-216;
// phys_constr utils.py:171-176; resol_circle_constr utils.py:229-256.
//
// The reference runs every step in numpy.  Its arrays have mixed precision
// and this file keeps the same types and rounding order:
//   * CG / Lasso-L1: x, r, p, Hp and v are float32; the inner products are
//     float32 results (accumulated here in double, then rounded); alpha =
//     <r,r> / (<p,Hp> + np.spacing(1)) is float64 under NumPy 2 promotion, so
//     the x and r updates are float64 expressions rounded to float32;
//   * Lasso-TV: Gt returns float64 (dense float64 matrices), so r and p are
//     float64, Hp is stored as float32 (the reference's Hp buffer), x stays
//     float32 and x += alpha p is evaluated in float64 and rounded;
//   * the scalars lambd1, lambd2 and mu are float32 (class_admm_param.py:67-69).
// Every product that numpy rounds before an addition is rounded here too
// (explicit __*_rn intrinsics, no contraction into FMA).
//
// Gt is the reference's dense g[1] . Gx + Gy . g[0]; every column of Gx and
// row of Gy has at most two non-zeros, so a radius-2 stencil gives the same
// float64 numbers.  Gt(G(y)) is evaluated in one pass from y.
//
// One CG iteration = forward + adjoint projection of p and three vector
// kernels (Hp, update, direction); each reduction is per slice, in a fixed
// order (per-block partials, summed by the last block of the slice), so runs
// are bitwise reproducible.  The per-slice scalars (alpha, beta) never leave
// the device, and one outer iteration (ADMM) or one CG iteration (plain CG)
// is captured once into a CUDA graph and replayed.
#include <cmath>

#include "tomo_internal.cuh"

namespace tomo {

Plan *plan_of(tomo_plan *p);
int plan_forward(Plan &p, const float *in, float *out, cudaStream_t s, const FwdEpi &ep);
int plan_adjoint(Plan &p, const float *in, float *out, cudaStream_t s, const AdjEpi &ep);

namespace {

constexpr int kThr = 256;
constexpr int kNq = 3;  // reduced quantities per kernel, at most

// per-slice scalars, sc[s][*]
enum : int { SC_RR = 0, SC_PHP, SC_RRN, SC_ROLD, SC_ERR, SC_DIFF, SC_XOLD, SC_N = 8 };

struct Red {
  double *part;   // [nz][kNq][bps] per-block partial sums
  unsigned *cnt;  // [nz] blocks finished, reset by the last one
  double *sc;     // [nz][SC_N]
  int bps;        // blocks per slice
};

struct Vec {
  int n0, n1, nz;
  size_t N;            // n0 * n1
  float *x;            // [nz][N]
  float *xold;         // [nz][N]
  const float *atb;    // A^T b
  const float *q;      // A^T A (x or p)
  float *v;            // TV: [nz][2][N], L1: [nz][N]
  float *alpha;        // same layout as v (ADMM multiplier)
  void *r, *p;         // float (CG, L1) or double (TV), [nz][N]
  float *p32;          // float32 copy of p handed to the projector
  float *hp;           // [nz][N]
  float l1, mu, c;     // lambd1, mu, lambd1 + mu (float32 sums as numpy forms them)
  float beta;          // lambd2 / mu (float32)
};

// ---- numpy.gradient and the reference's Gt ---------------------------------

__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float half_rn(float a) { return __fmul_rn(a, 0.5f); }  // == a / 2.0, exactly
__device__ __forceinline__ double half_rn(double a) { return __dmul_rn(a, 0.5); }

// numpy.gradient along axis 0 / axis 1 at (i, j) of an n0 x n1 array (n0, n1 >= 2)
template <typename T>
__device__ __forceinline__ T grad0(const T *m, int n0, int n1, int i, int j) {
  const size_t k = (size_t)i * n1 + j;
  if (i == 0) return sub_rn(m[k + n1], m[k]);
  if (i == n0 - 1) return sub_rn(m[k], m[k - n1]);
  return half_rn(sub_rn(m[k + n1], m[k - n1]));
}
template <typename T>
__device__ __forceinline__ T grad1(const T *m, int n1, int i, int j) {
  const size_t k = (size_t)i * n1 + j;
  if (j == 0) return sub_rn(m[k + 1], m[k]);
  if (j == n1 - 1) return sub_rn(m[k], m[k - 1]);
  return half_rn(sub_rn(m[k + 1], m[k - 1]));
}

// Entry (k, j) of numpy.gradient(I_n) along axis 0.
__device__ __forceinline__ double dgrad(int k, int j, int n) {
  if (k == 0) return j == 1 ? 1.0 : (j == 0 ? -1.0 : 0.0);
  if (k == n - 1) return j == n - 1 ? 1.0 : (j == n - 2 ? -1.0 : 0.0);
  return j == k + 1 ? 0.5 : (j == k - 1 ? -0.5 : 0.0);
}

// (g1 . Gx + Gy . g0)[i][j], g0(k, j) and g1(i, k) supplied by functors.
template <class G0, class G1>
__device__ __forceinline__ double gt_at(int i, int j, int n0, int n1, G0 g0, G1 g1) {
  double a = 0.0, b = 0.0;
  for (int k = max(j - 1, 0); k <= min(j + 1, n1 - 1); ++k) {
    const double w = dgrad(k, j, n1);
    if (w != 0.0) a = __dadd_rn(a, __dmul_rn((double)g1(i, k), w));
  }
  for (int k = max(i - 1, 0); k <= min(i + 1, n0 - 1); ++k) {
    const double w = dgrad(k, i, n0);
    if (w != 0.0) b = __dadd_rn(b, __dmul_rn(w, (double)g0(k, j)));
  }
  return __dadd_rn(a, b);
}

// Gt(G(y)) at (i, j): G in T arithmetic (float32 for x, float64 for p), Gt in float64.
template <typename T>
__device__ __forceinline__ double gtg_at(const T *y, int n0, int n1, int i, int j) {
  return gt_at(i, j, n0, n1, [&](int k, int jj) { return grad0<T>(y, n0, n1, k, jj); },
               [&](int ii, int k) { return grad1<T>(y, n1, ii, k); });
}

// ---- deterministic per-slice reductions -------------------------------------

// Block sums of v[0..NQ) (fixed order) into the partials of slice s; the last
// block of the slice to finish adds the partials in block order and stores
// the totals in sc[s][dst[q]].
template <int NQ>
__device__ void reduce_commit(const Red &R, int s, const double (&v)[NQ], const int (&dst)[NQ]) {
  __shared__ double sh[NQ][kThr / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double a = v[q];
    for (int off = 16; off; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
    if (lane == 0) sh[q][warp] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < NQ; ++q) {
      double a = 0.0;
      for (int w = 0; w < kThr / 32; ++w) a += sh[q][w];
      R.part[((size_t)s * kNq + q) * R.bps + blockIdx.x] = a;
    }
    __threadfence();
    last = atomicAdd(R.cnt + s, 1u) == (unsigned)R.bps - 1u;
  }
  __syncthreads();
  if (!last) return;  // block-uniform
  __threadfence();
  for (int q = 0; q < NQ; ++q) {
    double a = 0.0;
    for (int b = threadIdx.x; b < R.bps; b += kThr) a += __ldcg(R.part + ((size_t)s * kNq + q) * R.bps + b);
    for (int off = 16; off; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
    __syncthreads();
    if (lane == 0) sh[q][warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kThr / 32; ++w) t += sh[q][w];
      R.sc[(size_t)s * SC_N + dst[q]] = t;
    }
  }
  if (threadIdx.x == 0) R.cnt[s] = 0u;
}

#define FOR_PIXELS(V)                                                                         \
  const int s = blockIdx.y;                                                                   \
  for (size_t idx = (size_t)blockIdx.x * kThr + threadIdx.x; idx < (V).N;                     \
       idx += (size_t)gridDim.x * kThr)

// ---- CG kernels ---------------------------------------------------------------

// r0 = A^T b - A^T A x (CG); A^T b + v - (A^T A x + (l1 + mu) x) (L1);
// (A^T b + Gt(v)) - ((A^T A x + l1 x) + Gt(G(x))) (TV).  p0 = r0; sc[RR] = <r0, r0>.
template <int REG>
__global__ void __launch_bounds__(kThr) cg_init_kernel(Vec V, Red R) {
  double rr = 0.0;
  FOR_PIXELS(V) {
    const size_t o = (size_t)s * V.N + idx;
    if constexpr (REG == TOMO_REG_LASSO_TV) {
      const int i = (int)(idx / V.n1), j = (int)(idx - (size_t)i * V.n1);
      const float *vs = V.v + (size_t)s * 2 * V.N;
      const float *xs = V.x + (size_t)s * V.N;
      const double gtv = gt_at(i, j, V.n0, V.n1, [&](int k, int jj) { return vs[(size_t)k * V.n1 + jj]; },
                               [&](int ii, int k) { return vs[V.N + (size_t)ii * V.n1 + k]; });
      const double gtgx = gtg_at<float>(xs, V.n0, V.n1, i, j);
      const double t1 = __dadd_rn((double)V.atb[o], gtv);
      const float t2 = __fadd_rn(V.q[o], __fmul_rn(V.l1, V.x[o]));
      const double r = __dsub_rn(t1, __dadd_rn((double)t2, gtgx));
      ((double *)V.r)[o] = r;
      ((double *)V.p)[o] = r;
      V.p32[o] = __double2float_rn(r);
      rr = fma(r, r, rr);
    } else {
      float r;
      if constexpr (REG == TOMO_REG_LASSO)
        r = __fsub_rn(__fadd_rn(V.atb[o], V.v[o]), __fadd_rn(V.q[o], __fmul_rn(V.c, V.x[o])));
      else
        r = __fsub_rn(V.atb[o], V.q[o]);
      ((float *)V.r)[o] = r;
      ((float *)V.p)[o] = r;
      rr = fma((double)r, (double)r, rr);
    }
  }
  reduce_commit<1>(R, blockIdx.y, {rr}, {SC_RR});
}

// Hp = A^T A p (CG); + (l1 + mu) p (L1); (A^T A p + l1 p) + mu Gt(G(p)) (TV);
// sc[PHP] = <p, Hp>.
template <int REG>
__global__ void __launch_bounds__(kThr) cg_hp_kernel(Vec V, Red R) {
  double php = 0.0;
  FOR_PIXELS(V) {
    const size_t o = (size_t)s * V.N + idx;
    if constexpr (REG == TOMO_REG_LASSO_TV) {
      const int i = (int)(idx / V.n1), j = (int)(idx - (size_t)i * V.n1);
      const double *ps = (const double *)V.p + (size_t)s * V.N;
      const double pv = ps[idx];
      const double gtgp = gtg_at<double>(ps, V.n0, V.n1, i, j);
      const double h = __dadd_rn(__dadd_rn((double)V.q[o], __dmul_rn((double)V.l1, pv)),
                                 __dmul_rn((double)V.mu, gtgp));
      const float hf = __double2float_rn(h);
      V.hp[o] = hf;
      php = fma(pv, (double)hf, php);
    } else {
      const float pv = ((const float *)V.p)[o];
      float h = V.q[o];
      if constexpr (REG == TOMO_REG_LASSO) h = __fadd_rn(h, __fmul_rn(V.c, pv));
      V.hp[o] = h;
      php = fma((double)pv, (double)h, php);
    }
  }
  reduce_commit<1>(R, blockIdx.y, {php}, {SC_PHP});
}

// alpha = <r,r> / (<p,Hp> + spacing(1)); x += alpha p; r_old = r; r -= alpha Hp;
// sc[RRN] = <r,r>, sc[ROLD] = <r_old, r_old> (float32 r_old).
template <int REG>
__global__ void __launch_bounds__(kThr) cg_update_kernel(Vec V, Red R) {
  const int sl = blockIdx.y;
  const double rr = R.sc[(size_t)sl * SC_N + SC_RR];
  const double php = R.sc[(size_t)sl * SC_N + SC_PHP];
  double rrn = 0.0, rold = 0.0;
  if constexpr (REG == TOMO_REG_LASSO_TV) {
    const double alpha = __ddiv_rn(rr, __dadd_rn(php, kSpacing64));
    FOR_PIXELS(V) {
      const size_t o = (size_t)s * V.N + idx;
      const double pv = ((const double *)V.p)[o], rv = ((double *)V.r)[o];
      V.x[o] = __double2float_rn(__dadd_rn((double)V.x[o], __dmul_rn(alpha, pv)));
      const float ro = __double2float_rn(rv);
      rold = fma((double)ro, (double)ro, rold);
      const double rn = __dsub_rn(rv, __dmul_rn(alpha, (double)V.hp[o]));
      ((double *)V.r)[o] = rn;
      rrn = fma(rn, rn, rrn);
    }
  } else {
    // innpr of float32 arrays is a float32 number; + np.spacing(1) (a float64)
    // makes alpha float64, so x += alpha p and r -= alpha Hp are float64
    // expressions rounded to float32 (NumPy 2 promotion)
    const double alpha = __ddiv_rn((double)(float)rr, __dadd_rn((double)(float)php, kSpacing64));
    FOR_PIXELS(V) {
      const size_t o = (size_t)s * V.N + idx;
      const float pv = ((const float *)V.p)[o], rv = ((float *)V.r)[o];
      V.x[o] = __double2float_rn(__dadd_rn((double)V.x[o], __dmul_rn(alpha, (double)pv)));
      const float rn = __double2float_rn(__dsub_rn((double)rv, __dmul_rn(alpha, (double)V.hp[o])));
      ((float *)V.r)[o] = rn;
      rrn = fma((double)rn, (double)rn, rrn);
    }
    rold = 0.0;  // r_old == r exactly: <r_old, r_old> is sc[RR]
  }
  reduce_commit<2>(R, sl, {rrn, rold}, {SC_RRN, SC_ROLD});
}

// p = r + (<r,r> / <r_old,r_old>) p   (CG: <r_old,r_old> + spacing(1)).
template <int REG>
__global__ void __launch_bounds__(kThr) cg_dir_kernel(Vec V, Red R) {
  const int sl = blockIdx.y;
  const double rrn = R.sc[(size_t)sl * SC_N + SC_RRN];
  if constexpr (REG == TOMO_REG_LASSO_TV) {
    // innpr(r_old, r_old) of float32 arrays is a float32 number
    const double beta = __ddiv_rn(rrn, (double)(float)R.sc[(size_t)sl * SC_N + SC_ROLD]);
    FOR_PIXELS(V) {
      const size_t o = (size_t)s * V.N + idx;
      const double pn = __dadd_rn(((const double *)V.r)[o], __dmul_rn(beta, ((double *)V.p)[o]));
      ((double *)V.p)[o] = pn;
      V.p32[o] = __double2float_rn(pn);
    }
  } else {
    const float ro = (float)R.sc[(size_t)sl * SC_N + SC_RR];
    if constexpr (REG == TOMO_REG_CG) {
      // float32 / (float32 + float64): a float64 coefficient (cg.py:149)
      const double beta = __ddiv_rn((double)(float)rrn, __dadd_rn((double)ro, kSpacing64));
      FOR_PIXELS(V) {
        const size_t o = (size_t)s * V.N + idx;
        ((float *)V.p)[o] = __double2float_rn(
            __dadd_rn((double)((const float *)V.r)[o], __dmul_rn(beta, (double)((float *)V.p)[o])));
      }
    } else {
      const float beta = __fdiv_rn((float)rrn, ro);  // float32 / float32 (cg.py:236)
      FOR_PIXELS(V) {
        const size_t o = (size_t)s * V.N + idx;
        ((float *)V.p)[o] = __fadd_rn(((const float *)V.r)[o], __fmul_rn(beta, ((float *)V.p)[o]));
      }
    }
  }
}

// sc[RR] <- sc[RRN] for the next step, after the direction kernel has read
// sc[RR] (L1/CG: <r_old, r_old> == <r, r> of the step just taken).
__global__ void cg_advance_kernel(double *sc, int nz) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nz) sc[(size_t)s * SC_N + SC_RR] = sc[(size_t)s * SC_N + SC_RRN];
}

// ---- ADMM outer-step kernels ------------------------------------------------

// TV (admm.py:567-592): g = G(x); u = hard_thres(g + alpha/mu, lambd2/mu);
// r = g - u; alpha += r; v = mu u - alpha (the next CG's right-hand side);
// per slice |r|^2, |x - x_old|^2, |x_old|^2; then x_old = x.
__global__ void __launch_bounds__(kThr) admm_tv_update_kernel(Vec V, Red R) {
  double e2 = 0.0, d2 = 0.0, o2 = 0.0;
  FOR_PIXELS(V) {
    const size_t o = (size_t)s * V.N + idx;
    const int i = (int)(idx / V.n1), j = (int)(idx - (size_t)i * V.n1);
    const float *xs = V.x + (size_t)s * V.N;
    const float g[2] = {grad0<float>(xs, V.n0, V.n1, i, j), grad1<float>(xs, V.n1, i, j)};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const size_t k = ((size_t)s * 2 + c) * V.N + idx;
      const float a = V.alpha[k];
      const float t = __fadd_rn(g[c], __fdiv_rn(a, V.mu));
      const float u = __fsub_rn(fmaxf(0.0f, __fsub_rn(t, V.beta)), fmaxf(0.0f, __fsub_rn(-t, V.beta)));
      const float r = __fsub_rn(g[c], u);
      const float an = __fadd_rn(a, r);
      V.alpha[k] = an;
      V.v[k] = __fsub_rn(__fmul_rn(V.mu, u), an);
      e2 = fma((double)r, (double)r, e2);
    }
    const float xo = V.xold[o], xv = V.x[o];
    const float d = __fsub_rn(xv, xo);
    d2 = fma((double)d, (double)d, d2);
    o2 = fma((double)xo, (double)xo, o2);
    V.xold[o] = xv;
  }
  reduce_commit<3>(R, blockIdx.y, {e2, d2, o2}, {SC_ERR, SC_DIFF, SC_XOLD});
}

// L1 (admm.py:387-397): u = hard_thres(x + alpha/mu, lambd2/mu); r = x - u;
// alpha += r; v = mu u - alpha; the same statistics; x_old = x.
__global__ void __launch_bounds__(kThr) admm_l1_update_kernel(Vec V, Red R) {
  double e2 = 0.0, d2 = 0.0, o2 = 0.0;
  FOR_PIXELS(V) {
    const size_t o = (size_t)s * V.N + idx;
    const float xv = V.x[o], a = V.alpha[o];
    const float t = __fadd_rn(xv, __fdiv_rn(a, V.mu));
    const float u = __fsub_rn(fmaxf(0.0f, __fsub_rn(t, V.beta)), fmaxf(0.0f, __fsub_rn(-t, V.beta)));
    const float r = __fsub_rn(xv, u);
    const float an = __fadd_rn(a, r);
    V.alpha[o] = an;
    V.v[o] = __fsub_rn(__fmul_rn(V.mu, u), an);
    e2 = fma((double)r, (double)r, e2);
    const float xo = V.xold[o];
    const float d = __fsub_rn(xv, xo);
    d2 = fma((double)d, (double)d, d2);
    o2 = fma((double)xo, (double)xo, o2);
    V.xold[o] = xv;
  }
  reduce_commit<3>(R, blockIdx.y, {e2, d2, o2}, {SC_ERR, SC_DIFF, SC_XOLD});
}

// Physical constraints on x[:, i1:i2, i1:i2] (admm.py:374-384, 556-565):
// pc == 1: negatives times 0, then the resolution circle; pc == 2: the
// circle; otherwise negatives times pc.
__global__ void constrain_kernel(float *x, int n1, int nz, int i1, int i2, float pc) {
  const int m = i2 - i1;
  const size_t M = (size_t)m * m;
  const double ctr = m * 0.5 - 0.5;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < M * nz; t += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(t / M);
    const size_t rem = t - (size_t)s * M;
    const int a = (int)(rem / m), b = (int)(rem - (size_t)a * m);
    float &v = x[((size_t)s * n1 + (i1 + a)) * n1 + (i1 + b)];
    if (pc != 2.0f) {
      const float scale = pc == 1.0f ? 0.0f : pc;
      if (v < 0.0f) v = __fmul_rn(v, scale);
    }
    if (pc == 1.0f || pc == 2.0f) {
      const double dx = __dsub_rn((double)b, ctr), dy = __dsub_rn((double)a, ctr);
      if (__dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy))) > ctr) v = 0.0f;
    }
  }
}

// Appends sc[s][ERR, DIFF, XOLD] (ADMM) or sc[s][RRN] (CG) to hist[*counter].
__global__ void record_kernel(const double *sc, int nz, int cg, double *hist, int *counter, int cap) {
  const int k = *counter;
  __syncthreads();
  for (int s = threadIdx.x; s < nz; s += blockDim.x) {
    if (k >= cap) break;
    double *h = hist + ((size_t)k * nz + s) * 3;
    const double *c = sc + (size_t)s * SC_N;
    h[0] = cg ? c[SC_RRN] : c[SC_ERR];
    h[1] = cg ? 0.0 : c[SC_DIFF];
    h[2] = cg ? 0.0 : c[SC_XOLD];
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = k + 1;
}

__global__ void fill_zero_kernel(float *p, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = 0.0f;
}

unsigned flat_grid(size_t n) {
  const size_t b = (n + 255) / 256;
  return (unsigned)(b > 148 * 32 ? 148 * 32 : (b ? b : 1));
}

}  // namespace

struct Admm {
  tomo_plan *plan = nullptr;
  Plan *p = nullptr;
  int reg = 0;
  tomo_admm_params prm{};
  const float *b = nullptr;
  Vec V{};
  Red R{};
  float *sino = nullptr;
  float *q = nullptr;
  float *atb = nullptr;
  double *hist = nullptr;
  int *counter = nullptr;
  int cap = 0;
  dim3 grid;
  cudaGraphExec_t exec = nullptr;
  float *graph_x = nullptr;
  cudaStream_t own = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  bool started = false;  // CG state (r, p) valid for a continuing plain-CG run
};

}  // namespace tomo

using namespace tomo;

struct tomo_admm {
  Admm a;
};

static void admm_free(Admm &A) {
  if (A.exec) cudaGraphExecDestroy(A.exec);
  if (A.own) cudaStreamDestroy(A.own);
  if (A.ev_in) cudaEventDestroy(A.ev_in);
  if (A.ev_out) cudaEventDestroy(A.ev_out);
  cudaFree(A.sino);
  cudaFree(A.q);
  cudaFree(A.atb);
  cudaFree(A.V.xold);
  cudaFree(A.V.v);
  cudaFree(A.V.alpha);
  cudaFree(A.V.r);
  cudaFree(A.V.p);
  if (A.reg == TOMO_REG_LASSO_TV) cudaFree(A.V.p32);
  cudaFree(A.V.hp);
  cudaFree(A.R.part);
  cudaFree(A.R.cnt);
  cudaFree(A.R.sc);
  cudaFree(A.hist);
  cudaFree(A.counter);
}

template <int REG>
static int cg_start(Admm &A, cudaStream_t st) {
  Plan &p = *A.p;
  int rc = plan_forward(p, A.V.x, A.sino, st, FwdEpi());
  if (rc) return rc;
  if ((rc = plan_adjoint(p, A.sino, A.q, st, AdjEpi()))) return rc;
  cg_init_kernel<REG><<<A.grid, kThr, 0, st>>>(A.V, A.R);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

template <int REG>
static int cg_step(Admm &A, cudaStream_t st) {
  Plan &p = *A.p;
  int rc = plan_forward(p, A.V.p32, A.sino, st, FwdEpi());
  if (rc) return rc;
  if ((rc = plan_adjoint(p, A.sino, A.q, st, AdjEpi()))) return rc;
  cg_hp_kernel<REG><<<A.grid, kThr, 0, st>>>(A.V, A.R);
  cg_update_kernel<REG><<<A.grid, kThr, 0, st>>>(A.V, A.R);
  cg_dir_kernel<REG><<<A.grid, kThr, 0, st>>>(A.V, A.R);
  cg_advance_kernel<<<(A.V.nz + 127) / 128, 128, 0, st>>>(A.R.sc, A.V.nz);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

// One ADMM outer iteration (Lasso-L1 / Lasso-TV), or one plain CG iteration.
template <int REG>
static int admm_iteration(Admm &A, cudaStream_t st) {
  int rc;
  if constexpr (REG == TOMO_REG_CG) {
    if ((rc = cg_step<REG>(A, st))) return rc;
    record_kernel<<<1, 128, 0, st>>>(A.R.sc, A.V.nz, 1, A.hist, A.counter, A.cap);
  } else {
    if ((rc = cg_start<REG>(A, st))) return rc;
    for (int k = 0; k < A.prm.n_iter_pcg; ++k)
      if ((rc = cg_step<REG>(A, st))) return rc;
    if (A.prm.pc >= 0.0f) {
      const size_t m = (size_t)(A.prm.i2 - A.prm.i1);
      constrain_kernel<<<flat_grid(m * m * A.V.nz), 256, 0, st>>>(A.V.x, A.V.n1, A.V.nz, A.prm.i1, A.prm.i2,
                                                                  A.prm.pc);
    }
    if constexpr (REG == TOMO_REG_LASSO_TV) admm_tv_update_kernel<<<A.grid, kThr, 0, st>>>(A.V, A.R);
    else admm_l1_update_kernel<<<A.grid, kThr, 0, st>>>(A.V, A.R);
    record_kernel<<<1, 128, 0, st>>>(A.R.sc, A.V.nz, 0, A.hist, A.counter, A.cap);
  }
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

static int admm_iteration_any(Admm &A, cudaStream_t st) {
  switch (A.reg) {
    case TOMO_REG_CG: return admm_iteration<TOMO_REG_CG>(A, st);
    case TOMO_REG_LASSO: return admm_iteration<TOMO_REG_LASSO>(A, st);
    default: return admm_iteration<TOMO_REG_LASSO_TV>(A, st);
  }
}

extern "C" {

int tomo_admm_create(tomo_plan *plan, int reg, const float *d_b, const tomo_admm_params *prm, void *stream,
                     tomo_admm **out) {
  if (!plan || !d_b || !prm || !out) return fail(TOMO_EINVAL, "tomo_admm_create: NULL argument");
  *out = nullptr;
  if (reg != TOMO_REG_CG && reg != TOMO_REG_LASSO && reg != TOMO_REG_LASSO_TV)
    return fail(TOMO_EINVAL, "tomo_admm_create: reg must be TOMO_REG_CG, _LASSO or _LASSO_TV");
  Plan &p = *plan_of(plan);
  const int n = p.g.n, nz = p.g.nz;
  if (image_elems(p) != (size_t)nz * n * n || sino_elems(p) != (size_t)nz * p.g.na * n)
    return fail(TOMO_EINVAL, "tomo_admm_create: the plan must hold nz slices of one geometry");
  if (n < 2) return fail(TOMO_EINVAL, "tomo_admm_create: the image side must be >= 2 (numpy.gradient)");
  if (reg != TOMO_REG_CG && prm->n_iter_pcg < 0) return fail(TOMO_EINVAL, "tomo_admm_create: n_iter_pcg < 0");
  if (reg != TOMO_REG_CG && !(prm->mu != 0.0f)) return fail(TOMO_EINVAL, "tomo_admm_create: mu must be non-zero");
  if (prm->pc >= 0.0f && (prm->i1 < 0 || prm->i2 > n || prm->i1 >= prm->i2))
    return fail(TOMO_EINVAL, "tomo_admm_create: constraint region [i1, i2) outside the image");
  auto *h = new tomo_admm();
  Admm &A = h->a;
  A.plan = plan;
  A.p = &p;
  A.reg = reg;
  A.prm = *prm;
  A.b = d_b;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t N = (size_t)n * n, ni = image_elems(p), ns = sino_elems(p);
  Vec &V = A.V;
  V.n0 = V.n1 = n;
  V.nz = nz;
  V.N = N;
  V.l1 = prm->lambd1;
  V.mu = prm->mu;
  V.c = prm->lambd1 + prm->mu;  // float32 + float32
  V.beta = reg == TOMO_REG_CG ? 0.0f : prm->lambd2 / prm->mu;
  const size_t tsz = reg == TOMO_REG_LASSO_TV ? sizeof(double) : sizeof(float);
  const size_t vlen = (reg == TOMO_REG_LASSO_TV ? 2 : 1) * ni;
  A.R.bps = (int)std::min<size_t>((N + 1023) / 1024, 1184);
  A.grid = dim3((unsigned)A.R.bps, (unsigned)nz);
  A.cap = 1 << 16;
  auto bail = [&](cudaError_t e, const char *what) {
    admm_free(A);
    delete h;
    return cuda_fail(e, what);
  };
#define ADMM_CUDA(call)                           \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return bail(e_, #call); \
  } while (0)
  ADMM_CUDA(cudaStreamCreateWithFlags(&A.own, cudaStreamNonBlocking));
  ADMM_CUDA(cudaEventCreateWithFlags(&A.ev_in, cudaEventDisableTiming));
  ADMM_CUDA(cudaEventCreateWithFlags(&A.ev_out, cudaEventDisableTiming));
  ADMM_CUDA(cudaMalloc(&A.sino, sizeof(float) * ns));
  ADMM_CUDA(cudaMalloc(&A.q, sizeof(float) * ni));
  ADMM_CUDA(cudaMalloc(&A.atb, sizeof(float) * ni));
  ADMM_CUDA(cudaMalloc(&V.xold, sizeof(float) * ni));
  ADMM_CUDA(cudaMalloc(&V.v, sizeof(float) * vlen));
  ADMM_CUDA(cudaMalloc(&V.alpha, sizeof(float) * vlen));
  ADMM_CUDA(cudaMalloc(&V.r, tsz * ni));
  ADMM_CUDA(cudaMalloc(&V.p, tsz * ni));
  if (reg == TOMO_REG_LASSO_TV) ADMM_CUDA(cudaMalloc(&V.p32, sizeof(float) * ni));
  else V.p32 = (float *)V.p;
  ADMM_CUDA(cudaMalloc(&V.hp, sizeof(float) * ni));
  ADMM_CUDA(cudaMalloc(&A.R.part, sizeof(double) * (size_t)nz * kNq * A.R.bps));
  ADMM_CUDA(cudaMalloc(&A.R.cnt, sizeof(unsigned) * nz));
  ADMM_CUDA(cudaMalloc(&A.R.sc, sizeof(double) * (size_t)nz * SC_N));
  ADMM_CUDA(cudaMalloc(&A.hist, sizeof(double) * 3 * (size_t)nz * A.cap));
  ADMM_CUDA(cudaMalloc(&A.counter, sizeof(int)));
  ADMM_CUDA(cudaMemsetAsync(A.R.cnt, 0, sizeof(unsigned) * nz, st));
  ADMM_CUDA(cudaMemsetAsync(A.R.sc, 0, sizeof(double) * (size_t)nz * SC_N, st));
  V.atb = A.atb;
  V.q = A.q;
  // A^T b once (every CG start uses it)
  int rc = plan_adjoint(p, d_b, A.atb, st, AdjEpi());
  if (rc) {
    admm_free(A);
    delete h;
    return rc;
  }
  ADMM_CUDA(cudaGetLastError());
  ADMM_CUDA(cudaStreamSynchronize(st));
#undef ADMM_CUDA
  *out = h;
  return TOMO_OK;
}

int tomo_admm_run(tomo_admm *h, float *d_x, int iters, int reset, double *stats, int use_graph, void *stream) {
  if (!h || !d_x) return fail(TOMO_EINVAL, "tomo_admm_run: NULL argument");
  if (iters < 0) return fail(TOMO_EINVAL, "tomo_admm_run: iters must be >= 0");
  Admm &A = h->a;
  if (iters > A.cap) return fail(TOMO_EINVAL, "tomo_admm_run: at most 65536 iterations per call");
  if (!reset && !A.started) return fail(TOMO_EINVAL, "tomo_admm_run: nothing to continue (reset = 0 before a run)");
  if (!reset && A.V.x != d_x) return fail(TOMO_EINVAL, "tomo_admm_run: a continued run must use the same x");
  cudaStream_t caller = (cudaStream_t)stream, st = A.own;
  TOMO_CUDA(cudaEventRecord(A.ev_in, caller));
  TOMO_CUDA(cudaStreamWaitEvent(st, A.ev_in, 0));
  TOMO_CUDA(cudaMemsetAsync(A.counter, 0, sizeof(int), st));
  A.V.x = d_x;
  const size_t ni = image_elems(*A.p);
  if (reset) {
    if (A.reg == TOMO_REG_CG) {
      int rc = cg_start<TOMO_REG_CG>(A, st);
      if (rc) return rc;
    } else {
      // it == 0 (admm.py:366-369, 525-528): u = alpha = 0, hence v = 0; x_old = x
      const size_t vlen = (A.reg == TOMO_REG_LASSO_TV ? 2 : 1) * ni;
      fill_zero_kernel<<<flat_grid(vlen), 256, 0, st>>>(A.V.v, vlen);
      fill_zero_kernel<<<flat_grid(vlen), 256, 0, st>>>(A.V.alpha, vlen);
      TOMO_CUDA(cudaMemcpyAsync(A.V.xold, d_x, sizeof(float) * ni, cudaMemcpyDeviceToDevice, st));
    }
    TOMO_CUDA(cudaGetLastError());
    A.started = true;
  }
  if (use_graph && iters > 0) {
    if (!A.exec || A.graph_x != d_x) {
      if (A.exec) {
        cudaGraphExecDestroy(A.exec);
        A.exec = nullptr;
      }
      cudaGraph_t g = nullptr;
      TOMO_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      int rc = admm_iteration_any(A, st);
      cudaError_t e = cudaStreamEndCapture(st, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
      e = cudaGraphInstantiate(&A.exec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
      A.graph_x = d_x;
    }
    for (int k = 0; k < iters; ++k) TOMO_CUDA(cudaGraphLaunch(A.exec, st));
  } else {
    for (int k = 0; k < iters; ++k) {
      int rc = admm_iteration_any(A, st);
      if (rc) return rc;
    }
  }
  TOMO_CUDA(cudaEventRecord(A.ev_out, st));
  TOMO_CUDA(cudaStreamWaitEvent(caller, A.ev_out, 0));
  if (stats && iters > 0) {
    TOMO_CUDA(cudaMemcpyAsync(stats, A.hist, sizeof(double) * 3 * (size_t)A.V.nz * iters, cudaMemcpyDeviceToHost,
                              st));
    TOMO_CUDA(cudaStreamSynchronize(st));
  }
  return TOMO_OK;
}

int tomo_admm_destroy(tomo_admm *h) {
  if (!h) return TOMO_OK;
  admm_free(h->a);
  delete h;
  return TOMO_OK;
}

}  // extern "C"
