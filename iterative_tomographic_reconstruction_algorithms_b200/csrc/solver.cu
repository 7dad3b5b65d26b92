// Iterative solvers on a projector plan: SIRT, MLEM and SPS with their update
// arithmetic fused into the projector kernels (epilogue.cuh).
//
// References: SIRT algorithms/art.py:211-237 (R = 1/A1, C = 1/A^T1, zeros
// replaced by 1e-10; x <- x + C A^T (R (b - A x))); MLEM algorithms/sir.py
// :204-290 (d = A^T 1, zeros + 1e-10; x <- x * (1/d) * A^T(b / A x), A x == 0
// replaced by eps); SPS algorithms/sir.py:348-540 without regularisation
// (w = exp(-b / max b), den = A^T(w A 1); x <- clip(x - A^T(w (A x - b)) /
// (den + eps), 0, max x)).
//
// One iteration = one forward launch whose epilogue produces the sinogram the
// adjoint needs (and per-warp partial sums of |A x - b|^2), one adjoint launch
// whose epilogue writes the updated iterate in place, and two tiny kernels:
// the fixed-order residual reduction and (SPS) the clip fix-up.  The
// iteration is captured once into a CUDA graph and replayed.
#include <cmath>
#include <string>

#include "tomo_internal.cuh"

namespace tomo {
namespace {

__global__ void fill_kernel(float *p, size_t n, float v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// out = 1 / (in == 0 ? 1e-10 : in), float32 as numpy evaluates R[R==0] += 1e-10; 1.0/R
__global__ void recip_guard_kernel(const float *in, float *out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float v = in[i];
    if (v == 0.0f) v = 1e-10f;
    out[i] = __fdiv_rn(1.0f, v);
  }
}

__global__ void max_kernel(const float *in, size_t n, unsigned *out) {
  unsigned m = 0u;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = max(m, float_to_ordered(in[i]));
  for (int off = 16; off; off >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// w = exp(-b / max b) (sir.py:366-367), then aux = w * A1 in place of A1
__global__ void sps_weights_kernel(const float *b, const unsigned *bmax, float *w, float *a1, size_t n) {
  const float m = ordered_to_float(*bmax);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float wi = expf(__fdiv_rn(-b[i], m));
    w[i] = wi;
    a1[i] = __fmul_rn(wi, a1[i]);
  }
}

// Fixed-order sum of the residual partials into out[*counter]; ++*counter.
__global__ void reduce_resid_kernel(const double *part, size_t n, double *out, int *counter, int cap) {
  __shared__ double sh[1024];
  double s = 0.0;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int k = *counter;
    if (k < cap) out[k] = sh[0];
    *counter = k + 1;
  }
}

// clip(x, 0, M): the epilogue already wrote max(x, 0), which is the answer
// unless every updated value was negative (M < 0), where numpy gives M.
__global__ void sps_fixup_kernel(float *x, size_t n, const unsigned *mx) {
  const float m = ordered_to_float(*mx);
  if (!(m < 0.0f)) return;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = m;
}

unsigned grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b > 148 * 32 ? 148 * 32 : (b ? b : 1));
}

}  // namespace

struct Solver {
  tomo_plan *plan = nullptr;
  Plan *p = nullptr;
  int algo = 0;
  const float *b = nullptr;
  float *y = nullptr;       // forward epilogue output (sinogram)
  float *aux_f = nullptr;   // R (SIRT) / w (SPS)
  float *aux_a = nullptr;   // C (SIRT) / 1/d (MLEM) / den (SPS)
  double *part = nullptr;   // residual partial sums
  size_t nparts = 0;
  double *resid = nullptr;  // residual per iteration (device)
  int *counter = nullptr;
  int cap = 0;
  unsigned *sps_max = nullptr;
  cudaGraphExec_t exec = nullptr;
  float *graph_x = nullptr;
  cudaStream_t own = nullptr;  // iterations run (and are captured) here
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
};

}  // namespace tomo

using namespace tomo;

struct tomo_solver {
  Solver s;
};

// Plan accessors defined in tomo_abi.cu
namespace tomo {
Plan *plan_of(tomo_plan *p);
int plan_forward(Plan &p, const float *in, float *out, cudaStream_t s, const FwdEpi &ep);
int plan_adjoint(Plan &p, const float *in, float *out, cudaStream_t s, const AdjEpi &ep);
}  // namespace tomo

static void solver_free(Solver &S) {
  if (S.exec) cudaGraphExecDestroy(S.exec);
  if (S.own) cudaStreamDestroy(S.own);
  if (S.ev_in) cudaEventDestroy(S.ev_in);
  if (S.ev_out) cudaEventDestroy(S.ev_out);
  cudaFree(S.y);
  cudaFree(S.aux_f);
  cudaFree(S.aux_a);
  cudaFree(S.part);
  cudaFree(S.resid);
  cudaFree(S.counter);
  cudaFree(S.sps_max);
}

static int solver_iteration(Solver &S, float *x, cudaStream_t st) {
  Plan &p = *S.p;
  const size_t ni = image_elems(p);
  FwdEpi fe;
  fe.op = S.algo == TOMO_ALGO_SIRT ? EPI_SIRT : (S.algo == TOMO_ALGO_MLEM ? EPI_MLEM : EPI_SPS);
  fe.b = S.b;
  fe.w = S.aux_f;
  fe.resid = S.part;
  AdjEpi ae;
  ae.op = fe.op;
  ae.x = x;
  ae.aux = S.aux_a;
  ae.sps_max = S.sps_max;
  if (S.algo == TOMO_ALGO_SPS) TOMO_CUDA(cudaMemsetAsync(S.sps_max, 0, sizeof(unsigned), st));
  int rc = plan_forward(p, x, S.y, st, fe);
  if (rc) return rc;
  reduce_resid_kernel<<<1, 1024, 0, st>>>(S.part, S.nparts, S.resid, S.counter, S.cap);
  rc = plan_adjoint(p, S.y, x, st, ae);
  if (rc) return rc;
  if (S.algo == TOMO_ALGO_SPS) sps_fixup_kernel<<<grid_for(ni), 256, 0, st>>>(x, ni, S.sps_max);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

extern "C" {

int tomo_solver_create(tomo_plan *plan, int algo, const float *d_b, void *stream, tomo_solver **out) {
  if (!plan || !d_b || !out) return fail(TOMO_EINVAL, "tomo_solver_create: NULL argument");
  if (algo != TOMO_ALGO_SIRT && algo != TOMO_ALGO_MLEM && algo != TOMO_ALGO_SPS)
    return fail(TOMO_EINVAL, "tomo_solver_create: algo must be TOMO_ALGO_SIRT, _MLEM or _SPS");
  *out = nullptr;
  auto *ts = new tomo_solver();
  Solver &S = ts->s;
  S.plan = plan;
  S.p = plan_of(plan);
  S.algo = algo;
  S.b = d_b;
  Plan &p = *S.p;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t ni = image_elems(p), ns = sino_elems(p);
  S.nparts = p.fwd_warps;
  S.cap = 1 << 16;
  int rc = TOMO_OK;
  float *ones_i = nullptr, *ones_s = nullptr;
  auto bail = [&](int code) {
    cudaFree(ones_i);
    cudaFree(ones_s);
    solver_free(S);
    delete ts;
    return code;
  };
#define SOLVER_CUDA(call)                                \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return bail(cuda_fail(e_, #call)); \
  } while (0)
  SOLVER_CUDA(cudaStreamCreateWithFlags(&S.own, cudaStreamNonBlocking));
  SOLVER_CUDA(cudaEventCreateWithFlags(&S.ev_in, cudaEventDisableTiming));
  SOLVER_CUDA(cudaEventCreateWithFlags(&S.ev_out, cudaEventDisableTiming));
  SOLVER_CUDA(cudaMalloc(&S.y, sizeof(float) * ns));
  SOLVER_CUDA(cudaMalloc(&S.aux_f, sizeof(float) * ns));
  SOLVER_CUDA(cudaMalloc(&S.aux_a, sizeof(float) * ni));
  SOLVER_CUDA(cudaMalloc(&S.part, sizeof(double) * S.nparts));
  SOLVER_CUDA(cudaMalloc(&S.resid, sizeof(double) * S.cap));
  SOLVER_CUDA(cudaMalloc(&S.counter, sizeof(int)));
  SOLVER_CUDA(cudaMalloc(&S.sps_max, sizeof(unsigned)));
  SOLVER_CUDA(cudaMemsetAsync(S.counter, 0, sizeof(int), st));
  SOLVER_CUDA(cudaMalloc(&ones_i, sizeof(float) * ni));
  SOLVER_CUDA(cudaMalloc(&ones_s, sizeof(float) * ns));
  fill_kernel<<<grid_for(ni), 256, 0, st>>>(ones_i, ni, 1.0f);
  fill_kernel<<<grid_for(ns), 256, 0, st>>>(ones_s, ns, 1.0f);
  if (algo == TOMO_ALGO_SIRT) {
    // R = 1/(A 1), C = 1/(A^T 1)   (art.py:227-237)
    if ((rc = plan_forward(p, ones_i, S.y, st, FwdEpi()))) return bail(rc);
    recip_guard_kernel<<<grid_for(ns), 256, 0, st>>>(S.y, S.aux_f, ns);
    if ((rc = plan_adjoint(p, ones_s, S.aux_a, st, AdjEpi()))) return bail(rc);
    recip_guard_kernel<<<grid_for(ni), 256, 0, st>>>(S.aux_a, S.aux_a, ni);
  } else if (algo == TOMO_ALGO_MLEM) {
    // 1/d with d = A^T 1   (sir.py:215-217, 283)
    if ((rc = plan_adjoint(p, ones_s, S.aux_a, st, AdjEpi()))) return bail(rc);
    recip_guard_kernel<<<grid_for(ni), 256, 0, st>>>(S.aux_a, S.aux_a, ni);
  } else {
    // w = exp(-b / max b), den = A^T(w * A 1)   (sir.py:365-384)
    SOLVER_CUDA(cudaMemsetAsync(S.sps_max, 0, sizeof(unsigned), st));
    max_kernel<<<grid_for(ns), 256, 0, st>>>(d_b, ns, S.sps_max);
    if ((rc = plan_forward(p, ones_i, S.y, st, FwdEpi()))) return bail(rc);
    sps_weights_kernel<<<grid_for(ns), 256, 0, st>>>(d_b, S.sps_max, S.aux_f, S.y, ns);
    if ((rc = plan_adjoint(p, S.y, S.aux_a, st, AdjEpi()))) return bail(rc);
  }
  SOLVER_CUDA(cudaGetLastError());
  SOLVER_CUDA(cudaStreamSynchronize(st));
  cudaFree(ones_i);
  cudaFree(ones_s);
#undef SOLVER_CUDA
  *out = ts;
  return TOMO_OK;
}

int tomo_solver_run(tomo_solver *solver, float *d_x, int iters, double *residuals, int use_graph,
                    void *stream) {
  if (!solver || !d_x) return fail(TOMO_EINVAL, "tomo_solver_run: NULL argument");
  if (iters < 0) return fail(TOMO_EINVAL, "tomo_solver_run: iters must be >= 0");
  Solver &S = solver->s;
  if (iters > S.cap) return fail(TOMO_EINVAL, "tomo_solver_run: at most 65536 iterations per call");
  cudaStream_t caller = (cudaStream_t)stream, st = S.own;
  // order the solver's stream after the caller's work, and the caller's after ours
  TOMO_CUDA(cudaEventRecord(S.ev_in, caller));
  TOMO_CUDA(cudaStreamWaitEvent(st, S.ev_in, 0));
  TOMO_CUDA(cudaMemsetAsync(S.counter, 0, sizeof(int), st));
  if (use_graph && iters > 0) {
    if (!S.exec || S.graph_x != d_x) {
      if (S.exec) {
        cudaGraphExecDestroy(S.exec);
        S.exec = nullptr;
      }
      cudaGraph_t g = nullptr;
      TOMO_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      int rc = solver_iteration(S, d_x, st);
      cudaError_t e = cudaStreamEndCapture(st, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
      e = cudaGraphInstantiate(&S.exec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
      S.graph_x = d_x;
    }
    for (int k = 0; k < iters; ++k) TOMO_CUDA(cudaGraphLaunch(S.exec, st));
  } else {
    for (int k = 0; k < iters; ++k) {
      int rc = solver_iteration(S, d_x, st);
      if (rc) return rc;
    }
  }
  TOMO_CUDA(cudaEventRecord(S.ev_out, st));
  TOMO_CUDA(cudaStreamWaitEvent(caller, S.ev_out, 0));
  if (residuals && iters > 0) {
    TOMO_CUDA(cudaMemcpyAsync(residuals, S.resid, sizeof(double) * iters, cudaMemcpyDeviceToHost, st));
    TOMO_CUDA(cudaStreamSynchronize(st));
  }
  return TOMO_OK;
}

int tomo_solver_destroy(tomo_solver *solver) {
  if (!solver) return TOMO_OK;
  solver_free(solver->s);
  delete solver;
  return TOMO_OK;
}

}  // extern "C"
