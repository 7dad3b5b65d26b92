/*
 * tomo_b200.h -- C ABI of libtomo_b200.so, the B200 (sm_100a) projector pair
 * behind the reference's projector classes.
 *
 * Two layers:
 *
 * 1. Drop-in entry points (tomo_radon_*, tomo_gen_*, tomo_gridrec_*).  Each one
 *    has the argument list and meaning of one reference C function, so that a
 *    binding which used to call the reference C can call this instead.  Host
 *    pointers, synchronous, and -- like the reference C -- they ACCUMULATE into
 *    the output array (the reference's Cython shims always pass zeros).
 *    Differences: every function returns an int status instead of void (0 on
 *    success, see TOMO_E*), and inputs the reference C would read or write out
 *    of bounds are rejected with TOMO_EINVAL instead.
 *
 * 2. Plan API (tomo_plan_*, tomo_forward, tomo_adjoint, solver steps).  Device
 *    pointers and a caller stream (cudaStream_t passed as void*), stream-ordered,
 *    no allocation per call, a batch of nz slices per call.  Outputs are
 *    overwritten.  The *_host variants take host pointers and do the copies.
 *
 * Conventions shared by both layers (they are the reference's):
 *   image    float32 [n][n] row-major (C order), n = npix;
 *   sinogram float32 [na][n], one row per angle;
 *   angles   exactly the array the reference C function receives, i.e. AFTER
 *            its Cython shim: radians for pd/rd/dd/ss (fftshifted for pd and
 *            dd), degrees for the B-spline and gridding pairs.
 * Sine and cosine of every angle are evaluated on the host with the C
 * library's sincosf(), as the compiled reference does.
 *
 * Thread safety: a plan may be used from one host thread at a time; distinct
 * plans are independent.  The drop-in entry points serialise internally.
 */
#ifndef TOMO_B200_H
#define TOMO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define TOMO_OK 0
#define TOMO_ENOMEM 12      /* device or pinned-host allocation failed */
#define TOMO_EINVAL 22      /* bad shape, kind, angle or parameter */
#define TOMO_ETIMEDOUT 110  /* a bounded device wait gave up */
#define TOMO_ECUDA 1000     /* CUDA runtime error; message via tomo_last_error */

/* ---- projector kinds ---- */
#define TOMO_KIND_PD 0      /* pixel-driven, linear (radon_pd.c method 1) */
#define TOMO_KIND_RD 1      /* ray-driven / Siddon (radon_rd.c) */
#define TOMO_KIND_DD 2      /* distance-driven (radon_dd.c) */
#define TOMO_KIND_SS 3      /* slant-stacking, linear (radon_ss.c method 1) */
#define TOMO_KIND_BSPLINE 4 /* generalised Radon of B-splines (gen_forwproj.c) */
#define TOMO_KIND_GRID 5    /* gridding / Fourier slice (gridrec_v4_*.c) */

typedef struct tomo_plan tomo_plan;

typedef struct tomo_geom {
  int kind;             /* TOMO_KIND_* */
  int n;                /* image side = detector bins (reference: sino(nang, npix)) */
  int na;               /* number of angles */
  int nz;               /* slices per call (>= 1); arrays are [nz][...] */
  const float *angles;  /* host, na entries, see conventions above */
  /* B-spline pair (gen_forwproj.c:22-25): LUT [na][lut_size] and its support */
  const float *lut;
  int lut_size;
  float support;
  /* gridding pair (gridrec_v4.pyx:28-86): param[8], lut[len], deapod[pdim*pdim] */
  const float *grid_param;
  const float *grid_lut;
  int grid_lut_len;
  const float *grid_deapod;
  int grid_mode;        /* 0 = compat: the reference's arithmetic in both directions
                         *     (gridrec_v4_forwproj.c, gridrec_v4_backproj.c);
                         * 1 = matched: the forward unchanged, the adjoint its
                         *     exact transpose (the forward's kernel width, the
                         *     transpose of the crop, consistent Hermitian halves);
                         *     no reference counterpart */
} tomo_geom;

/* Last error message of the calling thread ("" if none).  Returns TOMO_OK. */
int tomo_last_error(char *buf, size_t len);

/* Library version string, e.g. "tomo_b200 0.1 sm_100a". */
const char *tomo_version(void);

/* Measures, on the current device and at its current clocks, the shared-memory
 * load bandwidth (16-byte conflict-free loads), the L1 load bandwidth (loads
 * that hit L1, each warp request one aligned block: 4-byte loads, one 128-byte
 * line per request; 16-byte loads, four lines) and the FP32 FMA rate.  These
 * are the roofline denominators of the projector kernels (gather- and
 * issue-bound, not HBM).  tomo_measure_onchip_peaks reports the larger of the
 * two L1 rates.  No reference counterpart. */
int tomo_measure_onchip_peaks(double *smem_gbs, double *l1_gbs, double *fp32_tflops);
int tomo_measure_onchip_peaks2(double *smem_gbs, double *l1_4_gbs, double *l1_16_gbs, double *fp32_tflops);

/* ---- plan API ---- */
int tomo_plan_create(const tomo_geom *geom, tomo_plan **plan);
int tomo_plan_destroy(tomo_plan *plan);

/* Batched plan over `count` distance-driven geometries of different sizes
 * (each geoms[i].kind == TOMO_KIND_DD, with its own n, na, angles and nz
 * slices).  No reference counterpart: the reference runs independent slices
 * in a process pool (art.py:289, sir.py:260).  Images and sinograms are packed
 * back to back in geometry order, slice after slice, each slice C-order; the
 * plan is then used with tomo_forward / tomo_adjoint / tomo_solver_* on those
 * packed arrays.  Every forward or adjoint is one persistent launch over all
 * instances (plus its prefix-sum pre-pass); results equal the per-geometry
 * plans' bit for bit. */
int tomo_plan_create_batch(const tomo_geom *geoms, int count, tomo_plan **plan);
/* Number of instances (slices) of a plan and, if the arrays are given
 * (cap >= instances + 1 entries), the offset in floats of each instance's
 * image and sinogram in the packed arrays; entry [instances] is the total. */
int tomo_plan_layout(tomo_plan *plan, int *instances, size_t *img_off, size_t *sino_off, size_t cap);
/* The launch shape the plan uses (for dd: warps per block of the persistent
 * kernels, chosen at plan creation by timing the candidates on the plan's own
 * scratch when the workload is large enough), as text. */
int tomo_plan_tuning(tomo_plan *plan, char *buf, size_t len);
/* Pins the launch shape of a distance-driven plan by name instead of the
 * tuned one (NULL keeps a direction as it is): forward "w2w" "w4w" "w8w"
 * "w2b" "w4b" "w8b" (warps per block, warp or block fetch of work items);
 * adjoint "t1" "t2" "t4" (pixel tiles per block, 4 warps per tile).  Every
 * shape gives the same result to the bit; other kinds: TOMO_EINVAL. */
int tomo_plan_set_tuning(tomo_plan *plan, const char *fwd, const char *adj);

/* Forward A: d_image [nz][n][n] -> d_sino [nz][na][n] (overwritten). */
int tomo_forward(tomo_plan *plan, const float *d_image, float *d_sino, void *stream);
/* Adjoint A^T: d_sino [nz][na][n] -> d_image [nz][n][n] (overwritten). */
int tomo_adjoint(tomo_plan *plan, const float *d_sino, float *d_image, void *stream);
/* Same, host arrays in and out (copies through pinned staging; synchronous). */
int tomo_forward_host(tomo_plan *plan, const float *h_image, float *h_sino);
int tomo_adjoint_host(tomo_plan *plan, const float *h_sino, float *h_image);

/* ---- iterative solvers with the update fused into the projector kernels ---- */
#define TOMO_ALGO_SIRT 1 /* art.py:211-237: x += C A^T(R (b - A x)), R = 1/A1, C = 1/A^T1 */
#define TOMO_ALGO_MLEM 2 /* sir.py:204-290: x *= (1/A^T1) A^T(b / A x) */
#define TOMO_ALGO_SPS 3  /* sir.py:348-540 (no penalty): x = clip(x - A^T(w(Ax-b))/(A^T(w A1)+eps), 0, max x) */

typedef struct tomo_solver tomo_solver;

/* Binds a solver to a plan and a measured sinogram d_b [nz][na][n] (device;
 * must stay valid while the solver lives) and precomputes its normalisation
 * (R, C; 1/A^T1; w and A^T(w A1)) exactly as the reference does in float32.
 * Replaces the set-up half of the reference's art.sirt / sir.em / sir.sps. */
int tomo_solver_create(tomo_plan *plan, int algo, const float *d_b, void *stream,
                       tomo_solver **solver);
/* Runs `iters` iterations in place on d_x [nz][n][n].  Each iteration is one
 * forward and one adjoint launch (plus a residual reduction), captured once
 * into a CUDA graph when use_graph != 0.  If residuals != NULL it receives
 * ||A x_k - b||^2 of the iterate entering iteration k (k = 0..iters-1).  The
 * work is ordered after, and before later work on, `stream`. */
int tomo_solver_run(tomo_solver *solver, float *d_x, int iters, double *residuals, int use_graph,
                    void *stream);
int tomo_solver_destroy(tomo_solver *solver);

/* ---- ADMM / conjugate-gradient solvers (algorithms/admm.py, algorithms/cg.py) ---- */
#define TOMO_REG_CG 1       /* cg.py:83-185: CG on A^T A x = A^T b (admm.py:245 conj_grad) */
#define TOMO_REG_LASSO 2    /* admm.py:291-457 lasso_l1, inner cg.py:189-253 cg_lasso_l1 */
#define TOMO_REG_LASSO_TV 3 /* admm.py:470-640 lasso_tv, inner cg.py:256-320 cg_lasso_tv */

typedef struct tomo_admm_params {
  float lambd1, lambd2, mu; /* class_admm_param.py:67-69 (float32) */
  int n_iter_pcg;           /* inner CG iterations per ADMM iteration (-n2) */
  float pc;                 /* -pc: < 0 off; 1: negatives to 0 and resolution circle;
                               2: circle only; otherwise negatives times pc */
  int i1, i2;               /* the constraint acts on x[:, i1:i2, i1:i2] */
} tomo_admm_params;

typedef struct tomo_admm tomo_admm;

/* Binds an ADMM (or plain CG) solver to a plan of nz slices of one geometry
 * and a measured sinogram d_b [nz][na][n] (device; must outlive the solver);
 * computes A^T b once.  The arithmetic keeps the reference's numpy types
 * (float32 x; float64 r, p for Lasso-TV; float32 scalars). */
int tomo_admm_create(tomo_plan *plan, int reg, const float *d_b, const tomo_admm_params *prm, void *stream,
                     tomo_admm **out);
/* Runs `iters` ADMM iterations (Lasso-L1 / Lasso-TV: n_iter_pcg CG steps,
 * the constraint, the shrinkage and the multiplier update) or `iters` CG
 * iterations (TOMO_REG_CG) in place on d_x [nz][n][n].  reset != 0 starts as
 * the reference's function does (u = alpha = 0, x_old = x; CG: r0 from x);
 * reset == 0 continues the previous call on the same d_x.  If stats != NULL
 * it receives [iters][nz][3]: per slice |r|^2, |x - x_old|^2, |x_old|^2 (ADMM,
 * r the multiplier update) or |r|^2, 0, 0 (CG, r the CG residual). */
int tomo_admm_run(tomo_admm *h, float *d_x, int iters, int reset, double *stats, int use_graph, void *stream);
int tomo_admm_destroy(tomo_admm *h);

/* Distance-driven forward projection that allocates no device memory, for
 * callers that cannot call cudaMalloc (their device memory belongs to another
 * allocator, or they must not allocate inside a latency-bound loop).  No
 * counterpart in the reference.  d_image [nz][npix][npix] and d_sino
 * [nz][nang][npix] are device pointers (the sinogram is overwritten); angles is
 * the host array tomo_radon_dd receives.  Scratch lives in static device arrays
 * of this library (16 MiB + 256 KiB per GPU, held until exit): nz*npix*npix
 * must be <= 4194304 and nang <= 16384, else TOMO_EINVAL.  The first call on a
 * device sets up the arrays' addresses; make it before any stream capture.
 * All calls share the arrays: calls that overlap on the GPU race. */
int tomo_radon_dd_forward_noalloc(const float *d_image, int npix, const float *angles, int nang,
                                  int nz, float *d_sino, void *stream);

/* ---- sinogram pre-processing on the device (common/myimage/my_image_process.py) ---- */

/* sino_edge_padding (my_image_process.py:142-157): d_out [nang][npix + 2*npad]
 * = npad copies of column 0, the sinogram, npad copies of column npix-1. */
int tomo_sino_edge_pad(const float *d_sino, int nang, int npix, int npad, float *d_out, void *stream);

/* sino_correct_rot_axis (my_image_process.py:87-117): d_out [nang][npix] = each
 * row shifted by ctr - npix/2.  Integer shifts: the reference's roll with the
 * wrapped columns replaced by the edge column (exact).  Fractional shifts: Keys
 * cubic convolution of the zero-extended row, where the reference uses scipy's
 * 2-D Clough-Tocher griddata (the two agree to ~1e-3 of the signal on smooth
 * data).  d_out must not alias d_sino. */
int tomo_sino_center(const float *d_sino, int nang, int npix, double ctr, float *d_out, void *stream);

/* ---- ADMM-TV / CG finite differences on the device (algorithms/cg.py:62-71) ---- */

/* G: numpy.gradient of d_m [n0][n1] (float32): d_g0 along axis 0, d_g1 along axis 1. */
int tomo_grad2d(const float *d_m, int n0, int n1, float *d_g0, float *d_g1, void *stream);
/* Gt: d_out [n0][n1] (float64) = g1 . Gx + Gy . g0 with Gx, Gy the gradient matrices of
 * identities, as the reference multiplies them densely; the same float64 numbers, O(n^2). */
int tomo_grad2d_adjoint(const float *d_g0, const float *d_g1, int n0, int n1, double *d_out, void *stream);

/* ---- drop-in entry points (reference C signatures; host pointers) ---- */

/* radon_pd.c:20 `void radon_pd(float* image, int npix, float* angles, int nang,
 * int oper, int method, float* sino)`, bound at radon_pixel_driven.pyx:7-8.
 * oper 0: sino += A image; oper 1: image += A^T sino.  Only method 1 (linear,
 * the one class_projectors_radon.py:62 uses) is provided: the reference's
 * method 0 indexes bins outside [0, npix) for edge pixels; it returns
 * TOMO_EINVAL. */
int tomo_radon_pd(float *image, int npix, const float *angles, int nang, int oper,
                  int method, float *sino);

/* radon_rd.c:76 `void radon_rd(float* image, int npix, float* angles, int nang,
 * int oper, float* sino)`, bound at radon_ray_driven.pyx:7-8. */
int tomo_radon_rd(float *image, int npix, const float *angles, int nang, int oper,
                  float *sino);

/* radon_dd.c:54 `void radon_dd(float* image, int npix, float* angles, int nang,
 * int oper, float* sino)`, bound at radon_distance_driven.pyx:7.  Angles must
 * lie in [-pi/2, pi] (outside it the reference's boundary merge is undefined). */
int tomo_radon_dd(float *image, int npix, const float *angles, int nang, int oper,
                  float *sino);

/* radon_ss.c:93 `void radon_ss(float* image, int npix, float* angles, int nang,
 * int oper, int method, float* sino)`, bound at radon_slant_stacking.pyx:7-8.
 * Only method 1 (linear, class_projectors_radon.py:68) is provided.  Rays that
 * miss the square [-nh, nh-1]^2 (within about 1/nh rad of 180 degrees) make the
 * reference index outside the image; here those rows contribute nothing. */
int tomo_radon_ss(float *image, int npix, const float *angles, int nang, int oper,
                  int method, float *sino);

/* gen_forwproj.c:22 `void gen_forwproj(float* image, int npix, float* angles,
 * int nang, float* lut, int lut_size, float support_bspline, int num_cores,
 * float* sino)`, bound at genradon.pyx:10-11.  Angles in degrees; lut is
 * [nang][lut_size]; num_cores is accepted and ignored. */
int tomo_gen_forwproj(const float *image, int npix, const float *angles, int nang,
                      const float *lut, int lut_size, float support_bspline,
                      int num_cores, float *sino);

/* gen_backproj.c:22 `void gen_backproj(float* sino, int npix, float* angles,
 * int nang, float* lut, int lut_size, float support_bspline, float* image)`,
 * bound at genradon.pyx:13-14. */
int tomo_gen_backproj(const float *sino, int npix, const float *angles, int nang,
                      const float *lut, int lut_size, float support_bspline,
                      float *image);

/* gridrec_v4_forwproj.c:59 `void gridrec_v4_forwproj(float *S, int npix, int nang,
 * float *angles, float *param, float *lut, float *deapod, float *I, char *fftwfn)`,
 * bound at gridrec_v4.pyx:10-11.  Angles in degrees; param[8] = {ctr, filter,
 * filter source, oversampling, interp (0 nearest, 1 linear), len(lut)-5, kernel
 * width, Radon degree}; deapod is [pdim][pdim].  Like the reference it OVERWRITES
 * S.  fftwfn (an FFTW wisdom file) is accepted and ignored. */
int tomo_gridrec_forwproj(float *S, int npix, int nang, const float *angles, const float *param,
                          const float *lut, const float *deapod, const float *I, const char *fftwfn);

/* gridrec_v4_backproj.c:64 `void gridrec_v4_backproj(float *sino, int npix, int nang,
 * float *angles, float *param, float *lut, float *deapod, float *filter_ext, float *rec,
 * char *fftwfn)`, bound at gridrec_v4.pyx:7-8.  Overwrites rec.  Only the built-in
 * filters (param[2] == 0, what the reference classes pass) are provided;
 * filter_ext and fftwfn are accepted and ignored. */
int tomo_gridrec_backproj(const float *sino, int npix, int nang, const float *angles,
                          const float *param, const float *lut, const float *deapod,
                          const float *filter_ext, float *rec, const char *fftwfn);

#ifdef __cplusplus
}
#endif

#endif /* TOMO_B200_H */
