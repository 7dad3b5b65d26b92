// Internal declarations shared by the CUDA translation units of libtomo_b200.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/tomo_b200.h"
#include "epilogue.cuh"

namespace tomo {

// ---------------------------------------------------------------------------
// Error plumbing: every entry point returns an int status; the message of the
// last failure is kept per host thread.
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define TOMO_CUDA(call)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return ::tomo::cuda_fail(e_, #call); \
  } while (0)

// ---------------------------------------------------------------------------
// Per-angle geometry, evaluated on the host exactly as the compiled reference
// evaluates it (glibc sincosf, reciprocal products) and uploaded once per plan.
// ---------------------------------------------------------------------------
enum DdMode : int {
  DD_NONE = 0,   // angle contributes nothing (theta == pi/2 exactly; unreachable)
  DD_ROWSUM = 1, // |sin| < 1e-7: detector i <- sum of image row i      (radon_dd.c:75-84)
  DD_COLSUM = 2, // |cos| < 1e-7: detector i <- sum of image column i   (radon_dd.c:87-96)
  DD_ROWS = 3,   // theta > pi/2: lines are image rows                  (radon_dd.c:99-190)
  DD_COLS = 4,   // 0 < theta < pi/2 or theta < 0: lines are columns    (radon_dd.c:194-283)
};

struct DdAngle {
  int mode;     // DdMode
  int out_row;  // sinogram row written for this angle (na - 1 - v)
  float r;      // 1/s (ROWS) or 1/c (COLS): detector boundary D_m = (m - nh) * r
  float k;      // c*r (ROWS) or s*r (COLS): line offset q_i = ((i - nh) + 0.5) * k
};

// Slant stacking (radon_ss.c): steep rays step y and interpolate x.
struct SsAngle {
  int out_row;  // na - 1 - v
  int steep;    // |sin| <= sqrt(1/2)
  float a;      // minor coordinate f = fma(-m, a, t) * rb: a = s (steep) or c
  float rb;     // 1/c (steep) or 1/s
  float wt;     // 1/|c| (steep) or 1/|s|
};

// Pixel-driven (radon_pd.c).
struct PdAngle {
  float s, c, rc;  // sin, cos, 1/c
  int flags;       // 1: theta < pi/2, 2: theta > pi/2, 4: theta == 0
};

// Ray-driven / Siddon (radon_rd.c).
struct RdAngle {
  float s, c, rc, rs;      // sin, cos, 1/c, 1/s
  float ns, nc, mns, mnc;  // nh*s, nh*c, -nh*s, -nh*c
  int mode;                // 0 general, 1 |s| < 1e-7, 2 |c| < 1e-7
  int lt, gt;              // theta < pi/2, theta > pi/2
  int tr;                  // |s| > |c|: walks run along image columns; use the transposed image
};

struct Plan {
  tomo_geom g{};
  int nh = 0;
  std::vector<float> angles;  // host copy of the angle array
  // device tables
  void *d_angles = nullptr;   // kind-specific per-angle table
  void *d_aux = nullptr;      // kind-specific extra table (ss ray limits, B-spline LUT)
  // scratch owned by the plan (e.g. transposed image for the dd forward)
  float *d_scratch = nullptr;
  size_t scratch_bytes = 0;
  // host-call staging
  float *d_in = nullptr, *d_out = nullptr;  // device buffers for *_host calls
  size_t d_in_bytes = 0, d_out_bytes = 0;
  // pinned staging for host calls (copies overlap their DMA chunk by chunk)
  char *h_stage = nullptr;
  size_t h_stage_bytes = 0;
  std::vector<cudaEvent_t> stage_events;
  cudaStream_t host_stream = nullptr;
  int device = 0;
  // distance-driven layout (radon_dd.cu)
  int dd_pads = 0, dd_w = 0, dd_wl = 0, dd_nR = 0, dd_nC = 0, dd_nS = 0;
  // warps of the forward launch that write residual partial sums (solver.cu)
  size_t fwd_warps = 0;
  // packed image / sinogram sizes in floats when they are not nz*n*n and
  // nz*na*n (batched plans of uneven geometries)
  size_t img_total = 0, sino_total = 0;
  // kind-specific state owned by the plan (gridding), freed with ext_free
  void *ext = nullptr;
  void (*ext_free)(void *) = nullptr;
};

size_t image_elems(const Plan &p);
size_t sino_elems(const Plan &p);

// One setup/forward/adjoint triple per projector kind.
#define TOMO_DECLARE_KIND(k)                                                    \
  int k##_setup(Plan &p);                                                       \
  int k##_forward(Plan &p, const float *d_img, float *d_sino, cudaStream_t s,    \
                  const FwdEpi &ep = FwdEpi());                                 \
  int k##_adjoint(Plan &p, const float *d_sino, float *d_img, cudaStream_t s,    \
                  const AdjEpi &ep = AdjEpi());
TOMO_DECLARE_KIND(dd)  // radon_dd.cu
TOMO_DECLARE_KIND(ss)  // radon_ss.cu
TOMO_DECLARE_KIND(pd)  // radon_pd.cu
TOMO_DECLARE_KIND(rd)  // radon_rd.cu
TOMO_DECLARE_KIND(bs)  // bspline.cu
TOMO_DECLARE_KIND(grid)  // grid.cu
#undef TOMO_DECLARE_KIND

// Batched distance-driven plans (radon_dd.cu): geometries of different sizes
// packed back to back, run by the same persistent kernels as a plan's slices.
int dd_setup_batch(Plan &p, const tomo_geom *geoms, int count);
int dd_layout(const Plan &p, int *instances, size_t *img_off, size_t *sino_off, size_t cap);
const std::string &dd_tuning(const Plan &p);
int dd_set_tuning(Plan &p, const char *fwd, const char *adj);

// Plan-less pieces of the dd forward (radon_dd.cu), used by dd_noalloc.cu.
int dd_build_table(const float *angles, int na, DdAngle *tab);
int dd_forward_launch(const float *d_img, float *d_scratch, float *d_sino, const DdAngle *d_tab,
                      int n, int na, int nz, cudaStream_t s);

}  // namespace tomo
