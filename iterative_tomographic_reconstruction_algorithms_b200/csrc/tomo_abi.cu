// C ABI of libtomo_b200: plans, dispatch, host-buffer calls and the drop-in
// entry points that mirror the reference C functions (include/tomo_b200.h).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>
#include <thread>
#include <atomic>
#include <algorithm>
#include <condition_variable>
#include <functional>

#include "tomo_internal.cuh"

namespace tomo {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  g_last_error = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) +
                 ") in " + what;
  return TOMO_ECUDA;
}

size_t image_elems(const Plan &p) { return p.img_total ? p.img_total : (size_t)p.g.nz * p.g.n * p.g.n; }
size_t sino_elems(const Plan &p) { return p.sino_total ? p.sino_total : (size_t)p.g.nz * p.g.na * p.g.n; }

static void release(Plan &p) {
  if (p.d_angles) cudaFree(p.d_angles);
  if (p.d_aux) cudaFree(p.d_aux);
  if (p.d_scratch) cudaFree(p.d_scratch);
  if (p.d_in) cudaFree(p.d_in);
  if (p.d_out) cudaFree(p.d_out);
  if (p.host_stream) cudaStreamDestroy(p.host_stream);
  if (p.h_stage) cudaFreeHost(p.h_stage);
  for (cudaEvent_t e : p.stage_events) cudaEventDestroy(e);
  p.stage_events.clear();
  p.h_stage = nullptr;
  if (p.ext && p.ext_free) p.ext_free(p.ext);
  p.ext = nullptr;
  p.d_angles = p.d_aux = nullptr;
  p.d_scratch = p.d_in = p.d_out = nullptr;
  p.host_stream = nullptr;
}

static int validate(const tomo_geom *g) {
  if (!g) return fail(TOMO_EINVAL, "geometry is NULL");
  if (g->n < 2 || g->n > 32767)
    return fail(TOMO_EINVAL, "n (npix) must be in [2, 32767], got " + std::to_string(g->n));
  if (g->na < 1 || g->na > 65535)
    return fail(TOMO_EINVAL, "na (nang) must be in [1, 65535], got " + std::to_string(g->na));
  if (g->nz < 1 || g->nz > 65535)
    return fail(TOMO_EINVAL, "nz must be in [1, 65535], got " + std::to_string(g->nz));
  if (!g->angles) return fail(TOMO_EINVAL, "angles pointer is NULL");
  for (int v = 0; v < g->na; ++v)
    if (!std::isfinite(g->angles[v]))
      return fail(TOMO_EINVAL, "angle " + std::to_string(v) + " is not finite");
  switch (g->kind) {
    case TOMO_KIND_PD:
    case TOMO_KIND_RD:
    case TOMO_KIND_DD:
    case TOMO_KIND_SS:
    case TOMO_KIND_BSPLINE:
    case TOMO_KIND_GRID:
      return TOMO_OK;
    default:
      return fail(TOMO_EINVAL, "projector kind " + std::to_string(g->kind) + " is not available");
  }
}

}  // namespace tomo

using namespace tomo;

struct tomo_plan {
  Plan p;
};

namespace tomo {
Plan *plan_of(tomo_plan *p) { return &p->p; }

int plan_forward(Plan &p, const float *in, float *out, cudaStream_t s, const FwdEpi &ep) {
  switch (p.g.kind) {
    case TOMO_KIND_PD: return pd_forward(p, in, out, s, ep);
    case TOMO_KIND_RD: return rd_forward(p, in, out, s, ep);
    case TOMO_KIND_DD: return dd_forward(p, in, out, s, ep);
    case TOMO_KIND_SS: return ss_forward(p, in, out, s, ep);
    case TOMO_KIND_BSPLINE: return bs_forward(p, in, out, s, ep);
    case TOMO_KIND_GRID: return grid_forward(p, in, out, s, ep);
  }
  return fail(TOMO_EINVAL, "forward: unsupported kind");
}

int plan_adjoint(Plan &p, const float *in, float *out, cudaStream_t s, const AdjEpi &ep) {
  switch (p.g.kind) {
    case TOMO_KIND_PD: return pd_adjoint(p, in, out, s, ep);
    case TOMO_KIND_RD: return rd_adjoint(p, in, out, s, ep);
    case TOMO_KIND_DD: return dd_adjoint(p, in, out, s, ep);
    case TOMO_KIND_SS: return ss_adjoint(p, in, out, s, ep);
    case TOMO_KIND_BSPLINE: return bs_adjoint(p, in, out, s, ep);
    case TOMO_KIND_GRID: return grid_adjoint(p, in, out, s, ep);
  }
  return fail(TOMO_EINVAL, "adjoint: unsupported kind");
}
}  // namespace tomo

extern "C" {

int tomo_last_error(char *buf, size_t len) {
  if (buf && len) {
    std::snprintf(buf, len, "%s", g_last_error.c_str());
  }
  return TOMO_OK;
}

const char *tomo_version(void) { return "tomo_b200 0.1 sm_100a"; }

int tomo_plan_create(const tomo_geom *geom, tomo_plan **out) {
  if (!out) return fail(TOMO_EINVAL, "plan output pointer is NULL");
  *out = nullptr;
  int rc = validate(geom);
  if (rc) return rc;
  auto *tp = new tomo_plan();
  Plan &p = tp->p;
  p.g = *geom;
  p.nh = (int)(geom->n * 0.5);
  p.angles.assign(geom->angles, geom->angles + geom->na);
  p.g.angles = nullptr;
  cudaGetDevice(&p.device);
  switch (p.g.kind) {
    case TOMO_KIND_PD: rc = pd_setup(p); break;
    case TOMO_KIND_RD: rc = rd_setup(p); break;
    case TOMO_KIND_DD: rc = dd_setup(p); break;
    case TOMO_KIND_SS: rc = ss_setup(p); break;
    case TOMO_KIND_BSPLINE: rc = bs_setup(p); break;
    case TOMO_KIND_GRID: rc = grid_setup(p); break;
    default:
      rc = fail(TOMO_EINVAL, "unsupported kind");
  }
  if (rc) {
    release(p);
    delete tp;
    return rc;
  }
  if (!p.fwd_warps) p.fwd_warps = (size_t)((p.g.n + 127) / 128) * 4 * p.g.na * p.g.nz;
  *out = tp;
  return TOMO_OK;
}

int tomo_plan_create_batch(const tomo_geom *geoms, int count, tomo_plan **out) {
  if (!out) return fail(TOMO_EINVAL, "plan output pointer is NULL");
  *out = nullptr;
  if (!geoms || count < 1) return fail(TOMO_EINVAL, "batch: need at least one geometry");
  size_t instances = 0;
  for (int i = 0; i < count; ++i) {
    int rc = validate(&geoms[i]);
    if (rc) return fail(rc, "batch geometry " + std::to_string(i) + ": " + g_last_error);
    if (geoms[i].kind != TOMO_KIND_DD)
      return fail(TOMO_EINVAL, "batch geometry " + std::to_string(i) +
                                   ": batched plans are available for the distance-driven pair only");
    instances += (size_t)geoms[i].nz;
  }
  if (instances > (1u << 24)) return fail(TOMO_EINVAL, "batch: more than 2^24 instances");
  auto *tp = new tomo_plan();
  Plan &p = tp->p;
  p.g = geoms[0];
  p.g.angles = nullptr;
  p.nh = (int)(p.g.n * 0.5);
  cudaGetDevice(&p.device);
  int rc = dd_setup_batch(p, geoms, count);
  if (rc) {
    release(p);
    delete tp;
    return rc;
  }
  *out = tp;
  return TOMO_OK;
}

int tomo_plan_layout(tomo_plan *plan, int *instances, size_t *img_off, size_t *sino_off, size_t cap) {
  if (!plan) return fail(TOMO_EINVAL, "layout: NULL plan");
  const Plan &p = plan->p;
  if (p.g.kind != TOMO_KIND_DD) {
    if (instances) *instances = p.g.nz;
    if (img_off || sino_off) {
      if (cap < (size_t)p.g.nz + 1) return fail(TOMO_EINVAL, "layout: arrays need instances + 1 entries");
      for (int z = 0; z <= p.g.nz; ++z) {
        if (img_off) img_off[z] = (size_t)z * p.g.n * p.g.n;
        if (sino_off) sino_off[z] = (size_t)z * p.g.na * p.g.n;
      }
    }
    return TOMO_OK;
  }
  return dd_layout(p, instances, img_off, sino_off, cap);
}

int tomo_plan_tuning(tomo_plan *plan, char *buf, size_t len) {
  if (!plan) return fail(TOMO_EINVAL, "tuning: NULL plan");
  const std::string t = plan->p.g.kind == TOMO_KIND_DD ? dd_tuning(plan->p) : std::string("fixed launch shape");
  if (buf && len) std::snprintf(buf, len, "%s", t.c_str());
  return TOMO_OK;
}

int tomo_plan_set_tuning(tomo_plan *plan, const char *fwd, const char *adj) {
  if (!plan) return fail(TOMO_EINVAL, "set_tuning: NULL plan");
  if (plan->p.g.kind != TOMO_KIND_DD) return fail(TOMO_EINVAL, "set_tuning: only distance-driven plans have shapes");
  return dd_set_tuning(plan->p, fwd, adj);
}

int tomo_plan_destroy(tomo_plan *plan) {
  if (!plan) return TOMO_OK;
  release(plan->p);
  delete plan;
  return TOMO_OK;
}

int tomo_forward(tomo_plan *plan, const float *d_image, float *d_sino, void *stream) {
  if (!plan || !d_image || !d_sino) return fail(TOMO_EINVAL, "tomo_forward: NULL argument");
  return plan_forward(plan->p, d_image, d_sino, (cudaStream_t)stream, FwdEpi());
}

int tomo_adjoint(tomo_plan *plan, const float *d_sino, float *d_image, void *stream) {
  if (!plan || !d_image || !d_sino) return fail(TOMO_EINVAL, "tomo_adjoint: NULL argument");
  return plan_adjoint(plan->p, d_sino, d_image, (cudaStream_t)stream, AdjEpi());
}

static int ensure_host_buffers(Plan &p) {
  if (!p.host_stream) TOMO_CUDA(cudaStreamCreateWithFlags(&p.host_stream, cudaStreamNonBlocking));
  const size_t ib = sizeof(float) * image_elems(p), sb = sizeof(float) * sino_elems(p);
  const size_t mb = ib > sb ? ib : sb;
  if (!p.d_in) {
    TOMO_CUDA(cudaMalloc(&p.d_in, mb));
    p.d_in_bytes = mb;
  }
  if (!p.d_out) {
    TOMO_CUDA(cudaMalloc(&p.d_out, mb));
    p.d_out_bytes = mb;
  }
  if (!p.h_stage) {
    // pinned staging; if the system refuses pinned memory the copies go
    // straight from the caller's (pageable) arrays instead
    if (cudaMallocHost(&p.h_stage, mb) == cudaSuccess) p.h_stage_bytes = mb;
    else {
      cudaGetLastError();
      p.h_stage = nullptr;
    }
  }
  return TOMO_OK;
}

// Host <-> device copies through the pinned staging buffer, in 1 MiB chunks:
// host threads copy chunks between the caller's array and the staging buffer,
// and each chunk's DMA is queued as soon as its host copy is done (and the
// host copy of an output chunk starts as soon as its DMA has landed), so the
// copies and the transfers overlap.  The threads are a pool kept across calls.
constexpr size_t kStageChunk = (size_t)1 << 20;

// A fixed pool of host threads; run(n, f) calls f(0 .. n-1) on the pool and on
// the calling thread and returns when every call has returned.  One run at a
// time; a worker claims tasks only of the run it was woken for.
class StagePool {
 public:
  static StagePool &get() {
    static StagePool pool;
    return pool;
  }

  void run(int n, const std::function<void(int)> &f) {
    std::lock_guard<std::mutex> one(run_mu_);
    unsigned g;
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &f;
      n_ = n;
      next_ = 0;
      done_ = 0;
      g = ++gen_;
    }
    cv_.notify_all();
    work(g);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return done_ == n_; });
    job_ = nullptr;
  }

  ~StagePool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : workers_) t.join();
  }

 private:
  StagePool() {
    const unsigned hc = std::thread::hardware_concurrency();
    const int nw = std::max(0, (int)std::min(8u, std::max(1u, hc / 2)) - 1);
    for (int i = 0; i < nw; ++i)
      workers_.emplace_back([this] {
        unsigned seen = 0;
        for (;;) {
          unsigned g;
          {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            g = seen = gen_;
          }
          work(g);
        }
      });
  }

  void work(unsigned g) {
    for (;;) {
      int t;
      const std::function<void(int)> *f;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (gen_ != g || job_ == nullptr || next_ >= n_) return;
        t = next_++;
        f = job_;
      }
      (*f)(t);
      std::lock_guard<std::mutex> lk(mu_);
      if (++done_ == n_) done_cv_.notify_all();
    }
  }

  std::mutex run_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  std::vector<std::thread> workers_;
  const std::function<void(int)> *job_ = nullptr;
  int n_ = 0, next_ = 0, done_ = 0;
  unsigned gen_ = 0;
  bool stop_ = false;
};

static int stage_in(Plan &p, const void *src, void *dst, size_t bytes) {
  const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
  std::atomic<int> err{0};
  StagePool::get().run((int)nch, [&](int c) {
    const size_t off = (size_t)c * kStageChunk, len = std::min(kStageChunk, bytes - off);
    std::memcpy(p.h_stage + off, (const char *)src + off, len);
    if (cudaMemcpyAsync((char *)dst + off, p.h_stage + off, len, cudaMemcpyHostToDevice, p.host_stream) !=
        cudaSuccess)
      err = 1;
  });
  if (err) return cuda_fail(cudaGetLastError(), "staged host-to-device copy");
  return TOMO_OK;
}

static int stage_out(Plan &p, const void *src, void *dst, size_t bytes) {
  const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
  while (p.stage_events.size() < nch) {
    cudaEvent_t e;
    TOMO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    p.stage_events.push_back(e);
  }
  for (size_t c = 0; c < nch; ++c) {
    const size_t off = c * kStageChunk, len = std::min(kStageChunk, bytes - off);
    TOMO_CUDA(cudaMemcpyAsync(p.h_stage + off, (const char *)src + off, len, cudaMemcpyDeviceToHost,
                              p.host_stream));
    TOMO_CUDA(cudaEventRecord(p.stage_events[c], p.host_stream));
  }
  std::atomic<int> err{0};
  StagePool::get().run((int)nch, [&](int c) {
    const size_t off = (size_t)c * kStageChunk, len = std::min(kStageChunk, bytes - off);
    if (cudaEventSynchronize(p.stage_events[c]) != cudaSuccess) {
      err = 1;
      return;
    }
    std::memcpy((char *)dst + off, p.h_stage + off, len);
  });
  if (err) return cuda_fail(cudaGetLastError(), "staged device-to-host copy");
  return TOMO_OK;
}

// Touches every page of the output array (one byte per 4 KiB, overwritten by
// the result later) on the pool while the projector runs: a freshly allocated
// array would otherwise take its first-touch page faults inside the copies
// out, after the device has finished.
static void prefault_out(void *dst, size_t bytes) {
  constexpr size_t kPage = 4096;
  const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
  volatile char *b = (volatile char *)dst;
  StagePool::get().run((int)nch, [&](int c) {
    const size_t off = (size_t)c * kStageChunk, end = std::min(bytes, off + kStageChunk);
    for (size_t o = off; o < end; o += kPage) b[o] = 0;
  });
}

static int host_call(tomo_plan *plan, const float *h_in, float *h_out, bool forward) {
  if (!plan || !h_in || !h_out) return fail(TOMO_EINVAL, "host call: NULL argument");
  Plan &p = plan->p;
  int rc = ensure_host_buffers(p);
  if (rc) return rc;
  const size_t ib = sizeof(float) * image_elems(p), sb = sizeof(float) * sino_elems(p);
  const size_t in_b = forward ? ib : sb, out_b = forward ? sb : ib;
  if (p.h_stage) rc = stage_in(p, h_in, p.d_in, in_b);
  else TOMO_CUDA(cudaMemcpyAsync(p.d_in, h_in, in_b, cudaMemcpyHostToDevice, p.host_stream));
  if (rc) return rc;
  rc = forward ? tomo_forward(plan, p.d_in, p.d_out, p.host_stream)
               : tomo_adjoint(plan, p.d_in, p.d_out, p.host_stream);
  if (rc) return rc;
  prefault_out(h_out, out_b);
  if (p.h_stage) {
    rc = stage_out(p, p.d_out, h_out, out_b);
    if (rc) return rc;
  } else {
    TOMO_CUDA(cudaMemcpyAsync(h_out, p.d_out, out_b, cudaMemcpyDeviceToHost, p.host_stream));
  }
  TOMO_CUDA(cudaStreamSynchronize(p.host_stream));
  return TOMO_OK;
}

int tomo_forward_host(tomo_plan *plan, const float *h_image, float *h_sino) {
  return host_call(plan, h_image, h_sino, true);
}

int tomo_adjoint_host(tomo_plan *plan, const float *h_sino, float *h_image) {
  return host_call(plan, h_sino, h_image, false);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Drop-in entry points.  A small cache keeps one plan per (kind, n, angles) so
// that repeated calls -- the reference solvers call the same projector every
// iteration -- do not rebuild geometry tables or reallocate buffers.
// ---------------------------------------------------------------------------
namespace {

std::mutex g_dropin_mu;

struct CacheKey {
  int kind, n, na;
  std::vector<float> angles;
  std::vector<float> extra;  // B-spline LUT and support
  bool operator<(const CacheKey &o) const {
    return std::tie(kind, n, na, angles, extra) < std::tie(o.kind, o.n, o.na, o.angles, o.extra);
  }
};

std::map<CacheKey, tomo_plan *> g_cache;

int cached_plan(int kind, int n, const float *angles, int na, tomo_plan **out,
                const float *lut = nullptr, int lut_size = 0, float support = 0.0f) {
  if (!angles || na < 1) return fail(TOMO_EINVAL, "angles missing");
  CacheKey key{kind, n, na, std::vector<float>(angles, angles + na), {}};
  if (lut) {
    key.extra.assign(lut, lut + (size_t)na * lut_size);
    key.extra.push_back(support);
    key.extra.push_back((float)lut_size);
  }
  auto it = g_cache.find(key);
  if (it != g_cache.end()) {
    *out = it->second;
    return TOMO_OK;
  }
  if (g_cache.size() >= 16) {
    for (auto &kv : g_cache) tomo_plan_destroy(kv.second);
    g_cache.clear();
  }
  tomo_geom g{};
  g.kind = kind;
  g.n = n;
  g.na = na;
  g.nz = 1;
  g.angles = angles;
  g.lut = lut;
  g.lut_size = lut_size;
  g.support = support;
  int rc = tomo_plan_create(&g, out);
  if (rc) return rc;
  g_cache[key] = *out;
  return TOMO_OK;
}

// out_host += A in_host (oper 0) or A^T (oper 1), like the reference C.
int dropin_radon(int kind, float *image, int npix, const float *angles, int nang, int oper,
                 float *sino, const float *lut = nullptr, int lut_size = 0, float support = 0.0f) {
  if (!image || !sino) return fail(TOMO_EINVAL, "image/sino pointer is NULL");
  if (oper != 0 && oper != 1) return fail(TOMO_EINVAL, "oper must be 0 (forward) or 1 (adjoint)");
  std::lock_guard<std::mutex> lk(g_dropin_mu);
  tomo_plan *plan = nullptr;
  int rc = cached_plan(kind, npix, angles, nang, &plan, lut, lut_size, support);
  if (rc) return rc;
  const size_t ni = (size_t)npix * npix, ns = (size_t)nang * npix;
  std::vector<float> tmp(oper == 0 ? ns : ni);
  rc = oper == 0 ? tomo_forward_host(plan, image, tmp.data()) : tomo_adjoint_host(plan, sino, tmp.data());
  if (rc) return rc;
  float *dst = oper == 0 ? sino : image;
  for (size_t i = 0; i < tmp.size(); ++i) dst[i] += tmp[i];
  return TOMO_OK;
}

}  // namespace

extern "C" int tomo_radon_dd(float *image, int npix, const float *angles, int nang, int oper,
                             float *sino) {
  return dropin_radon(TOMO_KIND_DD, image, npix, angles, nang, oper, sino);
}

extern "C" int tomo_radon_rd(float *image, int npix, const float *angles, int nang, int oper,
                             float *sino) {
  return dropin_radon(TOMO_KIND_RD, image, npix, angles, nang, oper, sino);
}

extern "C" int tomo_radon_pd(float *image, int npix, const float *angles, int nang, int oper,
                             int method, float *sino) {
  if (method != 1)
    return fail(TOMO_EINVAL, "radon_pd: only method 1 (linear interpolation) is provided; the "
                             "reference's method 0 writes outside the sinogram for edge pixels");
  return dropin_radon(TOMO_KIND_PD, image, npix, angles, nang, oper, sino);
}

extern "C" int tomo_radon_ss(float *image, int npix, const float *angles, int nang, int oper,
                             int method, float *sino) {
  if (method != 1)
    return fail(TOMO_EINVAL, "radon_ss: only method 1 (linear interpolation) is provided");
  return dropin_radon(TOMO_KIND_SS, image, npix, angles, nang, oper, sino);
}

extern "C" int tomo_gen_forwproj(const float *image, int npix, const float *angles, int nang,
                                 const float *lut, int lut_size, float support_bspline,
                                 int num_cores, float *sino) {
  (void)num_cores;
  if (!lut) return fail(TOMO_EINVAL, "gen_forwproj: lut is NULL");
  return dropin_radon(TOMO_KIND_BSPLINE, const_cast<float *>(image), npix, angles, nang, 0, sino,
                      lut, lut_size, support_bspline);
}

extern "C" int tomo_gen_backproj(const float *sino, int npix, const float *angles, int nang,
                                 const float *lut, int lut_size, float support_bspline,
                                 float *image) {
  if (!lut) return fail(TOMO_EINVAL, "gen_backproj: lut is NULL");
  return dropin_radon(TOMO_KIND_BSPLINE, image, npix, angles, nang, 1, const_cast<float *>(sino),
                      lut, lut_size, support_bspline);
}

// gridrec_v4.pyx:7-11 binds gridrec_v4_forwproj / gridrec_v4_backproj.  Unlike
// the Radon kernels these reference functions OVERWRITE their output.
namespace {
int gridrec_call(bool forward, const float *in, float *out, int npix, int nang, const float *angles,
                 const float *param, const float *lut, const float *deapod, int lut_len) {
  if (!in || !out || !angles || !param || !lut || !deapod)
    return fail(TOMO_EINVAL, "gridrec: NULL argument");
  std::lock_guard<std::mutex> lk(g_dropin_mu);
  tomo_geom g{};
  g.kind = TOMO_KIND_GRID;
  g.n = npix;
  g.na = nang;
  g.nz = 1;
  g.angles = angles;
  g.grid_param = param;
  g.grid_lut = lut;
  g.grid_lut_len = lut_len;
  g.grid_deapod = deapod;
  tomo_plan *plan = nullptr;
  int rc = tomo_plan_create(&g, &plan);
  if (rc) return rc;
  rc = forward ? tomo_forward_host(plan, in, out) : tomo_adjoint_host(plan, in, out);
  tomo_plan_destroy(plan);
  return rc;
}
}  // namespace

extern "C" int tomo_gridrec_forwproj(float *S, int npix, int nang, const float *angles,
                                     const float *param, const float *lut, const float *deapod,
                                     const float *I, const char *fftwfn) {
  (void)fftwfn;
  if (!param) return fail(TOMO_EINVAL, "gridrec: param is NULL");
  return gridrec_call(true, I, S, npix, nang, angles, param, lut, deapod, (int)param[5] + 5);
}

extern "C" int tomo_gridrec_backproj(const float *sino, int npix, int nang, const float *angles,
                                     const float *param, const float *lut, const float *deapod,
                                     const float *filter_ext, float *rec, const char *fftwfn) {
  (void)fftwfn;
  (void)filter_ext;  // only read by the reference when param[2] != 0, which is rejected
  if (!param) return fail(TOMO_EINVAL, "gridrec: param is NULL");
  return gridrec_call(false, sino, rec, npix, nang, angles, param, lut, deapod, (int)param[5] + 5);
}
