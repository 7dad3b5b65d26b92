// Distance-driven forward projection that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code whose device memory is owned by
// another allocator (a framework's caching allocator or a fixed arena sized
// at start-up), or code that must not allocate -- and so implicitly
// synchronise the device -- inside a latency-bound loop.  For them this file
// provides tomo_radon_dd_forward_noalloc: the caller passes the image and the
// sinogram; the scratch the forward needs (a transposed copy of the image and
// the per-angle geometry table) lives in the file-scope __device__ arrays
// below, which every GPU that loads this library holds until the process
// exits (16 MiB + 256 KiB).
//
// Limits: nz * npix * npix <= 4,194,304 (e.g. one 2048 x 2048 slice) and
// nang <= 16384; larger requests fail with TOMO_EINVAL.
//
// Set-up: the first call on a device, with that device current, looks up the
// device addresses of the arrays (cudaGetSymbolAddress).  Make that first call
// before any stream capture.
//
// Sharing: every call on a device uses the same arrays, which keep the last
// call's contents.  Both are fully rewritten by each call before they are read
// (the transpose covers all nz*npix*npix scratch words used, the table all
// nang entries), so nothing needs clearing.  Calls whose work overlaps on the
// GPU (different streams, or different host threads without ordering) race on
// the arrays: serialise them.
#include <cmath>
#include <mutex>
#include <string>

#include "tomo_internal.cuh"

namespace tomo {
namespace {

constexpr size_t kNoAllocScratchFloats = (size_t)4 << 20;  // 16 MiB
constexpr int kNoAllocMaxAngles = 16384;                   // 256 KiB
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];
static __device__ __align__(256) DdAngle g_noalloc_angles[kNoAllocMaxAngles];

std::mutex g_noalloc_mu;
float *g_scratch_addr[kNoAllocMaxDevices];
DdAngle *g_angles_addr[kNoAllocMaxDevices];
DdAngle g_host_table[kNoAllocMaxAngles];  // staging for the table upload (under the mutex)

}  // namespace
}  // namespace tomo

using namespace tomo;

extern "C" int tomo_radon_dd_forward_noalloc(const float *d_image, int npix, const float *angles,
                                             int nang, int nz, float *d_sino, void *stream) {
  if (!d_image || !d_sino || !angles)
    return fail(TOMO_EINVAL, "dd noalloc: NULL image, sinogram or angles");
  if (npix < 2 || npix > 32767)
    return fail(TOMO_EINVAL, "dd noalloc: npix must be in [2, 32767], got " + std::to_string(npix));
  if (nang < 1 || nang > kNoAllocMaxAngles)
    return fail(TOMO_EINVAL, "dd noalloc: nang must be in [1, " + std::to_string(kNoAllocMaxAngles) +
                                 "], got " + std::to_string(nang));
  if (nz < 1 || nz > 65535) return fail(TOMO_EINVAL, "dd noalloc: nz must be in [1, 65535]");
  const size_t need = (size_t)nz * npix * npix;
  if (need > kNoAllocScratchFloats)
    return fail(TOMO_EINVAL, "dd noalloc: nz*npix*npix = " + std::to_string(need) +
                                 " exceeds the static scratch of " +
                                 std::to_string(kNoAllocScratchFloats) + " floats");
  for (int v = 0; v < nang; ++v)
    if (!std::isfinite(angles[v])) return fail(TOMO_EINVAL, "dd noalloc: angle is not finite");
  int dev = 0;
  TOMO_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(TOMO_EINVAL, "dd noalloc: device ordinal too large");
  cudaStream_t s = (cudaStream_t)stream;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_scratch_addr[dev]) {
    void *a = nullptr, *b = nullptr;
    TOMO_CUDA(cudaGetSymbolAddress(&a, g_noalloc_scratch));
    TOMO_CUDA(cudaGetSymbolAddress(&b, g_noalloc_angles));
    g_scratch_addr[dev] = (float *)a;
    g_angles_addr[dev] = (DdAngle *)b;
  }
  int rc = dd_build_table(angles, nang, g_host_table);
  if (rc) return rc;
  // From pageable host memory this returns once the table is staged, so the
  // host array may be rewritten by the next call.
  TOMO_CUDA(cudaMemcpyAsync(g_angles_addr[dev], g_host_table, sizeof(DdAngle) * (size_t)nang,
                            cudaMemcpyHostToDevice, s));
  return dd_forward_launch(d_image, g_scratch_addr[dev], d_sino, g_angles_addr[dev], npix, nang, nz, s);
}
