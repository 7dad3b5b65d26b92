// Sinogram pre-processing on the device: edge padding and rotation-axis
// centring (reference: common/myimage/my_image_process.py:87-157).
//
// Edge padding (sino_edge_padding, :142-157): npad copies of the first
// detector column on the left and of the last on the right, per angle row.
//
// Rotation-axis centring (sino_correct_rot_axis, :87-117), shift =
// ctr - npix/2:
//   * integer shift: the row rolled left by shift, the wrapped-around
//     columns replaced by copies of the edge column the roll moved away from
//     (last column for shift > 0, first for shift < 0) -- exactly the
//     reference's arithmetic;
//   * fractional shift: out[v][j] = row_v interpolated at j + shift, the row
//     extended by zeros (the reference pads 100 zeros on each side).  The
//     reference evaluates scipy's 2-D Clough-Tocher interpolant
//     (griddata(method='cubic')) of the whole sinogram; here each row is
//     interpolated with the Keys cubic-convolution kernel (a = -1/2; R. Keys,
//     IEEE Trans. ASSP 29(6), 1981), which reproduces quadratics exactly.
//     The two interpolants agree to about 1e-3 of the signal on smooth data;
//     this is not a bit-exact restatement, nor can one be: the reference's
//     own result moves by as much when only the order of its input points
//     changes (Qhull's triangulation of the regular grid picks one of two
//     equally valid diagonals per cell, following that order).
// One thread per output element, coalesced along the detector axis.
#include <cmath>

#include "tomo_internal.cuh"

namespace tomo {
namespace {

__global__ void edge_pad_kernel(const float *__restrict__ in, int nang, int npix, int npad,
                                float *__restrict__ out) {
  const int w = npix + 2 * npad;
  const long long total = (long long)nang * w;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(i / w), c = (int)(i - (long long)v * w) - npad;
    const int src = c < 0 ? 0 : (c >= npix ? npix - 1 : c);
    out[i] = in[(long long)v * npix + src];
  }
}

__global__ void shift_int_kernel(const float *__restrict__ in, int nang, int npix, int shift,
                                 float *__restrict__ out) {
  const long long total = (long long)nang * npix;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(i / npix), j = (int)(i - (long long)v * npix);
    const float *row = in + (long long)v * npix;
    float o;
    if (shift >= 0) o = j < npix - shift ? row[j + shift] : row[npix - 1];
    else o = j >= -shift ? row[j + shift] : row[0];
    out[i] = o;
  }
}

__device__ __forceinline__ float keys(float t) {  // a = -1/2
  t = fabsf(t);
  if (t <= 1.0f) return (1.5f * t - 2.5f) * t * t + 1.0f;
  if (t < 2.0f) return ((-0.5f * t + 2.5f) * t - 4.0f) * t + 2.0f;
  return 0.0f;
}

__global__ void shift_cubic_kernel(const float *__restrict__ in, int nang, int npix, double shift,
                                   float *__restrict__ out) {
  const long long total = (long long)nang * npix;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(i / npix), j = (int)(i - (long long)v * npix);
    const float *row = in + (long long)v * npix;
    const double x = (double)j + shift;
    const int x0 = (int)floor(x);
    const float fr = (float)(x - (double)x0);
    float acc = 0.0f;
#pragma unroll
    for (int k = -1; k <= 2; ++k) {
      const int c = x0 + k;
      const float val = (c >= 0 && c < npix) ? row[c] : 0.0f;  // zero extension
      acc = fmaf(keys(fr - (float)k), val, acc);
    }
    out[i] = acc;
  }
}

int grid_for(long long total) {
  const long long b = (total + 255) / 256;
  return (int)(b < 148 * 32 ? (b < 1 ? 1 : b) : 148 * 32);
}

}  // namespace
}  // namespace tomo

using namespace tomo;

extern "C" {

int tomo_sino_edge_pad(const float *d_sino, int nang, int npix, int npad, float *d_out, void *stream) {
  if (!d_sino || !d_out || nang < 1 || npix < 1 || npad < 0)
    return fail(TOMO_EINVAL, "sino edge padding: bad arguments");
  const long long total = (long long)nang * (npix + 2LL * npad);
  edge_pad_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(d_sino, nang, npix, npad, d_out);
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

int tomo_sino_center(const float *d_sino, int nang, int npix, double ctr, float *d_out, void *stream) {
  if (!d_sino || !d_out || nang < 1 || npix < 1 || !std::isfinite(ctr))
    return fail(TOMO_EINVAL, "sino centring: bad arguments");
  if (d_sino == d_out) return fail(TOMO_EINVAL, "sino centring: output must not alias the input");
  const double shift = ctr - npix * 0.5;
  const long long total = (long long)nang * npix;
  if (shift == std::floor(shift)) {
    const double lim = (double)npix;
    if (std::fabs(shift) >= lim) return fail(TOMO_EINVAL, "sino centring: |shift| must be below npix");
    shift_int_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(d_sino, nang, npix, (int)shift, d_out);
  } else {
    shift_cubic_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(d_sino, nang, npix, shift, d_out);
  }
  TOMO_CUDA(cudaGetLastError());
  return TOMO_OK;
}

}  // extern "C"
