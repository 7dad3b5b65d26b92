"""Sinogram pre-processing on the GPU (reference: common/myimage/my_image_process.py).

``sino_correct_rot_axis(sino, ctr)`` and ``sino_edge_padding(sino, padding)``
keep the reference's names, arguments and output shapes
(my_image_process.py:87-117 and :142-157) and run as CUDA kernels of
``libtomo_b200.so`` (``csrc/sino_prep.cu``).  They take a numpy array (copied
to the device and back) or a CUDA float32 tensor (result on the same device).

Differences: a fractional rotation-axis shift is interpolated per row with the
Keys cubic-convolution kernel, where the reference evaluates scipy's 2-D
Clough-Tocher interpolant of the whole sinogram (``griddata(method='cubic')``);
integer shifts and the edge padding are exactly the reference's.  The reference's
fractional result is itself defined only up to the order of its input points
(the Delaunay triangulation of the regular grid, and the gradients fitted over
it, follow that order): listing the same points in another order moves it by
~1e-3 of the signal on smooth data, more than the kernel's distance to it.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_lib.lib.tomo_sino_edge_pad.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p]
_lib.lib.tomo_sino_center.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_void_p, ctypes.c_void_p]


def _on_device(x):
    import torch
    if isinstance(x, torch.Tensor):
        if not (x.is_cuda and x.dtype == torch.float32):
            raise TypeError("expected a CUDA float32 tensor or a numpy array")
        return x.contiguous(), False
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda(), True


def sino_correct_rot_axis(sino, ctr):
    """Shift each projection so that the rotation axis ``ctr`` sits at npix/2."""
    import torch
    s, was_np = _on_device(sino)
    nang, npix = s.shape
    out = torch.empty_like(s)
    stream = torch.cuda.current_stream(s.device).cuda_stream
    _lib.check(_lib.lib.tomo_sino_center(s.data_ptr(), nang, npix, float(ctr), out.data_ptr(), stream),
               "tomo_sino_center")
    return out.cpu().numpy() if was_np else out


def sino_edge_padding(sino, padding, verbose: bool = True):
    """Pad ``int(padding * npix)`` copies of the first / last detector column on each side."""
    import torch
    s, was_np = _on_device(sino)
    nang, npix = s.shape
    npad = int(padding * npix)
    if verbose:
        print("Padded pixels on one side = ", npad)
    out = torch.empty((nang, npix + 2 * npad), dtype=torch.float32, device=s.device)
    stream = torch.cuda.current_stream(s.device).cuda_stream
    _lib.check(_lib.lib.tomo_sino_edge_pad(s.data_ptr(), nang, npix, npad, out.data_ptr(), stream),
               "tomo_sino_edge_pad")
    return out.cpu().numpy() if was_np else out
