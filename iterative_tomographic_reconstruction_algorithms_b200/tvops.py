"""ADMM-TV / CG inner operators on the GPU (reference: algorithms/cg.py:62-71,
algorithms/utils.py:189-216).

``G(m)``      numpy.gradient of a 2-D image: [d/d axis 0, d/d axis 1], float32.
``Gt(g)``     the reference's adjoint, g[1] . Gx + Gy . g[0] with the gradient
              matrices of identities; the reference multiplies dense n x n
              matrices, here a stencil gives the same float64 numbers.
``hard_thres(x, beta)``, ``soft_thres(x, beta)``  the reference's shrinkage rules.

Inputs are numpy arrays (copied to the device and back, numpy out) or CUDA
tensors (results on the device).  ``G``/``Gt`` run as kernels of
``libtomo_b200.so`` (``csrc/tv_ops.cu``).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_lib.lib.tomo_grad2d.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_void_p]
_lib.lib.tomo_grad2d_adjoint.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p]


def _dev(x):
    import torch
    if isinstance(x, torch.Tensor):
        return x.to(torch.float32).contiguous(), False
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda(), True


def G(m):
    """numpy.gradient(m) of a 2-D float32 image: [gradient along axis 0, along axis 1]."""
    import torch
    md, was_np = _dev(m)
    n0, n1 = md.shape
    g0, g1 = torch.empty_like(md), torch.empty_like(md)
    stream = torch.cuda.current_stream(md.device).cuda_stream
    _lib.check(_lib.lib.tomo_grad2d(md.data_ptr(), n0, n1, g0.data_ptr(), g1.data_ptr(), stream), "tomo_grad2d")
    return [g0.cpu().numpy(), g1.cpu().numpy()] if was_np else [g0, g1]


def Gt(g):
    """The reference's Gt: g[1] . Gx + Gy . g[0] (float64 result)."""
    import torch
    g0, was_np = _dev(g[0])
    g1, _ = _dev(g[1])
    n0, n1 = g0.shape
    out = torch.empty((n0, n1), dtype=torch.float64, device=g0.device)
    stream = torch.cuda.current_stream(g0.device).cuda_stream
    _lib.check(_lib.lib.tomo_grad2d_adjoint(g0.data_ptr(), g1.data_ptr(), n0, n1, out.data_ptr(), stream),
               "tomo_grad2d_adjoint")
    return out.cpu().numpy() if was_np else out


def hard_thres(x, beta):
    """max(0, x - beta) - max(0, -x - beta) (utils.py:214-216)."""
    import torch
    if isinstance(x, torch.Tensor):
        return torch.clamp(x - beta, min=0) - torch.clamp(-x - beta, min=0)
    return np.maximum(0, x - beta) - np.maximum(0, -x - beta)


def soft_thres(x, beta):
    """x - beta where x > beta, 0 where |x| <= beta, x + beta where x < -beta (utils.py:189-203)."""
    if beta <= 0:
        raise ValueError("beta in soft thresholding has to be > 0")
    import torch
    lib = torch if isinstance(x, torch.Tensor) else np
    return lib.where(x > beta, x - beta, lib.where(x < -beta, x + beta, lib.zeros_like(x)))
