"""Device-resident SIRT, MLEM and SPS with the update fused into the projectors.

The arithmetic is the reference's (algorithms/art.py:211-237 for SIRT,
algorithms/sir.py:204-290 for MLEM, :348-540 for SPS without penalty), in the
same float32 rounding order; the loop runs on the GPU: one forward and one
adjoint launch per iteration, both with their solver arithmetic applied where
they store their result (csrc/epilogue.cuh), captured once into a CUDA graph.

    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.solvers import sirt
    tp = cpr.projectors(n, angles_deg, oper="rd")
    x, info = sirt(np.ones((n, n), np.float32), b, tp, n_iter=100)

``info`` holds ||A x_k - b||^2 for the iterate entering iteration k.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

ALGOS = {"sirt": 1, "em": 2, "mlem": 2, "sps": 3}

_lib.lib.tomo_solver_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
_lib.lib.tomo_solver_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_void_p]
_lib.lib.tomo_solver_destroy.argtypes = [ctypes.c_void_p]


def _as_device(a, torch, device):
    if isinstance(a, np.ndarray) or not hasattr(a, "is_cuda"):
        return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device), True
    return a.to(device=device, dtype=torch.float32).contiguous(), False


class Solver:
    """One solver (``algo`` in sirt / em / sps) bound to a projector and a sinogram."""

    def __init__(self, tp, algo: str, b, device=None):
        import torch
        self.torch = torch
        if algo not in ALGOS:
            raise ValueError(f"algo must be one of {sorted(ALGOS)}")
        self.algo = algo
        device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = device
        bd, _ = _as_device(b, torch, device)
        if isinstance(tp, _lib.Plan):  # a plan (e.g. a batched plan over packed arrays)
            self.plan = tp
            self.b = bd.reshape(tp.sino_shape).contiguous()
            self.nz = 0
        else:
            if bd.dim() == 2:
                bd = bd[None]
            self.b = bd.contiguous()
            self.nz = int(self.b.shape[0])
            self.plan = tp.plan(self.nz, device.index)
        h = ctypes.c_void_p()
        stream = torch.cuda.current_stream(device).cuda_stream
        _lib.check(_lib.lib.tomo_solver_create(self.plan._h, ALGOS[algo], self.b.data_ptr(), stream,
                                               ctypes.byref(h)), "tomo_solver_create")
        self._h = h

    def run(self, x, iters: int, use_graph: bool = True):
        """Run ``iters`` iterations from ``x`` (numpy or CUDA tensor); returns (x, residuals)."""
        torch = self.torch
        xd, was_np = _as_device(x, torch, self.device)
        in_shape = tuple(xd.shape)
        squeeze = self.nz > 0 and xd.dim() == 2
        xd = (xd[None] if squeeze else xd).clone()
        if self.nz == 0:
            xd = xd.reshape(self.plan.image_shape)
        res = (ctypes.c_double * max(iters, 1))()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(_lib.lib.tomo_solver_run(self._h, xd.data_ptr(), int(iters), res, int(use_graph), stream),
                   "tomo_solver_run")
        out = xd[0] if squeeze else xd
        if self.nz == 0:
            out = out.reshape(in_shape)
        if was_np:
            out = out.cpu().numpy()
        return out, np.array(res[:iters])

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib.tomo_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sirt(x, b, tp, n_iter: int = 200, use_graph: bool = True):
    """SIRT (art.py:211-365 without constraints): returns (x, residuals)."""
    return Solver(tp, "sirt", b).run(x, n_iter, use_graph)


def em(x, b, tp, n_iter: int = 100, use_graph: bool = True):
    """MLEM (sir.py:204-324): returns (x, residuals)."""
    return Solver(tp, "em", b).run(x, n_iter, use_graph)


def sps(x, b, tp, n_iter: int = 100, use_graph: bool = True):
    """SPS without penalty (sir.py:348-600): returns (x, residuals)."""
    return Solver(tp, "sps", b).run(x, n_iter, use_graph)
