"""ADMM (Lasso-L1, Lasso-TV) and conjugate-gradient reconstruction on the GPU.

Drop-in counterparts of the reference's solver functions
(algorithms/admm.py), with the same arguments and return values:

    conj_grad(x, b, tp, param)  -> (x, info)   admm.py:245-288 (cg.py:83-185)
    lasso_l1(x, b, tp, param)   -> (x, info)   admm.py:291-457 (cg.py:189-253)
    lasso_tv(x, b, tp, param)   -> (x, info)   admm.py:470-640 (cg.py:256-320)

``tp`` is any projector class of this package (``class_projectors_radon``,
``_grid`` or ``_bspline``); ``x`` [nz, n, n] and ``b`` [nz, na, n] are numpy
arrays (``x`` is updated in place and returned, as in the reference) or CUDA
float32 tensors.  ``param`` carries the reference's ``class_admm_param``
attributes that these functions read: lambd1, lambd2, mu, n_iter,
n_iter_pcg, eps, pc, edge_padding, index_start, index_end (``Param`` below
has them with the reference's command-line defaults).  ``info`` holds one
[err, diff, obj] per iteration as the reference computes it: err the norm of
the multiplier update (CG: of the residual), diff |x - x_old| (slice 0 for
Lasso-TV, relative for Lasso-L1, 0 for CG, whose reference value is always 0),
obj the objective of slice 0 (one extra forward projection per iteration;
``track=False`` skips it and reports obj = nan).

Every iteration runs on the device (csrc/admm.cu through libtomo_b200.so):
the CG steps with their float32 / float64 arithmetic, Gt(G(.)) as a stencil,
the shrinkage, the constraint and the multiplier update, one CUDA graph per
iteration.  The reference's masks (-mask, -mask_add) and plotting/check-point
output are not provided.  ``conj_grad`` reconstructs slice 0 only, as the
reference does (admm.py:276); ``AdmmSolver`` runs any number of slices.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

myfloat = np.float32
REGS = {"cg": 1, "lasso": 2, "lasso-tv": 3}


class _Params(ctypes.Structure):
    _fields_ = [("lambd1", ctypes.c_float), ("lambd2", ctypes.c_float), ("mu", ctypes.c_float),
                ("n_iter_pcg", ctypes.c_int), ("pc", ctypes.c_float), ("i1", ctypes.c_int), ("i2", ctypes.c_int)]


_lib.lib.tomo_admm_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(_Params),
                                      ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
_lib.lib.tomo_admm_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_void_p]
_lib.lib.tomo_admm_destroy.argtypes = [ctypes.c_void_p]


@dataclass
class Param:
    """The attributes of the reference's class_admm_param that the solvers read."""
    lambd1: float = 0.0
    lambd2: float = 0.0
    mu: float = 1.0
    n_iter: int | None = None      # -n1 (None: 200 for the ADMM solvers)
    n_iter_pcg: int = 4            # -n2
    eps: float | None = None       # None: 1e-10
    pc: float = -1.0               # -pc
    edge_padding: float = 0.0
    index_start: int = 0
    index_end: int = 0
    mask: object = None
    mask_add: object = None


class AdmmSolver:
    """One ADMM / CG solver (``reg`` in cg / lasso / lasso-tv) bound to a
    projector and a sinogram [nz, na, n] (numpy or CUDA tensor)."""

    def __init__(self, tp, reg: str, b, lambd1=0.0, lambd2=0.0, mu=1.0, n_iter_pcg: int = 4, pc: float = -1.0,
                 region=None, device=None):
        import torch
        if reg not in REGS:
            raise ValueError(f"reg must be one of {sorted(REGS)}")
        self.torch = torch
        self.reg = reg
        device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = device
        if hasattr(b, "is_cuda"):
            bd = b.to(device=device, dtype=torch.float32)
        else:
            bd = torch.from_numpy(np.ascontiguousarray(b, myfloat)).to(device)
        if bd.dim() == 2:
            bd = bd[None]
        self.b = bd.contiguous()
        self.nz = int(self.b.shape[0])
        self.tp = tp
        self.plan = tp.plan(self.nz, device.index)
        n = self.plan.image_shape[-1]
        i1, i2 = (0, n) if region is None else (int(region[0]), int(region[1]))
        self.prm = _Params(myfloat(lambd1), myfloat(lambd2), myfloat(mu), int(n_iter_pcg), myfloat(pc), i1, i2)
        h = ctypes.c_void_p()
        stream = torch.cuda.current_stream(device).cuda_stream
        _lib.check(_lib.lib.tomo_admm_create(self.plan._h, REGS[reg], self.b.data_ptr(), ctypes.byref(self.prm),
                                             stream, ctypes.byref(h)), "tomo_admm_create")
        self._h = h

    def run(self, x, iters: int, reset: bool = True, use_graph: bool = True):
        """``iters`` iterations in place on the CUDA float32 tensor ``x`` [nz, n, n];
        returns the statistics [iters, nz, 3] (tomo_admm_run)."""
        torch = self.torch
        if not (hasattr(x, "is_cuda") and x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()):
            raise ValueError("x must be a contiguous CUDA float32 tensor")
        stats = np.zeros((max(iters, 1), self.nz, 3), np.float64)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(_lib.lib.tomo_admm_run(self._h, x.data_ptr(), int(iters), int(bool(reset)),
                                          stats.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(use_graph),
                                          stream), "tomo_admm_run")
        return stats[:iters]

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib.tomo_admm_destroy(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _objective(tp, x0, b0, lambd1, lambd2, tv: bool) -> float:
    """0.5 |A x0 - b0|^2 + 0.5 lambd1 |x0| + lambd2 |T|_1 (admm.py:400-405, 599-604), with
    T = sqrt(G(x0)_0^2 + G(x0)_1^2) (TV) or x0 (L1) and |.|_1 numpy's matrix 1-norm."""
    import torch
    from . import tvops
    r = (tp.A(x0) - b0).double()
    obj_1 = float((r * r).sum())
    obj_2 = float(x0.double().norm())
    if tv:
        g0, g1 = tvops.G(x0)
        t = torch.sqrt(g0 * g0 + g1 * g1)
    else:
        t = x0
    obj_3 = float(t.double().abs().sum(dim=0).max())
    return 0.5 * obj_1 + 0.5 * float(myfloat(lambd1)) * obj_2 + float(myfloat(lambd2)) * obj_3


def _region(param, n):
    if getattr(param, "edge_padding", 0.0) != 0.0:
        return int(param.index_start), int(param.index_end)
    return 0, n


def _run(reg: str, x, b, tp, param, track: bool):
    import torch
    if getattr(param, "mask", None) is not None or getattr(param, "mask_add", None) is not None:
        raise NotImplementedError("masks (-mask / -mask_add) are not provided on the device")
    was_np = not hasattr(x, "is_cuda")
    device = torch.device("cuda", torch.cuda.current_device())
    xd = torch.from_numpy(np.ascontiguousarray(x, myfloat)).to(device) if was_np else x
    squeeze = xd.dim() == 2
    if squeeze:
        xd = xd[None]
    work = xd if (xd.is_contiguous() and xd.dtype == torch.float32) else xd.to(torch.float32).contiguous()
    bd = b if hasattr(b, "is_cuda") else torch.from_numpy(np.ascontiguousarray(b, myfloat)).to(device)
    if bd.dim() == 2:
        bd = bd[None]
    n = int(work.shape[-1])
    eps = 1e-10 if getattr(param, "eps", None) is None else float(param.eps)
    n1 = 200 if getattr(param, "n_iter", None) is None else int(param.n_iter)
    if reg == "cg":
        # the reference reconstructs slice 0 only (admm.py:276)
        target, bt = work[:1], bd[:1].contiguous()
        solver = AdmmSolver(tp, "cg", bt, device=device)
    else:
        target, bt = work, bd.contiguous()
        solver = AdmmSolver(tp, reg, bt, param.lambd1, param.lambd2, param.mu, int(param.n_iter_pcg),
                            float(getattr(param, "pc", -1.0)), _region(param, n), device=device)
    info = []
    it, err = 0, 1e20
    while it < n1 and (reg == "cg" or err > eps):
        st = solver.run(target, 1, reset=(it == 0))[0]
        if reg == "cg":
            err = float(np.sqrt(st[0, 0]))
            diff = 0.0
        elif reg == "lasso-tv":
            err = float(np.sqrt(st[:, 0].sum()))
            diff = float(np.sqrt(st[0, 1]))
        else:
            err = float(np.sqrt(st[:, 0].sum()))
            diff = float(np.sqrt(st[:, 1].sum()) / np.sqrt(st[:, 2].sum()))
        if not track:
            obj = float("nan")
        elif reg == "cg":  # cg.py:176-178: [err, diff, |A x - b|^2]
            obj = float(((tp.A(target[0]) - bt[0]).double() ** 2).sum())
        else:
            obj = _objective(tp, target[0], bt[0], param.lambd1, param.lambd2, reg == "lasso-tv")
        info.append([err, diff, obj])
        it += 1
        if reg == "cg" and err < 1e-12:
            break
    if work is not xd:
        xd.copy_(work)
    out = xd[0] if squeeze else xd
    if was_np:
        np.copyto(x, out.cpu().numpy().astype(x.dtype, copy=False))
        return x, info
    return out, info


def conj_grad(x, b, tp, param, track: bool = True):
    """Plain CG on A^T A x = A^T b for slice 0 (admm.py:245-288, cg.py:83-185)."""
    return _run("cg", x, b, tp, param, track)


def lasso_l1(x, b, tp, param, track: bool = True):
    """ADMM Lasso-L1 (admm.py:291-457)."""
    return _run("lasso", x, b, tp, param, track)


def lasso_tv(x, b, tp, param, track: bool = True):
    """ADMM Lasso-TV (admm.py:470-640)."""
    return _run("lasso-tv", x, b, tp, param, track)
