"""Drop-in replacement for the reference's ``algorithms/class_projectors_bspline.py``.

Same constructor, attributes and methods (class_projectors_bspline.py:41-108):

    tp = projectors(npix, angles, param, ctr=0.0, bspline_degree=3,
                    proj_support_y=4, nsamples_y=2048, radon_degree=1)
    tp.A(x), tp.At(b), tp.fbp(b)

As in the reference, the angles passed in are only counted: the projector uses
``arange(nang) * 180 / nang`` degrees (:48-50), and the look-up tables are
built from those degree values (bspline_functions.init_lut_bspline).  ``A``
and ``At`` use the table of Radon degree ``radon_degree``; ``fbp`` filters the
detector-reversed sinogram (ramp, or its Hilbert counterpart when
radon_degree != 0), backprojects it with the degree-0 table and normalises
(:83-108).  The projector kernels run on the GPU (libtomo_b200.so); inputs may
be numpy arrays or CUDA float32 torch tensors, with an optional leading slice
axis.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .bspline_functions import init_lut_bspline
from .filters import filter_proj, filter_proj_device

myfloat = np.float32


class projectors:
    """B-spline (generalised Radon) projector pair."""

    def __init__(self, npix, angles, param=None, ctr=0.0, bspline_degree=3, proj_support_y=4,
                 nsamples_y=2048, radon_degree=1):
        nang = len(angles)
        angles = np.arange(nang)
        angles = (angles * 180.0) / myfloat(nang)
        lut = init_lut_bspline(nsamples_y, angles, bspline_degree, radon_degree, proj_support_y)
        lut0 = init_lut_bspline(nsamples_y, angles, bspline_degree, 0, proj_support_y)
        self.nang = nang
        self.filt = "ramp"
        self.plot = True
        self.radon_degree = radon_degree
        self.lut = lut.astype(myfloat)
        self.lut0 = lut0.astype(myfloat)
        self.angles = angles.astype(myfloat)
        self.param_spline = np.array([lut.shape[1], proj_support_y], dtype=myfloat)
        self.npix = int(npix)
        self._plans = {}

    def _plan(self, nz: int, device, which: str):
        key = (nz, device, which)
        p = self._plans.get(key)
        if p is None:
            lut = self.lut if which == "lut" else self.lut0
            kw = dict(lut=lut, lut_size=int(self.param_spline[0]),
                      support=float(myfloat(self.param_spline[1])))
            if device is not None:
                import torch
                with torch.cuda.device(device):
                    p = _lib.Plan(_lib.KIND_BSPLINE, self.npix, self.angles, nz=nz, **kw)
            else:
                p = _lib.Plan(_lib.KIND_BSPLINE, self.npix, self.angles, nz=nz, **kw)
            self._plans[key] = p
        return p

    def plan(self, nz: int = 1, device=None):
        """The libtomo_b200 plan (table of Radon degree ``radon_degree``) for ``nz`` slices."""
        return self._plan(nz, device, "lut")

    def _apply(self, x, forward: bool, which: str = "lut"):
        if isinstance(x, np.ndarray) or not hasattr(x, "is_cuda"):
            x = np.ascontiguousarray(x, dtype=myfloat)  # no copy when already float32 (inputs are never modified)
            device = None
        else:
            device = x.device.index
        squeeze = x.ndim == 2
        nz = 1 if squeeze else int(x.shape[0])
        plan = self._plan(nz, device, which)
        y = plan.forward(x) if forward else plan.adjoint(x)
        return y[0] if squeeze else y

    def A(self, x):
        """Forward projection (class_projectors_bspline.py:71-72, gen_forwproj.c)."""
        return self._apply(x, True)

    def At(self, x):
        """Backprojection (class_projectors_bspline.py:77-78, gen_backproj.c)."""
        return self._apply(x, False)

    def fbp(self, x):
        """Filtered backprojection (class_projectors_bspline.py:83-108).

        numpy input follows the reference step by step (host filtering);
        a CUDA tensor [na, n] or [nz, na, n] is filtered on the device
        (filters.filter_proj_device) and stays there."""
        dpc = self.radon_degree != 0
        scale = np.pi / (1.0 * self.nang) if dpc else np.pi / (2.0 * self.nang)
        if hasattr(x, "is_cuda") and x.is_cuda:
            import torch
            x0 = filter_proj_device(torch.flip(x, dims=[-1]), ftype=self.filt, dpc=dpc)
            reco = self._apply(x0, False, which="lut0") * scale
            return torch.flip(reco, dims=[-2, -1]).contiguous()
        x0 = np.asarray(x)[:, ::-1].copy()
        x0[:] = filter_proj(x0, ftype=self.filt, dpc=dpc)
        reco = self._apply(x0.astype(myfloat), False, which="lut0")
        reco = reco * scale
        reco[:] = reco[::-1, ::-1]
        return reco
