"""Drop-in replacement for the reference's ``algorithms/class_projectors_radon.py``.

Same constructor, attributes and methods (class_projectors_radon.py:44-110):

    tp = projectors(npix, angles_deg, oper='pd'|'rd'|'dd'|'ss', ctr=0.0)
    tp.A(x)   # [npix, npix] image  -> [nang, npix] sinogram
    tp.At(b)  # [nang, npix] sinogram -> [npix, npix] image
    tp.nang, tp.angles (float32 radians), tp.filt, tp.plot, tp.oper

Each call runs the hand-written sm_100a kernels of libtomo_b200.so.  Inputs may
be numpy arrays (returned as numpy, like the reference) or CUDA float32 torch
tensors (returned on the same device, no host copies).  A leading slice axis
``[nz, ...]`` is accepted and runs all slices in one launch.

The angle array handed to the kernels is the one the reference's Cython shim
hands to its C function (radon_pixel_driven.pyx:89-92,
radon_ray_driven.pyx:25-26, radon_distance_driven.pyx:25-27,
radon_slant_stacking.pyx:25-28): degrees -> float32 radians here, a further
rescale if the maximum exceeds 2*pi, and an fftshift for pd and dd.
"""
from __future__ import annotations

import numpy as np

from . import _lib

myfloat = np.float32

_KIND = {"pd": _lib.KIND_PD, "rd": _lib.KIND_RD, "dd": _lib.KIND_DD, "ss": _lib.KIND_SS}
# (apply fftshift, rescale factor used when max(angles) > 2*pi) per shim
_SHIM = {"pd": (True, 2 * np.pi / 180.0), "rd": (False, np.pi / 180.0),
         "dd": (True, np.pi / 180.0), "ss": (False, 2 * np.pi / 180.0)}


def shim_angles(oper: str, angles_rad_f32: np.ndarray) -> np.ndarray:
    """The angle array the reference C function receives for projector ``oper``."""
    shift, factor = _SHIM[oper]
    a = np.array(angles_rad_f32, dtype=np.float32, copy=True)
    if np.max(a) > 2 * np.pi:
        a *= factor
    if shift:
        a = np.fft.fftshift(a)
    return np.ascontiguousarray(a, dtype=np.float32)


class projectors:
    """Radon projector pair (pixel-, ray-, distance-driven or slant-stacking)."""

    def __init__(self, npix, angles, oper="pd", ctr=0.0):
        if oper not in _KIND:
            raise ValueError(f"oper must be one of {sorted(_KIND)}, got {oper!r}")
        nang = len(angles)
        angles1 = np.asarray(angles) * np.pi / 180.0
        self.nang = nang
        self.filt = "ramp"
        self.plot = True
        self.angles = angles1.astype(myfloat)
        self.oper = oper
        self.npix = int(npix)
        self._angles_c = shim_angles(oper, self.angles)
        self._plans = {}

    # ---- plan cache: one per (slice count, device) ----
    def _plan(self, nz: int, device):
        key = (nz, device)
        p = self._plans.get(key)
        if p is None:
            if device is not None:
                import torch
                with torch.cuda.device(device):
                    p = _lib.Plan(_KIND[self.oper], self.npix, self._angles_c, nz=nz)
            else:
                p = _lib.Plan(_KIND[self.oper], self.npix, self._angles_c, nz=nz)
            self._plans[key] = p
        return p

    def plan(self, nz: int = 1, device=None):
        """The libtomo_b200 plan for ``nz`` slices on CUDA device ``device`` (None: host calls)."""
        return self._plan(nz, device)

    def _apply(self, x, forward: bool):
        is_np = isinstance(x, np.ndarray) or not hasattr(x, "is_cuda")
        if is_np:
            x = np.ascontiguousarray(x, dtype=myfloat)  # no copy when already float32 (inputs are never modified)
            device = None
        else:
            device = x.device.index
        squeeze = x.ndim == 2
        nz = 1 if squeeze else int(x.shape[0])
        plan = self._plan(nz, device)
        y = plan.forward(x) if forward else plan.adjoint(x)
        return y[0] if squeeze else y

    def A(self, x):
        """Forward projection (reference: class_projectors_radon.py:60-68)."""
        return self._apply(x, True)

    def At(self, x):
        """Backprojection, the exact transpose of A (class_projectors_radon.py:73-81)."""
        return self._apply(x, False)

    def fbp(self, x):
        """Not provided.

        The reference method (class_projectors_radon.py:86-110) reads an
        undefined name ``dpc`` and raises NameError before any computation, so
        no reference behaviour exists to reproduce.  Use the gridding
        projector's ``fbp`` for an analytic start.
        """
        raise NotImplementedError(
            "class_projectors_radon.fbp: the reference method raises NameError "
            "(undefined 'dpc'); use class_projectors_grid.projectors(...).fbp")
