"""Drop-in replacement for the reference's ``algorithms/class_projectors_grid.py``.

Same constructor, attributes and methods (class_projectors_grid.py:47-151):

    tp = projectors(npix, angles_deg, ctr=0.0, kernel='pswf', oversampl=2.0,
                    interp='nn', radon_degree=0, W=7.0, errs=1e-3, filt=None, args=None)
    tp.A(x), tp.At(b), tp.fbp(b)
    tp.lut, tp.deapod, tp.angles, tp.param_nofilt, tp.param_filt

The projector is the gridding (Fourier-slice) pair of gridrec_v4 with the
reference's arithmetic (including its asymmetries: the forward fixes the kernel
width at 2*7/pi while the adjoint uses the configured one, and the adjoint
edge-replicates the projections), run on the GPU (libtomo_b200.so: hand-written
interpolation, deapodisation and 1-D FFTs, cuFFT for the 2-D transform).
``fbp`` is the adjoint with the configured reconstruction filter (ramp by
default), as in the reference.

``adjoint="matched"`` (a keyword beyond the reference's) makes ``At`` the exact
transpose of ``A`` instead (same kernel width as the forward, zero-padded
projections, consistent Hermitian halves), so the pair passes the adjoint
dot-product test and its gradient is exact; ``A`` and ``fbp`` are unchanged.
On band-limited images supported in the inscribed circle both adjoints agree.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from . import gridrec_lut as glut

myfloat = np.float32

filter_list = np.array([["none", ""], ["ramp", ""], ["shepp-logan", "shlo"], ["hanning", "hann"],
                        ["hamming", "hamm"], ["lanczos", "lanc"], ["parzen", "parz"]])


class projectors:
    """Gridding projector pair (PSWF or Kaiser-Bessel interpolation)."""

    def __init__(self, npix, angles, ctr=0.0, kernel="pswf", oversampl=2.0, interp="nn",
                 radon_degree=0, W=7.0, errs=1e-3, filt=None, args=None, verbose=True, adjoint="compat"):
        if args is not None:
            kernel = args.kernel
            oversampl = args.oversampl
            interp = args.kernel_interp
            W = args.kernel_size
            errs = args.errs
            radon_degree = 1 if (hasattr(args, "dpc") and args.dpc is True) else 0
            if hasattr(args, "dbp") and args.dbp is True:
                radon_degree = 1
            filt = args.filt if hasattr(args, "filt") else None
        W, lut, deapod = glut.configure_regridding(npix, kernel, oversampl, interp, W, errs)
        interp1 = 0 if interp == "nn" else 1
        filt = 1 if filt is None else int(np.argwhere(filter_list == filt)[0][0])
        param_nofilt = np.array([ctr, 0, 0, oversampl, interp1, len(lut) - 5, W, radon_degree])
        param_filt = np.array([ctr, filt, 0, oversampl, interp1, len(lut) - 5, W, radon_degree])
        self.lut = lut.astype(myfloat)
        self.deapod = deapod.astype(myfloat)
        self.angles = np.asarray(angles).astype(myfloat)
        self.param_nofilt = param_nofilt.astype(myfloat)
        self.param_filt = param_filt.astype(myfloat)
        self.nang = len(angles)
        self.npix = int(npix)
        if adjoint not in ("compat", "matched"):
            raise ValueError("adjoint must be 'compat' or 'matched'")
        self.adjoint = adjoint
        self._plans = {}
        if verbose:
            print("\nSetting of the regridding projectors:")
            print("Kernel type: ", kernel)
            print("Oversampling: ", oversampl)
            print("Interpolation:", interp)
            print("LUT resolution: ", len(self.lut))
            print("Kernel size: ", W)
            print("Approx. error of LUT: ", errs)
            print("Filter for backprojection: ", filter_list[filt, 0])
            print("Radon transform degree: ", radon_degree)

    def _plan(self, nz: int, device, which: str):
        key = (nz, device, which)
        p = self._plans.get(key)
        if p is None:
            param = self.param_nofilt if which == "nofilt" else self.param_filt
            kw = dict(grid_param=param, grid_lut=self.lut, grid_lut_len=len(self.lut),
                      grid_deapod=self.deapod,
                      grid_mode=1 if (self.adjoint == "matched" and which == "nofilt") else 0)
            if device is not None:
                import torch
                with torch.cuda.device(device):
                    p = _lib.Plan(_lib.KIND_GRID, self.npix, self.angles, nz=nz, **kw)
            else:
                p = _lib.Plan(_lib.KIND_GRID, self.npix, self.angles, nz=nz, **kw)
            self._plans[key] = p
        return p

    def plan(self, nz: int = 1, device=None):
        """The libtomo_b200 plan of A / At for ``nz`` slices."""
        return self._plan(nz, device, "nofilt")

    def _apply(self, x, forward: bool, which: str):
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
        """Forward projection (class_projectors_grid.py:135-137, gridrec_v4_forwproj)."""
        return self._apply(x, True, "nofilt")

    def At(self, x):
        """Backprojection (class_projectors_grid.py:143-145, gridrec_v4_backproj)."""
        return self._apply(x, False, "nofilt")

    def fbp(self, x):
        """Filtered backprojection (class_projectors_grid.py:149-151)."""
        return self._apply(x, False, "filt")
