"""Interpolation kernel table and deapodiser of the gridding projector (host set-up).

Restates ``common/operators/gridrec_module/gridrec_lut.py`` of the reference:

* ``configure_regridding`` (:268-302): kernel width ``W *= 2/pi``; Fourier grid
  size ``nfreq = int(2^ceil(log2 npix) * oversampl)`` rounded up to a multiple
  of 4; the fixed 2048-entry table for prolate/os=2/nn.
* Kaiser-Bessel (:91-137): ``beta = pi sqrt(((W/alpha)(alpha - 1/2))^2 - 0.8)``,
  table of ``I0(beta sqrt(1 - (2 ns k / W)^2))`` normalised to its first entry,
  zero-padded by 4; deapodiser ``norm / |sin f / f|`` with the normalisation of
  ``normalize_kaiser_bessel`` (:149-182).
* Prolate spheroidal wave function (:194-241): Legendre series of the PSWF,
  zero-padded by 5, deapodiser from the table at ``i * ns_ker / (nh + 1/2)``.
* ``create_lut_deapod`` (:55-79): checkerboard sign (fftshift in Fourier space)
  and outer product to a ``[nfreq, nfreq]`` matrix.

The arithmetic follows the reference's numpy float32/float64 mix, so the
arrays are the reference's to rounding (pinned in tests/test_grid.py).
"""
from __future__ import annotations

import numpy as np

myfloat = np.float32
_EPS = 1e-8

_KB_LAMBDA = np.array([[2.0, 0.6735177854455913], [1.9, 0.6859972251713252],
                       [1.8, 0.7016852052327338], [1.7, 0.7186085894388523],
                       [1.6, 0.7391321589920385], [1.5, 0.7631378768943125],
                       [1.4, 0.7915122594523216], [1.3, 0.8296167052898601],
                       [1.2, 0.8762210440212161], [1.1, 0.9373402868152573]], dtype=myfloat)

_PSWF_COEFFS = np.array([0.5767616E+02, 0.0, -0.8931343E+02, 0.0, 0.4167596E+02, 0.0,
                         -0.1053599E+02, 0.0, 0.1662374E+01, 0.0, -0.1780527E-00, 0.0,
                         0.1372983E-01, 0.0, -0.7963169E-03, 0.0, 0.3593372E-04, 0.0,
                         -0.1295941E-05, 0.0, 0.3817796E-07])


def _nn(x):
    return np.round(x).astype(int)


def _kb_lambda(alpha: float) -> float:
    """Tabulated KB normalisation, with the reference's interpolation rule (:149-182)."""
    lut = _KB_LAMBDA[::-1, :].copy()
    d = np.abs(lut - alpha)
    ind = np.argwhere(d == np.min(d))
    r = ind[0, 0]
    if alpha != lut[r, 0]:
        if alpha > lut[r, 0]:
            dd = alpha - lut[r, 0]
            return (1 - dd) * lut[r, 1] + dd * lut[r, 1]
        dd = alpha - lut[r - 1, 0]
        return (1 - dd) * lut[r - 1, 1] + dd * lut[r, 1]
    return lut[r, 1]


def kaiser_bessel(W, alpha, err, interp, ns_grid):
    beta = np.pi * np.sqrt(((W / alpha) * (alpha - 0.5)) ** 2 - 0.8)
    if interp == "nn":
        ns_ker = int(0.91 / (err * alpha))
    else:
        ns_ker = int(np.sqrt(0.37 / err) * 1.0 / alpha)
    k_max = W / myfloat(2 * ns_grid)
    k = np.linspace(0, k_max, ns_ker)
    lut = ns_grid / myfloat(W) * np.i0(beta * np.sqrt(1 - (2 * ns_grid * k / W) ** 2))
    lut /= lut[0]
    lut = np.pad(lut, (0, 4), "constant", constant_values=0)
    nh = int(ns_grid * 0.5)
    x = np.linspace(-nh, nh, ns_grid)
    f = (np.pi * W * x / ns_grid) ** 2 - beta ** 2
    f = np.sqrt(f.astype(complex))
    deapod = np.abs(np.sin(f) / f)
    deapod[:] /= deapod[nh]
    deapod += _EPS
    norm = myfloat(np.sqrt(1.0 / (W * _kb_lambda(alpha))))
    deapod[:] = norm / deapod
    return lut, deapod


def prolate(W, alpha, err, interp, ns_grid, ns_ker):
    if ns_ker != 2048:
        if interp == "nn":
            ns_ker = int(0.91 / (err * alpha))
        else:
            ns_ker = int((0.37 / err) / alpha)
    x = np.arange(0, ns_ker) / myfloat(ns_ker)
    lut = np.polynomial.legendre.legval(x, _PSWF_COEFFS) / np.polynomial.legendre.legval(0.0, _PSWF_COEFFS)
    lut = np.pad(lut, (0, 5), "constant", constant_values=0)
    nh = int(ns_grid * 0.5)
    lmbda = 0.99998546
    norm = myfloat(np.sqrt(1.0 / (W * lmbda)))
    scale_ratio = myfloat(ns_ker) / myfloat(nh + 0.5)
    deapod = np.zeros(ns_grid, dtype=myfloat)
    deapod[nh] = norm / lut[_nn(0.0)]
    for i in range(1, nh + 1):
        v = norm / (lut[_nn(i * scale_ratio)] + _EPS)
        if i != nh:
            deapod[nh + i] = v
            deapod[nh - i] = v
        else:
            deapod[0] = v
    return lut, deapod


def create_lut_deapod(kernel, ns_grid, ns_ker, W, alpha, interp, err):
    if kernel in ("prolate", "pswf"):
        lut, deapod = prolate(W, alpha, err, interp, ns_grid, ns_ker)
    elif kernel in ("kaiser-bessel", "kb"):
        lut, deapod = kaiser_bessel(W, alpha, err, interp, ns_grid)
    else:
        raise ValueError(f"unknown gridding kernel {kernel!r}")
    nh = int(ns_grid * 0.5)
    sign = 1.0
    for i in range(1, nh + 1):
        sign = 1.0 if i % 2 == 0 else -1.0
        if i != nh:
            deapod[nh + i] *= sign
            deapod[nh - i] *= sign
        else:
            deapod[0] *= sign
    deapod[nh] *= sign
    return lut, np.outer(deapod, deapod)


def grid_size(npix: int, oversampl: float) -> int:
    nfreq = int(2 ** (np.ceil(np.log2(npix))) * oversampl)
    while nfreq % 4 != 0:
        nfreq += 1
    return nfreq


def configure_regridding(npix, kernel, oversampl, interp, W, errs):
    """(W in the projector's units, lut, deapod) as gridrec_lut.configure_regridding."""
    W *= 2 / np.pi
    nfreq = grid_size(npix, oversampl)
    ltbl = 2048 if (kernel == "prolate" and oversampl == 2.0 and interp == "nn") else None
    lut, deapod = create_lut_deapod(kernel, nfreq, ltbl, W, oversampl, interp, errs)
    return W, lut, deapod
