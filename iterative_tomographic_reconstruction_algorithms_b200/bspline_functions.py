"""Look-up table of the Radon transform of a tensor B-spline (host-side setup).

Restates ``common/operators/bspline_module/bspline_functions.py`` of the
reference: ``init_lut_bspline`` (:116-201) evaluates formula 28 of Nilchian et
al., "Fast iterative reconstruction of differential phase contrast X-ray
tomograms", Optics Express 2013,

    R^n{beta^m}(y, theta) = sum_{k1,k2=0}^{m+1} (-1)^(k1+k2) C(m+1,k1) C(m+1,k2)
        (y + ((m+1)/2 - k1) cos(theta) + ((m+1)/2 - k2) sin(theta))_+^(2m-n+1)
        / [ (2m-n+1)! cos(theta)^(m+1) sin(theta)^(m+1) ],

on ``nsamples_y`` points of y in [-support/2, support/2) and one row per angle.
Rows whose angle is 0, pi/2 or pi (within 1e-8) divide by zero in that form and
are filled instead by the repeated-finite-difference form of
``radon_n_bspline_general`` (:70-94), with the same float32/float64 mix as the
reference so that the table is the reference's to rounding.

The reference passes this function angles in DEGREES but evaluates sin/cos on
them as if they were radians (class_projectors_bspline.py:49-53).  That quirk is
part of the operator the reference solves with, so it is kept: callers pass the
same degree values, and the projector kernels convert degrees to radians for
the geometry exactly as the reference C does.

Setup only: the table is computed once per projector object, in float64, and
handed to the CUDA kernels as float32 ``[nang, nsamples_y]``.
"""
from __future__ import annotations

import math

import numpy as np

_EPS = 1e-8


def _comb(n: int, k: int) -> float:
    return float(math.comb(n, k))


def _general_row(y: np.float32, theta: float, m: int, n: int) -> float:
    """radon_n_bspline_general (bspline_functions.py:70-94) for one sample.

    Builds the same chain of closures as the reference: a positive power,
    optionally replaced by its analytic (m+1)-fold derivative when theta is
    0, pi/2 or pi, then m+1 centred finite differences with step cos(theta)
    and/or sin(theta).  Arithmetic types follow the reference under NumPy 2
    promotion rules (float32 samples, Python-float constants).
    """
    exponent = 2 * m - n + 1

    def positive_power(p):
        def f(x):
            xf = np.float32(x)
            if xf > 0.0:
                return np.power(xf, p)
            return 0.0
        return f

    def scaled(lam, f):
        return lambda x: float(lam) * f(x)

    def fdiff(f, h):
        return lambda x: (f(x + 0.5 * h) - f(x - 0.5 * h)) / np.float32(h)

    y_plus = positive_power(exponent)
    deriv = scaled(math.factorial(exponent) / math.factorial(exponent - (m + 1)),
                   positive_power(m - n))
    if theta == 0.0 or theta == np.pi / 2.0 or theta == np.pi:
        y_plus = deriv
    if abs(theta - np.pi / 2.0) > _EPS:
        for _ in range(m + 1):
            y_plus = fdiff(y_plus, np.cos(theta))
    if abs(theta) > _EPS and abs(theta - np.pi) > _EPS:
        for _ in range(m + 1):
            y_plus = fdiff(y_plus, np.sin(theta))
    return y_plus(y) / float(math.factorial(exponent))


def init_lut_bspline(nsamples_y: int, angles, bspline_degree: int, rt_degree: int,
                     proj_support_y: float) -> np.ndarray:
    """Table [len(angles), nsamples_y] (float64) of R^rt_degree of the B-spline."""
    m, n = int(bspline_degree), int(rt_degree)
    exponent = 2 * m - n + 1
    angles = np.asarray(angles, dtype=np.float64).reshape(-1)

    y = np.arange(nsamples_y).astype(np.float32)
    y -= nsamples_y / 2.0
    y /= np.float32(nsamples_y)
    y *= proj_support_y

    th = angles[:, None]
    sn, cs = np.sin(th), np.cos(th)
    divisor = np.float32(math.factorial(exponent)) * np.power(sn * cs, m + 1)
    special = [np.argwhere(np.abs(angles - a) < _EPS).reshape(-1) for a in (0.0, np.pi / 2.0, np.pi)]
    for idx in special:
        divisor[idx, :] = 1.0

    ym = y[None, :]
    res = np.zeros((len(angles), nsamples_y))
    for k1 in range(m + 2):
        for k2 in range(m + 2):
            num = ym + (m / 2.0 + 0.5 - k1) * cs + (m / 2.0 + 0.5 - k2) * sn
            num[num < 0.0] = 0.0
            res += np.power(num, exponent) * ((-1.0) ** (k1 + k2) * _comb(m + 1, k1) * _comb(m + 1, k2))
    res /= divisor

    for idx, a in zip(special, (0.0, np.pi / 2.0, np.pi)):
        if len(idx):
            row = np.array([_general_row(y[j], a, m, n) for j in range(nsamples_y)], dtype=np.float64)
            res[idx, :] = row[None, :]
    return res
