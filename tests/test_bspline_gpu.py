"""GPU parity tests of the B-spline (generalised Radon) projector pair."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _lut(na, deg, sup, rdeg=1):
    from iterative_tomographic_reconstruction_algorithms_b200.bspline_functions import init_lut_bspline
    return init_lut_bspline(2048, (np.arange(na) * 180.0) / np.float32(na), deg, rdeg, sup).astype(np.float32)


def test_matches_reference_golden(cuda, bspline_golden):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_bspline as cpb
    cases = sorted({k.split("/")[0] for k in bspline_golden.files})
    for case in cases:
        deg, sup = bspline_golden[f"{case}/deg_support"]
        img, sino = bspline_golden[f"{case}/image"], bspline_golden[f"{case}/sino"]
        na, n = sino.shape
        tp = cpb.projectors(n, np.zeros(na), None, bspline_degree=int(deg), proj_support_y=float(sup))
        assert rel_l2(tp.A(img), bspline_golden[f"{case}/fwd"]) <= TOL, case
        assert rel_l2(tp.At(sino), bspline_golden[f"{case}/adj"]) <= TOL, case


@pytest.mark.parametrize("n,na", [(128, 120), (129, 61), (256, 304)])
def test_matches_fp64_oracle_and_adjoint(cuda, oracle, n, na):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_bspline as cpb
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n)).astype(np.float32)
    y = rng.standard_normal((na, n)).astype(np.float32)
    tp = cpb.projectors(n, np.zeros(na), None)
    ax, aty = tp.A(x), tp.At(y)
    assert rel_l2(ax, oracle.bspline(0, x, tp.angles, tp.lut, tp.param_spline)) <= TOL
    assert rel_l2(aty, oracle.bspline(1, y, tp.angles, tp.lut, tp.param_spline)) <= TOL
    ax, aty = ax.astype(np.float64), aty.astype(np.float64)
    dot = abs(np.sum(ax * y) - np.sum(x * aty)) / (np.linalg.norm(ax) * np.linalg.norm(y))
    assert dot <= TOL


def test_dropin_entry_points(cuda, bspline_golden):
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    case = sorted({k.split("/")[0] for k in bspline_golden.files})[0]
    deg, sup = bspline_golden[f"{case}/deg_support"]
    img, sino = bspline_golden[f"{case}/image"], bspline_golden[f"{case}/sino"]
    na, n = sino.shape
    ang = bspline_golden[f"{case}/angles"]
    lut = _lut(na, int(deg), float(sup))
    fp = ctypes.POINTER(ctypes.c_float)
    out = np.zeros((na, n), np.float32)
    rc = _lib.lib.tomo_gen_forwproj(img.ctypes.data_as(fp), n, ang.ctypes.data_as(fp), na,
                                    lut.ctypes.data_as(fp), lut.shape[1], float(sup), 8,
                                    out.ctypes.data_as(fp))
    assert rc == 0, _lib.last_error()
    assert rel_l2(out, bspline_golden[f"{case}/fwd"]) <= TOL
    back = np.zeros((n, n), np.float32)
    rc = _lib.lib.tomo_gen_backproj(sino.ctypes.data_as(fp), n, ang.ctypes.data_as(fp), na,
                                    lut.ctypes.data_as(fp), lut.shape[1], float(sup),
                                    back.ctypes.data_as(fp))
    assert rc == 0, _lib.last_error()
    assert rel_l2(back, bspline_golden[f"{case}/adj"]) <= TOL


def test_fbp_runs_and_is_deterministic(cuda):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_bspline as cpb
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    n, na = 96, 90
    tp = cpb.projectors(n, np.zeros(na), None, radon_degree=0)
    b = tp.A(random_ellipses(n, seed=4))
    r1, r2 = tp.fbp(b), tp.fbp(b)
    assert r1.shape == (n, n) and np.array_equal(r1, r2) and np.isfinite(r1).all()
