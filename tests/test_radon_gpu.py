"""GPU parity tests of the Radon-family projector pairs (pixel/ray/distance-driven,
slant-stacking) through the C ABI.

Bars (written in each test):
  * vs the reference's own outputs (tests/golden): relative L2 <= 1e-5;
  * vs the FP64 oracle on the same inputs: relative L2 <= 1e-5;
  * adjoint dot test |<Ax,y> - <x,A^T y>| / (||Ax|| ||y||) <= 1e-5 (FP64 dots);
  * bit-identical results on repeated runs (no floating-point atomics on any path);
  * batched slices == slice-by-slice; device path == host path.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import rel_l2
from oracle.oracle import radon_angles

pytestmark = pytest.mark.gpu

KINDS = ("pd", "rd", "dd", "ss")
TOL = 1e-5


def _proj(kind, n, deg):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    return cpr.projectors(n, np.asarray(deg), oper=kind)


def _cases(golden, kind):
    cases = sorted({k.split("/")[0] for k in golden.files})
    return [c for c in cases if f"{c}/{kind}/fwd" in golden.files]


@pytest.mark.parametrize("kind", KINDS)
def test_matches_reference_golden(cuda, radon_golden, kind):
    for case in _cases(radon_golden, kind):
        deg = radon_golden[f"{case}/angles_deg"]
        img, sino = radon_golden[f"{case}/image"], radon_golden[f"{case}/sino"]
        tp = _proj(kind, img.shape[0], deg)
        assert rel_l2(tp.A(img), radon_golden[f"{case}/{kind}/fwd"]) <= TOL, case
        assert rel_l2(tp.At(sino), radon_golden[f"{case}/{kind}/adj"]) <= TOL, case


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n,na", [(128, 180), (129, 91), (256, 304)])
def test_matches_fp64_oracle(cuda, oracle, kind, n, na):
    rng = np.random.default_rng(n + na)
    deg = np.linspace(0, 180, na, endpoint=False)
    img = rng.standard_normal((n, n)).astype(np.float32)
    sino = rng.standard_normal((na, n)).astype(np.float32)
    tp = _proj(kind, n, deg)
    ang = radon_angles(deg)
    assert rel_l2(tp.A(img), oracle.radon(kind, 0, img, ang)) <= TOL
    assert rel_l2(tp.At(sino), oracle.radon(kind, 1, sino, ang)) <= TOL


@pytest.mark.parametrize("kind", KINDS)
def test_phantom_matches_oracle_tightly(cuda, oracle, kind):
    """Non-negative smooth data: no cancellation, so the bar is tighter."""
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    n, na = 192, 200
    deg = np.linspace(0, 180, na, endpoint=False)
    img = random_ellipses(n, seed=3)
    tp = _proj(kind, n, deg)
    b = tp.A(img)
    assert rel_l2(b, oracle.radon(kind, 0, img, radon_angles(deg))) <= 2e-6
    assert rel_l2(tp.At(b), oracle.radon(kind, 1, b, radon_angles(deg))) <= 2e-6


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n,na", [(256, 304), (97, 50)])
def test_adjoint_dot_product(cuda, kind, n, na):
    rng = np.random.default_rng(7)
    x = rng.standard_normal((n, n)).astype(np.float32)
    y = rng.standard_normal((na, n)).astype(np.float32)
    tp = _proj(kind, n, np.linspace(0, 180, na, endpoint=False))
    ax, aty = tp.A(x).astype(np.float64), tp.At(y).astype(np.float64)
    lhs, rhs = np.sum(ax * y), np.sum(x.astype(np.float64) * aty)
    assert abs(lhs - rhs) / (np.linalg.norm(ax) * np.linalg.norm(y)) <= TOL


@pytest.mark.parametrize("kind", KINDS)
def test_deterministic_and_batched(cuda, kind):
    torch = cuda
    n, na, nz = 160, 120, 3
    rng = np.random.default_rng(5)
    x = rng.standard_normal((nz, n, n)).astype(np.float32)
    y = rng.standard_normal((nz, na, n)).astype(np.float32)
    tp = _proj(kind, n, np.linspace(0, 180, na, endpoint=False))
    b1, b2 = tp.A(x), tp.A(x)
    assert np.array_equal(b1, b2)
    g1, g2 = tp.At(y), tp.At(y)
    assert np.array_equal(g1, g2)
    for z in range(nz):
        assert np.array_equal(tp.A(x[z]), b1[z])
        assert np.array_equal(tp.At(y[z]), g1[z])
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y).cuda()
    assert np.array_equal(tp.A(xd).cpu().numpy(), b1)
    assert np.array_equal(tp.At(yd).cpu().numpy(), g1)


def test_rd_thread_layouts_agree(cuda):
    """Both rd kernels pick their thread layout by grid size, and the layouts
    make the same arithmetic in the same order, so the results are the same
    bits.  The forward runs blocks of 128 bins x 4 angles once there are 8 or
    more such blocks per SM (148 SMs), else blocks of 32 bins x 4 angles; the
    adjoint runs one thread per bin when bins x angles x slices reach
    148 x 1024, else one thread per sub-ray.  Here the 12-slice batch of
    256 x 256 at 200 angles (1200 blocks; 614,400 threads) takes the first
    layout of each and a slice alone (100 blocks; 51,200 threads) the second.
    Non-finite values and the axis angles' row and column sums (made by a
    bin's first thread only in the adjoint) are included."""
    n, na, nz = 256, 200, 12
    assert 2 * (na // 4) * nz >= 148 * 8 > 2 * (na // 4)
    assert n * na * nz >= 148 * 1024 > n * na
    rng = np.random.default_rng(17)
    x = rng.standard_normal((nz, n, n)).astype(np.float32)
    y = rng.standard_normal((nz, na, n)).astype(np.float32)
    y[1, 7, 100] = np.inf
    y[2, 150, 31] = np.nan
    x[3, 60, 70] = -np.inf
    deg = np.linspace(0, 180, na, endpoint=False)  # includes 0 and 90 degrees
    tp = _proj("rd", n, deg)
    fwd, adj = tp.A(x), tp.At(y)
    for z in range(nz):
        assert np.array_equal(tp.A(x[z]).view(np.uint32), fwd[z].view(np.uint32)), z
        assert np.array_equal(tp.At(y[z]).view(np.uint32), adj[z].view(np.uint32)), z


@pytest.mark.parametrize("kind", KINDS)
def test_dropin_entry_point_accumulates(cuda, radon_golden, kind):
    """tomo_radon_<kind> has the reference C signature and accumulates like it."""
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    from iterative_tomographic_reconstruction_algorithms_b200.class_projectors_radon import shim_angles
    case = _cases(radon_golden, kind)[0]
    img = radon_golden[f"{case}/image"].copy()
    n = img.shape[0]
    ang = shim_angles(kind, radon_angles(radon_golden[f"{case}/angles_deg"]))
    fp = ctypes.POINTER(ctypes.c_float)
    sino = np.ones((len(ang), n), np.float32)
    fn = getattr(_lib.lib, f"tomo_radon_{kind}")
    extra = (1,) if kind in ("pd", "ss") else ()  # method 1 = linear interpolation
    rc = fn(img.ctypes.data_as(fp), n, ang.ctypes.data_as(fp), len(ang), 0, *extra,
            sino.ctypes.data_as(fp))
    assert rc == 0, _lib.last_error()
    assert rel_l2(sino - 1.0, radon_golden[f"{case}/{kind}/fwd"]) <= TOL


def test_dd_rejects_angles_outside_domain(cuda):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    with pytest.raises(ValueError, match="outside"):
        cpr.projectors(32, np.array([0.0, 200.0]), oper="dd").A(np.zeros((32, 32), np.float32))


def test_rd_adjoint_carries_non_finite_values(cuda, oracle):
    """inf and NaN in the sinogram reach the pixels their rays credit as the
    reference's float sums carry them: +-inf, or NaN where NaN, 0 * inf or both
    infinities meet (the FP64 oracle accumulates the same credits)."""
    n, na = 64, 60
    deg = np.linspace(0, 180, na, endpoint=False)          # 0 and 90 degrees: row / column sums
    rng = np.random.default_rng(3)
    y = rng.standard_normal((na, n)).astype(np.float32)
    y[5, 20], y[17, 40], y[33, 31] = np.inf, -np.inf, np.nan
    y[0, 10], y[30, 12], y[41, 22] = np.inf, -np.inf, np.inf
    got = _proj("rd", n, deg).At(y)
    ref = oracle.radon("rd", 1, y, radon_angles(deg))
    for test in (np.isnan, np.isposinf, np.isneginf):
        assert np.array_equal(test(got), test(ref)), test.__name__
    fin = np.isfinite(ref)
    assert fin.sum() > n * n // 4
    assert rel_l2(got[fin], ref[fin]) <= TOL


def test_pd_forward_carries_non_finite_values(cuda, oracle):
    """inf and NaN pixels reach the bins their sub-samples land in as the
    reference's float sums carry them, and every finite bin keeps its value
    (the fixed-point unit comes from the finite pixels only)."""
    n, na = 64, 60
    deg = np.linspace(0, 180, na, endpoint=False)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((n, n)).astype(np.float32)
    x[20, 11] = np.inf
    x[40, 50] = -np.inf
    x[33, 31] = np.nan
    got = _proj("pd", n, deg).A(x)
    ref = oracle.radon("pd", 0, x, radon_angles(deg))
    for test in (np.isnan, np.isposinf, np.isneginf):
        assert np.array_equal(test(got), test(ref)), test.__name__
    fin = np.isfinite(ref)
    assert fin.sum() > na * n // 2
    assert rel_l2(got[fin], ref[fin]) <= TOL


def test_bspline_forward_carries_non_finite_values(cuda, oracle):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_bspline as cpb
    n, na = 64, 60
    rng = np.random.default_rng(5)
    x = rng.standard_normal((n, n)).astype(np.float32)
    x[10, 12] = np.inf
    x[41, 43] = -np.inf
    x[30, 22] = np.nan
    tp = cpb.projectors(n, np.zeros(na), None)
    got = tp.A(x)
    ref = oracle.bspline(0, x, tp.angles, tp.lut, tp.param_spline)
    for test in (np.isnan, np.isposinf, np.isneginf):
        assert np.array_equal(test(got), test(ref)), test.__name__
    fin = np.isfinite(ref)
    assert fin.sum() > na * n // 2
    assert rel_l2(got[fin], ref[fin]) <= TOL


@pytest.mark.parametrize("kind", ("pd", "rd", "dd"))
def test_near_axis_angles_match_oracle_row_by_row(cuda, oracle, radon_golden, kind):
    """Angles within 0.001-0.5 degrees of 90 and 180 degrees (and 0.1, 0.5,
    44.9, 134.9): for the distance-driven pair the reference's pixel
    coordinates reach nh / |cos|, where pixels straddling a binade of the
    coordinate are wider or narrower than 1 by up to 1/16 (and beyond 2^22 the
    widths are 0 or 2).  Every row against the FP64 oracle and the reference."""
    case = "n256_nearaxis"
    deg = radon_golden[f"{case}/angles_deg"]
    img, sino = radon_golden[f"{case}/image"], radon_golden[f"{case}/sino"]
    tp = _proj(kind, img.shape[0], deg)
    got = tp.A(img)
    orc = oracle.radon(kind, 0, img, radon_angles(deg))
    ref = radon_golden[f"{case}/{kind}/fwd"]
    for r in range(len(deg)):
        floor = rel_l2(ref[r], orc[r])
        assert rel_l2(got[r], orc[r]) <= TOL + floor, (r, rel_l2(got[r], orc[r]), floor)
        assert rel_l2(got[r], ref[r]) <= TOL + floor, (r, rel_l2(got[r], ref[r]), floor)
    adj = tp.At(sino)
    assert rel_l2(adj, oracle.radon(kind, 1, sino, radon_angles(deg))) <= TOL
