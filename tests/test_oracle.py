"""CPU tests of the oracle: it must reproduce the reference before it may check the GPU.

* against the golden fixtures (reference outputs stored in tests/golden/);
* against the compiled reference itself on fresh random inputs and on
  impulses (where float accumulation error vanishes, so any geometry or bin
  decision that differs from the reference shows up as an O(1) error);
* the B-spline LUT restatement against the reference's own Python.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import REFERENCE_TREE, rel_l2
from oracle.oracle import radon_angles

RADON_KINDS = ("pd", "rd", "dd", "ss")


def _cases(golden):
    return sorted({k.split("/")[0] for k in golden.files})


@pytest.mark.parametrize("kind", RADON_KINDS)
def test_oracle_matches_golden_radon(oracle, radon_golden, kind):
    checked = 0
    for case in _cases(radon_golden):
        if f"{case}/{kind}/fwd" not in radon_golden.files:
            continue
        ang = radon_angles(radon_golden[f"{case}/angles_deg"])
        fwd = oracle.radon(kind, 0, radon_golden[f"{case}/image"], ang)
        adj = oracle.radon(kind, 1, radon_golden[f"{case}/sino"], ang)
        # reference accumulates in float32, the oracle in float64
        assert rel_l2(radon_golden[f"{case}/{kind}/fwd"], fwd) < 3e-6, case
        assert rel_l2(radon_golden[f"{case}/{kind}/adj"], adj) < 3e-6, case
        checked += 1
    assert checked >= 3


def test_oracle_matches_golden_bspline(oracle, bspline_golden):
    from iterative_tomographic_reconstruction_algorithms_b200.bspline_functions import init_lut_bspline
    for case in _cases(bspline_golden):
        deg, sup = bspline_golden[f"{case}/deg_support"]
        a32 = bspline_golden[f"{case}/angles"]
        na = len(a32)
        lut = init_lut_bspline(2048, (np.arange(na) * 180.0) / np.float32(na),
                               int(deg), 1, float(sup)).astype(np.float32)
        assert np.sum(lut, dtype=np.float64) == pytest.approx(bspline_golden[f"{case}/lut_sum"][0], rel=1e-12)
        param = bspline_golden[f"{case}/param"]
        fwd = oracle.bspline(0, bspline_golden[f"{case}/image"], a32, lut, param)
        adj = oracle.bspline(1, bspline_golden[f"{case}/sino"], a32, lut, param)
        assert rel_l2(bspline_golden[f"{case}/fwd"], fwd) < 3e-6, case
        assert rel_l2(bspline_golden[f"{case}/adj"], adj) < 3e-6, case


@pytest.mark.parametrize("kind", RADON_KINDS)
@pytest.mark.parametrize("n,na", [(40, 30), (57, 23)])
def test_oracle_matches_reference_impulses(oracle, reflib, kind, n, na):
    """Impulse inputs: each output is a sum of at most a few terms, so the
    oracle must agree with the compiled reference to float rounding."""
    rng = np.random.default_rng(n * 1000 + na)
    ang = radon_angles(np.linspace(0, 180, na, endpoint=False))
    if kind == "ss":
        ang = ang[:-1]  # keep rays inside the square (see make_golden.py)
    for _ in range(6):
        img = np.zeros((n, n), np.float32)
        img[rng.integers(n), rng.integers(n)] = 1.0
        d = np.abs(reflib.radon(kind, 0, img, ang) - oracle.radon(kind, 0, img, ang))
        assert d.max() < 1e-6
        sino = np.zeros((len(ang), n), np.float32)
        sino[rng.integers(len(ang)), rng.integers(n)] = 1.0
        d = np.abs(reflib.radon(kind, 1, sino, ang) - oracle.radon(kind, 1, sino, ang))
        assert d.max() < 1e-6


@pytest.mark.parametrize("kind", RADON_KINDS)
def test_oracle_matches_reference_random(oracle, reflib, kind):
    rng = np.random.default_rng(11)
    n, na = 96, 120
    ang = radon_angles(np.linspace(0, 180, na, endpoint=False))
    img = rng.standard_normal((n, n)).astype(np.float32)
    sino = rng.standard_normal((na, n)).astype(np.float32)
    assert rel_l2(reflib.radon(kind, 0, img, ang), oracle.radon(kind, 0, img, ang)) < 3e-6
    assert rel_l2(reflib.radon(kind, 1, sino, ang), oracle.radon(kind, 1, sino, ang)) < 3e-6


def test_bspline_lut_matches_reference_python():
    if not (REFERENCE_TREE / "common/operators/bspline_module/bspline_functions.py").exists():
        pytest.skip("reference tree not present")
    import importlib.util
    import sys
    import types

    import scipy
    import scipy.special as sp
    shim = types.ModuleType("scipy.misc")  # scipy.misc.factorial/comb were removed upstream
    shim.factorial, shim.comb = sp.factorial, sp.comb
    saved = sys.modules.get("scipy.misc")
    sys.modules["scipy.misc"] = shim
    scipy.misc = shim
    try:
        spec = importlib.util.spec_from_file_location(
            "ref_bspline_functions",
            REFERENCE_TREE / "common/operators/bspline_module/bspline_functions.py")
        ref = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(ref)
    finally:
        if saved is not None:
            sys.modules["scipy.misc"] = saved
    from iterative_tomographic_reconstruction_algorithms_b200.bspline_functions import init_lut_bspline
    for na, deg, rdeg, sup in [(60, 3, 1, 4), (60, 3, 0, 4), (17, 1, 1, 2)]:
        angles = (np.arange(na) * 180.0) / np.float32(na)
        a = ref.init_lut_bspline(512, angles, deg, rdeg, sup)
        b = init_lut_bspline(512, angles, deg, rdeg, sup)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("kind", RADON_KINDS)
def test_sinogram_row_of_angle_matches_reference(reflib, kind):
    """The row map that the large-geometry fixture relies on: the reference's
    full-angle forward holds, in row sinogram_row_of_angle(kind, na)[k], exactly
    the row that the reference computes from angle k alone."""
    from oracle.oracle import sinogram_row_of_angle
    n, na = 48, 37
    ang = radon_angles(np.linspace(0, 180, na, endpoint=False))
    img = np.random.default_rng(4).standard_normal((n, n)).astype(np.float32)
    full = reflib.radon(kind, 0, img, ang)
    rows = sinogram_row_of_angle(kind, na)
    for k in range(na):
        assert np.array_equal(full[rows[k]], reflib.radon(kind, 0, img, ang[k:k + 1])[0]), k


@pytest.mark.parametrize("kind", RADON_KINDS + ("bspline",))
def test_oracle_matches_large_golden_sparse_rows(oracle, kind):
    """At 2048 x 2048 the FP64 oracle reproduces the reference's rows of the
    sparse image (a few terms per bin, so no float32 accumulation error hides a
    geometry difference) on 3 of the sampled angles of large_golden.npz; the
    GPU test checks all of them on every input."""
    import importlib.util
    from conftest import GOLDEN
    g = np.load(GOLDEN / "large_golden.npz")
    spec = importlib.util.spec_from_file_location("make_large_golden", GOLDEN / "make_large_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    sparse = mk.large_inputs()[2]
    assert sparse.sum(dtype=np.float64) == g["sums"][2]
    ang = radon_angles(np.linspace(0, 180, mk.NA, endpoint=False))
    if kind == "bspline":
        from iterative_tomographic_reconstruction_algorithms_b200.bspline_functions import init_lut_bspline
        bdeg = (np.arange(mk.NA) * 180.0) / np.float32(mk.NA)
    for j in (1, 4, 7):                    # 0.1, 45.0 and 90.0 degrees
        k = int(g["angle_index"][j])
        if kind == "bspline":
            lut = init_lut_bspline(2048, bdeg[k:k + 1], 3, 1, 4.0).astype(np.float32)
            row = oracle.bspline(0, sparse, bdeg[k:k + 1].astype(np.float32), lut,
                                 np.array([lut.shape[1], 4.0], np.float32))[0]
        else:
            row = oracle.radon(kind, 0, sparse, ang[k:k + 1])[0]
        assert rel_l2(g[f"{kind}/fwd_sparse"][j], row) < 1e-6, k
