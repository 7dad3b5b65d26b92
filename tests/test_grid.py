"""Gridding pair: CPU pins of the host set-up and of the compiled reference, and
GPU parity of the CUDA path against the reference's outputs.

The reference's own golden vector for this path is data/shepp_logan_pix0256.tif
and its grid-PSWF sinogram data/shepp_logan_pix0256_ang0304_sino.tif (stored in
tests/golden/grid_golden.npz as "sl/*").  The reference gridding pair is not an
adjoint pair (its forward fixes the kernel width at 2*7/pi, its adjoint
edge-replicates the projections), so the compat mode has no dot-product test;
the matched mode (adjoint="matched": the forward's exact transpose) has one,
on N(0,1) data, to 1e-5.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import GOLDEN, REFERENCE_TREE, rel_l2

TOL = 1e-5


@pytest.fixture(scope="module")
def grid_golden():
    return np.load(GOLDEN / "grid_golden.npz")


def _cases(golden):
    return sorted({k.split("/")[0] for k in golden.files if k.count("/") == 1 and not k.startswith("sl/")})


def _proj(golden, case, verbose=False):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    n, na, os_, interp, W, errs, rdeg, filt = golden[f"{case}/cfg"]
    kernel = str(golden[f"{case}/kernel"])
    deg = np.linspace(0, 180, int(na), endpoint=False)
    return cpg.projectors(int(n), deg, kernel=kernel, oversampl=float(os_), interp="nn" if interp == 0 else "lin",
                          radon_degree=int(rdeg), W=float(W), errs=float(errs), verbose=verbose)


def test_compiled_reference_reproduces_golden_sinogram(reflib, grid_golden):
    from iterative_tomographic_reconstruction_algorithms_b200 import gridrec_lut as glut
    W, lut, deapod = glut.configure_regridding(256, "prolate", 2.0, "nn", 7.0, 1e-3)
    param = np.array([0.0, 0, 0, 2.0, 0, len(lut) - 5, W, 0], np.float32)
    ang = np.linspace(0, 180, 304, endpoint=False).astype(np.float32)
    out = reflib.gridrec(0, grid_golden["sl/image"], ang, param, lut.astype(np.float32), deapod.astype(np.float32))
    assert rel_l2(out, grid_golden["sl/sino"]) < 3e-6


def test_gridrec_lut_matches_reference_python():
    if not (REFERENCE_TREE / "common/operators/gridrec_module/gridrec_lut.py").exists():
        pytest.skip("reference tree not present")
    import importlib.util
    np.int = int  # the reference module uses np.int
    spec = importlib.util.spec_from_file_location(
        "ref_gridrec_lut", REFERENCE_TREE / "common/operators/gridrec_module/gridrec_lut.py")
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    from iterative_tomographic_reconstruction_algorithms_b200 import gridrec_lut as mine
    for args in [(256, "prolate", 2.0, "nn", 7.0, 1e-3), (200, "pswf", 2.0, "lin", 7.0, 1e-3),
                 (300, "kb", 1.5, "lin", 6.6, 6e-6), (96, "kb", 2.0, "nn", 6.0, 1e-3)]:
        a, b = ref.configure_regridding(*args), mine.configure_regridding(*args)
        assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


@pytest.mark.gpu
def test_forward_reproduces_reference_golden_sinogram(cuda, grid_golden):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    tp = cpg.projectors(256, np.linspace(0, 180, 304, endpoint=False), kernel="prolate", oversampl=2.0,
                        interp="nn", W=7.0, errs=1e-3, verbose=False)
    assert rel_l2(tp.A(grid_golden["sl/image"]), grid_golden["sl/sino"]) <= TOL


@pytest.mark.gpu
def test_matches_reference_outputs(cuda, grid_golden):
    for case in _cases(grid_golden):
        tp = _proj(grid_golden, case)
        filt = int(grid_golden[f"{case}/cfg"][7])
        assert rel_l2(tp.A(grid_golden[f"{case}/image"]), grid_golden[f"{case}/fwd"]) <= TOL, case
        back = tp.fbp(grid_golden[f"{case}/sino"]) if filt else tp.At(grid_golden[f"{case}/sino"])
        assert rel_l2(back, grid_golden[f"{case}/adj"]) <= TOL, case


@pytest.mark.gpu
def test_deterministic_batched_and_device(cuda, grid_golden):
    torch = cuda
    case = "n96_kb_lin"
    tp = _proj(grid_golden, case)
    x = np.stack([grid_golden[f"{case}/image"]] * 2)
    y = np.stack([grid_golden[f"{case}/sino"]] * 2)
    a1, a2 = tp.A(x), tp.A(x)
    b1, b2 = tp.At(y), tp.At(y)
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    assert np.array_equal(a1[0], a1[1]) and np.array_equal(a1[0], tp.A(x[0]))
    assert np.array_equal(tp.At(torch.from_numpy(y).cuda()).cpu().numpy(), b1)


@pytest.mark.gpu
def test_dropin_entry_points_overwrite(cuda, grid_golden):
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    case = "n64_pswf_nn"
    tp = _proj(grid_golden, case)
    fp = ctypes.POINTER(ctypes.c_float)
    img, sino = grid_golden[f"{case}/image"], grid_golden[f"{case}/sino"]
    na, n = sino.shape
    f = _lib.lib.tomo_gridrec_forwproj
    f.argtypes = [fp, ctypes.c_int, ctypes.c_int, fp, fp, fp, fp, fp, ctypes.c_char_p]
    out = np.full((na, n), 7.0, np.float32)
    rc = f(out.ctypes.data_as(fp), n, na, tp.angles.ctypes.data_as(fp), tp.param_nofilt.ctypes.data_as(fp),
           tp.lut.ctypes.data_as(fp), tp.deapod.ctypes.data_as(fp), img.ctypes.data_as(fp), b"/dev/null")
    assert rc == 0, _lib.last_error()
    assert rel_l2(out, grid_golden[f"{case}/fwd"]) <= TOL
    g = _lib.lib.tomo_gridrec_backproj
    g.argtypes = [fp, ctypes.c_int, ctypes.c_int, fp, fp, fp, fp, fp, fp, ctypes.c_char_p]
    rec = np.full((n, n), 7.0, np.float32)
    rc = g(sino.ctypes.data_as(fp), n, na, tp.angles.ctypes.data_as(fp), tp.param_nofilt.ctypes.data_as(fp),
           tp.lut.ctypes.data_as(fp), tp.deapod.ctypes.data_as(fp), None, rec.ctypes.data_as(fp), None)
    assert rc == 0, _lib.last_error()
    assert rel_l2(rec, grid_golden[f"{case}/adj"]) <= TOL


MATCHED_CASES = [  # n, na, kernel, oversampling, interp, W
    (64, 90, "pswf", 2.0, "nn", 7.0),
    (96, 120, "kb", 2.0, "lin", 6.0),
    (100, 75, "kb", 1.5, "lin", 6.6),      # pdim 192, not a power of two
    (129, 61, "prolate", 2.0, "nn", 7.0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("n,na,kernel,os_,interp,W", MATCHED_CASES)
def test_matched_adjoint_passes_dot_test(cuda, n, na, kernel, os_, interp, W):
    """<A x, y> = <x, A^T y> with float64 dot products, relative to |A x| |y|."""
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    tp = cpg.projectors(n, np.linspace(0, 180, na, endpoint=False), kernel=kernel, oversampl=os_,
                        interp=interp, W=W, verbose=False, adjoint="matched")
    rng = np.random.default_rng(7)
    x = rng.standard_normal((n, n)).astype(np.float32)
    y = rng.standard_normal((na, n)).astype(np.float32)
    ax, aty = tp.A(x).astype(np.float64), tp.At(y).astype(np.float64)
    lhs, rhs = float(np.sum(ax * y)), float(np.sum(x.astype(np.float64) * aty))
    assert abs(lhs - rhs) / (np.linalg.norm(ax) * np.linalg.norm(y)) <= TOL
    # A itself is the reference's forward in both modes
    tpc = cpg.projectors(n, np.linspace(0, 180, na, endpoint=False), kernel=kernel, oversampl=os_,
                         interp=interp, W=W, verbose=False)
    assert np.array_equal(tp.A(x), tpc.A(x))


@pytest.mark.gpu
def test_matched_adjoint_agrees_with_reference_on_band_limited_in_circle_data(cuda, grid_golden):
    """On a smooth image supported well inside the inscribed circle, and its
    sinogram, the matched adjoint and the reference's (compat, same kernel
    width for PSWF W = 7) differ only by what the reference does differently at
    the edges of the padded projections and the grid: compared on the disk."""
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    n, na = 128, 180
    deg = np.linspace(0, 180, na, endpoint=False)
    kw = dict(kernel="pswf", oversampl=2.0, interp="lin", W=7.0, verbose=False)
    tpm = cpg.projectors(n, deg, adjoint="matched", **kw)
    tpc = cpg.projectors(n, deg, **kw)
    c = (np.arange(n) - n / 2 + 0.5) / (n / 2)
    X, Y = np.meshgrid(c, c)
    img = np.exp(-((X - 0.1) ** 2 + (Y + 0.05) ** 2) / (2 * 0.15 ** 2)).astype(np.float32)
    y = tpc.A(img)
    disk = X ** 2 + Y ** 2 < 0.6 ** 2
    am, ac = tpm.At(y), tpc.At(y)
    assert rel_l2(am[disk], ac[disk]) <= 1e-2


@pytest.mark.gpu
def test_admm_size_sampled_angles_match_reference(cuda):
    """The gridding pair at the ADMM-TV configuration (1536 bins, 1500 angles,
    Kaiser-Bessel W = 6, oversampling 2: a 4096^2 Fourier grid, linear
    interpolation): the full 1500-angle application on the GPU, its rows at 14
    sampled angles and the adjoint of a sinogram zero outside them (at 32768
    seeded pixels) against the reference (tests/golden/large_grid_golden.npz,
    make_large_golden.py --grid)."""
    import importlib.util
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    spec = importlib.util.spec_from_file_location("make_large_golden", GOLDEN / "make_large_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    g = np.load(GOLDEN / "large_grid_golden.npz")
    phantom, noise, rows, pix = mk.grid_inputs()
    assert np.array_equal(np.array([x.sum(dtype=np.float64) for x in (phantom, noise, rows)]), g["sums"])
    idx = g["angle_index"]
    tp = cpg.projectors(mk.N_GRID, np.linspace(0, 180, mk.NA_GRID, endpoint=False), kernel="kb", oversampl=2.0,
                        W=6.0, errs=1e-3, interp="lin", verbose=False)
    for name, img in (("phantom", phantom), ("noise", noise)):
        got = tp.A(torch.from_numpy(img).cuda()).cpu().numpy()[idx]
        ref = g[f"fwd_{name}"]
        assert rel_l2(got, ref) <= TOL, (name, rel_l2(got, ref))
        for j in range(len(idx)):
            assert rel_l2(got[j], ref[j]) <= TOL, (name, int(idx[j]), rel_l2(got[j], ref[j]))
    y = torch.zeros((mk.NA_GRID, mk.N_GRID), dtype=torch.float32, device="cuda")
    y[torch.from_numpy(idx).cuda()] = torch.from_numpy(rows).cuda()
    adj = tp.At(y).cpu().numpy().ravel()[pix]
    assert rel_l2(adj, g["adj"]) <= TOL, rel_l2(adj, g["adj"])


@pytest.mark.gpu
def test_adjoint_is_additive_over_angles(cuda):
    """The adjoint gathers, for every grid point, the polar samples of the
    angles in an angular window around it; an angle's contribution must not
    depend on which other angles the plan holds.  A row alone in a 300-angle
    plan gives what it gives in a plan of that one angle (148.8 degrees at
    256^2 once lost 2.6 % there: the scan stopped at a boundary angle that
    float rounding put just outside the window)."""
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    n, na = 256, 300
    deg = np.linspace(0, 180, na, endpoint=False).astype(np.float32)
    kw = dict(kernel="kb", oversampl=2.0, W=6.0, errs=1e-3, interp="lin", verbose=False)
    tp = cpg.projectors(n, deg, **kw)
    rng = np.random.default_rng(1)
    for k in (0, 37, 150, 246, 247, 248, 249, 299):
        row = rng.standard_normal(n).astype(np.float32)
        y = np.zeros((na, n), np.float32)
        y[k] = row
        one = cpg.projectors(n, deg[k:k + 1], **kw).At(row[None])
        assert rel_l2(tp.At(y), one) <= 1e-6, k
