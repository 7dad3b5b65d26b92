"""Filtered backprojection: projection filtering, the B-spline ``fbp`` and the
gridding ``fbp`` with every built-in filter, against the reference's outputs
(tests/golden/fbp_golden.npz, made by make_golden.py from the reference's own
filters.filter_proj and the compiled reference C).

Tolerances: host filtering is bit-exact (same numpy float64 arithmetic); the
device filter (cuFFT in float64) is within float32 rounding of it (rel L2
1e-6); the backprojections are within the projector bar (rel L2 1e-5).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

TOL = 1e-5


@pytest.fixture(scope="module")
def fbp_golden():
    return np.load(GOLDEN / "fbp_golden.npz")


def _filter_cases(g):
    return sorted(k[:-3] for k in g.files if k.startswith("filter/") and k.endswith("/in"))


def _cases(g, prefix):
    return sorted({k.split("/")[1] for k in g.files if k.startswith(prefix + "/")})


def test_filter_proj_bit_exact(fbp_golden):
    from iterative_tomographic_reconstruction_algorithms_b200.filters import filter_proj
    for case in _filter_cases(fbp_golden):
        ftype, dpc = case.split("/")[1].rsplit("_", 1)
        out = filter_proj(fbp_golden[case + "/in"].copy(), ftype=ftype, dpc=bool(int(dpc)))
        assert np.array_equal(out, fbp_golden[case + "/out"]), case


def test_hilbert_with_apodisation_raises_like_reference():
    from iterative_tomographic_reconstruction_algorithms_b200.filters import calc_filter
    with pytest.raises(NameError):
        calc_filter(64, ftype="hanning", dpc=True)


@pytest.mark.gpu
def test_device_filter_matches_reference(cuda, fbp_golden):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200.filters import filter_proj_device
    for case in _filter_cases(fbp_golden):
        ftype, dpc = case.split("/")[1].rsplit("_", 1)
        x = torch.from_numpy(fbp_golden[case + "/in"]).cuda()
        out = filter_proj_device(x, ftype=ftype, dpc=bool(int(dpc)))
        assert out.dtype == torch.float32 and out.is_cuda
        assert rel_l2(out.cpu().numpy(), fbp_golden[case + "/out"]) <= 1e-6, case
        assert np.array_equal(x.cpu().numpy(), fbp_golden[case + "/in"])  # input untouched


@pytest.mark.gpu
def test_bspline_fbp_matches_reference(cuda, fbp_golden):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_bspline as cpb
    for case in _cases(fbp_golden, "bspline"):
        n, na, deg, sup, rdeg = fbp_golden[f"bspline/{case}/cfg"]
        tp = cpb.projectors(int(n), np.zeros(int(na)), None, bspline_degree=int(deg), proj_support_y=float(sup),
                            radon_degree=int(rdeg))
        sino, ref = fbp_golden[f"bspline/{case}/sino"], fbp_golden[f"bspline/{case}/fbp"]
        host = tp.fbp(sino)
        assert rel_l2(host, ref) <= TOL, case
        dev = tp.fbp(torch.from_numpy(sino).cuda())
        assert dev.is_cuda and rel_l2(dev.cpu().numpy(), ref) <= TOL, case
        two = tp.fbp(torch.from_numpy(np.stack([sino, 2 * sino])).cuda()).cpu().numpy()
        assert np.array_equal(two[0], dev.cpu().numpy()) and rel_l2(two[1], 2 * ref) <= TOL, case


@pytest.mark.gpu
def test_gridding_fbp_every_filter_matches_reference(cuda, fbp_golden):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    for case in _cases(fbp_golden, "grid"):
        n, na, os_, interp, W, errs, rdeg, filt = fbp_golden[f"grid/{case}/cfg"]
        name = cpg.filter_list[int(filt), 0]
        tp = cpg.projectors(int(n), np.linspace(0, 180, int(na), endpoint=False),
                            kernel=str(fbp_golden[f"grid/{case}/kernel"]), oversampl=float(os_),
                            interp="nn" if interp == 0 else "lin", radon_degree=int(rdeg), W=float(W),
                            errs=float(errs), filt=name, verbose=False)
        assert int(tp.param_filt[1]) == int(filt)
        out = tp.fbp(fbp_golden[f"grid/{case}/sino"])
        assert rel_l2(out, fbp_golden[f"grid/{case}/fbp"]) <= TOL, case
