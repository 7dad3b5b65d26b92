"""ADMM (Lasso-L1, Lasso-TV) and plain CG on the device (admm.py, csrc/admm.cu)
against the reference's own solver functions (algorithms/admm.py, cg.py).

tests/golden/admm_golden.npz holds the reference's outputs: admm.conj_grad,
admm.lasso_l1 and admm.lasso_tv imported from the reference tree and run over
the compiled reference projectors (tests/golden/make_admm_golden.py).
oracle/admm_oracle.py restates those loops; with numpy's inner products it
reproduces every case bit for bit (CPU test below), which pins the types and
rounding the kernels follow.

Tolerances (rel L2 of the final image): max(1e-4, 3 x floor), where each
case's floor (stored with the fixture) is how far the reference's OWN result
moves when its projector accumulates in float64 instead of float32, the same
solver and geometry otherwise.  The well-conditioned cases have floors of
2e-6 to 7e-6 and keep the 1e-4 solver bar; float32 CG (cg_n48, floor 9.0e-4)
and Lasso-L1 with a weak L2 term (l1_n48, floor 3.2e-4) amplify rounding of
1.5e-7 per projector application by three orders of magnitude, so a
projector that rounds differently from the reference's C -- as any GPU
accumulation order does -- can only be held to a few times that spread.
The gridding case has no float64 oracle (floor 0, bar 1e-4).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2


@pytest.fixture(scope="module")
def admm_golden():
    return np.load(GOLDEN / "admm_golden.npz")


def _cases(g):
    return sorted({k.split("/")[0] for k in g.files})


def _cfg(g, name):
    n, na, nz, l1, l2, mu, n1, n2, pc, e1, e2 = g[f"{name}/cfg"]
    return dict(n=int(n), na=int(na), nz=int(nz), l1=float(l1), l2=float(l2), mu=float(mu), n1=int(n1),
                n2=int(n2), pc=float(pc), edge=None if e1 < 0 else (int(e1), int(e2)), reg=str(g[f"{name}/reg"]))


def test_oracle_reproduces_reference(reflib, admm_golden):
    from oracle import admm_oracle as ao
    from oracle.oracle import radon_angles
    from iterative_tomographic_reconstruction_algorithms_b200 import gridrec_lut as glut
    for name in _cases(admm_golden):
        c = _cfg(admm_golden, name)
        deg = np.linspace(0, 180, c["na"], endpoint=False)
        if name.startswith("grid"):
            W, lut, deapod = glut.configure_regridding(c["n"], "kb", 1.5, "lin", 6.6, 6e-6)
            prm = np.array([0.0, 0, 0, 1.5, 1, len(lut) - 5, W, 0], np.float32)
            d32, l32, a32 = deg.astype(np.float32), lut.astype(np.float32), deapod.astype(np.float32)
            A = lambda x: reflib.gridrec(0, np.asarray(x).astype(np.float32), d32, prm, l32, a32)  # noqa: E731
            At = lambda y: reflib.gridrec(1, np.asarray(y).astype(np.float32), d32, prm, l32, a32)  # noqa: E731
        else:
            ang = radon_angles(deg)
            A = lambda x: reflib.radon("dd", 0, np.asarray(x).astype(np.float32), ang)  # noqa: E731
            At = lambda y: reflib.radon("dd", 1, np.asarray(y).astype(np.float32), ang)  # noqa: E731
        b = admm_golden[f"{name}/b"]
        x0 = np.ones((c["nz"], c["n"], c["n"]), np.float32)
        if c["reg"] == "cg":
            x = x0.copy()
            x[0] = ao.cg_plain(x0[0], b[0], A, At, c["n1"])
        else:
            x = ao.admm(x0, b, A, At, c["reg"], c["l1"], c["l2"], c["mu"], c["n1"], c["n2"], c["pc"], c["edge"])
        assert np.array_equal(x, admm_golden[f"{name}/x"]), name


def _projector(name, c):
    deg = np.linspace(0, 180, c["na"], endpoint=False)
    if name.startswith("grid"):
        from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
        return cpg.projectors(c["n"], deg, kernel="kb", oversampl=1.5, W=6.6, errs=6e-6, interp="lin", verbose=False)
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    return cpr.projectors(c["n"], deg, oper="dd")


def _param(c):
    from iterative_tomographic_reconstruction_algorithms_b200.admm import Param
    p = Param(lambd1=c["l1"], lambd2=c["l2"], mu=c["mu"], n_iter=c["n1"], n_iter_pcg=c["n2"], pc=c["pc"])
    if c["edge"] is not None:
        p.edge_padding, p.index_start, p.index_end = 1.0, c["edge"][0], c["edge"][1]
    return p


@pytest.mark.gpu
def test_device_solvers_match_reference(cuda, admm_golden):
    from iterative_tomographic_reconstruction_algorithms_b200 import admm
    fn = {"lasso-tv": admm.lasso_tv, "lasso": admm.lasso_l1, "cg": admm.conj_grad}
    for name in _cases(admm_golden):
        c = _cfg(admm_golden, name)
        tp = _projector(name, c)
        x0 = np.ones((c["nz"], c["n"], c["n"]), np.float32)
        x, info = fn[c["reg"]](x0, admm_golden[f"{name}/b"], tp, _param(c))
        assert x is x0  # updated in place, as the reference does
        floor = float(admm_golden[f"{name}/floor"][0])
        tol = max(1e-4, 3.0 * floor)
        assert rel_l2(x, admm_golden[f"{name}/x"]) <= tol, (name, rel_l2(x, admm_golden[f"{name}/x"]), tol)
        ref_info = admm_golden[f"{name}/info"]
        info = np.asarray(info)
        assert info.shape == ref_info.shape, name
        itol = 2e-2 if floor > 1e-4 else 2e-3
        for col in (0, 1, 2):
            if c["reg"] == "cg" and col == 1:
                assert np.all(info[:, 1] == 0.0)
                continue
            assert np.allclose(info[:, col], ref_info[:, col], rtol=itol, atol=1e-6), (name, col, info, ref_info)


@pytest.mark.gpu
def test_deterministic_graph_and_slices(cuda, admm_golden):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200.admm import AdmmSolver
    name = "tv_n48"
    c = _cfg(admm_golden, name)
    tp = _projector(name, c)
    b = torch.from_numpy(admm_golden[f"{name}/b"]).cuda()
    kw = dict(lambd1=c["l1"], lambd2=c["l2"], mu=c["mu"], n_iter_pcg=c["n2"])
    runs = []
    for use_graph in (True, True, False):
        s = AdmmSolver(tp, "lasso-tv", b, **kw)
        x = torch.ones((c["nz"], c["n"], c["n"]), device="cuda")
        st = s.run(x, 2, reset=True, use_graph=use_graph)
        st2 = s.run(x, 1, reset=False, use_graph=use_graph)
        runs.append((x.cpu().numpy(), np.concatenate([st, st2])))
    for x, st in runs[1:]:
        assert np.array_equal(x, runs[0][0]) and np.array_equal(st, runs[0][1])
    # slices are independent: slice 1 alone gives the same bits as in the batch of two
    s1 = AdmmSolver(tp, "lasso-tv", b[1:].contiguous(), **kw)
    x1 = torch.ones((1, c["n"], c["n"]), device="cuda")
    s1.run(x1, 2, reset=True)
    s1.run(x1, 1, reset=False)
    assert np.array_equal(x1.cpu().numpy()[0], runs[0][0][1])


@pytest.mark.gpu
def test_three_runs_equal_one_continued(cuda, admm_golden):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200.admm import AdmmSolver
    name = "l1_n48"
    c = _cfg(admm_golden, name)
    tp = _projector(name, c)
    b = torch.from_numpy(admm_golden[f"{name}/b"]).cuda()
    s = AdmmSolver(tp, "lasso", b, c["l1"], c["l2"], c["mu"], c["n2"])
    xa = torch.ones((c["nz"], c["n"], c["n"]), device="cuda")
    s.run(xa, 3, reset=True)
    xb = torch.ones_like(xa)
    for k in range(3):
        s.run(xb, 1, reset=(k == 0))
    assert torch.equal(xa, xb)
