"""The ray-driven adjoint is the transpose of the forward.

Both directions run the same walks and form the same float terms
0.2 * l * value (radon_rd.c:62-66).  For one-hot inputs the forward's entry
A[(v, b), p] (image e_p) adds a pixel's terms, at most five (one per sub-ray),
in float in walk order; the adjoint's pixel p for the sinogram e_(v, b) is
their exact sum, rounded once.  So the two matrices have the same support and
agree to within the forward's rounding (4 ulp), entry by entry; a missed or
extra visit, or a wrong credited length, shows as a larger difference.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _proj(n, deg):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    return cpr.projectors(n, np.asarray(deg, np.float64), oper="rd")


def _check_transpose(torch, F, G):
    """F, G: the same entries from the forward and the adjoint."""
    assert torch.count_nonzero(F).item() > 0
    assert torch.equal(F != 0, G != 0), "supports differ"
    tol = torch.maximum(F.abs(), G.abs()) * 2.0 ** -21
    bad = (F - G).abs() > tol
    assert not bad.any(), f"{int(bad.sum())} of {bad.numel()} entries differ by more than 4 ulp"


@pytest.mark.parametrize("n,deg", [
    (64, np.linspace(0, 180, 180, endpoint=False)),                       # 0, 45, 90, 135 included
    (65, np.sort(np.concatenate([np.random.default_rng(4).uniform(0, 180, 57), [0.0, 45.0, 90.0, 135.0]]))),
])
def test_full_matrix_transpose(cuda, n, deg):
    torch = cuda
    tp = _proj(n, deg)
    na = len(deg)
    X = torch.eye(n * n, device="cuda", dtype=torch.float32).view(n * n, n, n)
    F = tp.A(X).view(n * n, na * n)                  # F[p, (v, b)] = A[(v, b), p]
    del X
    Y = torch.eye(na * n, device="cuda", dtype=torch.float32).view(na * n, na, n)
    G = tp.At(Y).view(na * n, n * n)                 # G[(v, b), p] = (A^T e_(v,b))[p]
    del Y
    _check_transpose(torch, F.t(), G)


def test_sampled_transpose_2048(cuda):
    torch = cuda
    n, na = 2048, 1800
    tp = _proj(n, np.linspace(0, 180, na, endpoint=False))
    rng = np.random.default_rng(9)
    pix = [(1, 1), (1, n - 1), (n - 1, 1), (n - 1, n - 1), (n // 2, n // 2), (1, n // 2), (n // 2, n - 1)]
    pix += [tuple(int(v) for v in rng.integers(1, n, 2)) for _ in range(5)]
    X = torch.zeros((len(pix), n, n), device="cuda")
    for k, (r, c) in enumerate(pix):
        X[k, r, c] = 1.0
    F = tp.A(X)                                      # [P, na, n]
    del X
    # sinogram entries in each sampled column's support, 45 and 90 degrees among them
    ent = []
    for k in range(len(pix)):
        nzv, nzb = torch.nonzero(F[k], as_tuple=True)
        pick = rng.choice(nzv.numel(), 2, replace=False)
        ent += [(int(nzv[j]), int(nzb[j])) for j in pick]
        for v in (450, 900):
            row = torch.nonzero(F[k, v]).flatten()
            if row.numel():
                ent.append((v, int(row[0])))
    Y = torch.zeros((len(ent), na, n), device="cuda")
    for k, (v, b) in enumerate(ent):
        Y[k, v, b] = 1.0
    G = tp.At(Y)                                     # [E, n, n]
    del Y
    rows = torch.tensor([r for r, _ in pix], device="cuda")
    cols = torch.tensor([c for _, c in pix], device="cuda")
    vs = torch.tensor([v for v, _ in ent], device="cuda")
    bs = torch.tensor([b for _, b in ent], device="cuda")
    g = G[:, rows, cols]                             # [E, P]
    f = F[:, vs, bs].t()                             # [E, P]
    assert torch.count_nonzero(f).item() >= len(ent)
    _check_transpose(torch, f, g)
