"""Every projector pair's adjoint is the transpose of its forward, entry by entry.

The reference computes each pair's forward and adjoint with one routine and an
`oper` flag (radon_pd.c:63,81-83; radon_rd.c:62-66; radon_dd.c:181-183,273-275;
radon_ss.c:93-196; gen_backproj.c:69 against gen_forwproj.c), so its A^T is
A's transpose.  Here the two directions are separate kernels with their own
arithmetic and summation orders.  On one-hot inputs the forward's column for
pixel p and the adjoint's image for sinogram entry (v, b) give the same matrix
entry, up to float rounding and with the same support: relative L2 bars over
whole images can miss a single wrong entry, this cannot.

Tolerances per entry, relative to the entry (and, where the arithmetic of the
two directions differs, a floor relative to the largest entry):
  rd       forward adds at most five equal float terms 0.2 l in walk order, the
           adjoint sums them exactly: 4 ulp, no floor.
  pd, ss, B-spline: 2^-20 of the entry plus 2^-20 of the largest entry.
  dd       the forward's prefix tables take every pixel one unit wide; in the
           reference a pixel's width is P_j+1 - P_j between float boundaries,
           exactly 1 except where the line's boundaries cross a power of two
           (or zero), where it is off by up to one ulp of the coordinate.  The
           adjoint forms the reference's gaps.  Floor: two ulps of the largest
           boundary coordinate of the angle set, nh (1 + max(|cot|, |tan|)).
           test_dd_entries_match_reference pins each direction to the
           reference's own entries.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"rd": (2.0 ** -21, 0.0), "pd": (2.0 ** -20, 2.0 ** -20), "ss": (2.0 ** -20, 2.0 ** -20),
       "dd": (2.0 ** -20, 2.0 ** -20), "bspline": (2.0 ** -20, 2.0 ** -20)}


def _proj(kind, n, deg):
    if kind == "bspline":
        from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_bspline as cpb
        return cpb.projectors(n, np.asarray(deg, np.float64), None)   # angles arange(na) 180/na
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    return cpr.projectors(n, np.asarray(deg, np.float64), oper=kind)


def dd_coordinate_ulp(n, deg):
    """One ulp of the largest pixel/detector boundary coordinate of the dd lines."""
    th = np.radians(np.asarray(deg, np.float64))
    s, c = np.abs(np.sin(th)), np.abs(np.cos(th))
    axis = (s < 1e-7) | (c < 1e-7)                     # row / column sums: no boundaries
    ratio = np.maximum(c[~axis] / s[~axis], s[~axis] / c[~axis])
    m = (n // 2) * (1.0 + ratio.max())
    return 2.0 ** (np.floor(np.log2(m)) - 23)


def _check_transpose(torch, kind, F, G, abs_floor=None):
    """F, G: the same matrix entries from the forward and from the adjoint."""
    rel, floor = TOL[kind]
    m = torch.maximum(F.abs().max(), G.abs().max())
    assert m.item() > 0
    tol = torch.maximum(F.abs(), G.abs()) * rel + (m * floor if abs_floor is None else abs_floor)
    d = (F - G).abs()
    bad = d > tol
    if bad.any():
        k = int(torch.argmax(d - tol))
        raise AssertionError(f"{kind}: {int(bad.sum())} of {bad.numel()} entries differ beyond tolerance; "
                             f"worst flat index {k}: forward {float(F.flatten()[k])!r}, "
                             f"adjoint {float(G.flatten()[k])!r} (largest entry {float(m)!r})")


def _full_matrices(torch, tp, n, na):
    X = torch.eye(n * n, device="cuda", dtype=torch.float32).view(n * n, n, n)
    F = tp.A(X).reshape(n * n, na * n)               # F[p, (v, b)] = A[(v, b), p]
    del X
    Y = torch.eye(na * n, device="cuda", dtype=torch.float32).view(na * n, na, n)
    G = tp.At(Y).reshape(na * n, n * n)              # G[(v, b), p] = (A^T e_(v,b))[p]
    del Y
    return F.t(), G


@pytest.mark.parametrize("kind", ["rd", "pd", "ss", "dd", "bspline"])
def test_full_matrix_transpose_64(cuda, kind):
    torch = cuda
    n, na = 64, 180
    deg = np.linspace(0, 180, na, endpoint=False)      # 0, 45, 90, 135 included
    F, G = _full_matrices(torch, _proj(kind, n, deg), n, na)
    _check_transpose(torch, kind, F, G, 2 * dd_coordinate_ulp(n, deg) if kind == "dd" else None)


@pytest.mark.parametrize("kind", ["rd", "pd", "ss", "dd"])
def test_full_matrix_transpose_odd(cuda, kind):
    torch = cuda
    n = 65
    deg = np.sort(np.concatenate([np.random.default_rng(4).uniform(0, 180, 57), [0.0, 45.0, 90.0, 135.0]]))
    F, G = _full_matrices(torch, _proj(kind, n, deg), n, len(deg))
    _check_transpose(torch, kind, F, G, 2 * dd_coordinate_ulp(n, deg) if kind == "dd" else None)


def test_dd_entries_match_reference(cuda, dd_entries_golden):
    """Whole columns and rows of A from the reference's own dd routine
    (tests/golden/make_dd_entries_golden.py): the adjoint reproduces the
    reference's entries; the forward within the unit-width allowance above."""
    torch = cuda
    g = dd_entries_golden
    deg, pix, ent = g["angles_deg"], g["pixels"], g["entries"]
    n = g["fwd_columns"].shape[2]
    tp = _proj("dd", n, deg)
    X = torch.zeros((len(pix), n, n), device="cuda")
    for k, (r, c) in enumerate(pix):
        X[k, r, c] = 1.0
    Y = torch.zeros((len(ent), len(deg), n), device="cuda")
    for k, (v, b) in enumerate(ent):
        Y[k, v, b] = 1.0
    fwd = tp.A(X).cpu().numpy()
    adj = tp.At(Y).cpu().numpy()
    ref_f, ref_a = g["fwd_columns"], g["adj_rows"]
    da = np.abs(adj - ref_a)
    assert (da <= np.abs(ref_a) * 2.0 ** -21).all(), f"adjoint: max |diff| {da.max()!r}"
    df = np.abs(fwd - ref_f)
    floor = 2 * dd_coordinate_ulp(n, deg)
    off = int((df > np.abs(ref_f) * 2.0 ** -21).sum())
    assert (df <= np.abs(ref_f) * 2.0 ** -21 + floor).all(), \
        f"forward: max |diff| {df.max()!r} above the unit-width floor {floor!r}"
    # the pixels whose projection straddles a power of two or zero of the line
    # coordinate: 28 of the 1250 nonzero entries here (2.2 %)
    assert off <= 0.05 * (ref_f != 0).sum(), f"forward: {off} entries off the reference's widths"


def test_sampled_transpose_2048(cuda):
    torch = cuda
    n, na = 2048, 1800
    tp = _proj("rd", n, np.linspace(0, 180, na, endpoint=False))
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
    _check_transpose(torch, "rd", f, g)
