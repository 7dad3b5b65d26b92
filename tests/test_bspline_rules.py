"""CPU checks of the shortcuts the B-spline kernels (csrc/bspline.cu) take for
the reference's bin rule yi = trunc((double)fl(s + ps) + n/2)
(gen_forwproj.c:57-61), for even n:

* forward, per tap: floor(fl(s + ps)) + n/2, -1 folded onto bin 0, the double
  rule itself for t in (-1, 0);
* adjoint, per pixel and angle: floor(ps) + s + n/2 (-1 folded onto 0) for
  every tap when ps is at least 2^-12 from an integer.

Both must give the reference's bins on random and adversarial ps (next to
integers, small, half-integers)."""
from __future__ import annotations

import numpy as np
import pytest

f32 = np.float32


def _ps(n, rng):
    return np.concatenate([
        rng.uniform(-1.5 * n, 1.5 * n, 20000).astype(f32),
        (np.round(rng.uniform(-1.5 * n, 1.5 * n, 5000)) + rng.choice([-1, 1], 5000) * 2.0 ** -12).astype(f32),
        (np.round(rng.uniform(-1.5 * n, 1.5 * n, 5000)) + rng.choice([-1, 1], 5000) * 2.0 ** -24).astype(f32),
        rng.uniform(-4, 4, 5000).astype(f32), (rng.integers(-n, n, 2000) + f32(0.5)).astype(f32),
        np.array([0.0, -0.0, 1e-45, -1e-45, -1e-30, 2.0 ** -12, -(2.0 ** -12)], f32)])


@pytest.mark.parametrize("n", [4, 6, 64, 1536, 2048])
def test_bin_rules_match_the_double_rule(n):
    rng = np.random.default_rng(n)
    nh = n // 2
    ps = _ps(n, rng)
    fl = np.floor(ps)
    frac = (ps - fl).astype(f32)
    fast_ok = (frac >= f32(2.0 ** -12)) & (frac <= f32(1) - f32(2.0 ** -12))
    with np.errstate(over="ignore"):
        for s in range(-8, 9):
            t = (f32(s) + ps).astype(f32)
            exact = np.trunc(t.astype(np.float64) + nh).astype(np.int64)
            # forward rule
            fwd = np.floor(t).astype(np.int64) + nh
            fwd = np.where((fwd == -1) & (t > f32(-nh - 1)), 0, fwd)
            tiny_neg = (t < 0) & (t > -1)
            fwd = np.where(tiny_neg, exact, fwd)
            # only bins in [0, n) are used; below that both rules reject the tap
            mf = ((exact >= 0) & (exact < n)) | ((fwd >= 0) & (fwd < n))
            assert np.array_equal(fwd[mf], exact[mf])
            # adjoint rule, where it applies
            adj = fl.astype(np.int64) + s + nh
            adj = np.where(adj == -1, 0, adj)
            m = fast_ok & (((exact >= 0) & (exact < n)) | ((adj >= 0) & (adj < n)))
            assert np.array_equal(adj[m], exact[m])
