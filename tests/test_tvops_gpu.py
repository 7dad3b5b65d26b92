"""ADMM-TV / CG inner operators on the GPU (tvops.py, csrc/tv_ops.cu) against the
reference's formulas (algorithms/cg.py:62-71, utils.py:189-216) restated in
numpy: numpy.gradient, the dense-matrix Gt, and the two shrinkage rules.
G and Gt must agree bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ref_Gt(g):
    nx, ny = g[0].shape
    Gy = np.gradient(np.diag(np.ones(nx)))[1]
    Gx = np.gradient(np.diag(np.ones(ny)))[0]
    return np.dot(g[1], Gx) + np.dot(Gy, g[0])


@pytest.mark.parametrize("shape", [(2, 2), (3, 5), (64, 48), (257, 256)])
def test_gradient_and_adjoint_bit_exact(cuda, shape):
    from iterative_tomographic_reconstruction_algorithms_b200 import tvops
    rng = np.random.default_rng(0)
    m = rng.standard_normal(shape).astype(np.float32)
    g = tvops.G(m)
    ref = np.gradient(m)
    assert np.array_equal(g[0], ref[0]) and np.array_equal(g[1], ref[1])
    gg = [rng.standard_normal(shape).astype(np.float32) for _ in range(2)]
    assert np.array_equal(tvops.Gt(gg), _ref_Gt(gg))


def test_thresholds(cuda):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import tvops
    x = np.random.default_rng(1).standard_normal((2, 8, 8)).astype(np.float32)
    ref_h = np.maximum(0, x - 0.3) - np.maximum(0, -x - 0.3)
    assert np.array_equal(tvops.hard_thres(x, 0.3), ref_h)
    assert np.array_equal(tvops.hard_thres(torch.from_numpy(x).cuda(), 0.3).cpu().numpy(), ref_h)
    ref_s = x.copy()
    ref_s[x > 0.3] -= 0.3
    ref_s[np.abs(x) <= 0.3] = 0
    ref_s[x < -0.3] += 0.3
    assert np.array_equal(tvops.soft_thres(torch.from_numpy(x).cuda(), 0.3).cpu().numpy(), ref_s)
