"""GPU tests of batched distance-driven plans (uneven geometries, one persistent launch).

A batch plan must give, for every instance, exactly the result of a plan
built for that geometry alone (the kernels assign every output element to one
lane with a fixed summation order, whatever the mix of instances), and the
fused solvers must run on it unchanged.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

GEOMS = [(96, 120, 1), (33, 16, 2), (64, 48, 1), (65, 37, 3), (128, 45, 1)]


def _angles(na):
    from iterative_tomographic_reconstruction_algorithms_b200.class_projectors_radon import shim_angles
    deg = np.linspace(0, 180, na, endpoint=False)
    return shim_angles("dd", (deg * np.pi / 180).astype(np.float32))


def _batch():
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    return _lib.BatchPlan([(n, _angles(na), nz) for n, na, nz in GEOMS])


def test_layout_and_tuning(cuda):
    bp = _batch()
    assert bp.instances == sum(nz for _, _, nz in GEOMS)
    assert bp.img_total == sum(n * n * nz for n, _, nz in GEOMS)
    assert bp.sino_total == sum(na * n * nz for n, na, nz in GEOMS)
    assert "fwd w" in bp.tuning()


def test_batch_equals_per_geometry_plans(cuda):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    bp = _batch()
    rng = np.random.default_rng(3)
    imgs, sinos = [], []
    for n, na, nz in GEOMS:
        for z in range(nz):
            imgs.append(torch.from_numpy(random_ellipses(n, seed=100 + n + z)).cuda())
            sinos.append(torch.from_numpy(rng.standard_normal((na, n)).astype(np.float32)).cuda())
    fwd = bp.unpack(bp.forward(bp.pack(imgs)), "sino")
    adj = bp.unpack(bp.adjoint(bp.pack(sinos, "sino")), "img")
    i = 0
    for n, na, nz in GEOMS:
        single = _lib.Plan(_lib.KIND_DD, n, _angles(na), nz=nz)
        f1 = single.forward(torch.stack(imgs[i:i + nz]))
        a1 = single.adjoint(torch.stack(sinos[i:i + nz]))
        for z in range(nz):
            assert torch.equal(fwd[i + z], f1[z]), (n, na, z)
            assert torch.equal(adj[i + z], a1[z]), (n, na, z)
        i += nz


def test_batch_matches_oracle(cuda, oracle):
    torch = cuda
    bp = _batch()
    rng = np.random.default_rng(5)
    imgs = [rng.standard_normal((n, n)).astype(np.float32) for n, na, nz in GEOMS for _ in range(nz)]
    out = bp.unpack(bp.forward(bp.pack(imgs)), "sino")
    i = 0
    for n, na, nz in GEOMS:
        deg = np.linspace(0, 180, na, endpoint=False)
        ang = (deg * np.pi / 180).astype(np.float32)
        for z in range(nz):
            assert rel_l2(out[i], oracle.radon("dd", 0, imgs[i], ang)) <= 1e-5
            i += 1


def test_batched_sirt_equals_single_sirt(cuda):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    from iterative_tomographic_reconstruction_algorithms_b200.solvers import Solver
    bp = _batch()
    truth = [torch.from_numpy(random_ellipses(n, seed=7 + n + z)).cuda()
             for n, na, nz in GEOMS for z in range(nz)]
    b = bp.forward(bp.pack(truth))
    xb, res = Solver(bp, "sirt", b).run(torch.ones(bp.img_total, device="cuda"), 10)
    xs = bp.unpack(xb, "img")
    bs = bp.unpack(b, "sino")
    i = 0
    for n, na, nz in GEOMS:
        for z in range(nz):
            single = _lib.Plan(_lib.KIND_DD, n, _angles(na), nz=1)
            x1, _ = Solver(single, "sirt", bs[i].reshape(1, na, n).contiguous()).run(
                torch.ones((1, n, n), device="cuda"), 10)
            assert torch.equal(xs[i], x1[0]), (n, na, z)
            i += 1
    assert res[-1] < res[0]
