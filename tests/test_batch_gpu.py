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


FWD_SHAPES = ["w2w", "w4w", "w8w", "w2b", "w4b", "w8b"]
ADJ_SHAPES = ["t1", "t2", "t4"]


def test_every_launch_shape_gives_the_same_bits(cuda):
    """Every forward / adjoint launch shape the autotuner may pick, on single
    plans (odd and even sides, special angles, several slices) and on the
    uneven batch."""
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    rng = np.random.default_rng(11)
    special = np.array([0.0, 30.0, 45.0, 60.0, 90.0, 120.0, 135.0, 150.0, 179.5]) * np.pi / 180
    from iterative_tomographic_reconstruction_algorithms_b200.class_projectors_radon import shim_angles
    plans = [_lib.Plan(_lib.KIND_DD, 300, _angles(250), nz=2), _lib.Plan(_lib.KIND_DD, 97, _angles(61), nz=1),
             _lib.Plan(_lib.KIND_DD, 48, shim_angles("dd", special.astype(np.float32)), nz=1), _batch()]
    for p in plans:
        img = torch.from_numpy(rng.standard_normal(p.image_shape).astype(np.float32)).cuda()
        sino = torch.from_numpy(rng.standard_normal(p.sino_shape).astype(np.float32)).cuda()
        p.set_tuning("w2w", "t1")
        f0, a0 = p.forward(img), p.adjoint(sino)
        for s in ADJ_SHAPES:
            p.set_tuning(None, s)
            assert torch.equal(p.adjoint(sino), a0), (p.image_shape, s)
        for s in FWD_SHAPES:
            p.set_tuning(s, None)
            assert torch.equal(p.forward(img), f0), (p.image_shape, s)
        assert "set by the caller" in p.tuning()
        with pytest.raises(ValueError):
            p.set_tuning(None, "w2w")  # adjoint shapes are t1 / t2 / t4


def test_launch_shape_in_fused_solvers(cuda):
    """The solvers' adjoint epilogues (SIRT update, SPS clip, MLEM) under two adjoint shapes."""
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    from iterative_tomographic_reconstruction_algorithms_b200.solvers import Solver
    n, na = 128, 90
    x_true = torch.from_numpy(random_ellipses(n, seed=5)).cuda()[None].contiguous()
    for algo in ("sirt", "sps", "em"):
        out = []
        for adj in ("t1", "t4"):
            p = _lib.Plan(_lib.KIND_DD, n, _angles(na), nz=1)
            p.set_tuning(None, adj)
            b = p.forward(x_true)
            x, res = Solver(p, algo, b).run(torch.ones_like(x_true), 5)
            out.append((x, res))
        assert torch.equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1]), algo
