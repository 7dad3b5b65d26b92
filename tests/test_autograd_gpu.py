"""GPU tests of the differentiable projector (autograd.py).

* The gradient of A is the adjoint kernel (and of A^T the forward kernel),
  bit for bit.
* Central finite differences of a least-squares loss along a random
  direction agree with the autograd gradient (the loss is quadratic, so the
  difference quotient is exact up to rounding).
* The gradient agrees with the FP64 oracle's A^T (A x - b).
* Unrolled SIRT equals the fused solver's iterates; checkpointing changes
  nothing (bitwise); its gradient passes the finite-difference check.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

KINDS = ["pd", "rd", "dd", "ss"]


def _tp(kind, n=64, na=48):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    return cpr.projectors(n, np.linspace(0, 180, na, endpoint=False), oper=kind)


def _rand(torch, shape, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return torch.randn(shape, generator=g, dtype=torch.float32).cuda()


@pytest.mark.parametrize("kind", KINDS + ["bspline"])
def test_backward_is_the_adjoint_kernel(cuda, kind):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200.autograd import Projector
    if kind == "bspline":
        from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_bspline as cpb
        tp = cpb.projectors(64, np.zeros(48), None)
    else:
        tp = _tp(kind)
    op = Projector(tp)
    assert op.exact_gradient
    x = _rand(torch, (2, 64, 64), 1).requires_grad_(True)
    w = _rand(torch, (2, 48, 64), 2)
    (op(x) * w).sum().backward()
    assert torch.equal(x.grad, tp.At(w))
    y = _rand(torch, (48, 64), 3).requires_grad_(True)
    u = _rand(torch, (64, 64), 4)
    (op.T(y) * u).sum().backward()
    assert torch.equal(y.grad, tp.A(u))


@pytest.mark.parametrize("kind", KINDS)
def test_gradient_matches_finite_differences_and_oracle(cuda, oracle, kind):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200.autograd import Projector
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    tp = _tp(kind)
    op = Projector(tp)
    x = torch.from_numpy(random_ellipses(64, seed=5)).cuda().requires_grad_(True)
    b = 0.5 * tp.A(torch.from_numpy(random_ellipses(64, seed=6)).cuda())
    loss = 0.5 * ((op(x) - b) ** 2).sum()
    loss.backward()
    g = x.grad.detach()

    def L(xx):
        r = (tp.A(xx) - b).double()
        return 0.5 * float((r * r).sum())

    v = _rand(torch, (64, 64), 9)
    h = 1e-2
    fd = (L(x.detach() + h * v) - L(x.detach() - h * v)) / (2 * h)
    an = float((g.double() * v.double()).sum())
    assert abs(fd - an) <= 1e-4 * abs(an)

    xn = x.detach().cpu().numpy()
    r = oracle.radon(kind, 0, xn, tp.angles) - b.cpu().numpy().astype(np.float64)
    g_ref = oracle.radon(kind, 1, r.astype(np.float32), tp.angles)
    assert rel_l2(g.cpu().numpy(), g_ref) <= 1e-5


def test_gridding_gradient_is_flagged_inexact(cuda):
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    from iterative_tomographic_reconstruction_algorithms_b200.autograd import Projector
    tp = cpg.projectors(64, np.linspace(0, 180, 48, endpoint=False), verbose=False)
    assert not Projector(tp).exact_gradient
    tpm = cpg.projectors(64, np.linspace(0, 180, 48, endpoint=False), verbose=False, adjoint="matched")
    assert Projector(tpm).exact_gradient


def test_matched_gridding_gradient_matches_finite_differences(cuda):
    """With the matched adjoint the backward of A is A^T exactly: the gradient
    of 0.5 |A x - b|^2 along a random direction equals the central difference."""
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_grid as cpg
    from iterative_tomographic_reconstruction_algorithms_b200.autograd import Projector
    n, na = 64, 60
    tp = cpg.projectors(n, np.linspace(0, 180, na, endpoint=False), kernel="kb", W=6.0, interp="lin",
                        verbose=False, adjoint="matched")
    op = Projector(tp)
    g = torch.Generator().manual_seed(3)
    x = torch.randn((n, n), generator=g).cuda().requires_grad_(True)
    b = torch.randn((na, n), generator=g).cuda()
    d = torch.randn((n, n), generator=g).cuda()
    loss = 0.5 * ((op(x) - b) ** 2).sum(dtype=torch.float64)
    loss.backward()
    gd = float((x.grad.double() * d.double()).sum())
    eps = 1e-2
    with torch.no_grad():
        lp = 0.5 * ((op(x + eps * d) - b).double() ** 2).sum()
        lm = 0.5 * ((op(x - eps * d) - b).double() ** 2).sum()
    fd = float((lp - lm) / (2 * eps))
    assert abs(gd - fd) <= 1e-4 * abs(fd)


def test_unrolled_sirt_matches_fused_solver_and_checkpointing(cuda):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200.autograd import (Projector, sirt_unrolled,
                                                                               sirt_weights)
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    from iterative_tomographic_reconstruction_algorithms_b200.solvers import sirt
    tp = _tp("dd", 96, 120)
    op = Projector(tp)
    truth = torch.from_numpy(random_ellipses(96, seed=11)).cuda()
    b = tp.A(truth)
    x0 = torch.ones(96, 96, device="cuda")
    x_fused, _ = sirt(np.ones((96, 96), np.float32), b.cpu().numpy(), tp, n_iter=5)
    with torch.no_grad():
        x_unr = sirt_unrolled(op, b, x0, 5)
    assert rel_l2(x_unr.cpu().numpy(), x_fused) <= 1e-5

    W = sirt_weights(op, x0)
    grads = []
    for ck in (True, False):
        z = x0.clone().requires_grad_(True)
        out = sirt_unrolled(op, b, z, 5, weights=W, use_checkpoint=ck)
        ((out - truth) ** 2).sum().backward()
        grads.append(z.grad.clone())
    assert torch.equal(grads[0], grads[1])

    def J(z):
        with torch.no_grad():
            out = sirt_unrolled(op, b, z, 5, weights=W)
            return float(((out - truth).double() ** 2).sum())

    v = _rand(torch, (96, 96), 12)
    h = 1e-2
    fd = (J(x0 + h * v) - J(x0 - h * v)) / (2 * h)
    an = float((grads[0].double() * v.double()).sum())
    assert abs(fd - an) <= 1e-3 * abs(an)
