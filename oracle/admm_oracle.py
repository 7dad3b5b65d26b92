"""Oracle of the ADMM / CG solvers: TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's solver loops with the reference's
array types and NumPy 2 promotion -- only the test-suite may use it:

* ``cg_plain``      algorithms/cg.py:83-185 (as admm.py:245-288 calls it)
* ``cg_lasso``      algorithms/cg.py:189-253 (Lasso-L1 inner CG)
* ``cg_tv``         algorithms/cg.py:256-320 (Lasso-TV inner CG)
* ``admm``          algorithms/admm.py:291-457 (lasso_l1), :470-640 (lasso_tv)
* ``G`` / ``Gt``    algorithms/cg.py:62-71 (numpy.gradient; dense Gt)
* ``hard_thres``, ``phys_constr``, ``circle``  algorithms/utils.py:171-256

The inner products are numpy's (``np.inner``; float32 arrays give float32
numbers), so with a projector pair that reproduces the reference's, the
iterates are the reference's bit for bit (tests/test_admm.py pins this
against tests/golden/admm_golden.npz).  ``dots="double"`` accumulates every
inner product in float64 instead -- the choice the device kernels make -- to
measure how far the reference's float32 results move with that alone.
Masks, plotting and check-point output are not restated.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32
SPACING = np.spacing(1)  # a float64 scalar, as the reference adds it


def _dot(a, b, dots):
    if dots == "numpy":
        return np.inner(a.reshape(-1), b.reshape(-1))
    s = float(np.dot(a.reshape(-1).astype(np.float64), b.reshape(-1).astype(np.float64)))
    return f32(s) if (a.dtype == np.float32 and b.dtype == np.float32) else s


def G(m):
    return np.gradient(m)


def Gt(g):
    nx, ny = g[0].shape
    gy = np.gradient(np.diag(np.ones(nx)))[1]
    gx = np.gradient(np.diag(np.ones(ny)))[0]
    return np.dot(g[1], gx) + np.dot(gy, g[0])


def hard_thres(x, beta):
    return np.maximum(0, x - beta) - np.maximum(0, -x - beta)


def phys_constr(x, beta):
    x[x < 0] *= beta
    return x


def circle(img):
    """Zero outside the inscribed circle of the last two axes (utils.py:229-256)."""
    m, n = img.shape[-2:]
    cx, cy = m * 0.5 - 0.5, n * 0.5 - 0.5
    d = min(cx, cy)
    X, Y = np.meshgrid(np.arange(m), np.arange(n))
    i = np.argwhere(np.sqrt((X - cx) ** 2 + (Y - cy) ** 2) > d)
    img[..., i[:, 0], i[:, 1]] = 0
    return img


def cg_plain(x, b, A, At, niter, dots="numpy"):
    r = At(b) - At(A(x))
    p = r.copy()
    for _ in range(niter):
        hp = At(A(p))
        alpha = _dot(r, r, dots) / (_dot(p, hp, dots) + SPACING)
        x = (x + alpha * p).astype(f32)
        r_old = r.astype(f32)
        r = (r - alpha * hp).astype(f32)
        p = (r + _dot(r, r, dots) / (_dot(r_old, r_old, dots) + SPACING) * p).astype(f32)
    return x


def cg_lasso(x, b, A, At, niter, v, lambd1, mu, dots="numpy"):
    r = At(b) + v - (At(A(x)) + (lambd1 + mu) * x)
    p = r.copy()
    for _ in range(niter):
        hp = At(A(p)) + (lambd1 + mu) * p
        alpha = _dot(r, r, dots) / (_dot(p, hp, dots) + SPACING)
        x = (x + alpha * p).astype(f32)
        r_old = r.copy()
        r = (r - alpha * hp).astype(f32)
        p = r + _dot(r, r, dots) / _dot(r_old, r_old, dots) * p
    return x


def cg_tv(x, b, A, At, niter, v, lambd1, mu, dots="numpy"):
    r = At(b) + Gt(v) - (At(A(x)) + lambd1 * x + Gt(G(x)))
    p = r.copy()
    for _ in range(niter):
        hp = (At(A(p)) + lambd1 * p + mu * Gt(G(p))).astype(f32)
        alpha = _dot(r, r, dots) / (_dot(p, hp, dots) + SPACING)
        x = (x + alpha * p).astype(f32)
        r_old = r.astype(f32)
        r = r - alpha * hp
        p = r + _dot(r, r, dots) / _dot(r_old, r_old, dots) * p
    return x


def admm(x, b, A, At, reg, lambd1, lambd2, mu, n_iter, n_iter_pcg, pc=-1.0, region=None, dots="numpy"):
    """lasso_l1 (reg "lasso") or lasso_tv (reg "lasso-tv") from x [nz, n, n]; returns x."""
    lambd1, lambd2, mu, pc = f32(lambd1), f32(lambd2), f32(mu), f32(pc)
    x = np.array(x, f32)
    nz, n = x.shape[0], x.shape[-1]
    i1, i2 = (0, n) if region is None else region
    tv = reg == "lasso-tv"
    u = np.zeros((nz, 2, n, n) if tv else (nz, n, n), f32)
    alpha = u.copy()
    inner = cg_tv if tv else cg_lasso
    for _ in range(n_iter):
        for s in range(nz):
            x[s] = inner(x[s], b[s], A, At, n_iter_pcg, mu * u[s] - alpha[s], lambd1, mu, dots)
        if pc >= 0.0:
            sub = x[:, i1:i2, i1:i2]
            if pc == 1.0:
                phys_constr(sub, f32(0.0))
                circle(sub)
            if pc == 2.0:
                circle(sub)
            else:
                phys_constr(sub, pc)
        for s in range(nz):
            g = np.asarray(G(x[s])) if tv else x[s]
            u[s] = hard_thres(g + alpha[s] / mu, lambd2 / mu)
            alpha[s] += g - u[s]
    return x
