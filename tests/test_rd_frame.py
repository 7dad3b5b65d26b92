"""CPU check of the bound behind the ray-driven walks that run unchecked
(csrc/radon_rd.cu: rd_walk_framed, rd_walk_loop<false>).

Those walks read and write framed images that hold pixel rows and columns
-1 .. n+1 only, with no range test, so every pixel such a walk steps into must
lie there.  The kernel takes a walk unchecked when all four coordinates of its
entry and exit points are within nh + 1/4 of the centre and both extents have
|1/e| <= 2^64; it then also runs without the step guard, since the walk ends
after at most |ex| + |ey| + 4 steps.

This replays the reference's walk (radon_rd.c:15-71, the same arithmetic as the
FP64 oracle's orc_siddon: crossing parameters as double quotients rounded to
float) from the reference's own entry and exit points (the oracle's
orc_rd_endpoints, radon_rd.c:133-179) for every sub-ray of many angles, the
near-axis ones included, and checks both claims on every walk that qualifies
(for these geometries every walk does: the reference's end points lie on the
square up to its rounding).  Synthetic walks with end points exactly at the
threshold, nh + 1/4 off the centre, check the bound where it is tight, and
walks a little beyond it show that the threshold matters.
"""
from __future__ import annotations

import ctypes
import ctypes.util

import numpy as np
import pytest

from oracle.oracle import Oracle, radon_angles

f32, f64 = np.float32, np.float64


@pytest.fixture(scope="module")
def libs():
    L = Oracle().L
    L.orc_rd_endpoints.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                                   ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    L.orc_rd_offset.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float]
    L.orc_rd_offset.restype = ctypes.c_float
    m = ctypes.CDLL(ctypes.util.find_library("m"))
    m.sincosf.argtypes = [ctypes.c_float, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    return L, m


def endpoints(libs, theta: float, n: int):
    """Entry / exit points of every sub-ray of one general angle, float32 [M, 2] each."""
    L, m = libs
    s, c = ctypes.c_float(), ctypes.c_float()
    m.sincosf(ctypes.c_float(theta), ctypes.byref(s), ctypes.byref(c))
    if abs(s.value) < 1e-7 or abs(c.value) < 1e-7:
        return None  # row / column sums: no walk
    nh = n // 2
    p1s, p2s = [], []
    a, b = (ctypes.c_float * 2)(), (ctypes.c_float * 2)()
    for i in range(1, 6 * n):
        if i % 6 == 0:
            continue
        t = L.orc_rd_offset(i, n, ctypes.c_float(theta))
        L.orc_rd_endpoints(ctypes.c_float(theta), s, c, nh, ctypes.c_float(t), a, b)
        p1s.append((a[0], a[1]))
        p2s.append((b[0], b[1]))
    return np.array(p1s, f32), np.array(p2s, f32)


def round_half_away(x):
    return (np.sign(x) * np.floor(np.abs(x.astype(f64)) + 0.5)).astype(np.int64)


def walk(p1, p2, n):
    """The reference's walks, all at once: per walk the smallest and largest
    row and column index (plus nh) stepped into, the step count, and whether
    the walk ended (alpha > 1) within 4n + 16 steps."""
    nh = n // 2
    ex, ey = (p2[:, 0] - p1[:, 0]).astype(f32), (p2[:, 1] - p1[:, 1]).astype(f32)
    ii, jj = round_half_away(p1[:, 0]), round_half_away(p1[:, 1])
    dx = np.where(p2[:, 0] > p1[:, 0], 1, -1)
    dy = np.where(p2[:, 1] > p1[:, 1], 1, -1)
    alpha = np.zeros(len(p1), f32)
    lo_i = hi_i = ii + nh
    lo_j = hi_j = jj + nh
    steps = np.zeros(len(p1), np.int64)
    live = np.ones(len(p1), bool)
    with np.errstate(all="ignore"):
        for _ in range(4 * n + 16):
            if not live.any():
                break
            ay = ((jj.astype(f64) + 0.5 * dy - p1[:, 1].astype(f64)) / ey.astype(f64)).astype(f32)
            ax = ((ii.astype(f64) + 0.5 * dx - p1[:, 0].astype(f64)) / ex.astype(f64)).astype(f32)
            sx = live & (ax <= ay)
            sy = live & (ay <= ax)
            alpha = np.where(sx, ax, np.where(sy, ay, alpha))
            ii = ii + np.where(sx, dx, 0)
            jj = jj + np.where(sy, dy, 0)
            lo_i = np.minimum(lo_i, np.where(live, ii + nh, lo_i))
            hi_i = np.maximum(hi_i, np.where(live, ii + nh, hi_i))
            lo_j = np.minimum(lo_j, np.where(live, jj + nh, lo_j))
            hi_j = np.maximum(hi_j, np.where(live, jj + nh, hi_j))
            steps += live
            live = live & (sx | sy) & (alpha <= 1.0)
    return lo_i, hi_i, lo_j, hi_j, steps, ~live, ex, ey


def qualifies(p1, p2, ex, ey, n):
    nh = n // 2
    reach = np.maximum(np.maximum(np.abs(p1[:, 0]), np.abs(p1[:, 1])), np.maximum(np.abs(p2[:, 0]), np.abs(p2[:, 1])))
    with np.errstate(divide="ignore"):
        rx, ry = f32(1) / ex, f32(1) / ey
    return (reach <= f32(nh) + f32(0.25)) & (np.abs(rx) <= f32(2.0 ** 64)) & (np.abs(ry) <= f32(2.0 ** 64))


@pytest.mark.parametrize("n", [16, 33, 64, 128])
def test_unchecked_walks_stay_in_the_frame(libs, n):
    rng = np.random.default_rng(n)
    deg = np.concatenate([np.linspace(0, 180, 97, endpoint=False),
                          [0.001, 0.01, 0.1, 44.99, 45.0, 45.01, 89.9, 89.99, 89.999, 90.001, 90.01, 134.99,
                           135.0, 179.9, 179.99, 179.999],
                          rng.uniform(0, 180, 24)])
    total = taken = 0
    for theta in radon_angles(deg):
        ep = endpoints(libs, float(theta), n)
        if ep is None:
            continue
        p1, p2 = ep
        lo_i, hi_i, lo_j, hi_j, steps, ended, ex, ey = walk(p1, p2, n)
        q = qualifies(p1, p2, ex, ey, n)
        total += len(q)
        taken += int(q.sum())
        assert np.all(lo_i[q] >= -1) and np.all(hi_i[q] <= n + 1), theta
        assert np.all(lo_j[q] >= -1) and np.all(hi_j[q] <= n + 1), theta
        assert np.all(ended[q]), theta
        bound = np.abs(ex.astype(f64)) + np.abs(ey.astype(f64)) + 4
        assert np.all(steps[q] <= bound[q]), theta
    assert taken > 0.99 * total  # nearly every walk runs unchecked


def synthetic(rng, n, off, m=200_000):
    """Walks between random points on the sides of the square of half-size
    nh + off (entry on one side, exit on another)."""
    h = f32(n // 2 + off)
    sides = rng.integers(0, 4, (m, 2))
    sides[:, 1] = (sides[:, 0] + rng.integers(1, 4, m)) % 4
    u = rng.uniform(-1, 1, (m, 2)).astype(f32) * h

    def point(side, v):
        x = np.where(side == 0, -h, np.where(side == 1, h, v))
        y = np.where(side == 2, -h, np.where(side == 3, h, v))
        return np.stack([x, y], 1).astype(f32)

    return point(sides[:, 0], u[:, 0]), point(sides[:, 1], u[:, 1])


@pytest.mark.parametrize("n", [16, 64, 255, 256])
def test_bound_at_the_threshold(n):
    rng = np.random.default_rng(1000 + n)
    p1, p2 = synthetic(rng, n, 0.25)
    lo_i, hi_i, lo_j, hi_j, steps, ended, ex, ey = walk(p1, p2, n)
    q = qualifies(p1, p2, ex, ey, n)
    assert q.all()
    assert lo_i.min() >= -1 and hi_i.max() <= n + 1
    assert lo_j.min() >= -1 and hi_j.max() <= n + 1
    assert ended.all()
    assert np.all(steps <= np.abs(ex.astype(f64)) + np.abs(ey.astype(f64)) + 4)
    # beyond the threshold the frame no longer holds every walk
    p1, p2 = synthetic(rng, n, 0.75)
    lo_i, hi_i, lo_j, hi_j, *_ = walk(p1, p2, n)
    assert min(lo_i.min(), lo_j.min()) < -1 or max(hi_i.max(), hi_j.max()) > n + 1
