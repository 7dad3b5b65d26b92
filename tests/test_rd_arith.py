"""CPU checks of the float-only arithmetic of the ray-driven walk
(csrc/radon_rd.cu: rd_alpha_mf, rd_walk_loop's pixel range test, rd_round_i).

The reference computes each crossing parameter as a double quotient rounded to
float, alpha = (float)(((double)a - p) / (p2 - p1)) (radon_rd.c:41-42), and the
start pixel as (int)round(p1) (radon_rd.c:23-24).  The kernel evaluates both in
float arithmetic.  These tests replay its float steps in NumPy (every float32
operation rounds to nearest; the one FMA is evaluated exactly in 80-bit long
double, where -q1 e + h always fits, and rounded once) and require:
  * every result it accepts from the fast path equals the reference's float,
    on random inputs and on quotients constructed to lie exactly on a float
    rounding midpoint (which the fast path must refuse);
  * the fallback is rare;
  * the approximation is within 2^-22 (relative) of the exact quotient;
  * the round-down-add rounding equals roundf for |x| < 2^22.
"""
from __future__ import annotations

import numpy as np
import pytest

f32, f64 = np.float32, np.float64


def _rn(x):
    return np.asarray(x, dtype=f32)


def two_sum(a, p):
    """Knuth's TwoSum of a and -p: h + l == a - p exactly."""
    h = a - p
    bb = h - a
    return h, (a - (h - bb)) + (-p - bb)


def split_numerator(a, p):
    """The walk's numerator a - p as m - f: P = rint(p), f = p - P, m = a - P
    (rd_walk_loop), then Fast2Sum (rd_alpha_mf): h + l == m - f."""
    P = np.rint(p)
    f = p - P
    m = a - P
    h = m - f
    l = -f - (h - m)
    return m, f, h, l


def alpha_ff(a, p, e):
    """rd_alpha_mf's fast path on the numerator a - p: (value, accepted)."""
    a, p, e = _rn(a), _rn(p), _rn(e)
    with np.errstate(all="ignore"):
        r = f32(1.0) / e                              # __frcp_rn
        _, _, h, l = split_numerator(a, p)
        q1 = h * r
        fma = (-(q1.astype(np.longdouble)) * e.astype(np.longdouble) + h.astype(np.longdouble)).astype(f32)
        rho = fma + l
        q2 = rho * r
        d = np.abs(q1) * f32(2.0 ** -38)
        lo = q1 + (q2 - d)
        hi = q1 + (q2 + d)
        ok = lo == hi
        s = lo
    return s, ok


def reference_alpha(a, p, e):
    with np.errstate(all="ignore"):
        return ((f64(1) * _rn(a).astype(f64) - _rn(p).astype(f64)) / _rn(e).astype(f64)).astype(f32)


def _random_inputs(rng, m, n=4096):
    nh = n // 2
    a = (rng.integers(-nh - 1, nh + 1, m) + 0.5).astype(f32)
    kind = rng.integers(0, 4, m)
    p = rng.uniform(-nh, nh, m).astype(f32)
    p = np.where(kind == 1, (rng.integers(-1, 2, m) * nh).astype(f32), p)       # entry on a side
    ulps = rng.integers(1, 2 ** 12, m) * np.where(rng.random(m) < 0.5, -1, 1)
    near = (a.view(np.int32) + ulps).astype(np.int32).view(f32)                 # a - p tiny
    p = np.where(kind == 2, near, p)
    p = np.where(kind == 3, (rng.integers(-nh, nh, m) + 0.5).astype(f32), p)    # half-integer entry
    mag = 2.0 ** rng.uniform(-8, np.log2(2 * n), m)
    e = (np.where(rng.random(m) < 0.5, -1, 1) * mag).astype(f32)
    return a, p, e


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_fast_path_matches_double_quotient(seed):
    rng = np.random.default_rng(seed)
    a, p, e = _random_inputs(rng, 2_000_000)
    s, ok = alpha_ff(a, p, e)
    ref = reference_alpha(a, p, e)
    assert np.array_equal(s[ok].view(np.uint32), ref[ok].view(np.uint32))
    assert ok.mean() > 0.999   # the double division is the rare exception


def test_midpoint_quotients_are_refused_and_near_ones_exact():
    """a - p = num with num a float32 rounding midpoint (25 significant bits) and
    e a power of two: the exact quotient is a midpoint, where only the double
    division gives the reference's (ties-to-even) result."""
    rng = np.random.default_rng(11)
    m = 200_000
    mant = rng.integers(0, 2 ** 22, m) * 2 + 1                  # odd: a true midpoint
    num = 1.0 + mant * 2.0 ** -24                               # in [1, 1.5), 25 bits
    num = num[num < 1.5]
    p = (0.5 - num).astype(f32)
    assert np.array_equal(p.astype(f64), 0.5 - num)             # representable
    a = np.full(p.shape, 0.5, f32)
    k = rng.integers(-6, 13, p.size)
    e = (np.where(rng.random(p.size) < 0.5, -1.0, 1.0) * 2.0 ** k).astype(f32)
    s, ok = alpha_ff(a, p, e)
    assert not ok.any()
    # one float ulp of the numerator away from the midpoint: accepted and exact
    p2 = np.nextafter(p, np.where(rng.random(p.size) < 0.5, -np.inf, np.inf).astype(f32))
    s2, ok2 = alpha_ff(a, p2, e)
    ref2 = reference_alpha(a, p2, e)
    assert np.array_equal(s2[ok2].view(np.uint32), ref2[ok2].view(np.uint32))


def test_exact_and_degenerate_quotients():
    a = np.array([0.5, -0.5, 1024.5, 0.5, 0.5, 3.5, 3.5], f32)
    p = np.array([0.5, -0.5, 0.0, -1.5, 0.25, 1.0, 0.5], f32)
    e = np.array([3.0, -7.0, 0.0, 2.0, 0.0, 5.0, 2.0], f32)
    s, ok = alpha_ff(a, p, e)
    ref = reference_alpha(a, p, e)
    # zero extents go to the division; exact quotients, zero numerators (+0)
    # and powers of two do not
    assert list(ok) == [True, True, False, True, False, True, True]
    assert np.array_equal(s[ok], ref[ok])   # +0 == -0 for the zero numerators


def test_approximation_error_bound():
    rng = np.random.default_rng(3)
    a, p, e = _random_inputs(rng, 1_000_000)
    approx = (a - p) * (f32(1.0) / e)
    exact = (a.astype(f64) - p.astype(f64)) / e.astype(f64)
    nz = exact != 0
    rel = np.abs(approx[nz].astype(f64) - exact[nz]) / np.abs(exact[nz])
    assert rel.max() <= 2.0 ** -22


def _add_rd(x, y):
    v = x.astype(f64) + y.astype(f64)        # exact for these magnitudes
    r = v.astype(f32)
    return np.where(r.astype(f64) > v, np.nextafter(r, f32(-np.inf)), r)


def test_round_half_away_by_round_down_adds():
    rng = np.random.default_rng(5)
    k = rng.integers(-3000, 3000, 300_000).astype(f64)
    x = np.concatenate([
        rng.uniform(-4096, 4096, 300_000).astype(f32),
        (k + 0.5).astype(f32),
        np.nextafter((k + 0.5).astype(f32), f32(np.inf)),
        np.nextafter((k + 0.5).astype(f32), f32(-np.inf)),
        np.array([0.0, -0.0, 0.49999997, -0.49999997, 0.5, -0.5, 1.5, -2.5, 2.0 ** 21 + 0.5], f32),
    ]).astype(f32)
    f = _add_rd(_add_rd(np.abs(x), np.full_like(x, 0.5)), np.full_like(x, 12582912.0))
    got = f.view(np.int32) - 0x4B400000
    got = np.where(x < 0, -got, got)
    ref = (np.sign(x.astype(f64)) * np.floor(np.abs(x.astype(f64)) + 0.5)).astype(np.int64)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("seed", [0, 1])
def test_split_numerator_is_exact(seed):
    """m and f are exact, and Fast2Sum of (m, -f) gives TwoSum's (h, l) of
    (a, -p): the same float pair, so the same quotient and the same fallback."""
    rng = np.random.default_rng(100 + seed)
    a, p, _ = _random_inputs(rng, 2_000_000)
    m, f, h, l = split_numerator(a, p)
    P = np.rint(p).astype(f64)
    assert np.array_equal(f.astype(f64), p.astype(f64) - P)
    assert np.array_equal(m.astype(f64), a.astype(f64) - P)
    assert np.all(np.abs(m) >= 0.5) and np.all(np.abs(f) <= 0.5)
    h2, l2 = two_sum(a, p)
    assert np.array_equal(h.view(np.uint32), h2.view(np.uint32))
    assert np.array_equal(l, l2)    # equal as values (+0 and -0 alike)
    # and stepping m by +-1 keeps it exact: m - f stays a - p
    for k in (1, 7, 900):
        mk = m + f32(k)
        assert np.array_equal(mk.astype(f64), (a + f32(k)).astype(f64) - P)


@pytest.mark.parametrize("n", [2, 3, 64, 255, 256, 2048, 2049])
def test_pixel_range_test(n):
    """rd_walk_loop's |mx + kx| <= n/2 - 1 is the reference's
    0 < ii + nh < n, for every pixel a walk can reach and both directions."""
    rng = np.random.default_rng(n)
    nh = n // 2
    half = f32(0.5) * f32(n)
    lim = half - f32(1)
    for hx in (f32(0.5), f32(-0.5)):
        p1 = rng.uniform(-nh - 3, nh + 3, 4000).astype(f32)
        P = np.rint(p1)
        ii = np.arange(-nh - 8, nh + 9)
        II, PP = np.meshgrid(ii, P)
        mx = (II.astype(f32) + hx) - PP                 # the next x crossing's m
        kx = ((PP - hx) + f32(nh)) - half
        got = np.abs(mx + kx) <= lim
        pi = II + nh
        assert np.array_equal(got, (pi > 0) & (pi < n))
