"""Sinogram pre-processing (preprocess.py, csrc/sino_prep.cu) and DMP files (dmp_io.py).

Edge padding and integer rotation-axis shifts are compared exactly with a
numpy restatement of the reference's arithmetic
(common/myimage/my_image_process.py:87-157: roll, then the wrapped columns
replaced by the edge column; edge columns repeated).  Fractional shifts are
compared with the reference's own interpolant, scipy's griddata(method='cubic')
on the zero-padded sinogram, restated here, on smooth data (relative L2 <= 2e-3;
the kernel uses Keys cubic convolution), and must reproduce a quadratic
exactly away from the edges.  The reference's float mgrid bounds can give
npix + 1 output columns for some centres; only the first npix are compared.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2


def _ref_integer_shift(sino, ctr):
    nang, npix = sino.shape
    shift = int(ctr - npix / 2)
    if shift > 0:
        rolled = np.roll(sino, -shift, axis=1)
        block = np.ones((1, shift)) * sino[:, npix - 1].reshape(nang, 1)
        return np.concatenate((rolled[:, :npix - shift], block), axis=1)
    rolled = np.roll(sino, -shift, axis=1)
    block = np.ones((1, -shift)) * sino[:, 0].reshape(nang, 1)
    return np.concatenate((block, rolled[:, -shift:]), axis=1)


def _ref_fractional_shift(sino, ctr, order_seed=None):
    """The reference's fractional shift; ``order_seed`` lists the same data
    points in a random order (the interpolant's triangulation, and so its
    result, depends on that order)."""
    import scipy.interpolate as interp
    nang, npix = sino.shape
    shift = ctr - npix * 0.5
    npix_pad = npix + 200
    pad = np.zeros((nang, npix_pad), np.float32)
    i1 = int((npix_pad - npix) * 0.5)
    pad[:, i1:i1 + npix] = sino
    gx1, gy1 = np.meshgrid(np.arange(npix_pad), np.arange(nang))
    z = np.dstack((gy1, gx1)).reshape(npix_pad * nang, 2)
    v = pad.reshape(-1)
    if order_seed is not None:
        p = np.random.default_rng(order_seed).permutation(len(v))
        z, v = z[p], v[p]
    gx2, gy2 = np.mgrid[0:nang, i1 + shift:i1 + npix + shift]
    return interp.griddata(z, v, (gx2, gy2), method="cubic")[:, :npix]


def _order_spread(sino, ctr, seeds=(1, 2, 3)):
    """The reference's result in the natural point order, and how far (relative
    L2) the same call moves when only the order of its input points changes."""
    r0 = _ref_fractional_shift(sino, ctr)
    return r0, max(rel_l2(_ref_fractional_shift(sino, ctr, k), r0) for k in seeds)


def _noisy_sino():
    rng = np.random.default_rng(5)
    s = _smooth_sino()
    return (s + 0.05 * rng.standard_normal(s.shape)).astype(np.float32)


def _smooth_sino(nang=12, npix=64):
    x = np.arange(npix)
    return np.stack([np.exp(-((x - 30 - 5 * np.sin(a)) / 8.0) ** 2)
                     + 0.5 * np.exp(-((x - 20 - 3 * np.cos(a)) / 5.0) ** 2)
                     for a in np.linspace(0, np.pi, nang)]).astype(np.float32)


def test_dmp_roundtrip_and_header(tmp_path):
    from iterative_tomographic_reconstruction_algorithms_b200.dmp_io import read_dmp, write_dmp
    img = np.random.default_rng(0).standard_normal((37, 53)).astype(np.float32)
    p = tmp_path / "a.DMP"
    write_dmp(p, img)
    raw = p.read_bytes()
    assert np.frombuffer(raw[:6], np.int16).tolist() == [53, 37, 0]
    assert len(raw) == 6 + 4 * img.size
    assert np.array_equal(read_dmp(p), img)


@pytest.mark.gpu
def test_dmp_pinned_and_device_reads(cuda, tmp_path):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200.dmp_io import read_dmp, write_dmp
    img = np.random.default_rng(1).standard_normal((64, 96)).astype(np.float32)
    write_dmp(tmp_path / "b.dmp", img)
    h = read_dmp(tmp_path / "b.dmp", pinned=True)
    assert h.is_pinned() and np.array_equal(h.numpy(), img)
    d = read_dmp(tmp_path / "b.dmp", to_device=True)
    torch.cuda.synchronize()
    assert d.is_cuda and np.array_equal(d.cpu().numpy(), img)


@pytest.mark.gpu
def test_edge_padding_matches_reference(cuda):
    from iterative_tomographic_reconstruction_algorithms_b200.preprocess import sino_edge_padding
    s = np.random.default_rng(2).standard_normal((7, 33)).astype(np.float32)
    for padding in (0.0, 0.1, 0.5):
        npad = int(padding * 33)
        ref = np.concatenate((np.ones((1, npad)) * s[:, :1], s, np.ones((1, npad)) * s[:, -1:]), axis=1)
        assert np.array_equal(sino_edge_padding(s, padding, verbose=False), ref.astype(np.float32))


@pytest.mark.gpu
def test_integer_centre_shift_matches_reference(cuda):
    from iterative_tomographic_reconstruction_algorithms_b200.preprocess import sino_correct_rot_axis
    s = np.random.default_rng(3).standard_normal((9, 40)).astype(np.float32)
    for ctr in (20.0, 23.0, 17.0, 39.0, 1.0, 21.0):
        assert np.array_equal(sino_correct_rot_axis(s, ctr), _ref_integer_shift(s, ctr).astype(np.float32)), ctr


def test_reference_fractional_shift_depends_on_point_order():
    """The reference's fractional shift is defined only up to the order of its
    input points: scipy's Delaunay triangulation of the regular grid (Qhull)
    splits each cell along one of two equally valid diagonals, in a pattern
    that follows its processing order, and the Clough-Tocher gradients are
    fitted over that triangulation.  Listing the same points in another order
    moves the result by ~1e-3 (smooth data) to ~1e-2 (noisy data); this is the
    scale against which the kernel's residual is judged."""
    for data, lo in ((_smooth_sino(), 3e-4), (_noisy_sino(), 3e-3)):
        for ctr in (32.3, 31.5, 33.75):
            _, spread = _order_spread(data, ctr)
            assert spread > lo, (ctr, spread)


@pytest.mark.gpu
def test_fractional_centre_shift_close_to_reference(cuda):
    from iterative_tomographic_reconstruction_algorithms_b200.preprocess import sino_correct_rot_axis
    s = _smooth_sino()
    for ctr in (32.3, 31.5, 33.75, 30.1):
        assert rel_l2(sino_correct_rot_axis(s, ctr), _ref_fractional_shift(s, ctr)) <= 2e-3, ctr
    # within the reference's own spread under a reordering of its input points
    # (measured: 0.5-0.7 x the spread on smooth data, 1.1-1.2 x on noisy data)
    for data, factor in ((s, 1.0), (_noisy_sino(), 1.5)):
        for ctr in (32.3, 31.5, 33.75, 30.1):
            r0, spread = _order_spread(data, ctr)
            assert rel_l2(sino_correct_rot_axis(data, ctr), r0) <= factor * spread, ctr
    # cubic convolution reproduces quadratics exactly (interior, no edge effects)
    x = np.arange(64, dtype=np.float64)
    q = np.tile(0.01 * x ** 2 - 0.3 * x + 2.0, (3, 1)).astype(np.float32)
    out = sino_correct_rot_axis(q, 32.25)
    want = 0.01 * (x + 0.25) ** 2 - 0.3 * (x + 0.25) + 2.0
    assert np.abs(out[:, 2:-3] - want[2:-3]).max() < 1e-4
