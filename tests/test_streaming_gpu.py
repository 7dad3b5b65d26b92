"""GPU tests of the chunked multi-stream volume path (streaming.py): every
result is bit-identical to the slice-by-slice plan (a chunk runs the same
kernels on the same slices), with a slice count that is not a multiple of the
chunk, from page-locked and from pageable host memory."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["dd", "pd"])
def test_project_and_backproject_match_per_slice(cuda, kind):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.streaming import VolumeStreamer
    n, na, nz = 96, 70, 7
    tp = cpr.projectors(n, np.linspace(0, 180, na, endpoint=False), oper=kind)
    rng = np.random.default_rng(1)
    imgs = torch.from_numpy(rng.standard_normal((nz, n, n)).astype(np.float32)).pin_memory()
    sinos = torch.empty((nz, na, n), dtype=torch.float32).pin_memory()
    vs = VolumeStreamer(tp, chunk=3, slots=2)
    ms = vs.project(imgs, sinos)
    assert ms > 0
    for z in range(nz):
        assert np.array_equal(sinos[z].numpy(), tp.A(imgs[z].numpy())), z
    back = np.empty((nz, n, n), np.float32)          # pageable destination
    vs.backproject(sinos.numpy(), back)
    for z in range(nz):
        assert np.array_equal(back[z], tp.At(sinos[z].numpy())), z


def test_reconstruct_matches_per_slice_solver(cuda):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses
    from iterative_tomographic_reconstruction_algorithms_b200.solvers import sirt
    from iterative_tomographic_reconstruction_algorithms_b200.streaming import VolumeStreamer
    n, na, nz = 64, 60, 5
    tp = cpr.projectors(n, np.linspace(0, 180, na, endpoint=False), oper="dd")
    truth = np.stack([random_ellipses(n, seed=s) for s in range(nz)])
    b = tp.A(truth)
    out = torch.empty((nz, n, n), dtype=torch.float32).pin_memory()
    VolumeStreamer(tp, chunk=2, slots=3).reconstruct(torch.from_numpy(b).pin_memory(), out, "sirt", iters=7)
    for z in range(nz):
        x, _ = sirt(np.ones((n, n), np.float32), b[z], tp, n_iter=7)
        assert np.array_equal(out[z].numpy(), x), z
    with pytest.raises(ValueError):
        VolumeStreamer(tp).reconstruct(b, out.numpy(), "sps", iters=1)
