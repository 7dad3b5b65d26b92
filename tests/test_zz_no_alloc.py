"""GPU test of tomo_radon_dd_forward_noalloc, the distance-driven forward
projection for callers that cannot allocate device memory (their memory belongs
to another allocator, or they must not allocate inside a latency-bound loop).

The entry point is called through the C ABI on three inputs in a row, the
last one filling the static scratch exactly (one 2048 x 2048 slice), and each
result is compared with the plan-based forward (tomo_forward) and with the
FP64 oracle within the tolerance of the other projector tests.  Also checked:
requests beyond the static scratch are rejected with TOMO_EINVAL.
This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes on its own in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _noalloc(lib, x, n, ang, nz, out, stream):
    fp = ctypes.POINTER(ctypes.c_float)
    fn = lib.tomo_radon_dd_forward_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, fp, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                   ctypes.c_void_p]
    return fn(x.data_ptr(), n, ang.ctypes.data_as(fp), len(ang), nz, out.data_ptr(), stream)


def test_noalloc_forward_matches_plan_forward_and_oracle(cuda, oracle):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    from iterative_tomographic_reconstruction_algorithms_b200.class_projectors_radon import shim_angles
    from oracle.oracle import radon_angles
    rng = np.random.default_rng(99)
    stream = torch.cuda.current_stream().cuda_stream
    for n, na, nz in [(256, 304, 2), (193, 120, 1), (2048, 24, 1)]:
        deg = np.linspace(0, 180, na, endpoint=False)
        ang = shim_angles("dd", radon_angles(deg))
        x = torch.from_numpy(rng.standard_normal((nz, n, n)).astype(np.float32)).cuda()
        out = torch.full((nz, na, n), float("nan"), device="cuda")
        rc = _noalloc(_lib.lib, x, n, ang, nz, out, stream)
        assert rc == 0, _lib.last_error()
        plan = _lib.Plan(_lib.KIND_DD, n, ang, nz=nz)
        ref = plan.forward(x)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert rel_l2(got, ref.cpu().numpy()) <= TOL
        xh = x.cpu().numpy()
        for z in range(nz):
            assert rel_l2(got[z], oracle.radon("dd", 0, xh[z], radon_angles(deg))) <= TOL


def test_noalloc_rejects_oversized_requests(cuda):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    ang = np.linspace(0, 3.0, 8).astype(np.float32)
    x = torch.zeros(1, device="cuda")
    out = torch.zeros(1, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert _noalloc(_lib.lib, x, 2049, ang, 1, out, stream) == _lib.TOMO_EINVAL
    assert "static scratch" in _lib.last_error()
    assert _noalloc(_lib.lib, x, 1024, ang, 5, out, stream) == _lib.TOMO_EINVAL
