"""The property the angle-sharded slice rests on (sharding.AngleShardedProjector),
on the GPU with the real kernels: plans for contiguous shares of the angles give
the whole plan's rows bit for bit (each angle's row depends on that angle
alone), in one contiguous block of rows per share, and their adjoints sum to the
whole adjoint up to rounding (the same terms, summed in another order).  The
shares run one after another in one process on one GPU; the collectives
themselves are tested over gloo in tests/test_sharding.py.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

KINDS = {"pd": 0, "rd": 1, "dd": 2, "ss": 3}


@pytest.mark.parametrize("kind", list(KINDS))
def test_angle_shares_match_the_whole_plan(cuda, kind):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    from iterative_tomographic_reconstruction_algorithms_b200.sharding import _REVERSED_ROWS, angle_shards
    n, na, world = 128, 91, 3
    rng = np.random.default_rng(31)
    angles = np.linspace(0.0, np.pi, na, endpoint=False).astype(np.float32) + np.float32(0.013)
    x = torch.from_numpy(rng.standard_normal((n, n)).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.standard_normal((na, n)).astype(np.float32)).cuda()
    K = KINDS[kind]
    whole = _lib.Plan(K, n, angles)
    rows_whole = whole.forward(x).reshape(na, n)
    img_whole = whole.adjoint(y).reshape(n, n)
    img_sum = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    for a, b in angle_shards(na, world):
        part = _lib.Plan(K, n, angles[a:b])
        r0 = (na - b) if K in _REVERSED_ROWS else a
        rows = part.forward(x).reshape(b - a, n)
        assert torch.equal(rows, rows_whole[r0:r0 + b - a]), (kind, a, b)
        img_sum += part.adjoint(y[r0:r0 + b - a].contiguous()).reshape(n, n).double()
        part.close()
    whole.close()
    assert rel_l2(img_sum.cpu().numpy(), img_whole.cpu().numpy()) < 1e-6
