"""GPU tests of the learned warm start's tensor-core kernels (nn.py, libtomo_nn.so).

Every kernel is checked against a CPU FP64 torch computation on the same
BF16-rounded operands: the GEMM, the 3x3 convolution, its input and weight
gradients, the 1x1 head, Adam, and a whole U-Net forward/backward.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf(torch, shape, seed, scale=1.0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(shape, generator=g) * scale).to(torch.bfloat16)


def _relerr(torch, a, b):
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    return float((a - b).abs().max() / max(float(b.abs().max()), 1e-30))


@pytest.mark.parametrize("M,N,K", [(128, 32, 64), (200, 8, 96), (1000, 64, 264), (384, 96, 128),
                                   (256, 128, 512), (130, 256, 72)])
def test_gemm_matches_fp64(cuda, M, N, K):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import nn
    A, B = _bf(torch, (M, K), 1), _bf(torch, (N, K), 2)
    bias = torch.randn(N).float()
    ref = A.double() @ B.double().T + bias.double()
    out = nn.gemm(A.cuda(), B.cuda(), bias=bias.cuda())
    nn.check_status()
    assert _relerr(torch, out, ref) < 1e-5
    out_r = nn.gemm(A.cuda(), B.cuda(), bias=bias.cuda(), relu=True, out_dtype=torch.bfloat16)
    assert _relerr(torch, out_r, ref.clamp(min=0)) < 1e-2


@pytest.mark.parametrize("B,H,W,Cin,Cout", [(1, 16, 16, 8, 32), (2, 24, 40, 32, 64), (1, 64, 64, 64, 128),
                                            (2, 12, 8, 16, 256)])
def test_conv3x3_forward_and_gradients(cuda, B, H, W, Cin, Cout):
    torch = cuda
    import torch.nn.functional as F
    from iterative_tomographic_reconstruction_algorithms_b200 import nn
    X = _bf(torch, (B, H, W, Cin), 3)
    Wt = _bf(torch, (Cout, 3, 3, Cin), 4, scale=0.1)
    b = torch.randn(Cout).float()
    dY = _bf(torch, (B, H, W, Cout), 5)
    # FP64 reference on the BF16-rounded operands
    Xr = X.double().permute(0, 3, 1, 2).requires_grad_(True)
    Wr = Wt.double().permute(0, 3, 1, 2).requires_grad_(True)
    br = b.double().requires_grad_(True)
    Yr = F.conv2d(Xr, Wr, br, padding=1)
    Yr.backward(dY.double().permute(0, 3, 1, 2))
    Y = nn.conv3x3(X.cuda(), Wt.cuda(), b.cuda(), out_dtype=torch.float32)
    nn.check_status()
    assert _relerr(torch, Y.permute(0, 3, 1, 2), Yr) < 1e-5
    # input gradient: the same kernel over dY with flipped, transposed weights
    Wb, Wd = nn.prepare_weights(Wt.float().reshape(Cout, 9, Cin).cuda())
    assert torch.equal(Wb.cpu(), Wt.reshape(Cout, 9, Cin))
    dX = nn.conv3x3(dY.cuda(), Wd.reshape(Cin, 3, 3, Cout), out_dtype=torch.float32)
    assert _relerr(torch, dX.permute(0, 3, 1, 2), Xr.grad) < 1e-5
    dW, db = nn.wgrad(X.cuda(), dY.cuda(), 9)
    nn.check_status()
    assert _relerr(torch, dW.reshape(Cout, 3, 3, Cin).permute(0, 3, 1, 2), Wr.grad) < 1e-5
    assert _relerr(torch, db, br.grad) < 1e-5


def test_unet_matches_fp64_reference(cuda):
    torch = cuda
    import torch.nn.functional as F
    from iterative_tomographic_reconstruction_algorithms_b200 import nn
    net = nn.UNet(levels=3, base=16, seed=1).cuda()
    with torch.no_grad():  # a non-zero head so that every layer gets a gradient
        net.head_w.copy_(torch.randn(net.head_w.shape) * 0.1)
    x = torch.rand(2, 32, 32, device="cuda")
    tgt = torch.rand(2, 32, 32, device="cuda")
    out = net(x)
    loss = ((out - tgt) ** 2).sum()
    loss.backward()
    nn.check_status()

    # FP64 CPU re-statement of the same network (activations rounded to BF16 where the kernels round)
    def q(t):
        return t.to(torch.bfloat16).double()

    params = {n: p.detach().double().cpu().requires_grad_(True) for n, p in net.named_parameters()}
    h = torch.zeros(2, 8, 32, 32, dtype=torch.float64)
    h[:, 0] = q(x.cpu())
    skips = []
    for lvl in range(net.levels):
        for k in range(2):
            w = q(params[f"enc.{4 * lvl + 2 * k}"]).permute(0, 3, 1, 2)
            h = q(F.relu(F.conv2d(h, w, params[f"enc.{4 * lvl + 2 * k + 1}"], padding=1)))
        if lvl < net.levels - 1:
            skips.append(h)
            h = F.max_pool2d(h, 2)
    for j in range(net.levels - 1):
        h = torch.cat([F.interpolate(h, scale_factor=2, mode="nearest"), skips[-1 - j]], dim=1)
        for k in range(2):
            w = q(params[f"dec.{4 * j + 2 * k}"]).permute(0, 3, 1, 2)
            h = q(F.relu(F.conv2d(h, w, params[f"dec.{4 * j + 2 * k + 1}"], padding=1)))
    head = F.conv2d(h, q(params["head_w"])[:, :, None, None], params["head_b"])
    out_r = x.cpu().double() + head[:, 0]
    loss_r = ((out_r - tgt.cpu().double()) ** 2).sum()
    loss_r.backward()
    assert abs(float(loss.detach()) - float(loss_r.detach())) <= 2e-2 * float(loss_r.detach())
    for n, p in net.named_parameters():
        g, gr = p.grad.double().cpu().flatten(), params[n].grad.flatten()
        cos = float(g @ gr / (g.norm() * gr.norm() + 1e-30))
        assert cos > 0.99, (n, cos)


def test_adam_matches_torch(cuda):
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import nn
    p = torch.randn(1000, device="cuda")
    q = p.clone().requires_grad_(True)
    opt_ref = torch.optim.Adam([q], lr=1e-2)
    opt = nn.Adam([p], lr=1e-2)
    for step in range(3):
        g = torch.randn(1000, device="cuda")
        p.grad = g.clone()
        q.grad = g.clone()
        opt.step()
        opt_ref.step()
    assert torch.allclose(p, q.detach(), rtol=1e-5, atol=1e-6)


def test_pipeline_wait_gives_up_then_recovers(cuda):
    """With the pipeline wait limit at 0, every GEMM of more than two K blocks
    gives up at its first pipeline wait: it sets the status bit, stores nothing
    and still waits (with the long drain limit) for its committed MMAs before
    freeing its tensor memory, so nothing faults and nothing hangs.  The check
    raises, the status clears, and with the default limit restored the same
    GEMM is exact again."""
    torch = cuda
    from iterative_tomographic_reconstruction_algorithms_b200 import nn
    A, B = _bf(torch, (256, 512), 3), _bf(torch, (64, 512), 4)   # K = 512: 8 blocks of 64
    ref = A.double() @ B.double().T
    nn.check_status()
    try:
        nn.set_wait_limit(0)
        nn.gemm(A.cuda(), B.cuda())
        with pytest.raises(RuntimeError, match="wait gave up"):
            nn.check_status()
    finally:
        nn.set_wait_limit(-1)
    nn.check_status()                      # cleared by the read above
    out = nn.gemm(A.cuda(), B.cuda())
    nn.check_status()
    assert _relerr(torch, out, ref) < 1e-5
