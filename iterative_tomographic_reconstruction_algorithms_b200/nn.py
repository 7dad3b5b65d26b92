"""Learned warm start: tensor-core convolution kernels and a small U-Net.

The network maps a cheap reconstruction (2 SIRT iterations) to a start close
to the converged SIRT result; the plain solver then continues from it.  All
convolutions -- forward, input gradient and weight gradient -- are the
hand-written tcgen05 BF16 kernels of ``libtomo_nn.so`` (``csrc/nn_gemm.cu``,
``csrc/nn_ops.cu``) with FP32 accumulation and FP32 master weights; pooling,
upsampling and concatenation are layout operations left to torch.  Activations
are BF16 NHWC.

Layers (``UNet(levels=4, base=32)``): per level two 3x3 convolutions + ReLU,
2x2 max-pooling down, nearest 2x upsampling up with the skip connection
concatenated, a final 1x1 convolution, and the input added back (the network
predicts a correction).
"""
from __future__ import annotations

import ctypes
import math
import os
from pathlib import Path

import torch

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libtomo_nn.so"

__all__ = ["gemm", "conv3x3", "wgrad", "UNet", "Adam", "check_status"]


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR / 'csrc'}`")
    lib = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_GLOBAL)
    vp, i, f, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_size_t
    lib.tomo_nn_gemm.argtypes = [vp, i, vp, i, i, i, i, vp, vp, i, vp, i, vp]
    lib.tomo_nn_conv3x3.argtypes = [vp, i, i, i, i, vp, i, vp, vp, vp, i, vp]
    lib.tomo_nn_wgrad_workspace.argtypes = [i, i, i, i, i, i]
    lib.tomo_nn_wgrad_workspace.restype = sz
    lib.tomo_nn_wgrad.argtypes = [vp, vp, i, i, i, i, i, i, vp, vp, vp, sz, vp]
    lib.tomo_nn_prepare_weights.argtypes = [vp, i, i, i, vp, vp, vp]
    lib.tomo_nn_relu_bwd.argtypes = [vp, vp, sz, vp]
    lib.tomo_nn_adam.argtypes = [vp, vp, vp, vp, sz, f, f, f, f, i, vp]
    lib.tomo_nn_status.argtypes = [ctypes.POINTER(ctypes.c_uint)]
    return lib


lib = _load()


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


def _stream(t):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def set_wait_limit(spins: int) -> None:
    """Polls of a tensor-core pipeline wait before it gives up (tomo_nn.h:
    tomo_nn_set_wait_limit); a negative value restores the default."""
    lib.tomo_nn_set_wait_limit.argtypes = [ctypes.c_int]
    _check(lib.tomo_nn_set_wait_limit(int(spins)), "tomo_nn_set_wait_limit")


def check_status():
    """Raises if a tensor-core wait gave up in any kernel since the last check."""
    flags = ctypes.c_uint()
    _check(lib.tomo_nn_status(ctypes.byref(flags)), "tomo_nn_status")
    if flags.value:
        raise RuntimeError(f"tensor-core kernel reported status {flags.value:#x} (a wait gave up)")


def gemm(A, B, bias=None, relu=False, out_dtype=torch.float32):
    """A [M, K] . B [N, K]^T (BF16 CUDA tensors, K % 8 == 0) -> [M, N]."""
    M, K = A.shape
    N = B.shape[0]
    out = torch.empty((M, N), dtype=out_dtype, device=A.device)
    f32 = out_dtype == torch.float32
    _check(lib.tomo_nn_gemm(_p(A), A.stride(0), _p(B), B.stride(0), M, N, K, _p(out) if f32 else None,
                            None if f32 else _p(out), N, _p(bias), int(relu), _stream(A)), "tomo_nn_gemm")
    return out


def conv3x3(X, Wb, bias=None, relu=False, out_dtype=torch.bfloat16):
    """X [B, H, W, Cin] BF16, Wb [Cout, 3, 3, Cin] BF16 -> [B, H, W, Cout]."""
    B, H, W, Cin = X.shape
    Cout = Wb.shape[0]
    out = torch.empty((B, H, W, Cout), dtype=out_dtype, device=X.device)
    f32 = out_dtype == torch.float32
    _check(lib.tomo_nn_conv3x3(_p(X), B, H, W, Cin, _p(Wb), Cout, _p(out) if f32 else None,
                               None if f32 else _p(out), _p(bias), int(relu), _stream(X)), "tomo_nn_conv3x3")
    return out


def wgrad(X, dY, taps):
    """Weight and bias gradients of a 3x3 (taps=9) or 1x1 (taps=1) convolution."""
    B, H, W, Cin = X.shape
    Cout = dY.shape[-1]
    dW = torch.empty((Cout, taps, Cin), dtype=torch.float32, device=X.device)
    db = torch.empty((Cout,), dtype=torch.float32, device=X.device)
    nbytes = lib.tomo_nn_wgrad_workspace(B, H, W, Cin, Cout, taps)
    work = torch.empty((nbytes,), dtype=torch.uint8, device=X.device)
    _check(lib.tomo_nn_wgrad(_p(X), _p(dY), B, H, W, Cin, Cout, taps, _p(dW), _p(db), _p(work), nbytes,
                             _stream(X)), "tomo_nn_wgrad")
    return dW, db


def prepare_weights(W, with_transpose=True):
    """FP32 [Cout, taps, Cin] -> (BF16 copy, BF16 [Cin, taps, Cout] with the taps reversed)."""
    Cout, taps, Cin = W.shape
    Wb = torch.empty_like(W, dtype=torch.bfloat16)
    Wd = torch.empty((Cin, taps, Cout), dtype=torch.bfloat16, device=W.device) if with_transpose else None
    _check(lib.tomo_nn_prepare_weights(_p(W), Cout, Cin, taps, _p(Wb), _p(Wd), _stream(W)),
           "tomo_nn_prepare_weights")
    return Wb, Wd


class _Conv3x3(torch.autograd.Function):
    """3x3 convolution + bias (+ ReLU) with the tensor-core kernels in both directions."""

    @staticmethod
    def forward(ctx, X, W, b, relu, need_dx):
        Wb, Wd = prepare_weights(W.detach().reshape(W.shape[0], 9, W.shape[-1]), with_transpose=need_dx)
        Y = conv3x3(X, Wb.reshape(W.shape), b.detach(), relu=relu)
        ctx.save_for_backward(X, Y, Wd if need_dx else None)
        ctx.relu, ctx.need_dx = relu, need_dx
        return Y

    @staticmethod
    def backward(ctx, dY):
        X, Y, Wd = ctx.saved_tensors
        dZ = dY.to(torch.bfloat16).contiguous()
        if ctx.relu:
            _check(lib.tomo_nn_relu_bwd(_p(Y), _p(dZ), dZ.numel(), _stream(dZ)), "tomo_nn_relu_bwd")
        dW, db = wgrad(X, dZ, 9)
        dX = None
        if ctx.need_dx:
            dX = conv3x3(dZ, Wd.reshape(Wd.shape[0], 3, 3, Wd.shape[-1]))
        return dX, dW.reshape(dW.shape[0], 3, 3, dW.shape[-1]), db, None, None


class _Conv1x1(torch.autograd.Function):
    """1x1 convolution + bias, FP32 output (the network's last layer)."""

    @staticmethod
    def forward(ctx, X, W, b):
        Bn, H, Wd_, Cin = X.shape
        Wb, Wt = prepare_weights(W.detach().reshape(W.shape[0], 1, Cin), with_transpose=True)
        Y = gemm(X.reshape(-1, Cin), Wb.reshape(W.shape[0], Cin), bias=b.detach())
        ctx.save_for_backward(X, Wt)
        return Y.reshape(Bn, H, Wd_, W.shape[0])

    @staticmethod
    def backward(ctx, dY):
        X, Wt = ctx.saved_tensors
        Bn, H, W_, Cin = X.shape
        dZ = dY.to(torch.bfloat16).contiguous()
        dW, db = wgrad(X, dZ, 1)
        dX = gemm(dZ.reshape(-1, dZ.shape[-1]), Wt.reshape(Cin, -1), out_dtype=torch.bfloat16)
        return dX.reshape(X.shape), dW.reshape(dW.shape[0], Cin), db


def _pool(x):
    # NHWC view as channels-last NCHW for max-pooling
    return torch.nn.functional.max_pool2d(x.permute(0, 3, 1, 2), 2).permute(0, 2, 3, 1).contiguous()


def _up(x):
    return torch.nn.functional.interpolate(x.permute(0, 3, 1, 2), scale_factor=2, mode="nearest") \
        .permute(0, 2, 3, 1).contiguous()


class UNet(torch.nn.Module):
    """U-Net with ``levels`` resolutions and ``base`` channels at the top level.

    ``forward(x)``: x FP32 [B, H, W] (H, W divisible by 2^(levels-1)) -> FP32
    [B, H, W] = x + correction.  Input channels are padded to 8 with zeros.
    """

    CIN = 8

    def __init__(self, levels: int = 4, base: int = 32, seed: int = 0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.levels = levels
        ch = [base * 2 ** i for i in range(levels)]
        self.enc, self.dec = torch.nn.ParameterList(), torch.nn.ParameterList()

        def conv(cin, cout, store):
            w = torch.randn((cout, 3, 3, cin), generator=g) * math.sqrt(2.0 / (9 * cin))
            store.append(torch.nn.Parameter(w))
            store.append(torch.nn.Parameter(torch.zeros(cout)))

        cin = self.CIN
        for c in ch:
            conv(cin, c, self.enc)
            conv(c, c, self.enc)
            cin = c
        for c in reversed(ch[:-1]):
            conv(cin + c, c, self.dec)
            conv(c, c, self.dec)
            cin = c
        self.head_w = torch.nn.Parameter(torch.zeros((8, cin)))
        self.head_b = torch.nn.Parameter(torch.zeros(8))

    def forward(self, x, extra=None):
        """``extra``: optional further input channels, FP32 [B, H, W] or [B, H, W, k] (k <= 7)."""
        B, H, W = x.shape
        h = torch.zeros((B, H, W, self.CIN), dtype=torch.bfloat16, device=x.device)
        h[..., 0] = x.to(torch.bfloat16)
        if extra is not None:
            e = extra if extra.dim() == 4 else extra[..., None]
            h[..., 1:1 + e.shape[-1]] = e.to(torch.bfloat16)
        skips = []
        first = True
        for lvl in range(self.levels):
            w1, b1, w2, b2 = self.enc[4 * lvl:4 * lvl + 4]
            h = _Conv3x3.apply(h, w1, b1, True, not first)
            h = _Conv3x3.apply(h, w2, b2, True, True)
            first = False
            if lvl < self.levels - 1:
                skips.append(h)
                h = _pool(h)
        for j in range(self.levels - 1):
            w1, b1, w2, b2 = self.dec[4 * j:4 * j + 4]
            h = torch.cat([_up(h), skips[-1 - j]], dim=-1)
            h = _Conv3x3.apply(h, w1, b1, True, True)
            h = _Conv3x3.apply(h, w2, b2, True, True)
        out = _Conv1x1.apply(h, self.head_w, self.head_b)
        return x + out[..., 0]


class Adam:
    """Adam on FP32 parameters with the ``tomo_nn_adam`` kernel."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8):
        self.params = [p for p in params]
        self.lr, self.b1, self.b2, self.eps = lr, betas[0], betas[1], eps
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.t = 0

    def zero_grad(self):
        for p in self.params:
            p.grad = None

    @torch.no_grad()
    def step(self):
        self.t += 1
        for p, m, v in zip(self.params, self.m, self.v):
            if p.grad is None:
                continue
            g = p.grad.contiguous()
            _check(lib.tomo_nn_adam(_p(p), _p(g), _p(m), _p(v), p.numel(), self.lr, self.b1, self.b2, self.eps,
                                    self.t, _stream(p)), "tomo_nn_adam")
