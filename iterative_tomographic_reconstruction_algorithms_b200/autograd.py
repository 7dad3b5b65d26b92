"""Differentiable projector pair for PyTorch.

``Projector(tp)`` wraps a projector object of this package (radon, B-spline or
gridding class) as a ``torch.nn.Module``: ``op(x)`` is ``A x`` on CUDA float32
tensors, ``op.T(y)`` is ``A^T y``.  Gradients are the pair's own kernels: the
backward of ``A`` is the adjoint launch and the backward of ``A^T`` is the
forward launch -- no tape of the projector's internals, no float atomics, so
gradients are deterministic.  For the radon and B-spline pairs ``A^T`` is the
exact transpose of ``A`` (as in the reference C, where both directions walk the
same indices and weights), so these gradients are exact.  The gridding pair
by default reproduces the reference's asymmetric forward/adjoint (different
kernel widths, edge-replicated projections): there the backward is the
reference's adjoint, not the transpose, and is flagged with
``exact_gradient = False``; built with ``adjoint="matched"`` its adjoint is the
exact transpose and the flag is True.

``sirt_unrolled`` runs SIRT iterations (algorithms/art.py:211-237 of the
reference: ``x <- x + C A^T(R (b - A x))``, ``R = 1/A1``, ``C = 1/A^T 1``,
zeros replaced by 1e-10) as differentiable torch code, each iteration under
``torch.utils.checkpoint`` so that an unrolled chain keeps one iterate per step
instead of every intermediate sinogram.
"""
from __future__ import annotations

import torch
from torch.utils.checkpoint import checkpoint

__all__ = ["Projector", "sirt_weights", "sirt_unrolled"]


class _Forward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan):
        ctx.plan = plan
        return plan.forward(x.contiguous())

    @staticmethod
    def backward(ctx, g):
        return ctx.plan.adjoint(g.contiguous()), None


class _Adjoint(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y, plan):
        ctx.plan = plan
        return plan.adjoint(y.contiguous())

    @staticmethod
    def backward(ctx, g):
        return ctx.plan.forward(g.contiguous()), None


class Projector(torch.nn.Module):
    """``A`` of a projector object ``tp`` as a differentiable module.

    Inputs are CUDA float32 tensors of shape ``[n, n]`` (one slice) or
    ``[nz, n, n]`` (``A``) and ``[na, n]`` / ``[nz, na, n]`` (``A^T``).  One
    plan per (slice count, device) is created on first use and kept by ``tp``.
    """

    def __init__(self, tp):
        super().__init__()
        self.tp = tp
        self.n = int(getattr(tp, "npix", 0) or getattr(tp, "n"))
        self.na = int(tp.nang)
        is_grid = tp.__class__.__module__.split(".")[-1] == "class_projectors_grid"
        self.exact_gradient = (not is_grid) or getattr(tp, "adjoint", "compat") == "matched"

    def _plan(self, x, batched_ndim):
        if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float32):
            raise TypeError("Projector expects CUDA float32 tensors")
        nz = 1 if x.dim() == batched_ndim - 1 else int(x.shape[0])
        return self.tp.plan(nz, x.device.index)

    def forward(self, x):
        plan = self._plan(x, 3)
        y = _Forward.apply(x, plan)
        return y[0] if x.dim() == 2 else y

    def T(self, y):
        plan = self._plan(y, 3)
        x = _Adjoint.apply(y, plan)
        return x[0] if y.dim() == 2 else x


def sirt_weights(op: Projector, like: torch.Tensor):
    """(R, C) of art.py:227-233 for the slices of ``like`` (float32, zeros -> 1e-10)."""
    with torch.no_grad():
        ones = torch.ones_like(like)
        a1 = op(ones)
        a1 = torch.where(a1 == 0, torch.full_like(a1, 1e-10), a1)
        at1 = op.T(torch.ones_like(a1))
        at1 = torch.where(at1 == 0, torch.full_like(at1, 1e-10), at1)
        return 1.0 / a1, 1.0 / at1


def sirt_unrolled(op: Projector, b: torch.Tensor, x0: torch.Tensor, iters: int,
                  weights=None, use_checkpoint: bool = True) -> torch.Tensor:
    """``iters`` differentiable SIRT steps from ``x0`` towards data ``b``.

    With ``use_checkpoint`` each step is recomputed in the backward pass (one
    forward and one adjoint launch) instead of storing its sinograms.
    """
    R, C = weights if weights is not None else sirt_weights(op, x0)

    def step(x):
        return x + C * op.T(R * (b - op(x)))

    x = x0
    for _ in range(int(iters)):
        if use_checkpoint and torch.is_grad_enabled():
            x = checkpoint(step, x, use_reentrant=False)
        else:
            x = step(x)
    return x
