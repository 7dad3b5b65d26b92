"""Learned warm start for SIRT: training pairs, training and the time-to-residual test.

Problem (seeded, synthetic): random-ellipse phantoms of side ``side`` scaled to
attenuation in [0, ``mu_max``] per pixel, centred in an ``n_op`` x ``n_op``
operator (edge-padding convention), ``na`` angles on [0, 180), transmission
counts Poisson(I0 exp(-A x)), sinogram b = -log(max(counts, 1) / I0).  The
projector is the distance-driven pair; SIRT is the fused solver
(``solvers.Solver``), started from zero.

A training sample holds x2 (the 2-iteration SIRT image), the filtered
backprojection of b, x_ref (the ``ref_iters``-iteration SIRT image), the
phantom and b.  The network f (a ``nn.UNet``) sees x2 and the filtered
backprojection (ramp filter, the distance-driven adjoint), which carries the
data's high frequencies that SIRT recovers slowly, and is trained with

    loss = |f - x_true|^2 / |x_true|^2 + lam |A S5(f) - b|^2 / |A x_ref - b|^2,

S5 = five unrolled SIRT steps through the differentiable projector
(``autograd.sirt_unrolled``, checkpointed); the data term is relative to the
reference's own residual.  SIRT only changes an image within the row space of
A, so the start alone decides the null-space content of the result: the image
term pulls it towards the phantom, the data term makes a few SIRT steps from
it fit the data as well as the reference does.  At use, SIRT continues from
f; the plain start is kept when f has a larger data residual than x2 (the
fallback), and ``time_to_residual`` measures the GPU time each start needs to
reach the plain run's final data residual.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import nn
from .autograd import Projector, sirt_unrolled, sirt_weights
from .class_projectors_radon import projectors
from .phantom import random_ellipses_device
from .solvers import Solver


@dataclass
class Problem:
    side: int = 512
    n_op: int = 768
    na: int = 180
    I0: float = 5e3
    mu_max: float = 0.01
    ref_iters: int = 300
    start_iters: int = 2


def make_batch(pb: Problem, seeds, device="cuda"):
    """(x_true, b, tp) for the given phantom seeds: float32 CUDA tensors [B, n_op, n_op], [B, na, n_op]."""
    tp = projectors(pb.n_op, np.linspace(0, 180, pb.na, endpoint=False), oper="dd")
    # the phantoms of random_ellipses, drawn on the device (same values)
    ph = random_ellipses_device(pb.side, [int(s) for s in seeds], device)
    peak = ph.amax(dim=(1, 2), keepdim=True).clamp(min=1e-6)
    ph = ph / peak * np.float32(pb.mu_max)
    i1 = (pb.n_op - pb.side) // 2
    x_true = torch.zeros((len(seeds), pb.n_op, pb.n_op), dtype=torch.float32, device=device)
    x_true[:, i1:i1 + pb.side, i1:i1 + pb.side] = ph
    b_clean = tp.A(x_true)
    g = torch.Generator(device=device).manual_seed(int(seeds[0]) * 7919 + 1)
    counts = torch.poisson(pb.I0 * torch.exp(-b_clean), generator=g)
    b = -torch.log(torch.clamp(counts, min=1.0) / pb.I0)
    return x_true, b.contiguous(), tp


def fbp(tp, b):
    """Filtered backprojection: ramp-filtered sinogram rows, distance-driven adjoint, pi / na."""
    na, n = b.shape[-2], b.shape[-1]
    L = 1 << int(math.ceil(math.log2(2 * n)))
    ramp = torch.abs(torch.fft.rfftfreq(L, device=b.device)).to(torch.float32)
    f = torch.fft.irfft(torch.fft.rfft(b, n=L, dim=-1) * ramp, n=L, dim=-1)[..., :n].contiguous()
    return tp.At(f) * (math.pi / na)


def make_pairs(pb: Problem, seeds, chunk: int = 64, device="cuda", compact: bool = False):
    """Training samples on the GPU, ``chunk`` slices per batched solve: a dict of
    x2, fbp, x_ref, x_true, b and r_ref (the reference's data residual per slice).

    ``compact``: for large sample counts (20k samples at 768^2 hold ~200 GB in
    float32) x2, fbp and x_true are kept in bfloat16 (the network's operand
    type; ``train`` widens them to float32 per batch) and x_ref is not kept
    (training uses only r_ref): ~4 MB a sample."""
    keys = ("x2", "fbp", "x_true", "b", "r_ref") if compact else ("x2", "fbp", "x_ref", "x_true", "b", "r_ref")
    low = (lambda t: t.to(torch.bfloat16)) if compact else (lambda t: t)
    out = {k: [] for k in keys}
    for i in range(0, len(seeds), chunk):
        x_true, b, tp = make_batch(pb, seeds[i:i + chunk], device)
        zero = torch.zeros((b.shape[0], pb.n_op, pb.n_op), device=device)
        solver = Solver(tp, "sirt", b)
        x2, _ = solver.run(zero, pb.start_iters)
        xr, _ = solver.run(x2, pb.ref_iters - pb.start_iters)
        out["x2"].append(low(x2))
        out["fbp"].append(low(fbp(tp, b)))
        if not compact:
            out["x_ref"].append(xr)
        out["x_true"].append(low(x_true))
        out["b"].append(b)
        out["r_ref"].append(((tp.A(xr) - b) ** 2).sum(dim=(1, 2)))
        del solver, xr
    return {k: torch.cat(v) for k, v in out.items()}


def apply_net(net, pb: Problem, x2, fb):
    """The network's start image from x2 and the filtered backprojection."""
    scale = 1.0 / pb.mu_max
    return net(x2 * scale, fb * scale) / scale


def train(net, pb: Problem, data, steps: int = 1000, batch: int = 4, lr: float = 1e-3,
          lam: float = 0.03, unroll: int = 5, seed: int = 0, log_every: int = 100):
    """Trains ``net`` in place on ``make_pairs`` data; returns the loss history
    (one value per ``log_every`` steps).  The learning rate decays by cosine."""
    tp = projectors(pb.n_op, np.linspace(0, 180, pb.na, endpoint=False), oper="dd")
    op = Projector(tp)
    opt = nn.Adam(net.parameters(), lr=lr)
    g = torch.Generator().manual_seed(seed)
    n = data["x2"].shape[0]
    W = None
    hist = []
    for step in range(1, steps + 1):
        opt.lr = lr * 0.5 * (1.0 + math.cos(math.pi * (step - 1) / steps))
        idx = torch.randint(0, n, (batch,), generator=g).to(data["x2"].device)
        xi, fi, ti = data["x2"][idx].float(), data["fbp"][idx].float(), data["x_true"][idx].float()
        bi, rr = data["b"][idx].contiguous(), data["r_ref"][idx]
        if W is None:
            W = sirt_weights(op, xi)
        out = apply_net(net, pb, xi, fi)
        loss = ((out - ti) ** 2).sum() / (ti ** 2).sum()
        if lam > 0 and unroll > 0:
            xu = sirt_unrolled(op, bi, out, unroll, weights=W)
            loss = loss + lam * (((op(xu) - bi) ** 2).sum(dim=(1, 2)) / rr).mean()
        opt.zero_grad()
        loss.backward()
        opt.step()
        if step % log_every == 0 or step == steps:
            hist.append(float(loss.detach()))
    nn.check_status()
    return hist


@torch.no_grad()
def warm_start(net, pb: Problem, x2, tp, b, chunk: int = 64):
    """f(x2, fbp(b)), or x2 for the slices where f has the larger data residual
    (fallback).  The network runs on ``chunk`` slices at a time (its activations
    at 768^2 take ~50 MB a slice)."""
    fb = fbp(tp, b)
    xw = torch.empty_like(x2)
    for i in range(0, x2.shape[0], chunk):
        xw[i:i + chunk] = apply_net(net, pb, x2[i:i + chunk], fb[i:i + chunk])
    rw = ((tp.A(xw) - b) ** 2).sum(dim=(1, 2))
    r2 = ((tp.A(x2) - b) ** 2).sum(dim=(1, 2))
    keep = (rw <= r2)[:, None, None]
    return torch.where(keep, xw, x2), keep.flatten()


def _timed(fn):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


def time_to_residual(net, pb: Problem, seeds, device="cuda"):
    """Plain SIRT (ref_iters from zero) against warm-started SIRT on held-out seeds.

    Returns a dict with the GPU milliseconds of each, the iterations the warm
    start needed to reach the plain run's final data residual, and the images'
    relative errors to the phantom (float64).
    """
    x_true, b, tp = make_batch(pb, seeds, device)
    B = b.shape[0]
    zero = torch.zeros((B, pb.n_op, pb.n_op), device=device)
    solver = Solver(tp, "sirt", b)
    solver.run(zero, 1)  # graph capture and warm-up outside the timing
    (xp, resp), t_plain = _timed(lambda: solver.run(zero, pb.ref_iters))
    r_target = float(((tp.A(xp) - b).double() ** 2).sum())
    truth = x_true.double()

    def relerr(x):
        return float((x.double() - truth).norm() / truth.norm())

    # warm: x2, network, then SIRT; find the iteration count that reaches the target
    x2, _ = solver.run(zero, pb.start_iters)
    xw, kept = warm_start(net, pb, x2, tp, b)
    _, resw = solver.run(xw, pb.ref_iters)
    # residuals[k] is |A x_k - b|^2 of the iterate entering iteration k
    below = np.nonzero(resw <= r_target)[0]
    k = int(below[0]) if len(below) else pb.ref_iters
    curve = []
    for kk in (1, 2, 5, 10, 20, 50, 100):
        xkk, _ = solver.run(xw, kk)
        curve.append({"iters": kk, "residual": float(resw[kk]) if kk < len(resw) else None,
                      "err": relerr(xkk)})

    def warm_run():
        a, _ = solver.run(zero, pb.start_iters)
        w, _ = warm_start(net, pb, a, tp, b)
        return solver.run(w, k)[0] if k > 0 else w

    xk, t_warm = _timed(warm_run)
    r_warm = float(((tp.A(xk) - b).double() ** 2).sum())
    return {"slices": B, "plain_ms": t_plain, "warm_ms": t_warm, "ratio": t_warm / t_plain,
            "warm_iters": k, "plain_iters": pb.ref_iters, "residual_plain": r_target,
            "residual_warm": r_warm, "err_plain": relerr(xp), "err_warm": relerr(xk),
            "err_start": relerr(xw), "fallback_slices": int((~kept).sum()),
            "residual_start": {"x2": float(((tp.A(x2) - b).double() ** 2).sum()), "warm": float(resw[0])},
            "residual_curve_plain": [float(resp[i]) for i in (0, 2, 10, 50, 100, 200, pb.ref_iters - 1)
                                     if i < len(resp)],
            "warm_curve": curve, "x_plain": xp, "x_warm": xk, "b": b, "tp": tp}
