"""Seeded random-ellipse phantoms (synthetic stand-ins for the benchmark data).

Definition used by every workload of this package: ``count`` ellipses on the
square [-1, 1]^2 sampled at pixel centres ((j + 0.5) / side * 2 - 1); centres
uniform in the unit disk, semi-axes U(0.05, 0.5), rotation U(0, pi), additive
density U(-0.5, 1.0); the densities are summed and clipped at 0.  Generated
with ``numpy.random.default_rng(seed)`` so a seed names one phantom.
"""
from __future__ import annotations

import numpy as np


def random_ellipses(side: int, seed: int, count: int = 10, dtype=np.float32) -> np.ndarray:
    rng = np.random.default_rng(seed)
    c = (np.arange(side) + 0.5) / side * 2.0 - 1.0
    X, Y = np.meshgrid(c, c[::-1], indexing="xy")
    img = np.zeros((side, side), np.float64)
    for _ in range(count):
        rad = np.sqrt(rng.uniform(0.0, 1.0))
        ang = rng.uniform(0.0, 2 * np.pi)
        x0, y0 = rad * np.cos(ang), rad * np.sin(ang)
        a, b = rng.uniform(0.05, 0.5, size=2)
        phi = rng.uniform(0.0, np.pi)
        rho = rng.uniform(-0.5, 1.0)
        cp, sp = np.cos(phi), np.sin(phi)
        xr = (X - x0) * cp + (Y - y0) * sp
        yr = -(X - x0) * sp + (Y - y0) * cp
        img[(xr / a) ** 2 + (yr / b) ** 2 <= 1.0] += rho
    np.clip(img, 0.0, None, out=img)
    return img.astype(dtype)


def random_ellipses_device(side: int, seeds, device, count: int = 10):
    """``random_ellipses(side, seed)`` for every seed, drawn on the device: a
    float32 tensor [len(seeds), side, side].  The ellipse parameters come from
    the same numpy generator calls, and every pixel test is the same sequence of
    float64 operations (each rounded, no fused multiply-add), so the images
    equal the host ones."""
    import torch
    c = torch.from_numpy((np.arange(side) + 0.5) / side * 2.0 - 1.0).to(device)
    X = c[None, :].expand(side, side)
    Y = c.flip(0)[:, None].expand(side, side)
    out = torch.empty((len(seeds), side, side), dtype=torch.float32, device=device)
    for k, seed in enumerate(seeds):
        rng = np.random.default_rng(seed)
        img = torch.zeros((side, side), dtype=torch.float64, device=device)
        for _ in range(count):
            rad = np.sqrt(rng.uniform(0.0, 1.0))
            ang = rng.uniform(0.0, 2 * np.pi)
            x0, y0 = rad * np.cos(ang), rad * np.sin(ang)
            a, b = rng.uniform(0.05, 0.5, size=2)
            phi = rng.uniform(0.0, np.pi)
            rho = rng.uniform(-0.5, 1.0)
            cp, sp = np.cos(phi), np.sin(phi)
            dx, dy = X - x0, Y - y0
            xr = dx * cp + dy * sp
            yr = -dx * sp + dy * cp
            u, v = xr / a, yr / b
            img += (u * u + v * v <= 1.0).to(torch.float64) * rho   # rho or 0, exactly
        out[k] = img.clamp_(min=0.0).to(torch.float32)
    return out


def embed(img: np.ndarray, n_op: int) -> np.ndarray:
    """Centre ``img`` in an ``n_op`` x ``n_op`` zero canvas (edge-padding layout)."""
    side = img.shape[-1]
    if n_op < side:
        raise ValueError("operator side smaller than the phantom")
    i1 = (n_op - side) // 2
    out = np.zeros(img.shape[:-2] + (n_op, n_op), img.dtype)
    out[..., i1:i1 + side, i1:i1 + side] = img
    return out


def angles_deg(na: int) -> np.ndarray:
    """``na`` angles uniform on [0, 180) degrees (utils.create_projection_angles)."""
    return np.linspace(0.0, 180.0, na, endpoint=False)
