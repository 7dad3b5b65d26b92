"""Generate ``large_golden.npz``: reference outputs at the full 2048 x 2048,
1800-angle geometry, on a sample of the angles.

Needs the compiled reference C (``make -C oracle ref``):

    python tests/golden/make_large_golden.py           # Radon kinds and B-spline
    python tests/golden/make_large_golden.py --grid    # gridding, large_grid_golden.npz

A whole reference application at this size takes minutes (distance-driven:
about 13 minutes), so the fixture samples it.  Every Radon and B-spline kernel
of the reference computes each angle's sinogram row from that angle alone, and
its adjoint adds the angles' contributions one after the other, so

* forward: the row of a sampled angle is the reference called with that one
  angle (and, for B-spline, that angle's look-up-table row);
* adjoint: Aᵀ of a sinogram that is zero outside the sampled rows is the sum
  of the single-angle reference adjoints (summed here in float64; the
  reference's own float32 order differs from it by rounding only).

Sampled angles (indices into ``linspace(0, 180, 1800, endpoint=False)``): the
axis angles 0 and 90 degrees and their neighbours, the 45 and 135 degree
neighbourhoods, 179.9 degrees and two others.  Inputs: a 2048 x 2048
random-ellipse phantom (seed 11), an N(0,1) image (seed 12) and a sparse image
(4096 N(0,1) pixels at seeded places, seed 15) for the forward; N(0,1) values
on the sampled rows (seed 13) for the adjoint, whose result is stored at 32768
seeded pixel positions (seed 14).  The GPU test regenerates the images from the
seeds and checks their float64 sums against the ones stored.

At this size the reference's float32 sums are themselves off the exact sums by
more than 1e-5 on some rows (long rays: thousands of terms per bin), so its
rows on dense images carry that rounding; on the sparse image a bin holds a
few terms only, and the rows pin the geometry (which pixels reach which bin,
with which weight) with almost no rounding.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import RefLib, radon_angles  # noqa: E402
from iterative_tomographic_reconstruction_algorithms_b200.bspline_functions import init_lut_bspline  # noqa: E402
from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses  # noqa: E402

OUT = Path(__file__).resolve().parent / "large_golden.npz"
OUT_GRID = Path(__file__).resolve().parent / "large_grid_golden.npz"
N, NA = 2048, 1800
ANGLE_INDEX = np.array([0, 1, 263, 449, 450, 451, 899, 900, 901, 1117, 1349, 1350, 1351, 1799])
N_PIX = 32768


def large_inputs():
    """The seeded inputs of the fixture (also used by the GPU test)."""
    phantom = random_ellipses(N, seed=11)
    noise = np.random.default_rng(12).standard_normal((N, N), dtype=np.float32)
    rows = np.random.default_rng(13).standard_normal((len(ANGLE_INDEX), N), dtype=np.float32)
    pix = np.sort(np.random.default_rng(14).choice(N * N, size=N_PIX, replace=False))
    rng = np.random.default_rng(15)
    sparse = np.zeros(N * N, np.float32)
    sparse[rng.choice(N * N, size=4096, replace=False)] = rng.standard_normal(4096, dtype=np.float32)
    return phantom, noise, sparse.reshape(N, N), rows, pix


def main() -> None:
    R = RefLib()
    phantom, noise, sparse, rows, pix = large_inputs()
    deg = np.linspace(0, 180, NA, endpoint=False)
    ang = radon_angles(deg)
    data = {"angle_index": ANGLE_INDEX, "sums": np.array([phantom.sum(dtype=np.float64),
                                                          noise.sum(dtype=np.float64),
                                                          sparse.sum(dtype=np.float64),
                                                          rows.sum(dtype=np.float64)]),
            "pix": pix.astype(np.int64)}
    for kind in ("pd", "rd", "dd", "ss"):
        f_ph, f_no, f_sp, adj = [], [], [], np.zeros(N * N, np.float64)
        for j, k in enumerate(ANGLE_INDEX):
            a = ang[k:k + 1]
            f_ph.append(R.radon(kind, 0, phantom, a)[0])
            f_no.append(R.radon(kind, 0, noise, a)[0])
            f_sp.append(R.radon(kind, 0, sparse, a)[0])
            adj += R.radon(kind, 1, rows[j:j + 1], a).ravel()
        data[f"{kind}/fwd_phantom"] = np.array(f_ph, np.float32)
        data[f"{kind}/fwd_noise"] = np.array(f_no, np.float32)
        data[f"{kind}/fwd_sparse"] = np.array(f_sp, np.float32)
        data[f"{kind}/adj"] = adj[pix].astype(np.float32)
        print(kind, "done", flush=True)

    # B-spline pair as the class builds it: angles arange(na)*180/na degrees
    # (class_projectors_bspline.py:49-50), cubic, support 4, Radon degree 1.
    bdeg = (np.arange(NA) * 180.0) / np.float32(NA)
    lut = init_lut_bspline(2048, bdeg, 3, 1, 4.0).astype(np.float32)
    param = np.array([lut.shape[1], 4.0], np.float32)
    a32 = bdeg.astype(np.float32)
    f_ph, f_no, f_sp, adj = [], [], [], np.zeros(N * N, np.float64)
    for j, k in enumerate(ANGLE_INDEX):
        a, lk = a32[k:k + 1], lut[k:k + 1]
        f_ph.append(R.bspline(0, phantom, a, lk, param)[0])
        f_no.append(R.bspline(0, noise, a, lk, param)[0])
        f_sp.append(R.bspline(0, sparse, a, lk, param)[0])
        adj += R.bspline(1, rows[j:j + 1], a, lk, param).ravel()
    data["bspline/fwd_phantom"] = np.array(f_ph, np.float32)
    data["bspline/fwd_noise"] = np.array(f_no, np.float32)
    data["bspline/fwd_sparse"] = np.array(f_sp, np.float32)
    data["bspline/adj"] = adj[pix].astype(np.float32)
    np.savez_compressed(OUT, **data)
    print("wrote", OUT)


# Gridding at the ADMM-TV configuration: 1536 bins, 1500 angles on [0, 180),
# Kaiser-Bessel W = 6, oversampling 2 (a 4096^2 Fourier grid), linear
# interpolation, no filter.  The forward's 2-D transform does not depend on the
# angles and each angle's row is gathered from it alone, so the reference
# called with the sampled angles gives their rows; its adjoint (no filter: the
# filter factor is 1 whatever the angle count) is a sum over angles, so called
# with the sampled rows it gives A^T of a sinogram zero outside them.
N_GRID, NA_GRID = 1536, 1500
GRID_INDEX = np.array([0, 1, 187, 374, 375, 376, 749, 750, 751, 1000, 1124, 1125, 1126, 1499])


def grid_inputs():
    """The seeded inputs of the gridding fixture (also used by the GPU test)."""
    from iterative_tomographic_reconstruction_algorithms_b200.phantom import embed
    phantom = embed(random_ellipses(1024, seed=2), N_GRID)
    noise = np.random.default_rng(22).standard_normal((N_GRID, N_GRID), dtype=np.float32)
    rows = np.random.default_rng(23).standard_normal((len(GRID_INDEX), N_GRID), dtype=np.float32)
    pix = np.sort(np.random.default_rng(24).choice(N_GRID * N_GRID, size=N_PIX, replace=False))
    return phantom, noise, rows, pix


def grid_config():
    from iterative_tomographic_reconstruction_algorithms_b200 import gridrec_lut as glut
    Wp, lut, deapod = glut.configure_regridding(N_GRID, "kb", 2.0, "lin", 6.0, 1e-3)
    param = np.array([0.0, 0, 0, 2.0, 1, len(lut) - 5, Wp, 0], np.float32)
    return param, lut.astype(np.float32), deapod.astype(np.float32)


def main_grid() -> None:
    R = RefLib()
    phantom, noise, rows, pix = grid_inputs()
    param, lut, deapod = grid_config()
    deg = np.linspace(0, 180, NA_GRID, endpoint=False).astype(np.float32)[GRID_INDEX]
    data = {"angle_index": GRID_INDEX, "pix": pix.astype(np.int64),
            "sums": np.array([x.sum(dtype=np.float64) for x in (phantom, noise, rows)]),
            "fwd_phantom": R.gridrec(0, phantom, deg, param, lut, deapod),
            "fwd_noise": R.gridrec(0, noise, deg, param, lut, deapod),
            "adj": R.gridrec(1, rows, deg, param, lut, deapod).ravel()[pix]}
    np.savez_compressed(OUT_GRID, **data)
    print("wrote", OUT_GRID)


if __name__ == "__main__":
    if "--grid" in sys.argv:
        main_grid()
    else:
        main()
