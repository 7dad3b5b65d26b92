"""Matrix entries of the reference's distance-driven pair at 64x64, 180 angles.

Runs the compiled reference dd projector (oracle/_ref, ``make -C oracle ref``)
on one-hot inputs: its forward of six one-hot images (whole sinogram columns
of A) and its adjoint of six one-hot sinograms (whole image rows of A).  The
reference computes both with one routine (radon_dd.c:54-285, `oper` flag), so
each column and row holds A's entries exactly as the reference rounds them.
Pixel (5, 25) and angle 92, bin 5 are an entry where the reference's float
pixel width (P_j+1 - P_j) is not 1.  Writes dd_entries_golden.npz:

    python tests/golden/make_dd_entries_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import RefLib, radon_angles  # noqa: E402

N, NA = 64, 180
PIXELS = [(5, 25), (0, 0), (63, 63), (32, 32), (1, 62), (40, 7)]
ENTRIES = [(92, 5), (0, 10), (45, 32), (135, 60), (179, 1), (91, 33)]


def main() -> None:
    ref = RefLib()
    deg = np.linspace(0, 180, NA, endpoint=False)
    ang = radon_angles(deg)
    cols, rows = [], []
    for r, c in PIXELS:
        img = np.zeros((N, N), np.float32)
        img[r, c] = 1.0
        cols.append(ref.radon("dd", 0, img, ang))
    for v, b in ENTRIES:
        y = np.zeros((NA, N), np.float32)
        y[v, b] = 1.0
        rows.append(ref.radon("dd", 1, y, ang))
    out = Path(__file__).with_name("dd_entries_golden.npz")
    np.savez_compressed(out, angles_deg=deg, pixels=np.array(PIXELS), entries=np.array(ENTRIES),
                        fwd_columns=np.stack(cols), adj_rows=np.stack(rows))
    print(out, out.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
