"""Generate the golden fixtures in this directory from the REFERENCE itself.

Run in a tree where the reference C has been compiled into ``oracle/_ref``
(``make -C oracle ref``):

    python tests/golden/make_golden.py

For every projector pair and a set of small shapes (even and odd sides, dense
and sparse angle sets, special angles 0/45/90/135 degrees) it draws seeded
inputs, runs the reference C through a restatement of its Cython shim
(oracle/oracle.py: RefLib), and stores inputs and outputs (float32) in
``radon_golden.npz`` / ``bspline_golden.npz``.  The GPU parity tests compare
the CUDA path against these arrays, so the tests need neither the reference
tree nor the compiled reference on the machine that runs them.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import REFERENCE_TREE, RefLib, radon_angles  # noqa: E402
from iterative_tomographic_reconstruction_algorithms_b200.bspline_functions import init_lut_bspline  # noqa: E402

OUT = Path(__file__).resolve().parent

# (name, n, angle set in degrees[, own seed]); cases with their own seed draw
# their inputs from a separate generator, so adding one leaves the others as
# they were
RADON_CASES = [
    ("n64_a90", 64, np.linspace(0, 180, 90, endpoint=False)),
    ("n65_a37", 65, np.linspace(0, 180, 37, endpoint=False)),
    ("n48_special", 48, np.array([0.0, 30.0, 45.0, 60.0, 90.0, 120.0, 135.0, 150.0, 179.5])),
    ("n33_a16", 33, np.linspace(0, 180, 16, endpoint=False)),
    ("n128_a45", 128, np.linspace(0, 180, 45, endpoint=False)),
    # near-axis angles: pixel coordinates up to nh / |cos| (binade crossings of
    # P with large width errors; beyond 2^22 the widths are 0 or 2)
    ("n256_nearaxis", 256, np.array([0.1, 0.5, 44.9, 89.5, 89.9, 89.99, 89.999, 90.001, 90.1, 134.9,
                                     179.5, 179.9, 179.99, 179.999]), 256),
]


def main() -> None:
    R = RefLib()
    rng = np.random.default_rng(20240611)
    data = {}
    for name, n, deg, *own in RADON_CASES:
        ang = radon_angles(deg)
        na = len(ang)
        g = np.random.default_rng(own[0]) if own else rng
        img = g.standard_normal((n, n)).astype(np.float32)
        sino = g.standard_normal((na, n)).astype(np.float32)
        data[f"{name}/angles_deg"] = deg.astype(np.float64)
        data[f"{name}/image"] = img
        data[f"{name}/sino"] = sino
        for kind in ("pd", "rd", "dd", "ss"):
            sn = np.abs(np.sin(ang.astype(np.float64)))
            cs = np.abs(np.cos(ang.astype(np.float64)))
            nh = n // 2
            misses = (sn >= 1e-5) & (cs >= 1e-5) & ((nh - 1) * cs + nh * sn < nh + 0.5)
            if kind == "ss" and np.any(misses):
                # A ray of radon_ss.c that misses the square [-nh, nh-1]^2
                # (|sin| * nh < 1 near 180 degrees) makes ray_limits return
                # limits outside the image and the reference reads/writes out
                # of bounds (the adjoint corrupts the heap).  No golden values.
                continue
            data[f"{name}/{kind}/fwd"] = R.radon(kind, 0, img, ang)
            data[f"{name}/{kind}/adj"] = R.radon(kind, 1, sino, ang)
    np.savez_compressed(OUT / "radon_golden.npz", **data)
    if "--radon-only" in sys.argv:
        return

    data = {}
    for name, n, na, deg, sup in [("n64_a90_cubic", 64, 90, 3, 4.0), ("n65_a37_cubic", 65, 37, 3, 4.0),
                                  ("n48_a30_linear", 48, 30, 1, 2.0)]:
        ang = (np.arange(na) * 180.0) / np.float32(na)  # class_projectors_bspline.py:49-50
        lut = init_lut_bspline(2048, ang, deg, 1, sup).astype(np.float32)
        param = np.array([lut.shape[1], sup], np.float32)
        img = rng.standard_normal((n, n)).astype(np.float32)
        sino = rng.standard_normal((na, n)).astype(np.float32)
        a32 = ang.astype(np.float32)
        data[f"{name}/angles"] = a32
        data[f"{name}/deg_support"] = np.array([deg, sup], np.float64)
        data[f"{name}/lut_sum"] = np.array([np.sum(lut, dtype=np.float64)])
        data[f"{name}/param"] = param
        data[f"{name}/image"] = img
        data[f"{name}/sino"] = sino
        data[f"{name}/fwd"] = R.bspline(0, img, a32, lut, param)
        data[f"{name}/adj"] = R.bspline(1, sino, a32, lut, param)
    np.savez_compressed(OUT / "bspline_golden.npz", **data)

    # gridding pair: the reference's own golden pair (data/shepp_logan_pix0256.tif
    # and its grid-PSWF sinogram data/shepp_logan_pix0256_ang0304_sino.tif, made
    # by gridding_forward.py with its defaults: prolate kernel, W=7, os=2, nn,
    # errs=1e-3, 304 angles on [0, 180)), plus reference outputs on seeded inputs.
    from oracle.oracle import read_tiff_strip
    from iterative_tomographic_reconstruction_algorithms_b200 import gridrec_lut as glut
    ref_data = REFERENCE_TREE / "data"
    data = {"sl/image": read_tiff_strip(ref_data / "shepp_logan_pix0256.tif").astype(np.float32),
            "sl/sino": read_tiff_strip(ref_data / "shepp_logan_pix0256_ang0304_sino.tif")}
    for name, n, na, kernel, os_, interp, W, errs, rdeg, filt in [
            ("n64_pswf_nn", 64, 90, "pswf", 2.0, "nn", 7.0, 1e-3, 0, 0),
            ("n96_kb_lin", 96, 120, "kb", 2.0, "lin", 6.0, 6e-6, 0, 0),
            ("n100_kb_os15", 100, 75, "kb", 1.5, "lin", 6.6, 6e-6, 0, 0),
            ("n64_prolate_dpc", 64, 60, "prolate", 2.0, "nn", 7.0, 1e-3, 1, 0),
            ("n80_pswf_ramp", 80, 96, "pswf", 2.0, "nn", 7.0, 1e-3, 0, 1)]:
        Wp, lut, deapod = glut.configure_regridding(n, kernel, os_, interp, W, errs)
        param = np.array([0.0, filt, 0, os_, 0 if interp == "nn" else 1, len(lut) - 5, Wp, rdeg], np.float32)
        deg = np.linspace(0, 180, na, endpoint=False).astype(np.float32)
        img = rng.standard_normal((n, n)).astype(np.float32)
        sino = rng.standard_normal((na, n)).astype(np.float32)
        cfg = np.array([n, na, os_, 0 if interp == "nn" else 1, W, errs, rdeg, filt], np.float64)
        data[f"{name}/cfg"] = cfg
        data[f"{name}/kernel"] = np.array(kernel)
        data[f"{name}/image"] = img
        data[f"{name}/sino"] = sino
        data[f"{name}/fwd"] = R.gridrec(0, img, deg, param, lut.astype(np.float32), deapod.astype(np.float32))
        data[f"{name}/adj"] = R.gridrec(1, sino, deg, param, lut.astype(np.float32), deapod.astype(np.float32))
    np.savez_compressed(OUT / "grid_golden.npz", **data)
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))


def make_fbp() -> None:
    """fbp_golden.npz: filtered backprojection and projection filtering.

    * ``filter/<ftype>_<dpc>``: the reference's own filters.filter_proj
      (common/operators/filters_module/filters.py:89-113, imported from the
      reference tree) on seeded float32 projections;
    * ``bspline/<case>``: the reference's B-spline ``fbp`` pipeline
      (class_projectors_bspline.py:83-108): row flip, the reference's
      filter_proj, the compiled reference backprojector with the degree-0 LUT,
      pi/(2 na) or pi/na, 180-degree rotation;
    * ``grid/<case>``: the compiled reference gridding adjoint with every
      built-in filter (param[1] = 2..6) and with differential phase contrast
      (radon_degree 1).
    """
    import importlib.util
    R = RefLib()
    rng = np.random.default_rng(20261203)
    spec = importlib.util.spec_from_file_location(
        "ref_filters", REFERENCE_TREE / "common/operators/filters_module/filters.py")
    if not hasattr(np, "int"):
        np.int = int  # the reference module reads np.int at import
    ref_filters = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref_filters)
    data = {}
    for ftype, dpc in [("ramp", False), ("shepp-logan", False), ("cosine", False), ("hamming", False),
                       ("hanning", False), ("none", False), ("ramp", True), ("none", True)]:
        sino = rng.standard_normal((23, 77)).astype(np.float32)
        data[f"filter/{ftype}_{int(dpc)}/in"] = sino
        data[f"filter/{ftype}_{int(dpc)}/out"] = ref_filters.filter_proj(sino.copy(), ftype=ftype, dpc=dpc)

    for name, n, na, deg, sup, rdeg in [("n64_a90_cubic_dpc", 64, 90, 3, 4.0, 1), ("n65_a37_cubic", 65, 37, 3, 4.0, 0),
                                        ("n48_a30_linear", 48, 30, 1, 2.0, 0)]:
        ang = (np.arange(na) * 180.0) / np.float32(na)  # class_projectors_bspline.py:49-50
        lut = init_lut_bspline(2048, ang, deg, rdeg, sup).astype(np.float32)
        lut0 = init_lut_bspline(2048, ang, deg, 0, sup).astype(np.float32)
        param = np.array([lut.shape[1], sup], np.float32)
        sino = rng.standard_normal((na, n)).astype(np.float32)
        x0 = sino[:, ::-1].copy()
        x0[:] = ref_filters.filter_proj(x0, ftype="ramp", dpc=rdeg != 0)
        reco = R.bspline(1, x0.astype(np.float32), ang.astype(np.float32), lut0, param)
        reco = reco * (np.pi / (1.0 * na) if rdeg else np.pi / (2.0 * na))
        data[f"bspline/{name}/cfg"] = np.array([n, na, deg, sup, rdeg], np.float64)
        data[f"bspline/{name}/sino"] = sino
        data[f"bspline/{name}/fbp"] = reco[::-1, ::-1].copy()

    from iterative_tomographic_reconstruction_algorithms_b200 import gridrec_lut as glut
    for name, n, na, kernel, os_, interp, W, errs, rdeg, filt in [
            ("n72_pswf_shlo", 72, 64, "pswf", 2.0, "nn", 7.0, 1e-3, 0, 2),
            ("n72_pswf_hann", 72, 64, "pswf", 2.0, "nn", 7.0, 1e-3, 0, 3),
            ("n72_kb_hamm", 72, 64, "kb", 2.0, "lin", 6.0, 6e-6, 0, 4),
            ("n90_pswf_lanc", 90, 81, "pswf", 2.0, "nn", 7.0, 1e-3, 0, 5),
            ("n90_kb_parz", 90, 81, "kb", 1.5, "lin", 6.6, 6e-6, 0, 6),
            ("n64_prolate_dpc_ramp", 64, 60, "prolate", 2.0, "nn", 7.0, 1e-3, 1, 1),
            ("n64_pswf_dpc_hann", 64, 60, "pswf", 2.0, "nn", 7.0, 1e-3, 1, 3)]:
        Wp, lut, deapod = glut.configure_regridding(n, kernel, os_, interp, W, errs)
        param = np.array([0.0, filt, 0, os_, 0 if interp == "nn" else 1, len(lut) - 5, Wp, rdeg], np.float32)
        deg = np.linspace(0, 180, na, endpoint=False).astype(np.float32)
        sino = rng.standard_normal((na, n)).astype(np.float32)
        data[f"grid/{name}/cfg"] = np.array([n, na, os_, 0 if interp == "nn" else 1, W, errs, rdeg, filt], np.float64)
        data[f"grid/{name}/kernel"] = np.array(kernel)
        data[f"grid/{name}/sino"] = sino
        data[f"grid/{name}/fbp"] = R.gridrec(1, sino, deg, param, lut.astype(np.float32), deapod.astype(np.float32))
    np.savez_compressed(OUT / "fbp_golden.npz", **data)
    print("wrote fbp_golden.npz")


if __name__ == "__main__":
    if sys.argv[1:] == ["fbp"]:
        make_fbp()
    else:
        main()
        if "--radon-only" not in sys.argv:
            make_fbp()
