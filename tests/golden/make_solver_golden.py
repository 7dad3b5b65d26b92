"""Generate solver golden fixtures by running the REFERENCE solvers themselves.

Needs the reference tree and the compiled reference C (``make -C oracle ref``):

    python tests/golden/make_solver_golden.py

The reference's own ``algorithms/art.py`` (``sirt``, :215-365) and
``algorithms/sir.py`` (``em`` :204-324, ``sps`` :348-600) are imported
unchanged.  Only what they import for plotting, IO and the other projector
families is replaced by empty stand-in modules, ``multiprocessing.Pool`` by an
in-process pool (the computation is the same; only the forking is skipped),
and the projector object by one that calls the compiled reference C through a
restatement of its Cython shim (oracle/oracle.py: RefLib).  The resulting
reconstructions are stored in ``solver_golden.npz``:

* ``sirt_rd``: plain SIRT with the ray-driven pair, 256x256 random-ellipse
  phantom (seed 0), 304 angles on [0, 180), noiseless sinogram from the same
  projector, x0 = 1, 100 iterations;
* ``sps_dd``: SPS (no regularisation), 50 iterations, with the distance-driven
  pair on a reduced version of the transmission workload: 96x96 phantom scaled
  to mu in [0, 0.02] embedded in a 144x144 operator, 160 angles,
  counts ~ Poisson(1e4 exp(-Ax)) (seed 1), b = -log(max(counts,1)/1e4);
* ``em_dd``: MLEM, 50 iterations, same geometry on the noiseless sinogram
  b = A mu.  On the noisy data above b is negative where Ax ~ 0 and the
  multiplicative MLEM update from x0 = 1 diverges in the reference itself
  (relative residual 22 after 50 iterations), amplifying float rounding
  differences, so it cannot serve as a parity pin.

``python tests/golden/make_solver_golden.py --only em_dd`` regenerates one
entry and keeps the others.

``python tests/golden/make_solver_golden.py --c2 em`` (or ``--c2 sps``) runs the
transmission workload at its full size instead: 512x512 phantom (seed 1) scaled
to mu in [0, 0.02], embedded in a 768x768 operator, 720 angles on [0, 180),
768 bins, 50 iterations of the reference ``sir.em`` (noiseless b = A mu) or
``sir.sps`` (b from Poisson(1e4 exp(-A mu)) counts, seed 1), each in its own
file ``solver_c2_<algo>.npz`` with the sinogram, the result and the reference's
wall time.  One run takes about two hours on one core; the two can run at the
same time.
"""
from __future__ import annotations

import importlib.util
import sys
import time
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import REFERENCE_TREE as REF, RefLib, radon_angles  # noqa: E402
from iterative_tomographic_reconstruction_algorithms_b200.phantom import embed, random_ellipses  # noqa: E402

OUT = Path(__file__).resolve().parent / "solver_golden.npz"


class _Result:
    def __init__(self, v):
        self.v = v

    def get(self):
        return self.v


class InProcessPool:
    """multiprocessing.Pool stand-in: apply_async runs the call immediately."""

    def __init__(self, *a, **k):
        pass

    def apply_async(self, f, args=(), kwds=None):
        return _Result(f(*args, **(kwds or {})))

    def close(self):
        pass

    def join(self):
        pass


def load_reference_solvers():
    np.int = int  # the reference uses np.int (removed from NumPy)
    for name in ["matplotlib", "matplotlib.pyplot", "matplotlib.cm", "matplotlib.animation", "pylab",
                 "my_image_io", "my_image_process", "my_image_display", "my_image_denoise", "utils",
                 "class_projectors_grid", "class_projectors_bspline", "class_projectors_radon",
                 "class_art_param", "class_sir_param", "penalty"]:
        sys.modules.setdefault(name, types.ModuleType(name))
    mp = types.ModuleType("mproc_inprocess")
    mp.Pool = InProcessPool
    mods = {}
    for name in ("art", "sir"):
        spec = importlib.util.spec_from_file_location(f"reference_{name}", REF / "algorithms" / f"{name}.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.mproc = mp
        mods[name] = mod
    return mods["art"], mods["sir"]


class RefProjector:
    """tp.A / tp.At of class_projectors_radon, computed by the compiled reference C."""

    def __init__(self, R, kind, angles_deg):
        self.R, self.kind = R, kind
        self.angles = radon_angles(angles_deg)
        self.nang = len(angles_deg)

    def A(self, x):
        return self.R.radon(self.kind, 0, np.asarray(x, np.float32), self.angles)

    def At(self, y):
        return self.R.radon(self.kind, 1, np.asarray(y, np.float32), self.angles)


def transmission_sino(tp, mu, seed, i0=1e4):
    rng = np.random.default_rng(seed)
    counts = rng.poisson(i0 * np.exp(-tp.A(mu).astype(np.float64)))
    return (-np.log(np.maximum(counts, 1) / i0)).astype(np.float32)


def c2_transmission(algo: str) -> None:
    """MLEM or SPS with the distance-driven pair at the full transmission size."""
    art, sir = load_reference_solvers()
    R = RefLib()
    side, n_op, na = 512, 768, 720
    deg = np.linspace(0, 180, na, endpoint=False)
    tp = RefProjector(R, "dd", deg)
    ph = random_ellipses(side, seed=1)
    mu = embed(ph / max(float(ph.max()), 1e-12) * 0.02, n_op).astype(np.float32)
    bb = (tp.A(mu) if algo == "em" else transmission_sino(tp, mu, seed=1))[None]
    P = types.SimpleNamespace(eps=-1.0, n_iter=50, edge_padding=False, plot=False, num_cores=-1,
                              checkit=False, projector="dist-driv", reg=None, reg_cost=0.0,
                              huber_cost=None, index_start=0, index_end=n_op)
    t0 = time.time()
    x, info = getattr(sir, algo)(np.ones((1, n_op, n_op), np.float32), bb.copy(), tp, P)
    secs = time.time() - t0
    print(f"c2 {algo}: {secs:.1f} s")
    out = OUT.parent / f"solver_c2_{algo}.npz"
    np.savez_compressed(out, angles_deg=deg, b=bb[0], x50=np.asarray(x, np.float32)[0],
                        ref_seconds=np.array([secs]))
    print("wrote", out)


def main() -> None:
    if "--c2" in sys.argv:
        c2_transmission(sys.argv[sys.argv.index("--c2") + 1])
        return
    only = sys.argv[sys.argv.index("--only") + 1].split(",") if "--only" in sys.argv else None
    art, sir = load_reference_solvers()
    R = RefLib()
    data = dict(np.load(OUT)) if (only and OUT.exists()) else {}

    def want(name):
        return only is None or name in only

    # SIRT, ray-driven, 256^2 x 304, 100 iterations
    n, na = 256, 304
    deg = np.linspace(0, 180, na, endpoint=False)
    tp = RefProjector(R, "rd", deg)
    img = random_ellipses(n, seed=0)
    b = tp.A(img)[None]
    P = types.SimpleNamespace(npix_op=n, nz=1, nang=na, eps=None, n_iter=100, edge_padding=0.0,
                              plot=False, tv=0.0, mask=None, mask_add=None, pc=-1.0, checkit=False,
                              projector="ray-driv")
    if want("sirt_rd"):
        t0 = time.time()
        x, info = art.sirt(np.ones((1, n, n), np.float32), b.copy(), tp, P)
        print(f"sirt_rd: {time.time() - t0:.1f} s")
        data.update({"sirt_rd/angles_deg": deg, "sirt_rd/b": b[0],
                     "sirt_rd/x100": np.asarray(x, np.float32)[0],
                     "sirt_rd/obj": np.asarray(info, np.float64)[:, 1]})

    # MLEM and SPS, distance-driven, transmission data
    side, n_op, na = 96, 144, 160
    deg = np.linspace(0, 180, na, endpoint=False)
    tp = RefProjector(R, "dd", deg)
    ph = random_ellipses(side, seed=1)
    mu = embed(ph / max(float(ph.max()), 1e-12) * 0.02, n_op).astype(np.float32)
    b = transmission_sino(tp, mu, seed=1)[None]
    b_clean = tp.A(mu)[None]
    data.update({"mlsps/angles_deg": deg, "mlsps/b": b[0], "mlsps/mu": mu, "mlsps/b_clean": b_clean[0]})
    for algo, bb in (("em", b_clean), ("sps", b)):
        if not want(f"{algo}_dd"):
            continue
        P = types.SimpleNamespace(eps=-1.0, n_iter=50, edge_padding=False, plot=False, num_cores=-1,
                                  checkit=False, projector="dist-driv", reg=None, reg_cost=0.0,
                                  huber_cost=None, index_start=0, index_end=n_op)
        t0 = time.time()
        x, info = getattr(sir, algo)(np.ones((1, n_op, n_op), np.float32), bb.copy(), tp, P)
        print(f"{algo}_dd: {time.time() - t0:.1f} s")
        data[f"{algo}_dd/x50"] = np.asarray(x, np.float32)[0]
    np.savez_compressed(OUT, **data)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
