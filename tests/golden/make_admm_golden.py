"""Reference outputs of the ADMM / CG solvers on seeded distance-driven problems.

Runs the reference's own solver functions -- algorithms/admm.py conj_grad,
lasso_l1 and lasso_tv with their inner algorithms/cg.py loops and
algorithms/utils.py -- imported from the reference tree, over the compiled
reference dd projector (oracle/_ref, ``make -C oracle ref``).  Each case also
records its noise floor: the relative change of the reference's own result
when the same solver runs on the float64-accumulating dd oracle instead (only
the projector's float32 accumulation rounding differs).  The plotting,
image-IO and projector-class modules those files import but these functions
do not use are replaced by empty modules, and multiprocessing.Pool by an
in-process pool (apply_async runs the call at once), as the drop-in package
does.  Writes admm_golden.npz:

    python tests/golden/make_admm_golden.py
"""
from __future__ import annotations

import sys
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import REFERENCE_TREE, Oracle, RefLib, radon_angles  # noqa: E402

REF_ALGOS = REFERENCE_TREE / "algorithms"
from iterative_tomographic_reconstruction_algorithms_b200.phantom import random_ellipses  # noqa: E402

OUT = Path(__file__).resolve().parent


class _Result:
    def __init__(self, v):
        self.v = v

    def get(self):
        return self.v


class _Pool:
    def __init__(self, *a, **k):
        pass

    def apply_async(self, f, args=(), kwds=None):
        return _Result(f(*args, **(kwds or {})))

    def close(self):
        pass

    def join(self):
        pass


def load_reference():
    np.int = int  # the reference modules read np.int at import
    for name in ("pylab", "matplotlib", "matplotlib.pyplot", "matplotlib.cm", "matplotlib.animation",
                 "my_image_io", "my_image_process", "my_image_display", "my_image_denoise",
                 "bspline_functions", "class_projectors_grid", "class_projectors_bspline",
                 "class_projectors_radon", "class_admm_param"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.path.insert(0, str(REF_ALGOS))
    import admm  # noqa: E402  (the reference's)
    admm.mproc = types.SimpleNamespace(Pool=_Pool)
    return admm


class RefDD:
    """class_projectors_radon.projectors(n, angles, oper='dd') over the compiled reference C."""

    def __init__(self, R, n, deg):
        self.R, self.n, self.ang = R, n, radon_angles(deg)
        self.nang = len(deg)

    def A(self, x):
        return self.R.radon("dd", 0, np.asarray(x).astype(np.float32), self.ang)

    def At(self, y):
        return self.R.radon("dd", 1, np.asarray(y).astype(np.float32), self.ang)


class Fp64DD(RefDD):
    """The same dd geometry and bin decisions, accumulated in float64 (the
    project's oracle, oracle/tomo_oracle.c), rounded to float32: the reference
    operator without its float32 accumulation rounding."""

    def A(self, x):
        return self.R.radon("dd", 0, np.asarray(x).astype(np.float32), self.ang).astype(np.float32)

    def At(self, y):
        return self.R.radon("dd", 1, np.asarray(y).astype(np.float32), self.ang).astype(np.float32)


class RefGrid:
    """class_projectors_grid.projectors(n, angles, kernel='kb', oversampl=1.5, W=6.6, errs=6e-6,
    interp='lin') -- admm.py's 'grid-kb' projector (admm.py:885-887) -- over the compiled reference C."""

    def __init__(self, R, n, deg):
        from iterative_tomographic_reconstruction_algorithms_b200 import gridrec_lut as glut
        W, lut, deapod = glut.configure_regridding(n, "kb", 1.5, "lin", 6.6, 6e-6)
        self.R, self.deg = R, np.asarray(deg, np.float32)
        self.lut, self.deapod = lut.astype(np.float32), deapod.astype(np.float32)
        self.param = np.array([0.0, 0, 0, 1.5, 1, len(lut) - 5, W, 0], np.float32)
        self.nang = len(deg)

    def A(self, x):
        return self.R.gridrec(0, np.asarray(x).astype(np.float32), self.deg, self.param, self.lut, self.deapod)

    def At(self, y):
        return self.R.gridrec(1, np.asarray(y).astype(np.float32), self.deg, self.param, self.lut, self.deapod)


def param_ns(**kw):
    base = dict(lambd1=np.float32(0), lambd2=np.float32(0), mu=np.float32(1), n_iter=3, n_iter_pcg=4, eps=None,
                pc=np.float32(-1.0), edge_padding=0.0, index_start=0, index_end=0, mask=None, mask_add=None,
                plot=False, checkit=False, num_cores=1, projector="dist-driv", npix_op=0, nz=1)
    base.update(kw)
    return types.SimpleNamespace(**base)


def main() -> None:
    admm = load_reference()
    R = RefLib()
    O = Oracle()
    rng = np.random.default_rng(20261204)
    data = {}
    cases = [
        # name, reg, n, na, nz, lambd1, lambd2, mu, n1, n2, pc, edge (i1, i2) or None
        ("tv_n48", "lasso-tv", 48, 60, 2, 0.5, 2.0, 40.0, 3, 4, -1.0, None),
        ("tv_n37_pc", "lasso-tv", 37, 45, 1, 0.1, 1.0, 20.0, 3, 3, 0.0, None),
        ("tv_n40_circle", "lasso-tv", 40, 50, 1, 0.2, 0.5, 10.0, 2, 4, 1.0, (4, 36)),
        ("l1_n48", "lasso", 48, 60, 2, 0.5, 5.0, 30.0, 3, 4, -1.0, None),
        ("l1_n33_pc", "lasso", 33, 40, 1, 1.0, 2.0, 15.0, 3, 3, 0.5, (3, 30)),
        ("cg_n48", "cg", 48, 60, 1, 0.0, 0.0, 1.0, 6, 0, -1.0, None),
        ("grid_tv_n64", "lasso-tv", 64, 72, 1, 0.1, 1.0, 20.0, 2, 3, -1.0, None),
    ]
    for name, reg, n, na, nz, l1, l2, mu, n1, n2, pc, edge in cases:
        deg = np.linspace(0, 180, na, endpoint=False)
        tp = RefGrid(R, n, deg) if name.startswith("grid") else RefDD(R, n, deg)
        b = np.empty((nz, na, n), np.float32)
        for s in range(nz):
            ph = random_ellipses(n, seed=int(rng.integers(1 << 30))).astype(np.float32)
            bs = tp.A(ph)
            b[s] = bs + 0.01 * float(bs.max()) * rng.standard_normal(bs.shape).astype(np.float32)
        x0 = np.ones((nz, n, n), np.float32)  # admm.py:912
        kw = dict(lambd1=np.float32(l1), lambd2=np.float32(l2), mu=np.float32(mu), n_iter=n1, n_iter_pcg=n2,
                  pc=np.float32(pc), npix_op=n, nz=nz)
        if edge is not None:
            kw.update(edge_padding=1.0, index_start=edge[0], index_end=edge[1])
        prm = param_ns(**kw)
        fn = {"lasso-tv": admm.lasso_tv, "lasso": admm.lasso_l1, "cg": admm.conj_grad}[reg]
        x, info = fn(x0.copy(), b, tp, prm)
        data[f"{name}/cfg"] = np.array([n, na, nz, l1, l2, mu, n1, n2, pc,
                                        -1 if edge is None else edge[0], -1 if edge is None else edge[1]],
                                       np.float64)
        data[f"{name}/reg"] = np.array(reg)
        data[f"{name}/b"] = b
        data[f"{name}/x"] = np.asarray(x, np.float32)
        data[f"{name}/info"] = np.asarray(info, np.float64)
        # noise floor: how far the reference's own result moves when only its
        # projector's float32 accumulation rounding changes (the same solver on
        # the float64-accumulating dd oracle); no such oracle for gridding: 0
        floor = 0.0
        if not name.startswith("grid"):
            x64, _ = fn(x0.copy(), b, Fp64DD(O, n, deg), prm)
            floor = float(np.linalg.norm(np.asarray(x64, np.float64) - x) / np.linalg.norm(np.asarray(x, np.float64)))
        data[f"{name}/floor"] = np.array([floor])
        print(name, np.asarray(info)[-1], "floor", floor)
    np.savez_compressed(OUT / "admm_golden.npz", **data)
    print("wrote admm_golden.npz")


if __name__ == "__main__":
    main()
