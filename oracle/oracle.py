"""Oracle side of the projector pair: TEST INFRASTRUCTURE ONLY.

Two CPU implementations live behind this module, and only the test-suite,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may use them:

* ``RefLib`` drives the reference C kernels compiled from the reference tree into
  ``oracle/_ref/*.so`` (``make -C oracle ref``).  Each method restates the thin
  Cython shim that the reference puts in front of its C function (angle
  conversion, ``fftshift``, zeroed output), so a call here is what the
  reference's projector classes compute:
    - pd  radon_pixel_driven.pyx:15-41 (forward), :48-73 (adjoint)
    - rd  radon_ray_driven.pyx:15-35, :42-61
    - dd  radon_distance_driven.pyx:14-35, :42-62
    - ss  radon_slant_stacking.pyx:15-41, :48-73
    - bspline genradon.pyx:19-42, :48-68
    - gridrec gridrec_v4.pyx:28-54 (adjoint), :60-86 (forward)
* ``Oracle`` drives ``oracle/liboracle.so``, the project's own restatement of
  the same kernels (tomo_oracle.c, tomo_oracle_grid.c) with identical float32
  geometry and bin decisions but FP64 accumulation; outputs are float64.

Neither is ever on the product path: the package fails loudly when its CUDA
library is missing instead of falling back to anything here.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
# The reference source tree, read by the fixture generators, the CPU tests that
# import the reference's own Python, and `make -C oracle ref` (its REF variable).
# It is absent on machines that only run the GPU tests.
REFERENCE_TREE = Path(os.environ.get("TOMO_REFERENCE_TREE", "/root/reference"))
ORACLE_SO = HERE / "liboracle.so"

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)


def _fp(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_f32p)


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_f64p)


def radon_angles(angles_deg) -> np.ndarray:
    """Angle conversion of class_projectors_radon.py:49,54 (degrees -> float32 rad)."""
    a = np.asarray(angles_deg)
    return (a * np.pi / 180.0).astype(np.float32)


def sinogram_row_of_angle(kind: str, na: int) -> np.ndarray:
    """row[k] = the sinogram row that holds angle k (in the order passed to the
    class) in the reference's projector output.

    pd and dd shims pass ``fftshift(angles)`` to the C (radon_pixel_driven.pyx:30,
    radon_distance_driven.pyx:27); dd and ss write angle v of their C loop to row
    ``nang-1-v`` (radon_dd.c:181,273, radon_ss.c:111); pd and rd write row v.
    The B-spline pair keeps the class order (gen_forwproj.c:45-75)."""
    order = np.arange(na)
    if kind in ("pd", "dd"):
        order = np.fft.fftshift(order)           # C-loop index v -> class angle index
    rows = np.empty(na, np.int64)
    rows[order] = np.arange(na)
    if kind in ("dd", "ss"):
        rows = na - 1 - rows
    return rows


def ref_available(ref_dir: Path | None = None) -> bool:
    d = Path(ref_dir) if ref_dir else REF_DIR
    return all((d / f"ref_{k}.so").exists() for k in ("pd", "rd", "dd", "ss", "genradon", "gridrec"))


class RefLib:
    """The reference's compiled C kernels behind a restatement of their Cython shims."""

    def __init__(self, ref_dir: Path | None = None):
        d = Path(ref_dir) if ref_dir else REF_DIR
        L = {}
        for k in ("pd", "rd", "dd", "ss", "genradon", "gridrec"):
            p = d / f"ref_{k}.so"
            if not p.exists():
                raise FileNotFoundError(f"{p} missing: run `make -C oracle ref`")
            L[k] = ctypes.CDLL(str(p), mode=os.RTLD_LOCAL)
        self.L = L
        i, f = ctypes.c_int, ctypes.c_float
        L["pd"].radon_pd.argtypes = [_f32p, i, _f32p, i, i, i, _f32p]
        L["rd"].radon_rd.argtypes = [_f32p, i, _f32p, i, i, _f32p]
        L["dd"].radon_dd.argtypes = [_f32p, i, _f32p, i, i, _f32p]
        L["ss"].radon_ss.argtypes = [_f32p, i, _f32p, i, i, i, _f32p]
        L["genradon"].gen_forwproj.argtypes = [_f32p, i, _f32p, i, _f32p, i, f, i, _f32p]
        L["genradon"].gen_backproj.argtypes = [_f32p, i, _f32p, i, _f32p, i, f, _f32p]
        cp = ctypes.c_char_p
        L["gridrec"].gridrec_v4_forwproj.argtypes = [_f32p, i, i, _f32p, _f32p, _f32p, _f32p, _f32p, cp]
        L["gridrec"].gridrec_v4_backproj.argtypes = [_f32p, i, i, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, cp]

    # ---- Radon family: angles are the float32 radians held by the class ----
    @staticmethod
    def _shim_angles(angles: np.ndarray, shift: bool, factor: float) -> np.ndarray:
        a = np.ascontiguousarray(angles, dtype=np.float32).copy()
        if np.max(a) > 2 * np.pi:
            a *= factor
        if shift:
            a = np.fft.fftshift(a)
        return np.ascontiguousarray(a, dtype=np.float32)

    def radon(self, kind: str, oper: int, data: np.ndarray, angles: np.ndarray) -> np.ndarray:
        """oper 0: data is the [n,n] image, returns the [na,n] sinogram; oper 1: the reverse."""
        data = np.ascontiguousarray(data, dtype=np.float32)
        na = len(angles)
        if oper == 0:
            n = data.shape[0]
            img, sino = data, np.zeros((na, n), np.float32)
        else:
            n = data.shape[1]
            sino, img = data, np.zeros((n, n), np.float32)
        if kind == "pd":
            a = self._shim_angles(angles, True, 2 * np.pi / 180.0)
            self.L["pd"].radon_pd(_fp(img), n, _fp(a), na, oper, 1, _fp(sino))
        elif kind == "rd":
            a = self._shim_angles(angles, False, np.pi / 180.0)
            self.L["rd"].radon_rd(_fp(img), n, _fp(a), na, oper, _fp(sino))
        elif kind == "dd":
            a = self._shim_angles(angles, True, np.pi / 180.0)
            self.L["dd"].radon_dd(_fp(img), n, _fp(a), na, oper, _fp(sino))
        elif kind == "ss":
            a = self._shim_angles(angles, False, 2 * np.pi / 180.0)
            self.L["ss"].radon_ss(_fp(img), n, _fp(a), na, oper, 1, _fp(sino))
        else:
            raise ValueError(kind)
        return sino if oper == 0 else img

    # ---- B-spline pair: angles in degrees, LUT [na, lut_size] ----
    def bspline(self, oper: int, data, angles_deg, lut, param) -> np.ndarray:
        data = np.ascontiguousarray(data, dtype=np.float32)
        a = np.ascontiguousarray(angles_deg, dtype=np.float32)
        lut = np.ascontiguousarray(lut, dtype=np.float32)
        na = len(a)
        lut_size = int(param[0])
        support = float(np.float32(param[1]))
        if oper == 0:
            n = data.shape[0]
            sino = np.zeros((na, n), np.float32)
            self.L["genradon"].gen_forwproj(_fp(data), n, _fp(a), na, _fp(lut), lut_size,
                                            support, os.cpu_count() or 1, _fp(sino))
            return sino
        n = data.shape[1]
        img = np.zeros((n, n), np.float32)
        self.L["genradon"].gen_backproj(_fp(data), n, _fp(a), na, _fp(lut), lut_size, support, _fp(img))
        return img

    # ---- Gridding pair ----
    def gridrec(self, oper: int, data, angles_deg, param, lut, deapod, filt=None) -> np.ndarray:
        data = np.ascontiguousarray(data, dtype=np.float32)
        a = np.ascontiguousarray(angles_deg, dtype=np.float32)
        param = np.ascontiguousarray(param, dtype=np.float32)
        lut = np.ascontiguousarray(lut, dtype=np.float32)
        deapod = np.ascontiguousarray(deapod, dtype=np.float32)
        na = len(a)
        if oper == 0:
            n = data.shape[0]
            sino = np.zeros((na, n), np.float32)
            self.L["gridrec"].gridrec_v4_forwproj(_fp(sino), n, na, _fp(a), _fp(param), _fp(lut),
                                                  _fp(deapod), _fp(data), b"/dev/null")
            return sino
        n = data.shape[1]
        img = np.zeros((n, n), np.float32)
        fp = None if filt is None else _fp(np.ascontiguousarray(filt, dtype=np.float32))
        self.L["gridrec"].gridrec_v4_backproj(_fp(data), n, na, _fp(a), _fp(param), _fp(lut),
                                              _fp(deapod), fp, _fp(img), b"/dev/null")
        return img


class Oracle:
    """The project's FP64 restatement (liboracle.so); same shim semantics as ``RefLib``."""

    def __init__(self, so_path: Path | None = None):
        p = Path(so_path) if so_path else ORACLE_SO
        if not p.exists():
            raise FileNotFoundError(f"{p} missing: run `make -C oracle`")
        self.L = L = ctypes.CDLL(str(p), mode=os.RTLD_LOCAL)
        i = ctypes.c_int
        for k in ("pd", "rd", "dd", "ss"):
            getattr(L, f"orc_{k}").argtypes = [_f32p, i, _f32p, i, i, _f64p]
        L.orc_bspline.argtypes = [_f32p, i, _f32p, i, _f32p, i, ctypes.c_float, i, _f64p]

    def radon(self, kind: str, oper: int, data, angles) -> np.ndarray:
        data = np.ascontiguousarray(data, dtype=np.float32)
        na = len(angles)
        shift = kind in ("pd", "dd")
        factor = (2 * np.pi if kind in ("pd", "ss") else np.pi) / 180.0
        a = RefLib._shim_angles(angles, shift, factor)
        n = data.shape[0] if oper == 0 else data.shape[1]
        out = np.zeros((na, n) if oper == 0 else (n, n), np.float64)
        getattr(self.L, f"orc_{kind}")(_fp(data), n, _fp(a), na, oper, _dp(out))
        return out

    def bspline(self, oper: int, data, angles_deg, lut, param) -> np.ndarray:
        data = np.ascontiguousarray(data, dtype=np.float32)
        a = np.ascontiguousarray(angles_deg, dtype=np.float32)
        lut = np.ascontiguousarray(lut, dtype=np.float32)
        na = len(a)
        n = data.shape[0] if oper == 0 else data.shape[1]
        out = np.zeros((na, n) if oper == 0 else (n, n), np.float64)
        self.L.orc_bspline(_fp(data), n, _fp(a), na, _fp(lut), int(param[0]),
                           float(np.float32(param[1])), oper, _dp(out))
        return out


def read_tiff_strip(path) -> np.ndarray:
    """Minimal reader for the reference's uncompressed single-image TIFF data files
    (data/*.tif): little-endian, one strip or contiguous strips, float32/float64."""
    import struct
    raw = Path(path).read_bytes()
    assert raw[:2] == b"II", "big-endian TIFF not supported"
    off = struct.unpack_from("<I", raw, 4)[0]
    n = struct.unpack_from("<H", raw, off)[0]
    tags = {}
    types = {3: ("H", 2), 4: ("I", 4)}
    for i in range(n):
        tag, typ, cnt, val = struct.unpack_from("<HHII", raw, off + 2 + 12 * i)
        if typ in types:
            fmt, size = types[typ]
            if cnt * size <= 4:
                vals = struct.unpack_from("<" + fmt * cnt, raw, off + 2 + 12 * i + 8)
            else:
                vals = struct.unpack_from("<" + fmt * cnt, raw, val)
            tags[tag] = vals
    width, height = tags[256][0], tags[257][0]
    bits = tags.get(258, (32,))[0]
    fmt = tags.get(339, (3,))[0]
    assert fmt == 3 and tags.get(259, (1,))[0] == 1, "only uncompressed IEEE float supported"
    dtype = np.dtype("<f8") if bits == 64 else np.dtype("<f4")
    strips, counts = tags[273], tags[279]
    buf = b"".join(raw[o:o + c] for o, c in zip(strips, counts))
    return np.frombuffer(buf, dtype=dtype, count=width * height).reshape(height, width).copy()
