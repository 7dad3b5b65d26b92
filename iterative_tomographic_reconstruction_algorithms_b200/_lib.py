"""ctypes binding of libtomo_b200.so (include/tomo_b200.h).

The shared library is built in-tree (``csrc/Makefile``) and is the only
compute path: there is no CPU fallback.  Importing this module on a machine
without the library raises immediately; calling a projector on a machine
without a CUDA device raises at plan creation.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libtomo_b200.so"

TOMO_OK = 0
TOMO_ENOMEM = 12
TOMO_EINVAL = 22
TOMO_ETIMEDOUT = 110
TOMO_ECUDA = 1000

KIND_PD, KIND_RD, KIND_DD, KIND_SS, KIND_BSPLINE, KIND_GRID = range(6)
KIND_NAMES = {"pd": KIND_PD, "rd": KIND_RD, "dd": KIND_DD, "ss": KIND_SS,
              "bspline": KIND_BSPLINE, "grid": KIND_GRID}

_f32p = ctypes.POINTER(ctypes.c_float)


class TomoGeom(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("n", ctypes.c_int),
        ("na", ctypes.c_int),
        ("nz", ctypes.c_int),
        ("angles", _f32p),
        ("lut", _f32p),
        ("lut_size", ctypes.c_int),
        ("support", ctypes.c_float),
        ("grid_param", _f32p),
        ("grid_lut", _f32p),
        ("grid_lut_len", ctypes.c_int),
        ("grid_deapod", _f32p),
        ("grid_mode", ctypes.c_int),
    ]


class TomoError(RuntimeError):
    """A libtomo_b200 call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR / 'csrc'}` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    lib = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_GLOBAL)
    vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    lib.tomo_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.tomo_version.restype = ctypes.c_char_p
    lib.tomo_plan_create.argtypes = [ctypes.POINTER(TomoGeom), ctypes.POINTER(vp)]
    lib.tomo_plan_destroy.argtypes = [vp]
    for name in ("tomo_forward", "tomo_adjoint"):
        getattr(lib, name).argtypes = [vp, vp, vp, vp]
    for name in ("tomo_forward_host", "tomo_adjoint_host"):
        getattr(lib, name).argtypes = [vp, vp, vp]
    for name in ("tomo_radon_dd", "tomo_radon_rd"):
        getattr(lib, name).argtypes = [_f32p, i, _f32p, i, i, _f32p]
    for name in ("tomo_radon_pd", "tomo_radon_ss"):
        getattr(lib, name).argtypes = [_f32p, i, _f32p, i, i, i, _f32p]
    lib.tomo_gen_forwproj.argtypes = [_f32p, i, _f32p, i, _f32p, i, f, i, _f32p]
    lib.tomo_gen_backproj.argtypes = [_f32p, i, _f32p, i, _f32p, i, f, _f32p]
    lib.tomo_measure_onchip_peaks.argtypes = [ctypes.POINTER(ctypes.c_double)] * 3
    lib.tomo_plan_create_batch.argtypes = [ctypes.POINTER(TomoGeom), i, ctypes.POINTER(vp)]
    lib.tomo_plan_layout.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_size_t),
                                     ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t]
    lib.tomo_plan_tuning.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    lib.tomo_plan_set_tuning.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p]
    return lib


lib = _load()


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib.tomo_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, what: str = "") -> None:
    if rc != TOMO_OK:
        msg = last_error()
        if rc == TOMO_EINVAL:
            raise ValueError(f"{what}: {msg}")
        raise TomoError(rc, f"{what}: {msg}")


def _torch():
    import torch  # deferred: numpy-only users never pay the import
    return torch


class Plan:
    """One projector geometry on one device (a ``tomo_plan``).

    ``angles_c`` is the angle array exactly as the reference C function
    receives it (after its Cython shim).  ``forward``/``adjoint`` accept either
    numpy arrays (host path: copies in and out, returns numpy) or CUDA float32
    torch tensors (device path on the current stream, returns a tensor).
    """

    def __init__(self, kind: int, n: int, angles_c: np.ndarray, nz: int = 1, **extra):
        self.kind, self.n, self.nz = int(kind), int(n), int(nz)
        self.angles_c = np.ascontiguousarray(angles_c, dtype=np.float32)
        self.na = len(self.angles_c)
        self._keep = [self.angles_c]
        g = TomoGeom()
        g.kind, g.n, g.na, g.nz = self.kind, self.n, self.na, self.nz
        g.angles = self.angles_c.ctypes.data_as(_f32p)
        for key, val in extra.items():
            if isinstance(val, np.ndarray):
                arr = np.ascontiguousarray(val, dtype=np.float32)
                self._keep.append(arr)
                setattr(g, key, arr.ctypes.data_as(_f32p))
            else:
                setattr(g, key, val)
        self._lock = threading.Lock()
        h = ctypes.c_void_p()
        check(lib.tomo_plan_create(ctypes.byref(g), ctypes.byref(h)), "tomo_plan_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.tomo_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def image_shape(self):
        return (self.nz, self.n, self.n)

    @property
    def sino_shape(self):
        return (self.nz, self.na, self.n)

    def _run(self, x, fwd: bool, out=None):
        in_shape = self.image_shape if fwd else self.sino_shape
        out_shape = self.sino_shape if fwd else self.image_shape
        if isinstance(x, np.ndarray):
            xin = np.ascontiguousarray(x, dtype=np.float32)
            if xin.size != int(np.prod(in_shape)):
                raise ValueError(f"expected {in_shape} elements, got shape {x.shape}")
            out = np.empty(out_shape, np.float32)
            fn = lib.tomo_forward_host if fwd else lib.tomo_adjoint_host
            with self._lock:
                check(fn(self._h, xin.ctypes.data, out.ctypes.data), "host projector call")
            return out
        torch = _torch()
        if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float32):
            raise TypeError("expected a numpy array or a CUDA float32 torch tensor")
        if x.numel() != int(np.prod(in_shape)):
            raise ValueError(f"expected {in_shape} elements, got shape {tuple(x.shape)}")
        xin = x.contiguous()
        if out is None:
            out = torch.empty(out_shape, dtype=torch.float32, device=x.device)
        elif not (isinstance(out, torch.Tensor) and out.is_cuda and out.dtype == torch.float32
                  and out.is_contiguous() and out.numel() == int(np.prod(out_shape)) and out.device == x.device):
            raise ValueError(f"out must be a contiguous CUDA float32 tensor of {out_shape} elements on x's device")
        stream = torch.cuda.current_stream(x.device).cuda_stream
        fn = lib.tomo_forward if fwd else lib.tomo_adjoint
        with self._lock:
            check(fn(self._h, xin.data_ptr(), out.data_ptr(), stream), "device projector call")
        return out

    def forward(self, x, out=None):
        """A x; ``out`` (device path only) receives the result in place of a new tensor."""
        return self._run(x, True, out)

    def adjoint(self, y, out=None):
        """A^T y; ``out`` (device path only) receives the result in place of a new tensor."""
        return self._run(y, False, out)

    def tuning(self) -> str:
        return plan_tuning(self)

    def set_tuning(self, fwd: str | None = None, adj: str | None = None) -> None:
        """Pins the distance-driven launch shapes by name (``tomo_plan_set_tuning``)."""
        check(lib.tomo_plan_set_tuning(self._h, fwd.encode() if fwd else None, adj.encode() if adj else None),
              "tomo_plan_set_tuning")


class BatchPlan(Plan):
    """Distance-driven plan over geometries of different sizes (``tomo_plan_create_batch``).

    ``geoms`` is a list of ``(n, angles_c)`` or ``(n, angles_c, nz)``.  Images
    and sinograms are packed back to back in that order (each slice C-order)
    into flat float32 arrays of ``img_total`` / ``sino_total`` elements;
    ``img_off`` / ``sino_off`` give each instance's start.  All instances run
    in one persistent launch per forward or adjoint.
    """

    def __init__(self, geoms):
        self.kind = KIND_DD
        self._keep = []
        arr = (TomoGeom * len(geoms))()
        for g, spec in zip(arr, geoms):
            n, ang = int(spec[0]), np.ascontiguousarray(spec[1], dtype=np.float32)
            self._keep.append(ang)
            g.kind, g.n, g.na = KIND_DD, n, len(ang)
            g.nz = int(spec[2]) if len(spec) > 2 else 1
            g.angles = ang.ctypes.data_as(_f32p)
        self._lock = threading.Lock()
        h = ctypes.c_void_p()
        check(lib.tomo_plan_create_batch(arr, len(geoms), ctypes.byref(h)), "tomo_plan_create_batch")
        self._h = h
        cnt = ctypes.c_int()
        check(lib.tomo_plan_layout(h, ctypes.byref(cnt), None, None, 0), "tomo_plan_layout")
        io = (ctypes.c_size_t * (cnt.value + 1))()
        so = (ctypes.c_size_t * (cnt.value + 1))()
        check(lib.tomo_plan_layout(h, None, io, so, cnt.value + 1), "tomo_plan_layout")
        self.instances = cnt.value
        self.img_off = np.array(io[:], dtype=np.int64)
        self.sino_off = np.array(so[:], dtype=np.int64)
        self.img_total, self.sino_total = int(self.img_off[-1]), int(self.sino_off[-1])
        self.n = self.na = self.nz = 0
        self._geoms = [(int(sp[0]), len(sp[1]), int(sp[2]) if len(sp) > 2 else 1) for sp in geoms]

    def pack(self, arrays, which: str = "img"):
        """Concatenate per-instance images (``which='img'``) or sinograms into the packed layout."""
        shapes = _batch_shapes(self, which)
        if len(arrays) != len(shapes):
            raise ValueError(f"expected {len(shapes)} arrays, got {len(arrays)}")
        for a, sh in zip(arrays, shapes):
            if tuple(a.shape) != sh:
                raise ValueError(f"expected shape {sh}, got {tuple(a.shape)}")
        if isinstance(arrays[0], np.ndarray):
            return np.concatenate([np.asarray(a, np.float32).ravel() for a in arrays])
        torch = _torch()
        return torch.cat([a.reshape(-1) for a in arrays])

    def unpack(self, flat, which: str = "img"):
        """Split a packed image or sinogram array into per-instance views."""
        off = self.img_off if which == "img" else self.sino_off
        shapes = _batch_shapes(self, which)
        return [flat[int(off[i]):int(off[i + 1])].reshape(sh) for i, sh in enumerate(shapes)]

    @property
    def image_shape(self):
        return (self.img_total,)

    @property
    def sino_shape(self):
        return (self.sino_total,)


def plan_tuning(plan: Plan) -> str:
    """The launch shape the plan chose (``tomo_plan_tuning``)."""
    buf = ctypes.create_string_buffer(512)
    check(lib.tomo_plan_tuning(plan._h, buf, len(buf)), "tomo_plan_tuning")
    return buf.value.decode()


def _batch_shapes(plan: BatchPlan, which: str):
    out = []
    for g in plan._geoms:
        n, na, nz = g
        out += [(n, n) if which == "img" else (na, n)] * nz
    return out
