"""CPU tests of the C ABI: the library loads and exports what its header declares.

No projector is run here (there is no GPU on the CPU runner); plan creation
without a device must fail with a status, not crash.
"""
from __future__ import annotations

import ctypes
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "tomo_b200.h"
LIB = ROOT / "iterative_tomographic_reconstruction_algorithms_b200" / "libtomo_b200.so"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tomo_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("tomo_plan_create", "tomo_forward", "tomo_adjoint", "tomo_radon_dd",
              "tomo_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    assert LIB.exists(), "build libtomo_b200.so first (make -C iterative_tomographic_reconstruction_algorithms_b200/csrc)"
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, f"declared in {HEADER.name} but not exported: {missing}"


def test_nn_library_exports_every_declared_symbol():
    header = ROOT / "include" / "tomo_nn.h"
    lib = ROOT / "iterative_tomographic_reconstruction_algorithms_b200" / "libtomo_nn.so"
    assert lib.exists(), "build libtomo_nn.so first (make -C iterative_tomographic_reconstruction_algorithms_b200/csrc)"
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    declared = sorted(set(re.findall(r"\b(tomo_nn_[a-z0-9_]+)\s*\(", text)))
    assert "tomo_nn_conv3x3" in declared and "tomo_nn_wgrad" in declared
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, f"declared in {header.name} but not exported: {missing}"


def test_library_loads_and_reports_version():
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    assert b"sm_100a" in _lib.lib.tomo_version()


def test_invalid_geometry_is_rejected_without_a_device():
    """Validation happens before any CUDA call, so it works on a CPU host."""
    import numpy as np
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    for kwargs, msg in [(dict(n=1), "n (npix)"), (dict(na=0), "na"), (dict(nz=0), "nz"),
                        (dict(kind=99), "kind")]:
        g = _lib.TomoGeom()
        g.kind, g.n, g.na, g.nz = kwargs.get("kind", _lib.KIND_DD), kwargs.get("n", 16), \
            kwargs.get("na", 4), kwargs.get("nz", 1)
        ang = np.zeros(4, np.float32)
        g.angles = ang.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        h = ctypes.c_void_p()
        rc = _lib.lib.tomo_plan_create(ctypes.byref(g), ctypes.byref(h))
        assert rc == _lib.TOMO_EINVAL
        assert msg in _lib.last_error()
    nan = np.array([0.0, np.nan], np.float32)
    g = _lib.TomoGeom()
    g.kind, g.n, g.na, g.nz = _lib.KIND_DD, 16, 2, 1
    g.angles = nan.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    h = ctypes.c_void_p()
    assert _lib.lib.tomo_plan_create(ctypes.byref(g), ctypes.byref(h)) == _lib.TOMO_EINVAL


def test_null_arguments_are_rejected():
    from iterative_tomographic_reconstruction_algorithms_b200 import _lib
    assert _lib.lib.tomo_forward(None, None, None, None) == _lib.TOMO_EINVAL
    assert _lib.lib.tomo_adjoint(None, None, None, None) == _lib.TOMO_EINVAL
