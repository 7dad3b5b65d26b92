"""Shared test configuration.

Markers:
  gpu  -- needs a CUDA device (the B200); everything else runs on CPU.

Fixtures under tests/golden/ hold reference outputs on seeded inputs
(tests/golden/make_golden.py), so the parity tests need neither the reference
tree nor the compiled reference on the machine that runs them.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"
from oracle.oracle import REFERENCE_TREE  # noqa: E402,F401


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA device")


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def radon_golden():
    return np.load(GOLDEN / "radon_golden.npz")


@pytest.fixture(scope="session")
def dd_entries_golden():
    return np.load(GOLDEN / "dd_entries_golden.npz")


@pytest.fixture(scope="session")
def bspline_golden():
    return np.load(GOLDEN / "bspline_golden.npz")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reflib():
    from oracle.oracle import RefLib, ref_available
    if not ref_available():
        pytest.skip("compiled reference (oracle/_ref) not present")
    return RefLib()


@pytest.fixture(scope="session")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
