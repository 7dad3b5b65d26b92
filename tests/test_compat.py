"""The launcher that runs the reference's solver scripts unchanged on this
package (run.py, compat.py): the projector classes under their bare module
names, an in-process multiprocessing.Pool (CUDA cannot run in the forked
workers the scripts create), the NumPy aliases they read and inert stand-ins
for absent plotting modules.  The scripts are exercised through a stand-in
written the same way (tests/compat_scripts/fake_solver.py), in a fresh
interpreter."""
from __future__ import annotations

import subprocess
import sys

import pytest

from conftest import ROOT

SCRIPT = ROOT / "tests" / "compat_scripts" / "fake_solver.py"


def _run(*args):
    return subprocess.run([sys.executable, "-m", "iterative_tomographic_reconstruction_algorithms_b200.run",
                           str(SCRIPT), *args], cwd=ROOT, capture_output=True, text=True, timeout=600)


def test_launcher_runs_a_reference_style_script():
    p = _run()
    assert p.returncode == 0, p.stderr
    assert ("RESULT [0, 2, 4] iterative_tomographic_reconstruction_algorithms_b200.class_projectors_radon True"
            in p.stdout), p.stdout


def test_in_process_pool_semantics():
    from iterative_tomographic_reconstruction_algorithms_b200.compat import InProcessPool
    pool = InProcessPool(8)
    assert pool.apply_async(pow, (2, 5)).get() == 32
    assert pool.map(abs, [-1, 2, -3]) == [1, 2, 3]
    assert pool.starmap(pow, [(2, 2), (3, 2)]) == [4, 9]
    r = pool.apply_async(int, ("x",))
    with pytest.raises(ValueError):
        r.get()
    with InProcessPool() as p2:
        assert p2.apply(max, (1, 7)) == 7


def test_launcher_usage_errors():
    p = subprocess.run([sys.executable, "-m", "iterative_tomographic_reconstruction_algorithms_b200.run",
                        str(ROOT / "tests" / "compat_scripts" / "missing.py")], cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert p.returncode == 2 and "no such script" in p.stderr


@pytest.mark.gpu
def test_projector_through_the_pool_equals_the_batched_call(cuda):
    p = _run("gpu")
    assert p.returncode == 0, p.stderr
    assert "GPU True" in p.stdout, p.stdout


def test_reference_art_script_reaches_the_drop_in_projector(tmp_path):
    """The reference's own algorithms/art.py (SIRT, ray-driven projector) runs
    unchanged through the launcher on the reference's own Shepp-Logan sinogram
    (data/shepp_logan_pix0256_ang0304_sino.tif): imports, argument parsing,
    TIFF reading and the parameter classes all pass, and its first projector
    call reaches this package's class.  Where no CUDA device is present that
    call must fail loudly in libtomo_b200 (there is no CPU fallback); with a
    device the run completes and writes its reconstruction."""
    from conftest import REFERENCE_TREE
    script = REFERENCE_TREE / "algorithms" / "art.py"
    if not script.exists():
        pytest.skip("reference tree not present")
    import torch
    p = subprocess.run([sys.executable, "-m", "iterative_tomographic_reconstruction_algorithms_b200.run", str(script),
                        "-Di", str(REFERENCE_TREE / "data") + "/", "-i", "shepp_logan_pix0256_ang0304_sino.tif",
                        "-Do", str(tmp_path) + "/", "-o", "reco.tif", "-n", "2", "-a", "sirt", "-pr", "ray-driv"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    if torch.cuda.is_available():
        assert p.returncode == 0, p.stderr[-2000:]
        assert any(tmp_path.iterdir())
    else:
        assert p.returncode != 0
        assert "class_projectors_radon.py" in p.stderr and "TomoError" in p.stderr, p.stderr[-2000:]
        assert "tomo_plan_create" in p.stderr
