"""Launcher for the reference's solver scripts on this package's projectors.

    python -m iterative_tomographic_reconstruction_algorithms_b200.run path/to/sir.py [script arguments]

Installs the compatibility layer (compat.install: drop-in projector classes
under the reference's module names, an in-process multiprocessing.Pool, the
removed NumPy/SciPy aliases, inert plotting modules), changes to the script's
directory -- the scripts extend sys.path with ``../common/...`` relative to it --
and runs the script as ``__main__`` with the remaining arguments.
"""
from __future__ import annotations

import os
import runpy
import sys


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] in ("-h", "--help"):
        print(__doc__.strip())
        return 0 if argv else 2
    script = os.path.abspath(argv[0])
    if not os.path.isfile(script):
        print(f"run: no such script: {script}", file=sys.stderr)
        return 2
    # keep this package importable after the change of directory
    pkg_root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if pkg_root not in sys.path:
        sys.path.insert(0, pkg_root)
    from .compat import install
    install()
    sys.argv = [script] + argv[1:]
    here = os.path.dirname(script)
    os.chdir(here)
    sys.path.insert(0, here)
    # the reference's own Python modules next to the scripts (../common/...),
    # which the scripts add to sys.path themselves, some only after importing
    # from them (cg.py:28 before :42-44)
    common = os.path.join(os.path.dirname(here), "common")
    for sub in ("myimage", "operators/bspline_module", "operators/regularization_module", "operators/filters_module"):
        d = os.path.join(common, sub)
        if os.path.isdir(d) and d not in sys.path:
            sys.path.append(d)
    runpy.run_path(script, run_name="__main__")
    return 0


if __name__ == "__main__":
    sys.exit(main())
