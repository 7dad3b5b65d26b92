"""Run the reference's own solver scripts (algorithms/sir.py, art.py, admm.py,
...) on this package's projectors, unchanged.

``install()`` prepares the interpreter the way those scripts need it:

* the projector classes: ``class_projectors_radon``, ``class_projectors_bspline``
  and ``class_projectors_grid`` resolve to this package's drop-in modules, so
  every ``tp.A`` / ``tp.At`` / ``tp.fbp`` runs on the GPU;
* the process model: the scripts fork a ``multiprocessing.Pool`` per iteration
  after the parent has used the projector (art.py:227-235, then :289), and CUDA
  cannot be used in a forked child.  ``multiprocessing.Pool`` becomes an
  in-process pool whose ``apply_async(f, args)`` calls ``f(*args)`` at once (all
  slices can instead be passed as one [nz, n, n] array to the classes);
* NumPy and SciPy names the scripts use that later releases removed:
  ``np.int``, ``np.float``, ``np.bool``, ``np.complex``, ``np.object`` (read at
  import, e.g. sir.py:68) and ``scipy.misc.factorial`` / ``comb``
  (bspline_functions.py:76,155,183);
* plotting and image modules that are absent (matplotlib, pylab, skimage)
  become inert stand-ins: every attribute is a callable that returns another
  stand-in, so ``plt.figure().add_subplot(111).imshow(...)`` does nothing.

``python -m iterative_tomographic_reconstruction_algorithms_b200.run
path/to/sir.py [args]`` installs all of this, changes to the script's directory
(the scripts append ``../common/...`` to sys.path relative to it) and runs it as
``__main__``.
"""
from __future__ import annotations

import importlib
import sys
import types


class _Result:
    def __init__(self, value=None, error=None):
        self._value, self._error = value, error

    def get(self, timeout=None):
        if self._error is not None:
            raise self._error
        return self._value

    def wait(self, timeout=None):
        return None

    def ready(self):
        return True

    def successful(self):
        return self._error is None


class InProcessPool:
    """multiprocessing.Pool stand-in that runs every task in the calling process."""

    def __init__(self, processes=None, *args, **kwargs):
        self._processes = processes

    def apply(self, func, args=(), kwds=None):
        return func(*args, **(kwds or {}))

    def apply_async(self, func, args=(), kwds=None, callback=None, error_callback=None):
        try:
            value = func(*args, **(kwds or {}))
        except Exception as e:  # delivered by get(), as multiprocessing does
            if error_callback is not None:
                error_callback(e)
            return _Result(error=e)
        if callback is not None:
            callback(value)
        return _Result(value)

    def map(self, func, iterable, chunksize=None):
        return [func(x) for x in iterable]

    def map_async(self, func, iterable, chunksize=None, callback=None, error_callback=None):
        return self.apply_async(lambda it: [func(x) for x in it], (list(iterable),), callback=callback,
                                error_callback=error_callback)

    def starmap(self, func, iterable, chunksize=None):
        return [func(*x) for x in iterable]

    def imap(self, func, iterable, chunksize=1):
        return (func(x) for x in iterable)

    imap_unordered = imap

    def close(self):
        pass

    def join(self):
        pass

    def terminate(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class _Inert(types.ModuleType):
    """A module (or object) on which every attribute is an inert callable."""

    def __init__(self, name="inert"):
        super().__init__(name)

    def __getattr__(self, name):
        if name.startswith("__") and name.endswith("__"):
            raise AttributeError(name)
        return _Inert(f"{self.__name__}.{name}")

    def __call__(self, *args, **kwargs):
        return _Inert(f"{self.__name__}()")

    def __iter__(self):
        return iter(())

    def __getitem__(self, key):
        return _Inert(f"{self.__name__}[]")


def _stub_if_absent(name: str) -> bool:
    try:
        importlib.import_module(name)
        return False
    except Exception:
        parts = name.split(".")
        for i in range(1, len(parts) + 1):
            sub = ".".join(parts[:i])
            if sub not in sys.modules or not isinstance(sys.modules[sub], _Inert):
                sys.modules[sub] = _Inert(sub)
        return True


def install(classes: bool = True, pool: bool = True, stubs: bool = True) -> dict:
    """Prepares the interpreter for the reference's scripts; returns what it did."""
    import numpy as np
    done = {"numpy_aliases": [], "stubs": [], "classes": [], "pool": False}
    for name, val in (("int", int), ("float", float), ("bool", bool), ("complex", complex), ("object", object)):
        if not hasattr(np, name) or getattr(np, name) is not val:
            try:
                setattr(np, name, val)
                done["numpy_aliases"].append(name)
            except Exception:
                pass
    try:
        import scipy.misc
        import scipy.special
        for name in ("factorial", "comb"):
            if not hasattr(scipy.misc, name):
                setattr(scipy.misc, name, getattr(scipy.special, name))
    except Exception:
        pass
    if stubs:
        for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.cm", "matplotlib.animation", "pylab",
                     "skimage", "skimage.io", "skimage.transform"):
            if _stub_if_absent(name):
                done["stubs"].append(name)
    if classes:
        from . import class_projectors_bspline, class_projectors_grid, class_projectors_radon
        for mod in (class_projectors_radon, class_projectors_bspline, class_projectors_grid):
            short = mod.__name__.rsplit(".", 1)[1]
            sys.modules[short] = mod
            done["classes"].append(short)
    if pool:
        import multiprocessing
        multiprocessing.Pool = InProcessPool
        try:
            import multiprocessing.pool as mpp
            mpp.Pool = InProcessPool
        except Exception:
            pass
        done["pool"] = True
    return done
