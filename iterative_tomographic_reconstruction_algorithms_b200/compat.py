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
  ``np.int``, ``np.float``, ``np.complex``, ``np.object`` (and ``np.bool`` on a
  NumPy that lacks it; read at import, e.g. sir.py:68) and
  ``scipy.misc.factorial`` / ``comb`` (bspline_functions.py:76,155,183);
* plotting and image modules that are absent (matplotlib, pylab, skimage)
  become inert stand-ins: every attribute is a callable that returns another
  stand-in, so ``plt.figure().add_subplot(111).imshow(...)`` does nothing;
  except ``skimage.io.imread`` / ``imsave``, which read and write the scripts'
  uncompressed float TIFFs;
* the reference's compiled extensions outside the projector path that are not
  built (its penalty module and split-Bregman NL-TV denoiser) import as
  stand-ins whose functions raise when called.

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


class _MissingExtension(types.ModuleType):
    """Stand-in for a compiled extension of the reference that is outside the
    projector path (its regularisation penalties and its split-Bregman NL-TV
    denoiser): importing it succeeds, so scripts that do not use it run; using
    any of its functions raises."""

    def __getattr__(self, name):
        if name.startswith("__") and name.endswith("__"):
            raise AttributeError(name)
        mod = self.__name__

        def missing(*args, **kwargs):
            raise NotImplementedError(
                f"{mod}.{name}: a compiled extension of the reference outside the projector path, "
                f"which this package does not provide (build the reference's own module to use it)")
        return missing


class _ExtensionFinder:
    """Meta-path finder, consulted after every other finder, that supplies
    _MissingExtension modules for the reference's compiled extensions that are
    not built: ``penalty`` (sir.py:46) and
    ``pymodule_split_bregman_nltv.split_bregman_nltv`` (my_image_denoise.py:44)."""

    NAMES = ("penalty", "pymodule_split_bregman_nltv.split_bregman_nltv")

    def find_spec(self, fullname, path=None, target=None):
        if fullname not in self.NAMES:
            return None
        import importlib.machinery
        return importlib.machinery.ModuleSpec(fullname, self)

    def create_module(self, spec):
        return _MissingExtension(spec.name)

    def exec_module(self, module):
        pass


def _tiff_imread(path):
    """Reads a single-image, uncompressed TIFF of 32- or 64-bit floats (the
    format the reference's scripts read and write with skimage.io), as a 2-D
    numpy array."""
    import struct

    import numpy as np
    raw = open(path, "rb").read()
    end = "<" if raw[:2] == b"II" else ">"
    off = struct.unpack_from(end + "I", raw, 4)[0]
    count = struct.unpack_from(end + "H", raw, off)[0]
    tags = {}
    sizes = {3: ("H", 2), 4: ("I", 4)}
    for i in range(count):
        tag, typ, cnt, val = struct.unpack_from(end + "HHII", raw, off + 2 + 12 * i)
        if typ in sizes:
            fmt, size = sizes[typ]
            at = off + 2 + 12 * i + 8 if cnt * size <= 4 else val
            tags[tag] = struct.unpack_from(end + fmt * cnt, raw, at)
    width, height = tags[256][0], tags[257][0]
    bits, fmt = tags.get(258, (32,))[0], tags.get(339, (3,))[0]
    if tags.get(259, (1,))[0] != 1:
        raise ValueError(f"{path}: compressed TIFF is not supported")
    kind = {1: "u", 2: "i", 3: "f"}[fmt]
    dtype = np.dtype(f"{end}{kind}{bits // 8}")
    data = b"".join(raw[o:o + c] for o, c in zip(tags[273], tags[279]))
    return np.frombuffer(data, dtype=dtype, count=width * height).reshape(height, width).astype(dtype.newbyteorder("="))


def _tiff_imsave(path, arr, **kwargs):
    """Writes a 2-D float array as an uncompressed little-endian TIFF (float32
    or float64)."""
    import struct

    import numpy as np
    a = np.ascontiguousarray(arr)
    if a.dtype not in (np.float32, np.float64):
        a = a.astype(np.float32)
    h, w = a.shape
    body = a.astype(a.dtype.newbyteorder("<")).tobytes()
    entries = [(256, 4, 1, w), (257, 4, 1, h), (258, 3, 1, a.itemsize * 8), (259, 3, 1, 1), (262, 3, 1, 1),
               (273, 4, 1, 0), (277, 3, 1, 1), (278, 4, 1, h), (279, 4, 1, len(body)), (339, 3, 1, 3)]
    ifd_off = 8
    data_off = ifd_off + 2 + 12 * len(entries) + 4
    out = bytearray(b"II*\x00" + struct.pack("<I", ifd_off) + struct.pack("<H", len(entries)))
    for tag, typ, cnt, val in entries:
        val = data_off if tag == 273 else val
        out += struct.pack("<HHI", tag, typ, cnt) + (struct.pack("<HH", val, 0) if typ == 3 else struct.pack("<I", val))
    out += struct.pack("<I", 0) + body
    open(path, "wb").write(bytes(out))


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
    # only names NumPy no longer has: NumPy 2 defines np.bool again (its own
    # bool scalar type, which numpy.ma relies on), so it is left alone
    for name, val in (("int", int), ("float", float), ("bool", bool), ("complex", complex), ("object", object)):
        if name not in vars(np):
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
        if isinstance(sys.modules.get("skimage.io"), _Inert):
            # the scripts read and write their float TIFFs with skimage.io
            sys.modules["skimage.io"].imread = _tiff_imread
            sys.modules["skimage.io"].imsave = _tiff_imsave
            sys.modules["skimage"].io = sys.modules["skimage.io"]
        if not any(isinstance(f, _ExtensionFinder) for f in sys.meta_path):
            sys.meta_path.append(_ExtensionFinder())
            done["stubs"] += list(_ExtensionFinder.NAMES)
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
