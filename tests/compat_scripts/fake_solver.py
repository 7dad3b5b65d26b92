# A solver script written the way the reference's are (algorithms/sir.py,
# art.py): module-level imports of plotting modules and of the projector class
# by its bare name, np.int, and a multiprocessing.Pool per step whose workers
# call the projector.  tests/test_compat.py runs it through the launcher.
from __future__ import division, print_function

import multiprocessing as mproc
import sys

import matplotlib.pyplot as plt
import numpy as np
import pylab as py

sys.path.append('../common/myimage/')
import class_projectors_radon as cpj3  # noqa: E402

myint = np.int


def double(x):
    return 2 * x


def main():
    pool = mproc.Pool(4)
    res = [pool.apply_async(double, args=(i,)) for i in range(3)]
    out = [r.get() for r in res]
    pool.close()
    pool.join()
    plt.figure().add_subplot(111).imshow(np.zeros((2, 2)))
    py.ion()
    print("RESULT", out, cpj3.__name__, myint is int)
    if len(sys.argv) > 1 and sys.argv[1] == "gpu":
        n, na, nz = 64, 45, 3
        tp = cpj3.projectors(n, np.linspace(0, 180, na, endpoint=False), oper="dd")
        rng = np.random.default_rng(0)
        x = rng.standard_normal((nz, n, n)).astype(np.float32)
        pool = mproc.Pool()
        parts = [pool.apply_async(tp.A, args=(x[i],)) for i in range(nz)]
        per_slice = np.array([r.get() for r in parts])
        pool.close()
        pool.join()
        print("GPU", bool(np.array_equal(per_slice, tp.A(x))))


if __name__ == "__main__":
    main()
