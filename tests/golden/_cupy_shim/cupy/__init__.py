"""Minimal numpy-backed stand-in for CuPy, used only by tests/golden/make_golden.py to run the
reference's Python SHT path on the CPU of the build container (test infrastructure only).
Arrays are numpy arrays with a ``get()`` method; scalar indexing yields 0-d arrays so the
reference's ``x[r].get()`` idiom works.  ``RawModule`` is absent on purpose: the generator
patches the reference's kernel loaders with the host-compiled kernels in oracle/_ref."""
import numpy as _np
from numpy import *  # noqa: F401,F403


class GArr(_np.ndarray):
    def get(self):
        return _np.asarray(self)

    def __getitem__(self, k):
        r = _np.ndarray.__getitem__(self, k)
        if not isinstance(r, _np.ndarray):
            r = _np.asarray(r).view(GArr)
        return r


def _wrap(f):
    def g(*a, **k):
        r = f(*a, **k)
        return _np.asarray(r).view(GArr) if isinstance(r, (_np.ndarray, _np.generic)) else r
    return g


for _name in ("asarray", "array", "zeros", "empty", "ones", "zeros_like", "empty_like", "ones_like",
              "arange", "cos", "sin", "sqrt", "power", "exp", "concatenate", "abs", "real", "conj", "sum"):
    globals()[_name] = _wrap(getattr(_np, _name))

asrealarray = _wrap(_np.real)       # isht.py:25 calls cp.asrealarray (not a CuPy function)


def asnumpy(a):
    return _np.asarray(a)


class fft:  # noqa: N801
    fft = staticmethod(_wrap(_np.fft.fft))
    ifft = staticmethod(_wrap(_np.fft.ifft))


class random:  # noqa: N801
    RandomState = _np.random.RandomState
    normal = staticmethod(_np.random.normal)
    seed = staticmethod(_np.random.seed)
