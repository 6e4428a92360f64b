"""NumPy-backed stand-in for the subset of CuPy that realworld/polar_gpu.py uses.

Used only by tests/golden/make_golden.py to run the unmodified reference on CPU.
argsort is forced stable: CuPy's GPU sort is stable, NumPy's default is not."""
import numpy as _np
from numpy import *  # noqa: F401,F403


def asarray(a, dtype=None):
    """Host->device copy semantics: CuPy copies a host array, so the caller's array is
    never aliased (polar_gpu.py mutates its device copy of F)."""
    return _np.array(a, dtype=dtype, copy=True)


def asnumpy(a):
    return _np.asarray(a)


ARGSORT_LOG = []


def argsort(a, axis=-1, kind=None):
    """Stable, as CuPy's; records each input so the generator can keep the proxy scores."""
    ARGSORT_LOG.append(_np.array(a, copy=True))
    return _np.argsort(a, axis=axis, kind="stable")


ARGMAX_LOG = []


def argmax(a, axis=None):
    """Records each argmax input so the generator can keep the re-rank scores."""
    ARGMAX_LOG.append(_np.array(a, copy=True))
    return _np.argmax(a, axis=axis)


class _Device:
    def synchronize(self):
        pass


class _Runtime:
    @staticmethod
    def getDeviceProperties(i):
        return {"name": b"numpy-standin"}


class cuda:  # noqa: N801
    Device = _Device
    runtime = _Runtime


__version__ = "standin"
