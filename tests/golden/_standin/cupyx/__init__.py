"""NumPy-backed stand-in for cupyx.scatter_add."""
import numpy as _np


def scatter_add(a, idx, vals):
    _np.add.at(a, idx, vals)
