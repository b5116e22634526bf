"""Gauss-point shape-function data (drop-in for core/shape_functions.py).
Convention: wq (q, 1), N (q, I), Nderiv (q, dim, I); evaluated on the device."""
from .. import _lib
from ..context import empty, f64, ptr, stream

_DIMS = {_lib.SHAPE_QUAD4: (4, 4, 2), _lib.SHAPE_QUAD9: (9, 9, 2), _lib.SHAPE_HEX8: (8, 8, 3),
         _lib.SHAPE_LIN2: (2, 2, 1), _lib.SHAPE_LIN3: (3, 3, 1)}


def _eval(family, coords):
    nq, nen, dim = _DIMS[family]
    c = f64(coords).reshape(-1)
    wq, N, dN = empty(nq), empty(nq * nen), empty(nq * dim * nen)
    _lib.call("fem_shape_functions", family, ptr(c), ptr(wq), ptr(N), ptr(dN), stream())
    return wq.view(nq, 1), N.view(nq, nen), dN.view(nq, dim, nen)


def lin2_shape_functions(coords):
    """core/shape_functions.py:11."""
    return _eval(_lib.SHAPE_LIN2, coords)


def quad4_shape_functions(coords):
    """core/shape_functions.py:27."""
    return _eval(_lib.SHAPE_QUAD4, coords)


def hex8_shape_functions(coords):
    """core/shape_functions.py:47."""
    return _eval(_lib.SHAPE_HEX8, coords)


def lin3_shape_functions(coords):
    """core/shape_functions.py:89."""
    return _eval(_lib.SHAPE_LIN3, coords)


def quad9_shape_functions(coords):
    """core/shape_functions.py:108."""
    return _eval(_lib.SHAPE_QUAD9, coords)
