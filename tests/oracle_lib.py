"""Loader of the CPU oracle (oracle/_ref/libt3ns_oracle.so) for the tests.

The oracle is the checker only; nothing in the product imports this file."""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_lib = None


def lib():
    global _lib
    if _lib is None:
        p = os.path.join(ROOT, "oracle", "_ref", "libt3ns_oracle.so")
        if not os.path.exists(p):
            import pytest
            pytest.skip("oracle not built (make -C oracle)")
        _lib = C.CDLL(p)
    return _lib


def matvec(desc, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    lib().t3ns_oracle_matvec(C.byref(desc.desc), x.ctypes.data_as(C.POINTER(C.c_double)),
                             y.ctypes.data_as(C.POINTER(C.c_double)))
    return y


def diagonal(desc):
    d = np.empty(desc.size)
    lib().t3ns_oracle_diagonal(C.byref(desc.desc), d.ctypes.data_as(C.POINTER(C.c_double)))
    return d
