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


def matvec_blocks(desc, x, blocks):
    """The oracle matvec on the new blocks ``blocks`` only: returns y with
    those blocks filled and NaN elsewhere."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.full_like(x, np.nan)
    b = np.ascontiguousarray(blocks, dtype=np.int32)
    rc = lib().t3ns_oracle_matvec_blocks(C.byref(desc.desc), x.ctypes.data_as(C.POINTER(C.c_double)),
                                         y.ctypes.data_as(C.POINTER(C.c_double)),
                                         b.ctypes.data_as(C.POINTER(C.c_int)), C.c_int(b.size))
    assert rc == 0
    return y


def sample_blocks(s, k=8, seed=0):
    """A reproducible sample of new blocks of a step for oracle checks in
    bounded CPU time: the two smallest, k-4 from the middle of the size
    distribution and two from its top 5% (large blocks are the ones the
    engine tiles)."""
    off = s["beginblock"].astype(np.int64)
    sz = np.diff(off)
    order = np.argsort(sz, kind="stable")
    n = len(order)
    rng = np.random.default_rng(seed)
    mid = order[int(0.3 * n):max(int(0.6 * n), int(0.3 * n) + 1)]
    tail = order[int(0.95 * n):]
    pick = list(order[:2]) + list(rng.choice(mid, min(k - 4, len(mid)), replace=False)) + \
        list(rng.choice(tail, min(2, len(tail)), replace=False))
    return np.unique(np.array(pick, dtype=np.int32))
