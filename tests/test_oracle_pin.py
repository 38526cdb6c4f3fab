"""The CPU oracle reproduces the reference's own matvec and diagonal on the
golden step files (captured from the reference build), which pins it."""
import numpy as np
import pytest

import oracle_lib
from conftest import golden_steps
from t3ns_b200.native import StepDesc
from t3ns_b200.stepfile import read_step


@pytest.mark.parametrize("path", golden_steps(), ids=lambda p: p.split("/")[-1])
def test_oracle_matches_reference(path):
    s = read_step(path)
    d = StepDesc(s)
    for v in range(2):
        x, yref = s[f"x{v}"], s[f"y{v}"]
        y = oracle_lib.matvec(d, x)
        assert np.linalg.norm(y - yref) <= 1e-14 * np.linalg.norm(yref)
    dg = oracle_lib.diagonal(d)
    assert np.abs(dg - s["diag"]).max() <= 1e-14 * np.abs(s["diag"]).max()


def test_oracle_detects_planted_error():
    """A wrong prefactor in the oracle's input must show up in the check."""
    path = [p for p in golden_steps() if "qc12_t3ns" in p][0]
    s = read_step(path)
    s["sr.combo_pref"] = s["sr.combo_pref"].copy()
    s["sr.combo_pref"][::7] *= 1.0 + 1e-9
    y = oracle_lib.matvec(StepDesc(s), s["x0"])
    assert np.linalg.norm(y - s["y0"]) > 1e-14 * np.linalg.norm(s["y0"])


@pytest.mark.parametrize("path", golden_steps(), ids=lambda p: p.split("/")[-1])
def test_block_sampled_oracle_equals_full_oracle(path):
    """The block-restricted oracle (used on steps too large for the full one)
    gives exactly the full oracle's values on the blocks it computes."""
    s = read_step(path)
    d = StepDesc(s)
    full = oracle_lib.matvec(d, s["x0"])
    blocks = oracle_lib.sample_blocks(s, k=6)
    part = oracle_lib.matvec_blocks(d, s["x0"], blocks)
    off = s["beginblock"].astype(np.int64)
    for b in blocks:
        assert np.array_equal(part[off[b]:off[b + 1]], full[off[b]:off[b + 1]])


def _ref_lib():
    import ctypes as C
    import os

    from conftest import ROOT
    p = os.path.join(ROOT, "oracle", "_ref", "libt3ns_ref.so")
    if not os.path.exists(p):
        pytest.skip("reference library not built (make -C oracle)")
    return C.CDLL(p, mode=C.RTLD_GLOBAL)


@pytest.mark.parametrize("theta", [0.7, -1.25])
def test_preconditioner_oracle_matches_reference(theta):
    """oracle/precond_oracle.py against the reference's own
    davidson_diagonal_preconditioner (src/davidson.c:223-257) from the
    reference build, including diagonal entries exactly at theta (the
    1e-12 cutoff branch)."""
    import ctypes as C
    import os
    import sys

    from conftest import ROOT
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import precond_oracle
    f = _ref_lib().davidson_diagonal_preconditioner
    f.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
    f.restype = None
    rng = np.random.default_rng(5)
    n = 50_001
    r = rng.standard_normal(n)
    r /= np.linalg.norm(r)
    dg = rng.uniform(-3.0, 5.0, n)
    dg[::977] = theta
    dg[1::1013] = theta + 5e-13          # inside the cutoff, positive side
    dg[2::1019] = theta - 5e-13          # inside the cutoff, negative side
    t = rng.standard_normal(n) * 1e-3
    out = t.copy()
    f(r.ctypes.data, theta, n, dg.ctypes.data, out.ctypes.data)
    want = precond_oracle.precondition(r, theta, dg, t)
    assert np.linalg.norm(out - want) <= 1e-14 * np.linalg.norm(want)
