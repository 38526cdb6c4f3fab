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
