"""Host-side checks of the matvec work plan (no GPU): output tiling, the
contraction sequence of each pair and the operator row offsets of tiles,
emulated with numpy and compared with the reference's own matvec output."""
import numpy as np
import pytest

import plan_emulator as pe
from conftest import captured_steps, golden_steps
from t3ns_b200.native import StepDesc
from t3ns_b200.stepfile import read_step


def _check(path, nunits):
    s = read_step(path)
    plan = pe.dump_plan(StepDesc(s))
    units = plan["plan.units"].reshape(-1, 5)
    rng = np.random.default_rng(0)
    ids = sorted(set(range(min(nunits, len(units)))) |
                 set(rng.choice(len(units), min(nunits, len(units)), replace=False).tolist()))
    scale = max(np.abs(s["y0"]).max(), 1e-300)
    for u, t in zip(ids, pe.emulate_units(s, plan, s["x0"], ids)):
        r = pe.reference_tile(s, plan, s["y0"], u)
        assert np.abs(t - r).max() <= 1e-13 * scale, u
    # the executed FLOPs never undercut the reference's contraction order
    fl = plan["plan.flops"]
    assert fl[1] >= fl[0] * (1 - 1e-12)
    return plan


@pytest.mark.parametrize("path", golden_steps(), ids=lambda p: p.split("/")[-1])
def test_plan_emulation_golden(path):
    _check(path, 8)


def test_plan_emulation_tiled_blocks():
    """A D=512 step whose large output blocks are split into tiles."""
    cands = [p for p in captured_steps(max_bytes=1 << 30) if "qc24_D512" in p]
    if not cands:
        pytest.skip("no D=512 step file captured")
    plan = _check(sorted(cands)[0], 3)
    units = plan["plan.units"].reshape(-1, 5)
    edims = plan["plan.edims"].reshape(-1, 3)
    tiled = (units[:, 2] < edims[units[:, 0], 1]) | (units[:, 4] < edims[units[:, 0], 2])
    assert tiled.any()
    # tiled units come first in the schedule (heaviest first): emulate some
    s = read_step(sorted(cands)[0])
    ids = np.nonzero(tiled)[0][:4].tolist()
    scale = max(np.abs(s["y0"]).max(), 1e-300)
    for u, t in zip(ids, pe.emulate_units(s, plan, s["x0"], ids)):
        assert np.abs(t - pe.reference_tile(s, plan, s["y0"], u)).max() <= 1e-13 * scale
