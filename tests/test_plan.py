"""Host-side checks of the matvec work plan (no GPU): output tiling, pair
splitting, the contraction sequence of each pair and the operator row
offsets of tiles, emulated with numpy and compared with the reference's own
matvec output."""
import numpy as np
import pytest

import plan_emulator as pe
from conftest import captured_steps, golden_steps
from t3ns_b200.native import StepDesc
from t3ns_b200.stepfile import read_step


def _check(s, plan, blocks):
    scale = max(np.abs(s["y0"]).max(), 1e-300)
    got = pe.emulate_blocks(s, plan, s["x0"], blocks)
    for nb, blk in got.items():
        assert np.abs(blk - pe.reference_block(s, s["y0"], nb)).max() <= 1e-13 * scale, nb
    # executed FLOPs: below the reference's only through shared first stages
    fl = plan["plan.flops"]
    assert fl[1] >= pe.shared_flops_lower_bound(plan) * (1 - 1e-12)


# the engine's kernel configurations (3, 4: contraction-ordered; 5, 7: BF16x3
# tilings with twice the elements per buffer)
CONFIGS = (0, 1, 2, 3, 4, 5, 7)


@pytest.mark.parametrize("config", CONFIGS)
@pytest.mark.parametrize("path", golden_steps(), ids=lambda p: p.split("/")[-1])
def test_plan_emulation_golden(path, config):
    s = read_step(path)
    plan = pe.dump_plan(StepDesc(s), config)
    _check(s, plan, range(int(s["nrblocks"][0])))


@pytest.mark.parametrize("config", CONFIGS)
def test_plan_emulation_tiled_and_split_blocks(config):
    """A D=512 step: large output blocks are tiled (in the small-tile
    configuration at least), heavy tiles split."""
    cands = [p for p in captured_steps(max_bytes=1 << 30) if "qc24_D512/step_006" in p]
    if not cands:
        pytest.skip("D=512 step 6 not captured")
    s = read_step(cands[0])
    plan = pe.dump_plan(StepDesc(s), config)
    u = pe.units_of(plan)
    e = plan["plan.edims"].reshape(-1, 3)
    tiled = (u[:, 2] < e[u[:, 0], 1]) | (u[:, 4] < e[u[:, 0], 2]) | (u[:, 6] < e[u[:, 0], 0])
    split = u[:, 9] != 0
    if config in (0, 5, 7) and not tiled.any():
        tiled = split
    assert tiled.any()
    blocks = sorted({int(u[np.nonzero(tiled)[0][0], 0])} |
                    ({int(u[np.nonzero(split)[0][0], 0])} if split.any() else set()))
    _check(s, plan, blocks)
