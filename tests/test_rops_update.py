"""Physical renormalised-operator update (reference update_rOperators_physical,
src/rOperators_pUpdate.c:364-387) against the reference's own output.

Each capture holds the update's inputs, the drop-in's compiled schedule for
them and the reference's result.  CPU: a numpy replay of the schedule
reproduces the reference (so the schedule compiler is right).  GPU: the
engine's kernel, through the C ABI, reproduces it to 1e-12 of the largest
element, with the same surviving blocks after zero-block removal."""
import numpy as np
import pytest

import rops_check as rc
from conftest import pupdate_captures
from t3ns_b200.stepfile import read_step

CAPS = pupdate_captures()
SAMPLE = CAPS[::4] + [p for p in CAPS if p.endswith("_002.t3c")]


def _load(p):
    return read_step(p), read_step(p.replace(".t3c", ".sched"))


@pytest.mark.skipif(not CAPS, reason="no update captures")
def test_both_orientations_captured():
    kinds = {int(_load(p)[1]["pu.is_left"][0]) for p in CAPS}
    assert kinds == {0, 1}


@pytest.mark.parametrize("path", sorted(set(SAMPLE)), ids=lambda p: "/".join(p.split("/")[-2:]))
def test_pupdate_schedule_emulation(path):
    rec, sch = _load(path)
    assert rc.kick_and_compare(rec, sch, rc.emulate_pupdate(rec, sch)) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("path", CAPS, ids=lambda p: "/".join(p.split("/")[-2:]))
def test_pupdate_gpu_matches_reference(path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rec, sch = _load(path)
    assert rc.kick_and_compare(rec, sch, rc.run_pupdate_gpu(rec, sch)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.skipif(not CAPS, reason="no update captures")
def test_pupdate_workspace_reuse_is_exact():
    """The host calls stage through a per-thread workspace that keeps the
    largest call's buffers: every call gives the same bits whatever ran
    before it on the thread (calls in both size orders), so no output of an
    earlier call leaks into a later one."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    loaded = [_load(p) for p in CAPS]
    order = sorted(range(len(loaded)), key=lambda i: loaded[i][0]["T.tel"].size)
    first = {i: rc.run_pupdate_gpu(*loaded[i]) for i in order[::-1]}     # largest first
    for i in order:                                                      # then smallest first
        assert np.array_equal(rc.run_pupdate_gpu(*loaded[i]), first[i]), CAPS[i]
