"""Branching renormalised-operator update (reference
update_rOperators_branching, src/rOperators_bUpdate.c:229-248) against the
reference's own output.

Each capture holds both input operator sets, the branching tensor, the
drop-in's compiled schedule for them and the reference's result (after its
sum over unique operators and zero-block removal).  CPU: a numpy replay of
the schedule, summed as sum_unique_rOperators does, reproduces the reference
(so the schedule compiler is right).  GPU: the engine's kernel, through the C
ABI, reproduces it to 1e-12 of the largest element, with the same surviving
blocks."""
import numpy as np
import pytest

import rops_check as rc
from conftest import pupdate_captures
from t3ns_b200.stepfile import read_step

CAPS = pupdate_captures("bupdate")


def _load(p):
    return read_step(p), read_step(p.replace(".t3c", ".sched"))


@pytest.mark.skipif(not CAPS, reason="no update captures")
def test_all_update_cases_captured():
    """Captures cover every update case the networks produce: the new
    operator on the first, second or third bond of the branching site."""
    cases = {int(_load(p)[1]["bu.ax"][2]) for p in CAPS}
    assert len(cases) >= 2, cases


@pytest.mark.parametrize("path", CAPS, ids=lambda p: "/".join(p.split("/")[-2:]))
def test_bupdate_schedule_emulation(path):
    rec, sch = _load(path)
    assert len(sch["bu.pref"]) > 0
    pre = rc.sum_unique(rec, sch, rc.emulate_bupdate(rec, sch))
    assert rc.kick_compare(rec, 2, pre) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("path", CAPS, ids=lambda p: "/".join(p.split("/")[-2:]))
def test_bupdate_gpu_matches_reference(path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rec, sch = _load(path)
    got = rc.run_bupdate_gpu(rec, sch)
    ref = rc.emulate_bupdate(rec, sch)
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.abs(got - ref).max() / scale <= 1e-12
    assert rc.kick_compare(rec, 2, rc.sum_unique(rec, sch, got)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("path", CAPS, ids=lambda p: "/".join(p.split("/")[-2:]))
def test_bupdate_with_device_sum_matches_reference(path):
    """The branching update with the sum over unique operators and the
    zero-block removal on the device (t3ns_bupdate_sum_host, as the drop-in
    runs it) gives the reference's new set: the same surviving blocks, the
    elements to 1e-12 of the largest."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from t3ns_b200 import updates
    rec, sch = _load(path)
    assert rc.compare_summed(rec, 2, updates.bupdate_sum_host(rec, sch)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("path", CAPS[::3], ids=lambda p: "/".join(p.split("/")[-2:]))
def test_sum_unique_alone_matches_reference(path):
    """t3ns_sum_unique_host (the drop-in's sum_unique_rOperators) on the
    unique operators of the numpy replay gives the reference's new set."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from t3ns_b200 import updates
    rec, sch = _load(path)
    d, keep = updates.bupdate_sum_desc(rec, sch)
    got = updates.sum_unique_host(d, keep, rc.emulate_bupdate(rec, sch))
    assert rc.compare_summed(rec, 2, got) <= 1e-12


@pytest.mark.parametrize("path", CAPS[:4], ids=lambda p: "/".join(p.split("/")[-2:]))
def test_sum_descriptor_is_consistent(path):
    """Host-side descriptor of the device sum: every instruction appears once
    under the new operator it writes, sizes and layouts agree with the
    unique operators' (no GPU)."""
    from t3ns_b200 import updates
    rec, sch = _load(path)
    d, keep = updates.bupdate_sum_desc(rec, sch)
    instr = sch["bu.instr"].reshape(-1, 3)
    assert keep["instr_ptr"][-1] == len(instr)
    assert np.array_equal(np.diff(keep["instr_ptr"]), np.bincount(instr[:, 2], minlength=d.nnew))
    sizes = np.diff(keep["new_base"])
    lasts = keep["begin"][keep["begin_ptr"][1:] - 1]
    assert np.array_equal(sizes, lasts)
    assert np.all(keep["instr_src"] + np.repeat(sizes, np.diff(keep["instr_ptr"])) <= d.unique_elems)
