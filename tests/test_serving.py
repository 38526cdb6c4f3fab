"""The engine's request loop (t3ns_server_*): admission against a device
memory budget, concurrent solves, and the same result for a request alone
and in a mix of concurrent requests."""
import os

import numpy as np
import pytest

from conftest import ROOT
from t3ns_b200 import native
from t3ns_b200.serving import Server, Workload, estimate_bytes, request_steps, run_stream

STEPS = request_steps([os.path.join(ROOT, "oracle", "_ref", "captures", "*", "step_*.t3c"),
                       os.path.join(ROOT, "tests", "golden", "*.t3c")])


def test_estimate_covers_operators_and_basis():
    """The admission estimate (host only) holds at least the operators, the
    basis of the subspace and the vectors, and grows with the subspace and
    with the FP32 operator copy of split precision."""
    if not STEPS:
        pytest.skip("no captured steps")
    w = Workload(STEPS[0])
    n = w.diag.size
    ops = sum(int(w.step[f"ops{i}.tel"].size) for i in range(2 if int(w.step["isdmrg"][0]) else 3))
    e64 = estimate_bytes(w.desc, native.T3NS_PREC_FP64, 30)
    assert e64 >= 8 * ops + 8 * n * 60
    assert estimate_bytes(w.desc, native.T3NS_PREC_FP64, 10) < e64
    assert estimate_bytes(w.desc, native.T3NS_PREC_3XTF32, 30) >= e64 + 4 * ops


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [native.T3NS_PREC_FP64, native.T3NS_PREC_3XTF32])
def test_same_result_alone_and_in_the_mix(precision, torch_cuda):
    """Each request gives the same energy and vector alone (one in flight)
    as among 8 concurrent ones (4 in flight), within 1e-10 (the matvec's
    split-unit atomics may round differently), and the reference energy
    within 1e-8 Ha."""
    wls = [Workload(p) for p in STEPS[:: max(1, len(STEPS) // 8)]][:8]
    alone = []
    srv = Server(8 << 30, 1)
    for w in wls:
        g = w.guess_for(np.random.default_rng(0))
        r = srv.wait(srv.submit(w.desc, g, w.diag, precision, w.tol, 100, w.max_vecs, w.keep))
        alone.append((r["energy"], g))
    srv.close()
    srv = Server(8 << 30, 4)
    guesses = [w.guess_for(np.random.default_rng(0)) for w in wls]
    ids = [srv.submit(w.desc, g, w.diag, precision, w.tol, 100, w.max_vecs, w.keep)
           for w, g in zip(wls, guesses)]
    mixed = [srv.wait(i)["energy"] for i in ids]
    srv.close()
    for w, (ea, ga), em, gm in zip(wls, alone, mixed, guesses):
        assert abs(ea - em) <= 1e-10
        assert abs(abs(float(ga @ gm)) - 1.0) <= 1e-10
        assert abs(em - w.ref_energy) <= 1e-8


@pytest.mark.gpu
def test_admission_rejects_oversize_and_respects_budget(torch_cuda):
    wls = [Workload(p) for p in STEPS[:6]]
    est = [estimate_bytes(w.desc, native.T3NS_PREC_FP64, w.max_vecs) for w in wls]
    small = Server(min(est) - 1, 2)
    w0 = wls[int(np.argmin(est))]
    with pytest.raises(RuntimeError, match="budget"):
        small.submit(w0.desc, w0.guess_for(np.random.default_rng(0)), w0.diag,
                     native.T3NS_PREC_FP64)
    small.close()
    budget = 2 * max(est)               # at most two of these fit at once
    srv = Server(budget, 4)
    ids = []
    for w in wls * 2:
        ids.append(srv.submit(w.desc, w.guess_for(np.random.default_rng(1)), w.diag,
                              native.T3NS_PREC_FP64, w.tol, 100, w.max_vecs, w.keep))
    res = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    assert all(r["status"] >= 0 for r in res)
    assert 0 < st["peak"] <= budget
    assert st["in_use"] == 0 and st["queued"] == 0


@pytest.mark.gpu
def test_poisson_stream_reports_latency(torch_cuda):
    wls = [Workload(p) for p in STEPS]
    recs, s = run_stream(wls, n_requests=24, rate=200.0, budget_bytes=4 << 30, max_inflight=4,
                         precision="3xtf32", seed=3)
    assert s["failed"] == 0 and len(recs) == 24
    assert 0 < s["latency_p50_s"] <= s["latency_p99_s"]
    assert s["max_abs_dE_vs_reference"] <= 1e-8
    assert s["peak_admitted_bytes"] <= 4 << 30
