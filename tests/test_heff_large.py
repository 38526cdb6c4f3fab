"""Parity of the CUDA matvec on the large steps: the D=512 step with the
reference's own outputs, and the structure-only benchmark workloads (D=512
steps of the 24-orbital synthetic QC Hamiltonian, SITE_SIZE 2, and the
three-site D=1024 steps), whose operator elements are drawn from a fixed seed.
The latter are checked against the CPU oracle (pinned to the reference on
every golden step) on a sample of new blocks that includes tiled ones, so the
oracle finishes in seconds.  Calls go through the C ABI."""
import glob
import os

import numpy as np
import pytest

import oracle_lib
from conftest import ROOT
from t3ns_b200.native import T3NS_PREC_3XTF32, T3NS_PREC_BF16X3, HeffPlan, StepDesc
from t3ns_b200.stepfile import read_step

pytestmark = pytest.mark.gpu

MATVEC_RTOL = 1e-12
SPLIT_RTOL = 5e-6          # as tests/test_heff_gpu.py (3xTF32, FP32 accumulation)
BF16_RTOL = 2e-4           # as tests/test_bf16x3.py (BF16x3, FP32 accumulation)

D512 = os.path.join(ROOT, "oracle", "_ref", "captures", "qc24_D512", "step_006.t3c")
WORKLOADS = sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "workloads", "*.t3c")))


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def d512(cuda):
    if not os.path.exists(D512):
        pytest.skip("D=512 capture not built (oracle/captures.py d512)")
    s = read_step(D512)
    return s, StepDesc(s)


@pytest.mark.parametrize("config", [0, 1, 2, 3, 4])
def test_d512_matvec_matches_reference(d512, config):
    s, d = d512
    plan = HeffPlan(d)
    plan.set_config(config)
    for v in range(2):
        assert _rel(plan.matvec_host(s[f"x{v}"]), s[f"y{v}"]) <= MATVEC_RTOL
    plan.close()


def test_d512_diagonal_matches_reference(d512):
    s, d = d512
    plan = HeffPlan(d)
    dg = plan.diagonal_host()
    assert np.abs(dg - s["diag"]).max() <= MATVEC_RTOL * np.abs(s["diag"]).max()
    plan.close()


@pytest.mark.parametrize("config", [0, 1, 2, 3, 4])
def test_d512_split_precision_error(d512, config):
    s, d = d512
    plan = HeffPlan(d, T3NS_PREC_3XTF32)
    plan.set_config(config)
    for v in range(2):
        err = _rel(plan.matvec_host(s[f"x{v}"]), s[f"y{v}"])
        assert err <= SPLIT_RTOL, err
    plan.close()


@pytest.mark.parametrize("config", [0, 1, 2, 5, 6, 7])
def test_d512_bf16x3_error(d512, config):
    s, d = d512
    plan = HeffPlan(d, T3NS_PREC_BF16X3)
    plan.set_config(config)
    for v in range(2):
        err = _rel(plan.matvec_host(s[f"x{v}"]), s[f"y{v}"])
        assert err <= BF16_RTOL, err
    plan.close()


@pytest.mark.parametrize("path", WORKLOADS, ids=os.path.basename)
def test_workload_matches_oracle_on_sampled_blocks(path, cuda):
    s = read_step(path)
    d = StepDesc(s)
    x = np.random.default_rng(7).standard_normal(d.size)
    x /= np.linalg.norm(x)
    blocks = oracle_lib.sample_blocks(s)
    yo = oracle_lib.matvec_blocks(d, x, blocks)
    off = s["beginblock"].astype(np.int64)
    sel = np.concatenate([np.arange(off[b], off[b + 1]) for b in blocks])
    plan = HeffPlan(d)
    for config in range(5):
        plan.set_config(config)
        y = plan.matvec_host(x)
        assert np.isfinite(y).all()
        assert _rel(y[sel], yo[sel]) <= MATVEC_RTOL, config
    plan.close()
    split = HeffPlan(d, T3NS_PREC_3XTF32)
    err = _rel(split.matvec_host(x)[sel], yo[sel])
    split.close()
    assert err <= SPLIT_RTOL, err
    bf = HeffPlan(d, T3NS_PREC_BF16X3)
    for config in (0, 5, 7):
        bf.set_config(config)
        err = _rel(bf.matvec_host(x)[sel], yo[sel])
        assert err <= BF16_RTOL, (config, err)
    bf.close()
