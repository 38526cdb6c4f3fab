"""The BF16x3 matvec (T3NS_PREC_BF16X3): {hi, lo} BF16 operand pairs, three
products on the BF16 tensor pipe, FP32 accumulation.

Its error against the reference's FP64 output comes from the 16 significant
bits of an operand pair (2^-17 relative), the dropped lo*lo products
(~2^-16 each) and FP32 sums over three contraction stages; the stated
tolerance is BF16_RTOL (norm-wise relative).  With FP64 defect correction the
Davidson energy still meets the reference's to 1e-8 Ha.  Calls go through the
C ABI (libt3ns_b200.so)."""
import numpy as np
import pytest

from conftest import captured_steps, golden_steps
from t3ns_b200.native import T3NS_PREC_BF16X3, T3NS_PREC_FP64, HeffPlan, StepDesc
from t3ns_b200.stepfile import read_step

pytestmark = pytest.mark.gpu

BF16_RTOL = 2e-4
ENERGY_TOL = 1e-8

STEPS = golden_steps() + captured_steps(max_bytes=64 << 20)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("config", [0, 1, 2, 5, 6, 7])
@pytest.mark.parametrize("path", STEPS[::2], ids=lambda p: "/".join(p.split("/")[-2:]))
def test_bf16x3_matvec_error(path, config, torch_cuda):
    s = read_step(path)
    plan = HeffPlan(StepDesc(s), T3NS_PREC_BF16X3)
    plan.set_config(config)
    for v in range(2):
        err = _rel(plan.matvec_host(s[f"x{v}"]), s[f"y{v}"])
        assert err <= BF16_RTOL, err
    # conversion of x to pairs + the matvec
    assert plan.last_launches() == 2
    plan.close()


def test_configs_reject_other_precisions(torch_cuda):
    """3 and 4 do not run BF16x3, 5-7 run only BF16x3; switching the
    precision falls back to configuration 0 from one that does not run it."""
    s = read_step(golden_steps()[0])
    plan = HeffPlan(StepDesc(s), T3NS_PREC_BF16X3)
    for c in (3, 4):
        with pytest.raises(RuntimeError):
            plan.set_config(c)
    plan.set_config(5)
    assert _rel(plan.matvec_host(s["x0"]), s["y0"]) <= BF16_RTOL
    plan.set_precision(T3NS_PREC_FP64)      # 5 is BF16x3 only
    assert plan.config() == 0
    for c in (5, 6, 7):
        with pytest.raises(RuntimeError):
            plan.set_config(c)
    plan.set_config(3)
    assert _rel(plan.matvec_host(s["x0"]), s["y0"]) <= 1e-12
    plan.set_precision(T3NS_PREC_BF16X3)   # 3 does not run BF16x3
    assert plan.config() == 0
    assert _rel(plan.matvec_host(s["x0"]), s["y0"]) <= BF16_RTOL
    plan.close()


@pytest.mark.parametrize("path", [p for p in STEPS if "eig.energy" in read_step(p)][::3],
                         ids=lambda p: "/".join(p.split("/")[-2:]))
def test_bf16x3_davidson_defect_corrected(path, torch_cuda):
    """BF16x3 iterations followed by FP64 defect correction reach the
    reference's Davidson energy to 1e-8 Ha with an FP64 residual below tol."""
    s = read_step(path)
    tol = float(s["eig.tol"][0])
    plan = HeffPlan(StepDesc(s), T3NS_PREC_BF16X3)
    res = s["eig.guess"].copy()
    e, ret, info = plan.davidson_host(res, s["diag"], tol=tol, max_its=int(s["eig.max_its"][0]),
                                      max_vecs=int(s["eig.max_vecs"][0]),
                                      keep=int(s["eig.keep"][0]))
    plan.close()
    if int(s["eig.ret"][0]) == 0:
        assert ret == 0
    assert abs(e - float(s["eig.energy"][0])) <= ENERGY_TOL
    assert info["fp64_iterations"] >= 1
    fp64 = HeffPlan(StepDesc(s))
    r = fp64.matvec_host(res) - e * res
    assert np.linalg.norm(r) <= tol * 1.01
    fp64.close()


@pytest.mark.parametrize("config", [5, 6, 7])
def test_bf16x3_only_config_runs_fp64_defect_correction(config, torch_cuda):
    """With a BF16x3-only configuration active, the FP64 iterations of the
    defect correction (and FP64 matvecs after switching back) run in the
    configuration of the same launch shape."""
    cands = [p for p in STEPS if "eig.energy" in read_step(p)]
    s = read_step(cands[len(cands) // 2])
    plan = HeffPlan(StepDesc(s), T3NS_PREC_BF16X3)
    plan.set_config(config)
    res = s["eig.guess"].copy()
    tol = float(s["eig.tol"][0])
    e, ret, info = plan.davidson_host(res, s["diag"], tol=tol, max_its=int(s["eig.max_its"][0]),
                                      max_vecs=int(s["eig.max_vecs"][0]),
                                      keep=int(s["eig.keep"][0]))
    assert info["fp64_iterations"] >= 1
    assert abs(e - float(s["eig.energy"][0])) <= ENERGY_TOL
    assert plan.config() == config
    plan.close()
