"""The drop-in (libt3ns_dropin.so) behind the reference's own sweep driver.

CPU: its schedule compiler reproduces the reference's replay schedule
(exec_firstrun's struct secondrun) exactly, pair by pair, with bit-identical
prefactors, on Hubbard and quantum-chemistry steps (DMRG and T3NS types).

GPU: the unchanged reference sweep driver linked against the drop-in gives
the reference's energies: config 1 (Hubbard L=10, D=128) against the
reference CPU run to 1e-8 Ha, and the reference's own test1/test2 energy pin
(N2 STO-3G, -107.648250974014 Ha at 1e-8, tests/test1.c.in:99).
"""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from schedule_compare import compare
from t3ns_b200.stepfile import read_step
from t3ns_b200.workloads import synthetic_qc_fcidump

REF = os.path.join(ROOT, "oracle", "_ref")
RUN_REF = os.path.join(REF, "t3ns_run_ref")
RUN_DROPIN = os.path.join(REF, "t3ns_run_dropin")
DROPIN = os.path.join(ROOT, "t3ns_b200", "_lib", "libt3ns_dropin.so")
NET = os.path.join(ROOT, "tests", "golden", "networks")
HUB10 = ["--net", os.path.join(NET, "t3ns_10.netw"), "--inter", "NN_HUBBARD ( t = 1 U = 4 )",
         "--symm", "Z2,U1,SU2", "--ts", "0,10,0"]


def need(*paths):
    for p in paths:
        if not os.path.exists(p):
            pytest.skip(f"not built: {p}")


def run(exe, args, env_extra=None, timeout=1200):
    env = dict(os.environ, OMP_NUM_THREADS="4", OPENBLAS_NUM_THREADS="1")
    env.update(env_extra or {})
    r = subprocess.run([exe, *args], capture_output=True, text=True, env=env, timeout=timeout)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def energy(out):
    return float(re.findall(r"FINAL_ENERGY (\S+)", out)[-1])


@pytest.mark.parametrize("case", ["hub10", "qc12"])
def test_schedule_compiler_matches_reference(case, tmp_path):
    need(RUN_REF, DROPIN)
    if case == "hub10":
        args = HUB10 + ["--regime", "128,128,0,2,1e-5,100,1,1e-8,0"]
    else:
        fc = synthetic_qc_fcidump(tmp_path / "qc12.FCIDUMP", 12, 12, 0, 72)
        args = ["--net", os.path.join(NET, "t3ns_12.netw"), "--inter", fc, "--symm",
                "Z2,U1,SU2", "--ts", "0,12,0", "--regime", "64,64,0,2,1e-5,100,1,1e-8,0"]
    cap = tmp_path / "cap"
    cap.mkdir()
    run(RUN_REF, args + ["--init", "c", "--capture", str(cap), "--capture-limit", "7",
                         "--capture-stop", "--capture-noeig", "--capture-nvec", "1",
                         "--schedule-lib", DROPIN])
    steps = sorted(glob.glob(str(cap / "*.t3c")))
    assert len(steps) == 7
    kinds = set()
    for t in steps:
        ref = read_step(t)
        mine = read_step(t.replace(".t3c", ".sched"))
        isd = int(ref["isdmrg"][0])
        kinds.add(isd)
        assert np.array_equal(ref["sr.dims"], mine["my.dims"])
        missing, extra, diff = compare(ref, mine, isd)
        assert not missing and not extra and not diff, (t, missing[:3], extra[:3], diff[:3])
    if case == "hub10":
        assert kinds == {0, 1}   # DMRG-type and T3NS-type steps both covered


@pytest.mark.gpu
def test_sweep_energy_hubbard_config1():
    """Config 1: NN_HUBBARD t=1 U=4, 10 electrons, T3NS tree of 10 sites,
    U1 x SU2, D=128, SITE_SIZE 2, 6 sweeps, E_CONV 1e-8."""
    need(RUN_REF, RUN_DROPIN)
    args = HUB10 + ["--regime", "128,128,0,2,1e-5,100,6,1e-8,0", "--init", "c"]
    e_ref = energy(run(RUN_REF, args))
    out = run(RUN_DROPIN, args)
    assert "Davidson: (iter:" in out
    assert abs(energy(out) - e_ref) <= 1e-8
    assert abs(energy(out) - (-6.194800043519880)) <= 1e-8   # exact diagonalisation


@pytest.mark.gpu
def test_sweep_energy_hubbard_config1_split_precision():
    """Config 1 with split-precision (3xTF32) matvecs and FP64 defect
    correction in every Davidson solve: the final energy stays within 1e-8 Ha
    of exact diagonalisation."""
    need(RUN_DROPIN)
    args = HUB10 + ["--regime", "128,128,0,2,1e-5,100,6,1e-8,0", "--init", "c"]
    out = run(RUN_DROPIN, args, {"T3NS_B200_PRECISION": "3xtf32"})
    assert abs(energy(out) - (-6.194800043519880)) <= 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("net", ["10_T3NS", "10_DMRG"])
@pytest.mark.parametrize("symm,ts", [("Z2,U1,SU2", "0,14,0"), ("Z2,U1,SU2,D2h", "0,14,0,0"),
                                     ("Z2,U1,U1", "0,7,7")])
def test_reference_energy_pin_n2(net, symm, ts):
    """The reference's test1/test2 (tests/test1.c.in, tests/test2.c.in):
    N2/STO-3G, two regimes, energy -107.648250974014 within 1e-8."""
    fcidump = os.path.join(REF, "data", "N2.STO3G.FCIDUMP")
    netw = os.path.join(REF, "data", net + ".netw")
    need(RUN_DROPIN, fcidump, netw)
    out = run(RUN_DROPIN, ["--net", netw, "--inter", fcidump, "--symm", symm, "--ts", ts,
                           "--regime", "1000,1000,1e-4,2,1e-6,4,2,1e-8,0",
                           "--regime", "1000,1000,1e-4,2,1e-6,100,10,1e-8,0", "--init", "c"])
    assert abs(energy(out) + 107.648250974014) < 1e-8


@pytest.mark.gpu
def test_dropin_preconditioner_matches_restated_reference(tmp_path):
    """The drop-in's davidson_diagonal_preconditioner (the unchanged driver's
    symbol, linked into t3ns_run_dropin) against the numpy restatement of
    reference src/davidson.c:223-257 (oracle/precond_oracle.py, itself pinned
    to the reference build on the CPU), cutoff branch included."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import precond_oracle
    need(RUN_DROPIN)
    rng = np.random.default_rng(11)
    n, theta = 200_003, 0.35
    r = rng.standard_normal(n)
    r /= np.linalg.norm(r)
    dg = rng.uniform(-3.0, 5.0, n)
    dg[::977] = theta
    t = rng.standard_normal(n) * 1e-3
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as f:
        f.write(np.array([n], np.int64).tobytes())
        f.write(np.array([theta]).tobytes())
        for a in (r, dg, t):
            f.write(a.tobytes())
    subprocess.run([RUN_DROPIN, "--precond-file", str(fin), str(fout)], check=True, timeout=300)
    got = np.fromfile(fout, np.float64)
    want = precond_oracle.precondition(r, theta, dg, t)
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["hub10", "qc12"])
def test_dropin_append_matches_reference_every_call(case, tmp_path):
    """The drop-in's rOperators_append_phys (GPU scaled copies, device sum of
    the unique operators, zero-block removal) against the reference's on
    every call of a sweep: the reference harness runs both on the same input
    in one process (--check-dropin) and compares the new sets -- the same
    operators, sectors and surviving blocks, the elements to 1e-12 of the
    largest (reference src/rOperators_pUpdate.c:665-673)."""
    need(RUN_REF, DROPIN)
    if case == "hub10":
        args = HUB10 + ["--regime", "128,128,0,2,1e-5,100,1,1e-8,0"]
    else:
        fc = synthetic_qc_fcidump(tmp_path / "qc12.FCIDUMP", 12, 12, 0, 72)
        args = ["--net", os.path.join(NET, "t3ns_12.netw"), "--inter", fc, "--symm",
                "Z2,U1,SU2", "--ts", "0,12,0", "--regime", "64,64,0,2,1e-5,100,1,1e-8,0"]
    out = run(RUN_REF, args + ["--init", "c", "--check-dropin", DROPIN])
    diffs = [float(v) for v in re.findall(r"CHECK_APPEND \d+ (\S+)", out)]
    assert len(diffs) >= 10
    assert all(0.0 <= v <= 1e-12 for v in diffs), max(diffs)
