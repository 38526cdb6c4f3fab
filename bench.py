"""Benchmark of the effective-Hamiltonian matvec (Heff TFLOP/s).

One step = one matvec Psi' = Heff Psi over one optimisation step of the
synthetic 24-orbital quantum-chemistry Hamiltonian at D=512 (U1 x SU2,
SITE_SIZE 2): block structure, instruction set and schedule captured from
the reference sweep; the operator values (0.9 GB, too large to ship) are
drawn from a fixed seed, which leaves cost and schedule unchanged.

Besides the FP64 line it reports the split-precision (3xTF32) matvec on the
same step (`split_precision`), whole sweeps of the reference driver linked
against the drop-in with FP64 and with split-precision matvecs plus FP64
defect correction (`sweep`: sweep seconds and final-energy difference), and
the engine's request loop under a Poisson stream of solves (`serving`:
p50/p99 latency, solves/s), and the renormalised-operator updates and the
decomposition's SVDs through their host calls on the captured sweep calls
(`updates_and_decomposition`).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

The engine arm times K matvecs with CUDA events on the launching stream
(inputs resident in HBM; L2 flushed between iterations by writing a 256 MiB
buffer), then the same through the host-buffer C-ABI call (`e2e`: pinned
host x -> device -> matvec -> host y).  The reference arm times the
reference's own matvecT3NS (exec_secondrun, OpenMP + OpenBLAS) on the host
cores for the same step.  Multi-GPU runs are independent replicas (the
matvec of one step is not sharded), value = total FLOPs / max time.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import re
import subprocess
import sys
import tempfile
import time

# the reference LAPACK timed below is called from a pool of host threads:
# keep OpenBLAS from starting its own threads under them
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Heff TFLOP/s"
WORKLOAD_NAME = ("synthetic QC 24 orbitals, 24 e-, U1xSU2, D=512, SITE_SIZE 2: "
                 "one step's Heff matvec")
UNIT = "TFLOP/s"
DEFAULT_WORKLOAD_DIR = os.path.join(ROOT, "oracle", "_ref", "workloads")


# the headline step: the 24-orbital QC Hamiltonian at D=512, SITE_SIZE 2
DEFAULT_WORKLOAD = "qc24_D512_step005.t3c"
# the microbenchmark steps: three-site D=1024 steps of the same Hamiltonian
MICRO_PATTERN = "qc24_D1024_s3_step*.t3c"


def pick_workload(path: str | None) -> str:
    if path:
        return path
    p = os.path.join(DEFAULT_WORKLOAD_DIR, DEFAULT_WORKLOAD)
    if os.path.exists(p):
        return p
    cands = sorted(glob.glob(os.path.join(DEFAULT_WORKLOAD_DIR, "*.t3c")),
                   key=os.path.getsize)
    if not cands:
        raise SystemExit(f"no step files under {DEFAULT_WORKLOAD_DIR}; run "
                         "python -m oracle.captures in the build container")
    return cands[-1]


def step_stats(s):
    bb = s["beginblock"]
    sizes = np.diff(bb)
    return {"blocks": int(s["nrblocks"][0]), "psi_elems": int(bb[-1]),
            "block_median": float(np.median(sizes)), "block_max": int(sizes.max()),
            "merge_instr": int(s["iset.nr_instr"][0])}


class Clocks:
    """nvidia-smi sampler during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="t3ns_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if not self.proc:
            return None
        rows = []
        with open(self.path) as f:
            lines = f.readlines()
        os.unlink(self.path)
        for line in lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measure_fp64_peak(torch):
    """cuBLAS DGEMM 8192^3 through torch (best of 5): the FP64 roofline."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def max_over_ranks(values, world, device):
    """Each value's maximum over the ranks (the slowest rank's time); the
    values unchanged on one rank.  A collective: every rank calls it."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def run_engine(args, rank, world):
    import torch

    from t3ns_b200.native import HeffPlan, StepDesc
    from t3ns_b200.stepfile import read_step

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    path = pick_workload(args.workload)
    s = read_step(path)
    desc = StepDesc(s)
    plan = HeffPlan(desc)
    st = plan.stats
    n = plan.size
    g = torch.Generator(device="cpu").manual_seed(1234 + rank)
    x = torch.randn(n, generator=g, dtype=torch.float64)
    x /= x.norm()
    x = x.cuda()
    y = torch.empty_like(x)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream

    peak = measure_fp64_peak(torch) if rank == 0 else None
    if args.kernel_config is None:
        tune_ms = plan.autotune(reps=2)    # the engine's autotuner picks the configuration
    else:
        tune_ms = None
        plan.set_config(args.kernel_config)

    for _ in range(args.warmup):
        plan.matvec_device(x.data_ptr(), y.data_ptr(), sh)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()

    times = []
    with Clocks(dev) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.matvec_device(x.data_ptr(), y.data_ptr(), sh)
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize()
    t_steps = [a.elapsed_time(b) * 1e-3 for a, b in times]
    t_total = float(sum(t_steps))
    launches = plan.last_launches() * args.steps

    # split precisions (3xTF32, BF16x3) on the same step: time, and error
    # against FP64
    from t3ns_b200.native import T3NS_PREC_3XTF32, T3NS_PREC_BF16X3, T3NS_PREC_FP64
    y64 = y.clone()

    def time_precision(prec, fixed_config):
        plan.set_precision(prec)
        if fixed_config is None:
            tune = plan.autotune(reps=1)
        else:
            tune = None
            plan.set_config(fixed_config)
        for _ in range(args.warmup):
            plan.matvec_device(x.data_ptr(), y.data_ptr(), sh)
        torch.cuda.synchronize()
        ts = []
        for _ in range(args.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.matvec_device(x.data_ptr(), y.data_ptr(), sh)
            e1.record(stream)
            ts.append((e0, e1))
        torch.cuda.synchronize()
        t = float(sum(a.elapsed_time(b) * 1e-3 for a, b in ts))
        return t, float((y - y64).norm() / y64.norm()), plan.config(), tune

    t_split, split_err, split_cfg, split_tune = time_precision(T3NS_PREC_3XTF32,
                                                              args.split_kernel_config)
    t_bf, bf_err, bf_cfg, bf_tune = time_precision(T3NS_PREC_BF16X3, args.bf16_kernel_config)
    plan.set_precision(T3NS_PREC_FP64)
    if args.kernel_config is None:
        plan.autotune(reps=1, force=False)
    else:
        plan.set_config(args.kernel_config)
    y.copy_(y64)

    # e2e: host buffers (pinned) through the C-ABI host entry point
    xh = x.cpu().pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    import ctypes as C
    lib = plan.lib
    f64p = C.POINTER(C.c_double)
    for _ in range(max(1, args.warmup // 2)):
        lib.t3ns_heff_matvec_host(plan.h, C.cast(xh.data_ptr(), f64p), C.cast(yh.data_ptr(), f64p))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rc = lib.t3ns_heff_matvec_host(plan.h, C.cast(xh.data_ptr(), f64p),
                                       C.cast(yh.data_ptr(), f64p))
        if rc < 0:
            raise RuntimeError(lib.t3ns_last_error())
    t_e2e = time.perf_counter() - t0
    err = float((yh.cuda() - y).norm() / y.norm())
    assert err < 1e-12, err

    # every rank takes this collective, in the same order
    t_total, t_e2e, t_split, t_bf = max_over_ranks([t_total, t_e2e, t_split, t_bf], world, "cuda")
    if rank != 0:
        return None
    flops = st["flops_ref"]
    value = flops * args.steps * world / t_total / 1e12
    achieved = flops / (t_total / args.steps) / 1e12
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME + " (" + os.path.basename(path) + ")",
                   **step_stats(s), "flops_per_matvec": flops,
                   "parallelism": f"replicas{world}", "l2": "flushed between iterations",
                   "precision": "fp64", "kernel_config": plan.config(),
                   "autotune_ms": tune_ms},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "traffic": traffic_from_profile(path, plan.config()),
                     "peak_source": "measured this run: cuBLAS DGEMM 8192^3 via torch (FP64 "
                                    "peak; MEASURED_PEAKS.json has no FP64 figure)"},
        "e2e": {"value": flops * args.steps * world / t_e2e / 1e12, "unit": UNIT,
                "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
        "split_precision": {"value": flops * args.steps * world / t_split / 1e12, "unit": UNIT,
                            "ms_per_step": 1e3 * t_split / args.steps,
                            "speedup_vs_fp64": t_total / t_split,
                            "rel_err_vs_fp64": split_err, "kernel_config": split_cfg,
                            "autotune_ms": split_tune,
                            "arithmetic": "3xTF32 products of pre-split {hi, lo} TF32 pairs, "
                                          "FP32 accumulation"},
        "bf16x3": {"value": flops * args.steps * world / t_bf / 1e12, "unit": UNIT,
                   "ms_per_step": 1e3 * t_bf / args.steps, "speedup_vs_fp64": t_total / t_bf,
                   "rel_err_vs_fp64": bf_err, "kernel_config": bf_cfg, "autotune_ms": bf_tune,
                   "arithmetic": "3 BF16 products of pre-split {hi, lo} BF16 pairs "
                                 "(4 bytes an element), FP32 accumulation"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    return out


def sweep_comparison(timeout=900):
    """Whole sweeps of the reference's own driver linked against the drop-in,
    once with the FP64 matvec and once with the split-precision (3xTF32)
    matvec plus FP64 defect correction: sweep seconds of each and the
    final-energy difference.  Cases: the Hubbard tree (D=128, SITE_SIZE 2,
    6 sweeps; E_exact = -6.194800043519880) and the synthetic 12-orbital QC
    Hamiltonian (D=128, 2 sweeps).  None if the driver is not built."""
    exe = os.path.join(ROOT, "oracle", "_ref", "t3ns_run_dropin")
    if not os.path.exists(exe):
        return None
    from t3ns_b200.workloads import synthetic_qc_fcidump
    net = os.path.join(ROOT, "tests", "golden", "networks")
    tmp = tempfile.mkdtemp(prefix="t3ns_bench_")
    fcid = synthetic_qc_fcidump(os.path.join(tmp, "qc12.FCIDUMP"), 12, 12, 0, 72)
    cases = {
        "hubbard10_D128_6sweeps": ["--net", os.path.join(net, "t3ns_10.netw"), "--inter",
                                   "NN_HUBBARD ( t = 1 U = 4 )", "--symm", "Z2,U1,SU2", "--ts",
                                   "0,10,0", "--regime", "128,128,0,2,1e-5,100,6,1e-8,0"],
        "qc12_D128_2sweeps": ["--net", os.path.join(net, "t3ns_12.netw"), "--inter", fcid,
                              "--symm", "Z2,U1,SU2", "--ts", "0,12,0",
                              "--regime", "128,128,0,2,1e-5,100,2,1e-8,0"],
    }
    out = {}
    for name, args in cases.items():
        rec = {}
        for prec in ("fp64", "3xtf32", "bf16x3"):
            env = dict(os.environ, T3NS_B200_PRECISION=prec, OMP_NUM_THREADS="8",
                       OPENBLAS_NUM_THREADS="1")
            r = subprocess.run([exe, *args, "--init", "c"], capture_output=True, text=True,
                               env=env, timeout=timeout)
            if r.returncode != 0:
                tail = (r.stdout + r.stderr).strip().splitlines()[-3:]
                rec[prec] = {"error": f"exit {r.returncode}: " + " | ".join(tail)}
                continue
            rec[prec] = parse_sweep_run(r.stdout)
        f = rec["fp64"]
        if "error" not in f:
            for prec, key in (("3xtf32", "mixed"), ("bf16x3", "bf16x3")):
                m = rec[prec]
                if "error" in m:
                    continue
                rec[f"speedup_{key}_vs_fp64"] = f["sweep_seconds"] / m["sweep_seconds"]
                rec[f"matvec_bucket_speedup_{key}_vs_fp64"] = (
                    f["timers"].get("Heff T3NS: matvec", 0) + f["timers"].get("Heff DMRG: matvec", 0)) / max(
                    m["timers"].get("Heff T3NS: matvec", 0) + m["timers"].get("Heff DMRG: matvec", 0), 1e-12)
                rec[f"abs_dE_{key}_vs_fp64"] = abs(m["energy"] - f["energy"])
        out[name] = rec
    out["note"] = ("timers are the reference's own buckets over the whole scheme "
                   "(src/optimize_network.c:43-95): 'Heff ...: matvec' is the Davidson solves, "
                   "'prepare data' holds the plan build and the autotuner, so the matvec bucket "
                   "is the mixed-vs-FP64 comparison; davidson_iterations counts matvecs, "
                   "fp64_iterations those in FP64")
    return out


def sweep_qc24(D, precisions=("fp64", "bf16x3", "3xtf32"), timeout=3000):
    """One whole sweep (SITE_SIZE 2) of the reference driver linked against
    the drop-in on the 24-orbital synthetic QC Hamiltonian at bond dimension
    D, once per arithmetic mode: sweep seconds, the reference's own timer
    buckets, Davidson iteration counts, final energies and their differences
    from the FP64 run.  Run on request (--sweep-qc24 D): at D=512 one FP64
    sweep takes tens of minutes on one GPU."""
    exe = os.path.join(ROOT, "oracle", "_ref", "t3ns_run_dropin")
    if not os.path.exists(exe):
        return None
    from t3ns_b200.workloads import synthetic_qc_fcidump
    tmp = tempfile.mkdtemp(prefix="t3ns_bench_")
    fcid = synthetic_qc_fcidump(os.path.join(tmp, "qc24.FCIDUMP"), 24, 24, 0, 72)
    args = ["--net", os.path.join(ROOT, "tests", "golden", "networks", "t3ns_24.netw"),
            "--inter", fcid, "--symm", "Z2,U1,SU2", "--ts", "0,24,0",
            "--regime", f"{D},{D},0,2,1e-5,100,1,1e-8,0", "--init", "c"]
    out = {"D": D, "sweeps": 1, "site_size": 2}
    for prec in precisions:
        env = dict(os.environ, T3NS_B200_PRECISION=prec, OMP_NUM_THREADS="16",
                   OPENBLAS_NUM_THREADS="1")
        r = subprocess.run([exe, *args], capture_output=True, text=True, env=env, timeout=timeout)
        if r.returncode != 0:
            out[prec] = {"error": f"exit {r.returncode}"}
            continue
        rec = parse_sweep_run(r.stdout)
        rec["init_seconds"] = float(re.findall(r"INIT_SECONDS (\S+)", r.stdout)[-1])
        out[prec] = rec
    f = out.get("fp64", {})
    for prec in precisions[1:]:
        m = out.get(prec, {})
        if "sweep_seconds" in f and "sweep_seconds" in m:
            out[f"speedup_{prec}_vs_fp64"] = f["sweep_seconds"] / m["sweep_seconds"]
            out[f"abs_dE_{prec}_vs_fp64"] = abs(m["energy"] - f["energy"])
    return out


_TIMER = re.compile(r"^ \* (.+?)\s+:: ([0-9.]+) sec", re.M)


def parse_sweep_run(stdout: str) -> dict:
    """Final energy, sweep seconds, sweeps executed, the reference's timers
    for the whole optimisation scheme, and the Davidson iteration counts
    (all and FP64) of one run of the drop-in driver."""
    tail = stdout.split("TIMERS FOR OPTIMIZATION SCHEME")[-1]
    timers = {k.strip(): float(v) for k, v in _TIMER.findall(tail)}
    return {
        "sweep_seconds": float(re.findall(r"SWEEP_SECONDS (\S+)", stdout)[-1]),
        "energy": float(re.findall(r"FINAL_ENERGY (\S+)", stdout)[-1]),
        "sweeps": sum(int(k) for k in re.findall(r"END OF REGIME \d+ AFTER (\d+)/\d+ SWEEPS", stdout)),
        "timers": timers,
        "timers_total_vs_sweep_seconds": timers.get("Total time", 0.0) /
        max(float(re.findall(r"SWEEP_SECONDS (\S+)", stdout)[-1]), 1e-12),
        "davidson_solves": len(re.findall(r"Davidson: \(iter: ", stdout)),
        "davidson_iterations": sum(int(x) for x in re.findall(r"Davidson: \(iter: (\d+)\)", stdout)),
        "fp64_iterations": sum(int(x) for x in re.findall(r"\(fp64 iter: (\d+)\)", stdout)),
    }


def davidson_comparison(path=None, max_its=100, seed=7):
    """One Davidson solve of a real D=512 step (the 24-orbital QC
    Hamiltonian's step 6, 645,595 elements, operators as the reference built
    them) to tol 1e-5, with FP64 matvecs and with split-precision matvecs
    plus FP64 defect correction: seconds, iterations and the energy
    difference.  The guess stands in for the previous step's state the sweep
    would pass: an untimed FP64 solve to 3e-3 from a seeded random vector.
    None if the step is not present."""
    path = path or os.path.join(ROOT, "oracle", "_ref", "captures", "qc24_D512", "step_006.t3c")
    if not os.path.exists(path):
        return None
    from t3ns_b200.native import (HeffPlan, StepDesc, T3NS_PREC_3XTF32, T3NS_PREC_BF16X3,
                                  T3NS_PREC_FP64)
    from t3ns_b200.stepfile import read_step
    s = read_step(path)
    desc = StepDesc(s)
    g0 = np.random.default_rng(seed).standard_normal(s["diag"].size)
    g0 /= np.linalg.norm(g0)
    pre = HeffPlan(desc)
    _, _, pinfo = pre.davidson_host(g0, s["diag"], tol=3e-3, max_its=200)
    pre.close()
    out = {"step": os.path.relpath(path, ROOT), "psi_elems": int(s["diag"].size), "tol": 1e-5,
           "max_its": max_its,
           "guess": "FP64 solve from seeded N(0,1) to residual %.1e (%d iterations)"
                    % (pinfo["residual"], pinfo["iterations"])}
    for name, prec in (("fp64", T3NS_PREC_FP64), ("3xtf32", T3NS_PREC_3XTF32),
                       ("bf16x3", T3NS_PREC_BF16X3)):
        plan = HeffPlan(desc, prec)
        plan.autotune(reps=1, force=False)
        g = g0.copy()
        t0 = time.perf_counter()
        e, rc, info = plan.davidson_host(g, s["diag"], tol=1e-5, max_its=max_its)
        out[name] = {"seconds": time.perf_counter() - t0, "energy": e, "return": rc,
                     "iterations": info["iterations"], "fp64_iterations": info["fp64_iterations"],
                     "residual": info["residual"]}
        plan.close()
    out["speedup_mixed_vs_fp64"] = out["fp64"]["seconds"] / out["3xtf32"]["seconds"]
    out["abs_dE_mixed_vs_fp64"] = abs(out["3xtf32"]["energy"] - out["fp64"]["energy"])
    out["speedup_bf16x3_vs_fp64"] = out["fp64"]["seconds"] / out["bf16x3"]["seconds"]
    out["abs_dE_bf16x3_vs_fp64"] = abs(out["bf16x3"]["energy"] - out["fp64"]["energy"])
    return out


def other_rows_measurement(reps=3):
    """The renormalised-operator updates and the decomposition's
    factorisations through their host C-ABI calls (host arrays in and out,
    uploads, device allocations and the kernel: what the drop-in pays per
    call), on every captured call of the Hubbard and 12-orbital QC sweeps:
    algorithmic GFLOP and GPU seconds (best of `reps` per call); the SVDs
    also timed through the reference's LAPACK (OpenBLAS LAPACKE_dgesdd) on the
    host for comparison, one call at a time and all calls from a pool of host
    threads (the reference decomposes a split's sectors in an OpenMP loop,
    src/siteTensor_decompose.c:1413).  None if the captures are absent."""
    import ctypes as C
    from t3ns_b200 import native, updates
    from t3ns_b200.stepfile import read_step
    caps = os.path.join(ROOT, "oracle", "_ref", "captures")
    out = {}

    def bound_call(fn, a_in, jobz, m, n):
        """One SVD call with its own input copy and output arrays."""
        k = min(m, n)
        s_, u, vt = np.zeros(k), np.zeros(max(m * k, 1)), np.zeros(max(k * n, 1))

        def go():
            a = np.array(a_in)
            fn(jobz.encode(), m, n, a.ctypes.data, m, s_.ctypes.data, u.ctypes.data, m,
               vt.ctypes.data, k)
        return go

    def best(fn):
        t = []
        for _ in range(reps + 1):
            t0 = time.perf_counter()
            fn()
            t.append(time.perf_counter() - t0)
        return min(t[1:])

    for kind in ("pupdate", "bupdate"):
        files = sorted(glob.glob(os.path.join(caps, "pupdate_*", f"{kind}_*.t3c")))
        files = [f for f in files if os.path.exists(f.replace(".t3c", ".sched"))]
        if not files:
            return None
        flops = secs = 0.0
        for f in files:
            rec, sch = read_step(f), read_step(f.replace(".t3c", ".sched"))
            if kind == "pupdate":
                flops += updates.pupdate_flops(sch)
                secs += best(lambda: updates.pupdate_host(sch, rec["T.tel"], rec["ops0.tel"]))
            else:
                flops += updates.bupdate_flops(sch)
                secs += best(lambda: updates.bupdate_host(sch, rec["T.tel"], rec["ops0.tel"],
                                                          rec["ops1.tel"]))
        out[kind] = {"calls": len(files), "gflop": flops / 1e9, "gpu_seconds_e2e": secs,
                     "gflop_per_s_e2e": flops / secs / 1e9}

    lib = native.load()
    lib.t3ns_gesdd_host.argtypes = [C.c_char, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    libdir = os.path.join(os.path.dirname(np.__file__), "..", "opencv_python_headless.libs")
    blas = glob.glob(os.path.join(libdir, "libopenblas*.so"))
    for pat in ("libquadmath*.so*", "libgfortran*.so*"):   # OpenBLAS's Fortran runtime
        for dep in glob.glob(os.path.join(libdir, pat)):
            C.CDLL(dep, mode=C.RTLD_GLOBAL)
    cpu = C.CDLL(blas[0]) if blas else None
    if cpu is not None:
        cpu.LAPACKE_dgesdd.argtypes = [C.c_int, C.c_char, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                       C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    files = sorted(glob.glob(os.path.join(caps, "dense_*", "gesdd_*.t3c")))
    gpu_s = cpu_s = 0.0
    largest = (0, 0)
    pool_calls = []          # (GPU call, LAPACK call), each with its own arrays
    for f in files:
        r = read_step(f)
        m, n = int(r["gesdd.m"][0]), int(r["gesdd.n"][0])
        jobz = chr(int(r["gesdd.jobz"][0]))
        k = min(m, n)
        if k == 0:
            continue
        largest = max(largest, (m, n), key=lambda x: x[0] * x[1])
        gpu_call = bound_call(lambda *x: native.check(lib.t3ns_gesdd_host(*x), "gesdd"),
                              r["gesdd.a"], jobz, m, n)
        cpu_call = bound_call(lambda *x: cpu.LAPACKE_dgesdd(102, *x), r["gesdd.a"], jobz, m, n) \
            if cpu is not None else None
        gpu_s += best(gpu_call)
        if cpu_call is not None:
            cpu_s += best(cpu_call)
        pool_calls.append((gpu_call, cpu_call))

    from concurrent.futures import ThreadPoolExecutor
    workers = min(16, os.cpu_count() or 1)

    def pooled(fns):
        with ThreadPoolExecutor(workers) as ex:
            return best(lambda: list(ex.map(lambda fn: fn(), fns)))
    out["gesdd"] = {"calls": len(files), "largest": list(largest), "gpu_seconds_e2e": gpu_s,
                    "reference_lapack_seconds": cpu_s if cpu is not None else None,
                    "host_threads": workers,
                    "gpu_seconds_e2e_threads": pooled([g for g, _ in pool_calls]),
                    "reference_lapack_seconds_threads":
                        pooled([c for _, c in pool_calls]) if cpu is not None else None}
    return out


# request sources of the serving measurement: the captured small steps and
# the golden steps (each carries its reference Davidson energy)
REQUEST_SOURCES = [os.path.join(ROOT, "oracle", "_ref", "captures", "*", "step_*.t3c"),
                   os.path.join(ROOT, "tests", "golden", "*.t3c")]


def serving_stream():
    """The engine's request loop under a Poisson stream of 128 independent
    ground-state solves (mean 4 arrivals/s; solves drawn from the captured
    Hubbard and 12-orbital QC steps, with the reference's operators), 8 GiB
    admission budget, 4 in flight, split precision with FP64 defect
    correction: p50/p99 latency and solves/s."""
    from t3ns_b200.serving import Workload, request_steps, run_stream
    steps = request_steps(REQUEST_SOURCES)
    if not steps:
        return None
    _, summary = run_stream([Workload(p) for p in steps], n_requests=128, rate=4.0,
                            budget_bytes=8 << 30, max_inflight=4, precision="3xtf32", seed=0)
    summary["requests_from"] = "%d captured steps (Hubbard L=10 tree, 12-orbital QC)" % len(steps)
    return summary


def microbench_d1024(args, peak, reps=None):
    """The batched matvec microbenchmark: the three-site D=1024 steps of the
    24-orbital Hamiltonian (structure from the reference sweep, operator
    values from a fixed seed).  Per step: block statistics, F, the grouped
    persistent FP64 launch (autotuned), the same kernel dispatched block by
    block, and the split-precision (3xTF32) matvec with its error against
    FP64; CUDA events, L2 flushed between iterations."""
    import torch

    from t3ns_b200.native import (T3NS_PREC_3XTF32, T3NS_PREC_BF16X3, T3NS_PREC_FP64, HeffPlan,
                                  StepDesc)
    from t3ns_b200.stepfile import read_step
    files = sorted(glob.glob(os.path.join(DEFAULT_WORKLOAD_DIR, MICRO_PATTERN)))
    if not files:
        return None
    reps = reps or max(3, min(args.steps, 5))
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            ts.append((e0, e1))
        torch.cuda.synchronize()
        return float(np.median([a.elapsed_time(b) for a, b in ts]))

    out = []
    for f in files:
        s = read_step(f)
        sizes = np.diff(s["beginblock"].astype(np.int64))
        plan = HeffPlan(StepDesc(s))
        F = plan.stats["flops_ref"]
        g = torch.Generator(device="cpu").manual_seed(5)
        x = torch.randn(plan.size, generator=g, dtype=torch.float64)
        x = (x / x.norm()).cuda()
        y = torch.empty_like(x)
        sh = stream.cuda_stream
        tune = plan.autotune(reps=1)
        t64 = timed(lambda: plan.matvec_device(x.data_ptr(), y.data_ptr(), sh))
        cfg64 = plan.config()
        y64 = y.clone()
        tblk = timed(lambda: plan.matvec_device_per_block(x.data_ptr(), y.data_ptr(), sh))
        nblk = plan.last_launches()
        plan.set_precision(T3NS_PREC_3XTF32)
        stune = plan.autotune(reps=1)
        tsp = timed(lambda: plan.matvec_device(x.data_ptr(), y.data_ptr(), sh))
        err = float((y - y64).norm() / y64.norm())
        cfgsp = plan.config()
        plan.set_precision(T3NS_PREC_BF16X3)
        btune = plan.autotune(reps=1)
        tbf = timed(lambda: plan.matvec_device(x.data_ptr(), y.data_ptr(), sh))
        bf_err = float((y - y64).norm() / y64.norm())
        cfgbf = plan.config()
        plan.set_precision(T3NS_PREC_FP64)
        plan.close()
        out.append({
            "step": os.path.basename(f), "blocks": int(s["nrblocks"][0]), "psi_elems": int(sizes.sum()),
            "block_size_quantiles": {q: int(np.quantile(sizes, q)) for q in (0.5, 0.9, 1.0)},
            "merge_instr": int(s["iset.nr_instr"][0]), "flops_per_matvec": F,
            "fp64_grouped": {"ms": t64, "tflops": F / t64 / 1e9, "kernel_config": cfg64,
                             "autotune_ms": tune,
                             "roofline_frac": (F / t64 / 1e9) / peak if peak else None},
            "fp64_per_block_dispatch": {"ms": tblk, "tflops": F / tblk / 1e9, "launches": nblk},
            "grouped_speedup_vs_per_block": tblk / t64,
            "split_3xtf32": {"ms": tsp, "tflops": F / tsp / 1e9, "kernel_config": cfgsp,
                             "autotune_ms": stune, "speedup_vs_fp64": t64 / tsp,
                             "rel_err_vs_fp64": err},
            "bf16x3": {"ms": tbf, "tflops": F / tbf / 1e9, "kernel_config": cfgbf,
                       "autotune_ms": btune, "speedup_vs_fp64": t64 / tbf,
                       "rel_err_vs_fp64": bf_err},
        })
        del x, y, y64
        torch.cuda.empty_cache()
    return {"steps": out, "l2": "flushed between iterations",
            "data": "block structure and schedule from the reference's three-site D=1024 sweep of "
                    "the synthetic 24-orbital Hamiltonian; operator values from a fixed seed"}


def traffic_from_profile(workload_path, kernel_config):
    """DRAM bytes (read + write) of one FP64 heff_kernel launch in kernel
    configuration `kernel_config` on this workload, from the ncu capture
    summarised under profiles/ (None if that workload and configuration have
    not been profiled)."""
    p = os.path.join(ROOT, "profiles", "heff_kernel_traffic.json")
    if not os.path.exists(p):
        return None
    rec = json.load(open(p)).get(os.path.basename(workload_path))
    if rec is None or rec.get("kernel_config") != kernel_config:
        return None
    return rec["dram_bytes_per_launch"]


def cpu_baseline(path, samples=1, stride=None, target_s=15.0):
    """The reference's own matvecT3NS (exec_secondrun, OpenMP over all host
    cores, OpenBLAS) on every `stride`-th output block of the step: a bounded
    sample of about `target_s` seconds, found by a short calibration run on
    every 64th block."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_matvec_bench")
    if not os.path.exists(exe):
        return None
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(ncores), OPENBLAS_NUM_THREADS="1")

    def run(n, st):
        r = subprocess.run([exe, path, str(n), str(st)], capture_output=True, text=True, env=env)
        if r.returncode != 0:
            return None
        return json.loads(r.stdout.strip().splitlines()[-1])

    if stride is None:
        cal = run(1, 64)
        if cal is None:
            return None
        full_s = cal["seconds_per_matvec"] * 64
        stride = max(1, int(round(full_s / target_s)))
    res = run(samples, stride)
    if res is None:
        return None
    res["cores"] = ncores
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default=None)
    ap.add_argument("--kernel-config", type=int, default=None,
                    help="run the FP64 matvec in this kernel configuration instead of the "
                         "autotuner's choice (profiling: the autotuner's event timing is "
                         "distorted under a profiler)")
    ap.add_argument("--split-kernel-config", type=int, default=None,
                    help="the same for the 3xTF32 matvec")
    ap.add_argument("--bf16-kernel-config", type=int, default=None,
                    help="the same for the BF16x3 matvec")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sweep", action="store_true",
                    help="skip the whole-sweep FP64 vs split-precision comparison")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the request-stream (serving) measurement")
    ap.add_argument("--no-micro", action="store_true",
                    help="skip the three-site D=1024 matvec microbenchmark")
    ap.add_argument("--sweep-qc24", type=int, default=None, metavar="D",
                    help="also run one whole sweep of the 24-orbital QC Hamiltonian at bond "
                         "dimension D through the drop-in in each arithmetic mode (long)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))

    if args.impl == "reference":
        if rank != 0:
            return
        path = pick_workload(args.workload)
        from t3ns_b200.stepfile import read_step
        s = read_step(path)
        flops = None
        res = cpu_baseline(path, samples=max(1, min(args.steps, 3)))
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU build "
                              "(oracle/_ref/ref_matvec_bench) missing"}))
            return
        flops = res["flops"]
        v = flops / res["seconds_per_matvec"] / 1e12
        sample = (f"{res['calls']} calls (median taken) of the reference matvecT3NS "
                  f"(exec_secondrun) restricted to every {res['stride']}-th output block of "
                  f"this step ({res['sampled_blocks']} of {res['blocks']} blocks, "
                  f"{flops / res['flops_full']:.3f} of the full matvec's FLOPs); the full "
                  f"matvec's time is estimated at this rate")
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": res["calls"], "warmup": 0,
            "ms_per_step": 1e3 * res["seconds_per_matvec"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME + " (" + os.path.basename(path) + ")",
                       **step_stats(s), "flops_per_matvec": res["flops_full"],
                       "parallelism": f"replicas{world}", "precision": "fp64"},
            "sample": {"stride": res["stride"], "calls": res["calls"],
                       "flops_per_call": flops, "flops_full_matvec": res["flops_full"],
                       "ms_per_call": 1e3 * res["seconds_per_matvec"],
                       "ms_per_full_matvec_est": 1e3 * res["seconds_per_matvec"] *
                       res["flops_full"] / flops},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": res["cores"], "kind": "reference",
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    out = run_engine(args, rank, world)
    if world > 1:
        # the CPU baseline, Davidson, sweep, serving and update figures are
        # single-GPU measurements, taken at N=1 only
        args.no_cpu_baseline = args.no_sweep = args.no_serving = args.no_micro = True
    if rank == 0:
        if not args.no_micro:
            out["microbench_D1024"] = microbench_d1024(args, out["roofline"]["peak"])
        if not args.no_cpu_baseline:
            cb = cpu_baseline(pick_workload(args.workload), samples=1)
            if cb:
                v = cb["flops"] / cb["seconds_per_matvec"] / 1e12
                out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cb["cores"],
                                       "kind": "reference",
                                       "sample": "1 call of the reference matvecT3NS "
                                                 "(exec_secondrun) on every %d-th output block "
                                                 "of the same step" % cb["stride"]}
            else:
                out["cpu_baseline"] = None
        if not args.no_sweep:
            out["davidson_D512"] = davidson_comparison()
            out["sweep"] = sweep_comparison()
        if not args.no_serving:
            out["serving"] = serving_stream()
        if not args.no_sweep:
            out["updates_and_decomposition"] = other_rows_measurement()
        if args.sweep_qc24:
            out["sweep_qc24"] = sweep_qc24(args.sweep_qc24)
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
    # the JSON line is out: leave without the interpreter's teardown, where
    # the threads and runtimes this process loaded (OpenBLAS, two CUDA
    # runtimes, per-thread engine workspaces) are torn down in no fixed order
    sys.stdout.flush()
    sys.stderr.flush()
    os._exit(0)
