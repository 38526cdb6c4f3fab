"""Request stream over the engine's request loop (``t3ns_server_*``).

Independent ground-state solves (one Davidson solve of an effective
Hamiltonian each) arrive as a Poisson stream; the engine admits them against
a fixed device-memory budget, runs up to ``max_inflight`` at once on separate
streams, and this module reports p50 / p99 latency (arrival to result) and
solves per second.

    python -m t3ns_b200.serving [--requests N] [--rate R] [--budget-gib B]
                                [--inflight K] [--precision fp64|3xtf32]

Requests are drawn (seeded) from the captured optimisation steps under
``oracle/_ref/captures`` (Hubbard chain and tree, 12-orbital QC): each step
file carries the reference's operators, its diagonal and its Davidson guess.
"""
from __future__ import annotations

import argparse
import ctypes as C
import glob
import json
import os
import time

import numpy as np

from . import native
from .native import RequestResult, StepDesc
from .stepfile import read_step

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PRECISIONS = {"fp64": native.T3NS_PREC_FP64, "3xtf32": native.T3NS_PREC_3XTF32}


class Server:
    """Owner of one engine request loop."""

    def __init__(self, budget_bytes: int, max_inflight: int):
        self.lib = native.load()
        h = C.c_void_p()
        native.check(self.lib.t3ns_server_create(int(budget_bytes), int(max_inflight),
                                                 C.byref(h)), "server_create")
        self.h = h
        self._keep = {}

    def submit(self, desc: StepDesc, guess: np.ndarray, diag: np.ndarray, precision: int,
               tol: float = 1e-5, max_its: int = 100, max_vecs: int = 30, keep: int = 2) -> int:
        """Queues a solve; `guess` (float64, C-contiguous) receives the result."""
        assert guess.dtype == np.float64 and guess.flags.c_contiguous
        diag = np.ascontiguousarray(diag, dtype=np.float64)
        rid = C.c_int64()
        native.check(self.lib.t3ns_server_submit(
            self.h, C.byref(desc.desc), precision, guess.ctypes.data_as(C.POINTER(C.c_double)),
            diag.ctypes.data_as(C.POINTER(C.c_double)), tol, max_its, max_vecs, keep,
            C.byref(rid)), "server_submit")
        self._keep[rid.value] = (desc, guess, diag)      # alive until waited for
        return rid.value

    def wait(self, rid: int) -> dict:
        res = RequestResult()
        rc = self.lib.t3ns_server_wait(self.h, rid, C.byref(res))
        self._keep.pop(rid, None)
        native.check(rc, "server_wait")
        out = {f: getattr(res, f) for f, _ in RequestResult._fields_ if f != "info"}
        out["info"] = {f: getattr(res.info, f) for f, _ in native.DavidsonInfo._fields_}
        return out

    def stats(self) -> dict:
        a, b, q = C.c_int64(), C.c_int64(), C.c_int()
        native.check(self.lib.t3ns_server_stats(self.h, C.byref(a), C.byref(b), C.byref(q)))
        return {"in_use": a.value, "peak": b.value, "queued": q.value}

    def close(self):
        if getattr(self, "h", None):
            self.lib.t3ns_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def estimate_bytes(desc: StepDesc, precision: int, max_vecs: int = 30) -> int:
    return int(native.load().t3ns_server_estimate_bytes(C.byref(desc.desc), precision, max_vecs))


def request_steps(patterns: list[str]) -> list[str]:
    """Step files matching the glob `patterns` (the caller's request
    sources) that carry a diagonal, a Davidson guess and a Davidson energy,
    so every result can be checked against the energy recorded with it."""
    out = []
    cands = []
    for pat in patterns:
        cands += sorted(glob.glob(pat))
    for p in cands:
        if os.path.getsize(p) < (256 << 20) and "eig.energy" in read_step(p):
            out.append(p)
    return out


class Workload:
    """A step's descriptor and the inputs of its solve, loaded once."""

    def __init__(self, path: str):
        self.path = path
        self.step = read_step(path)
        self.desc = StepDesc(self.step)
        self.diag = np.ascontiguousarray(self.step["diag"])
        self.guess = np.ascontiguousarray(self.step["eig.guess"]) if "eig.guess" in self.step \
            else None
        self.tol = float(self.step["eig.tol"][0]) if "eig.tol" in self.step else 1e-5
        self.max_vecs = int(self.step["eig.max_vecs"][0]) if "eig.max_vecs" in self.step else 30
        self.keep = int(self.step["eig.keep"][0]) if "eig.keep" in self.step else 2
        self.ref_energy = float(self.step["eig.energy"][0]) if "eig.energy" in self.step else None

    def guess_for(self, rng: np.random.Generator) -> np.ndarray:
        if self.guess is not None:
            return self.guess.copy()
        g = rng.standard_normal(self.diag.size)
        return g / np.linalg.norm(g)


def run_stream(workloads, n_requests=128, rate=4.0, budget_bytes=8 << 30, max_inflight=4,
               precision="3xtf32", seed=0):
    """Poisson arrivals (mean `rate` per second) of `n_requests` solves drawn
    from `workloads`; returns per-request records and the summary."""
    rng = np.random.default_rng(seed)
    picks = rng.integers(0, len(workloads), n_requests)
    gaps = rng.exponential(1.0 / rate, n_requests)
    prec = PRECISIONS[precision]
    srv = Server(budget_bytes, max_inflight)
    t0 = time.perf_counter()
    ids = []
    arrival = 0.0
    for k in range(n_requests):
        arrival += gaps[k]
        delay = t0 + arrival - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        w = workloads[picks[k]]
        g = w.guess_for(rng)
        ids.append((srv.submit(w.desc, g, w.diag, prec, tol=w.tol, max_vecs=w.max_vecs,
                               keep=w.keep), w, g))
    recs = []
    for rid, w, g in ids:
        r = srv.wait(rid)
        r["step"] = os.path.relpath(w.path, ROOT)
        r["ref_energy"] = w.ref_energy
        recs.append(r)
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    lat = np.array([r["latency_seconds"] for r in recs])
    errs = [abs(r["energy"] - r["ref_energy"]) for r in recs if r["ref_energy"] is not None]
    summary = {
        "requests": n_requests, "rate_per_s": rate, "max_inflight": max_inflight,
        "budget_bytes": int(budget_bytes), "peak_admitted_bytes": st["peak"],
        "precision": precision, "wall_seconds": wall, "solves_per_s": n_requests / wall,
        "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
        "queue_p99_s": float(np.percentile([r["queue_seconds"] for r in recs], 99)),
        "max_abs_dE_vs_reference": max(errs) if errs else None,
        "failed": sum(1 for r in recs if r["status"] < 0),
    }
    return recs, summary


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--requests", type=int, default=128)
    ap.add_argument("--rate", type=float, default=4.0)
    ap.add_argument("--budget-gib", type=float, default=8.0)
    ap.add_argument("--inflight", type=int, default=4)
    ap.add_argument("--precision", default="3xtf32", choices=sorted(PRECISIONS))
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    wls = [Workload(p) for p in request_steps()]
    _, summary = run_stream(wls, a.requests, a.rate, int(a.budget_gib * (1 << 30)), a.inflight,
                            a.precision, a.seed)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
