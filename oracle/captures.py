"""Captured step files of the reference sweep (test infrastructure).

``ensure_small()`` runs the reference sweep (oracle/_ref/t3ns_run_ref, built
by oracle/Makefile) in capture mode for the small cases the GPU parity tests
use: the Hubbard config (L=10, D=128, all steps of one sweep) and the
12-orbital synthetic QC Hamiltonian (D=64).  ``ensure_d512()`` captures
steps 4-6 of the 24-orbital synthetic QC Hamiltonian at D=512 (about ten
minutes on 8 cores: the initial renormalised operators dominate) and writes
the structure-only benchmark workloads of steps 5 and 6.  Outputs go to
oracle/_ref/ (git-ignored).

``ensure_d1024_s3()`` captures the three-site D=1024 microbenchmark steps
with the reference on the CPU (hours on 8 cores); ``d1024_s3_on_gpu()``
builds the same steps' structure with the drop-in driver on a GPU machine
(``python -m oracle.captures d1024-gpu``, minutes).

``trim(path)`` rewrites a captured step file keeping only the operator
blocks that the step's schedule references (every other block is marked
empty, its elements dropped).  The matvec, its diagonal and the reference's
own replay are unchanged by this: an operator block is only ever read
through a schedule entry, and an entry whose blocks are all present keeps
them all.  It shrinks D=512 step files several-fold so they travel.
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from t3ns_b200.stepfile import read_step, write_step  # noqa: E402


def referenced_blocks(s):
    """Per operator set: boolean mask over (op, block) of referenced blocks,
    plus the per-op block counts and offsets into the flat beginblock array."""
    isd = int(s["isdmrg"][0])
    nops = 2 if isd else 3
    cp = s["sr.combo_ptr"]
    npairs = len(s["sr.pair_old"])
    sb = s["sr.combo_sbops"].reshape(-1, 3)
    mpo = s["sr.combo_mpo"]
    beg = s["iset.MPOc_beg"]
    ins = s["iset.instr"].reshape(-1, 3)
    sets = []
    for i in range(nops):
        hss = s[f"ops{i}.hss_of_ops"]
        bbh = s[f"ops{i}.begin_blocks_of_hss"]
        nbl = (bbh[hss + 1] - bbh[hss]).astype(np.int64)
        bstart = np.concatenate([[0], np.cumsum(nbl + 1)[:-1]])
        sets.append((nbl, bstart, s[f"ops{i}.beginblock"]))
    # expand combos x instructions
    ncombo = len(mpo)
    cnt = beg[mpo + 1] - beg[mpo]
    cidx = np.repeat(np.arange(ncombo), cnt)
    first = np.repeat(beg[mpo], cnt)
    within = np.arange(len(cidx)) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    k = first + within
    present = np.ones(len(k), bool)
    loc = []
    for i in range(nops):
        nbl, bstart, bb = sets[i]
        op = ins[k, i]
        b = sb[cidx, i]
        pos = bstart[op] + b
        present &= bb[pos] != bb[pos + 1]
        loc.append(pos)
    masks = []
    for i in range(nops):
        nbl, bstart, bb = sets[i]
        m = np.zeros(len(bb), bool)
        m[loc[i][present]] = True
        masks.append(m)
    return masks, sets


def trim(path, out=None):
    s = read_step(path)
    masks, sets = referenced_blocks(s)
    for i, (m, (nbl, bstart, bb)) in enumerate(zip(masks, sets)):
        tel = s[f"ops{i}.tel"]
        nbb = np.empty_like(bb)
        keep = []
        telpos = 0
        newpos = 0
        for o in range(len(nbl)):
            b0 = int(bstart[o])
            n = int(nbl[o])
            seg = bb[b0:b0 + n + 1]
            sizes = np.diff(seg)
            km = m[b0:b0 + n]
            newsizes = np.where(km, sizes, 0)
            nbb[b0] = 0
            nbb[b0 + 1:b0 + n + 1] = np.cumsum(newsizes)
            starts = telpos + seg[:-1]
            for st, sz in zip(starts[km], sizes[km]):
                keep.append(tel[st:st + sz])
            telpos += int(seg[-1])
            newpos += int(newsizes.sum())
        s[f"ops{i}.beginblock"] = nbb.astype(np.int32)
        s[f"ops{i}.tel"] = np.concatenate(keep) if keep else np.zeros(0)
    write_step(out or path, s)


def structure_only(path, out, compress=False):
    """Writes the step's structure without operator values or vectors: each
    ops{i}.tel record becomes ops{i}.tel_len, and the loaders fill the
    operator elements from a fixed seed (the matvec's cost and schedule depend
    only on the structure).  Used for benchmark workloads too large to ship
    with their values; compress: arrays above 1 MiB zlib-compressed (Python
    readers only)."""
    s = read_step(path)
    rec = {}
    for k, v in s.items():
        if k.startswith(("x", "y", "diag", "eig.")):
            continue
        if k.endswith(".tel"):
            rec[k + "_len"] = np.array([v.size], np.int64)
            continue
        rec[k] = v
    write_step(out, rec, compress_above=(1 << 20) if compress else None)


def structure_from_capture(t3c, sched, out, compress=True):
    """Joins a structure capture (t3ns_run --capture-structure: the step's
    structure with ops{i}.tel_len) and its compiled schedule (the .sched
    file, records my.*) into one structure-only step file with the
    schedule under the reference's names (sr.*)."""
    rec = dict(read_step(t3c))
    for k, v in read_step(sched).items():
        if k.startswith("my.") and k != "my.nr_qnB":
            rec["sr." + k[3:]] = v
    write_step(out, rec, compress_above=(1 << 20) if compress else None)


HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF = os.path.join(HERE, "_ref")
RUN = os.path.join(REF, "t3ns_run_ref")
NETS = os.path.join(ROOT, "tests", "golden", "networks")


def _fcidump(n):
    from t3ns_b200.workloads import synthetic_qc_fcidump
    os.makedirs(os.path.join(REF, "fcidump"), exist_ok=True)
    return synthetic_qc_fcidump(os.path.join(REF, "fcidump", f"syn{n}.FCIDUMP"), n, n, 0, 72)


def _capture(outdir, args, extra, threads, steps=True):
    import subprocess
    os.makedirs(outdir, exist_ok=True)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
    cap = ["--capture", outdir] if steps else []
    with open(os.path.join(outdir, "run.log"), "w") as log:
        subprocess.run([RUN, *args, "--init", "c", *cap, *extra], check=True,
                       env=env, stdout=log, stderr=subprocess.STDOUT)


def ensure_small(threads=None):
    threads = threads or os.cpu_count() or 1
    hub = os.path.join(REF, "captures", "hub10_D128")
    if not os.path.exists(os.path.join(hub, "step_013.t3c")):
        _capture(hub, ["--net", os.path.join(NETS, "t3ns_10.netw"), "--inter",
                       "NN_HUBBARD ( t = 1 U = 4 )", "--symm", "Z2,U1,SU2", "--ts", "0,10,0",
                       "--regime", "128,128,0,2,1e-5,100,6,1e-8,0"],
                 ["--capture-limit", "14", "--capture-stop"], threads)
    qc = os.path.join(REF, "captures", "qc12_D64")
    if not os.path.exists(os.path.join(qc, "step_017.t3c")):
        _capture(qc, ["--net", os.path.join(NETS, "t3ns_12.netw"), "--inter", _fcidump(12),
                      "--symm", "Z2,U1,SU2", "--ts", "0,12,0",
                      "--regime", "64,64,0,2,1e-5,100,2,1e-8,0"],
                 ["--capture-limit", "18", "--capture-stop"], threads)


def ensure_updates(threads=None):
    """Physical-update captures (inputs, the drop-in's compiled schedule,
    the reference output) over one sweep of the Hubbard and QC12 cases."""
    threads = threads or os.cpu_count() or 1
    lib = os.path.join(ROOT, "t3ns_b200", "_lib", "libt3ns_dropin.so")
    for name, args in [
        ("pupdate_hub10", ["--net", os.path.join(NETS, "t3ns_10.netw"), "--inter",
                           "NN_HUBBARD ( t = 1 U = 4 )", "--symm", "Z2,U1,SU2", "--ts", "0,10,0",
                           "--regime", "128,128,0,2,1e-5,100,1,1e-8,0"]),
        ("pupdate_qc12", ["--net", os.path.join(NETS, "t3ns_12.netw"), "--inter", _fcidump(12),
                          "--symm", "Z2,U1,SU2", "--ts", "0,12,0",
                          "--regime", "64,64,0,2,1e-5,100,1,1e-8,0"])]:
        d = os.path.join(REF, "captures", name)
        if os.path.exists(os.path.join(d, "run.log")):
            continue
        _capture(d, args, ["--capture-pupdate", d, "--capture-pupdate-limit", "60",
                           "--schedule-lib", lib], threads, steps=False)


def ensure_dense(threads=None):
    """Dense-factorisation captures: the LAPACKE_dgesdd / dgeqrf / dorgqr
    calls of the site-tensor decomposition with the reference LAPACK's
    outputs, over one sweep of the Hubbard and QC12 cases (the first calls
    of each run; the calls come from OpenMP threads, so their numbering is
    not deterministic)."""
    threads = threads or os.cpu_count() or 1
    for name, args in [
        ("dense_hub10", ["--net", os.path.join(NETS, "t3ns_10.netw"), "--inter",
                         "NN_HUBBARD ( t = 1 U = 4 )", "--symm", "Z2,U1,SU2", "--ts", "0,10,0",
                         "--regime", "128,128,0,2,1e-5,100,1,1e-8,0"]),
        ("dense_qc12", ["--net", os.path.join(NETS, "t3ns_12.netw"), "--inter", _fcidump(12),
                        "--symm", "Z2,U1,SU2", "--ts", "0,12,0",
                        "--regime", "64,64,0,2,1e-5,100,1,1e-8,0"])]:
        d = os.path.join(REF, "captures", name)
        if os.path.exists(os.path.join(d, "run.log")):
            continue
        _capture(d, args, ["--capture-dense", d, "--capture-dense-limit", "80"], threads,
                 steps=False)


def ensure_d512(threads=None):
    threads = threads or os.cpu_count() or 1
    d = os.path.join(REF, "captures", "qc24_D512")
    if not os.path.exists(os.path.join(d, "step_006.t3c")):
        _capture(d, ["--net", os.path.join(NETS, "t3ns_24.netw"), "--inter", _fcidump(24),
                     "--symm", "Z2,U1,SU2", "--ts", "0,24,0",
                     "--regime", "512,512,0,2,1e-5,100,1,1e-8,0"],
                 ["--capture-min", "60000", "--capture-max", "3000000", "--capture-limit", "3",
                  "--capture-stop", "--capture-noeig", "--capture-nvec", "2"], threads)
    wl = os.path.join(REF, "workloads")
    os.makedirs(wl, exist_ok=True)
    for step in ("005", "006"):
        out = os.path.join(wl, f"qc24_D512_step{step}.t3c")
        src = os.path.join(d, f"step_{step}.t3c")
        if not os.path.exists(out) and os.path.exists(src):
            structure_only(src, out)


def ensure_d1024_s3(threads=None):
    """The three-site microbenchmark steps: the 24-orbital synthetic QC
    Hamiltonian at D=1024 with SITE_SIZE 3 (branching site plus two physical
    sites, reference src/network.c:605-616), the first three steps of the
    sweep whose site tensor has 4e6 to 1.8e7 elements (one reference matvec
    each, to build the replay schedule; no Davidson).  The full captures
    (several GB) stay in oracle/_ref/captures/qc24_D1024_s3; the benchmark
    reads their compressed structure-only copies in oracle/_ref/workloads.
    About an hour on 8 cores: the initial renormalised operators and one
    reference matvec per step before the last capture dominate."""
    threads = threads or os.cpu_count() or 1
    d = os.path.join(REF, "captures", "qc24_D1024_s3")
    if not any(f.startswith("step_") for f in (os.listdir(d) if os.path.isdir(d) else [])):
        _capture(d, ["--net", os.path.join(NETS, "t3ns_24.netw"), "--inter", _fcidump(24),
                     "--symm", "Z2,U1,SU2", "--ts", "0,24,0",
                     "--regime", "1024,1024,0,3,1e-5,100,1,1e-8,0"],
                 ["--capture-min", "4000000", "--capture-max", "18000000",
                  "--capture-limit", "3", "--capture-stop", "--capture-noeig",
                  "--capture-nvec", "1"], threads)
    wl = os.path.join(REF, "workloads")
    os.makedirs(wl, exist_ok=True)
    for f in sorted(os.listdir(d)):
        if f.startswith("step_") and f.endswith(".t3c"):
            out = os.path.join(wl, "qc24_D1024_s3_" + f.replace("_", ""))
            if not os.path.exists(out):
                structure_only(os.path.join(d, f), out, compress=True)


def d1024_s3_on_gpu(outdir, threads=16, timeout=1700, limit=2):
    """The same three-site D=1024 steps, built on a GPU machine: the drop-in
    driver (oracle/_ref/t3ns_run_dropin) builds the initial operators and
    runs the updates and decompositions on the GPU (about five minutes for
    the initial operators, eleven to reach the second step: steps 3 and 5,
    2,661 and 3,420 blocks) and, with --capture-structure, writes each
    selected step's structure and the product's schedule for it without
    solving it; the pairs are joined into compressed structure-only
    workloads in outdir (about 1 and 2.3 GB: their schedules hold tens of
    millions of terms, too large to travel, so they are built where they
    are used).  Returns the workload paths."""
    import glob
    import subprocess
    import tempfile
    exe = os.path.join(REF, "t3ns_run_dropin")
    tmp = tempfile.mkdtemp(prefix="t3ns_d1024_")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1",
               T3NS_B200_AUTOTUNE="0")
    with open(os.path.join(tmp, "run.log"), "w") as log:
        subprocess.run([exe, "--net", os.path.join(NETS, "t3ns_24.netw"), "--inter", _fcidump(24),
                        "--symm", "Z2,U1,SU2", "--ts", "0,24,0",
                        "--regime", "1024,1024,0,3,1e-5,100,1,1e-8,0", "--init", "c",
                        "--capture-structure", tmp, "--capture-min", "4000000",
                        "--capture-max", "18000000", "--capture-limit", str(limit),
                        "--capture-stop"],
                       env=env, stdout=log, stderr=subprocess.STDOUT, timeout=timeout)
    os.makedirs(outdir, exist_ok=True)
    out = []
    for t in sorted(glob.glob(os.path.join(tmp, "step_*.t3c"))):
        sched = t.replace(".t3c", ".sched")
        if os.path.exists(sched):
            o = os.path.join(outdir, "qc24_D1024_s3_" + os.path.basename(t).replace("_", ""))
            structure_from_capture(t, sched, o, compress=True)
            out.append(o)
    return out


if __name__ == "__main__":
    if sys.argv[1] == "d1024":
        ensure_d1024_s3()
        sys.exit(0)
    if sys.argv[1] == "d1024-gpu":
        print(d1024_s3_on_gpu(os.path.join(REF, "workloads")))
        sys.exit(0)
    if sys.argv[1] == "small":
        ensure_small()
        sys.exit(0)
    if sys.argv[1] == "updates":
        ensure_updates()
        sys.exit(0)
    if sys.argv[1] == "dense":
        ensure_dense()
        sys.exit(0)
    if sys.argv[1] == "d512":
        ensure_d512()
        sys.exit(0)
    if sys.argv[1] in ("structure", "structure-z"):
        structure_only(sys.argv[2], sys.argv[3], compress=sys.argv[1] == "structure-z")
        print(sys.argv[3], os.path.getsize(sys.argv[3]) >> 20, "MiB")
    else:
        for p in sys.argv[1:]:
            before = os.path.getsize(p)
            trim(p)
            print(p, before >> 20, "MiB ->", os.path.getsize(p) >> 20, "MiB")
