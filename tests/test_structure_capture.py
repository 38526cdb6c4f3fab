"""Structure-only step capture (the benchmark workloads' recipe, CPU).

The sweep driver's --capture-structure mode writes a step's structure (site
tensor blocks, symsecs, the operator sets' block layout with element counts
instead of values, the merge instruction set) and the product's schedule for
it; oracle/captures.structure_from_capture joins the two into a
structure-only step file.  On the first steps of the 12-orbital QC sweep
(D=64) the joined file must equal the reference's full capture of the same
steps in every structural record: the same symmetry sectors, the same
instructions per MPO combination, the same schedule pairs with bit-identical
prefactors (orders within a block may differ; they change no sum), and the
same operator element counts.  Test infrastructure only (oracle/)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT
from t3ns_b200.stepfile import read_step

sys.path.insert(0, os.path.join(ROOT, "oracle"))

REF = os.path.join(ROOT, "oracle", "_ref")
RUN_REF = os.path.join(REF, "t3ns_run_ref")
DROPIN = os.path.join(ROOT, "t3ns_b200", "_lib", "libt3ns_dropin.so")
FULL = os.path.join(REF, "captures", "qc12_D64")


def _groups(s):
    beg = s["iset.MPOc_beg"]
    ins = s["iset.instr"].reshape(-1, 3)
    pr = s["iset.pref"]
    return ([sorted((tuple(ins[k]), pr[k]) for k in range(beg[m], beg[m + 1]))
             for m in range(len(beg) - 1)], list(s["iset.MPOc"]))


def _schedule(s):
    pp, po, pord = s["sr.pair_ptr"], s["sr.pair_old"], s["sr.pair_order"]
    cp, sb = s["sr.combo_ptr"], s["sr.combo_sbops"].reshape(-1, 3)
    mpo, pref = s["sr.combo_mpo"], s["sr.combo_pref"]
    out = []
    for n in range(len(pp) - 1):
        out.append({(int(po[p]), int(pord[p]),
                     tuple(sorted((tuple(sb[c]), int(mpo[c]), float(pref[c]))
                                  for c in range(cp[p], cp[p + 1]))))
                    for p in range(pp[n], pp[n + 1])})
    return out


def test_structure_capture_matches_full_capture(tmp_path):
    for p in (RUN_REF, DROPIN, os.path.join(FULL, "step_001.t3c")):
        if not os.path.exists(p):
            pytest.skip(f"not built: {p}")
    import captures
    env = dict(os.environ, OMP_NUM_THREADS="2", OPENBLAS_NUM_THREADS="1")
    fcid = captures._fcidump(12)
    subprocess.run([RUN_REF, "--net", os.path.join(ROOT, "tests", "golden", "networks",
                                                   "t3ns_12.netw"),
                    "--inter", fcid, "--symm", "Z2,U1,SU2", "--ts", "0,12,0",
                    "--regime", "64,64,0,2,1e-5,100,1,1e-8,0", "--init", "c",
                    "--capture-structure", str(tmp_path), "--capture-limit", "2",
                    "--capture-stop", "--schedule-lib", DROPIN],
                   check=True, env=env, capture_output=True, timeout=600)
    # step 0 is captured before any Davidson solve, so its structure is the
    # full capture's; later steps follow the (unsolved) guess's truncation
    out = str(tmp_path / "joined.t3c")
    captures.structure_from_capture(str(tmp_path / "step_000.t3c"),
                                    str(tmp_path / "step_000.sched"), out)
    a = read_step(out)
    b = read_step(os.path.join(FULL, "step_000.t3c"))
    for k in ("nrblocks", "beginblock", "qnumbers", "sites", "posB", "rOperators_on_site",
              "isdmrg", "sr.dims", "sr.pair_ptr"):
        assert np.array_equal(a[k], b[k]), k
    nsym = int(b["nrSyms"][0])
    for k in b:
        if k.endswith(".irreps"):
            assert np.array_equal(a[k].reshape(-1, 5)[:, :nsym], b[k].reshape(-1, 5)[:, :nsym]), k
    for i in range(3):
        assert a[f"ops{i}.tel"].size == b[f"ops{i}.tel"].size
        assert np.array_equal(a[f"ops{i}.beginblock"], b[f"ops{i}.beginblock"])
    assert _groups(a) == _groups(b)
    assert _schedule(a) == _schedule(b)
