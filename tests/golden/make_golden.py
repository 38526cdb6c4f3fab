"""Regenerates the committed golden step files under tests/golden/.

Runs the reference sweep (oracle/_ref/t3ns_run_ref, built from the reference
sources by oracle/Makefile) in capture mode and keeps a few small steps:

* ``hub10_*``: Hubbard t=1, U=4, 10 electrons on the 10-site T3NS tree,
  Z2 x U1 x SU2, D=128, SITE_SIZE 2 (the reference's CPU-runnable config);
* ``qc12_*``: the seeded synthetic 12-orbital quantum-chemistry Hamiltonian
  (t3ns_b200.workloads, seed 0), 12 electrons, S=0, D=64, SITE_SIZE 2.

Each step file holds the reference's inputs to init_Heffdata, its replay
schedule, its matvec outputs on two seeded vectors, its diagonal and its
Davidson result on that step.  Needs the reference checkout (only here).
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from t3ns_b200.workloads import synthetic_qc_fcidump  # noqa: E402

RUN = os.path.join(ROOT, "oracle", "_ref", "t3ns_run_ref")
NET = os.path.join(HERE, "networks")

CASES = {
    "hub10": dict(net="t3ns_10.netw", inter="NN_HUBBARD ( t = 1 U = 4 )", ts="0,10,0",
                  regime="128,128,0,2,1e-5,100,1,1e-8,0", keep={0: "dmrg", 1: "t3ns_a", 2: "t3ns_b"}),
    "qc12": dict(net="t3ns_12.netw", inter=None, ts="0,12,0",
                 regime="64,64,0,2,1e-5,100,1,1e-8,0", keep={0: "dmrg", 1: "t3ns_a"}),
}


def main():
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
    for name, c in CASES.items():
        with tempfile.TemporaryDirectory() as tmp:
            inter = c["inter"]
            if inter is None:
                inter = synthetic_qc_fcidump(os.path.join(tmp, "qc12.FCIDUMP"), 12, 12, 0, 72)
            cap = os.path.join(tmp, "cap")
            os.makedirs(cap)
            last = max(c["keep"])
            subprocess.run([RUN, "--net", os.path.join(NET, c["net"]), "--inter", inter,
                            "--symm", "Z2,U1,SU2", "--ts", c["ts"], "--regime", c["regime"],
                            "--init", "c", "--capture", cap, "--capture-limit", str(last + 1),
                            "--capture-stop"], check=True, env=env, stdout=subprocess.DEVNULL)
            for step, tag in c["keep"].items():
                shutil.copy(os.path.join(cap, "step_%03d.t3c" % step),
                            os.path.join(HERE, f"{name}_{tag}.t3c"))
                print("wrote", f"{name}_{tag}.t3c")


if __name__ == "__main__":
    main()
