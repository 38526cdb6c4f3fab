"""Build of the native libraries (nvcc for sm_100a, gcc for the drop-in shim).

Outputs (in-tree, git-ignored, shipped with the repository snapshot):

* ``t3ns_b200/_lib/libt3ns_b200.so``: the engine (include/t3ns_b200.h);
* ``t3ns_b200/_lib/libt3ns_dropin.so``: the reference-ABI drop-in
  (include/t3ns_dropin.h) on top of the engine; built only when the
  reference headers are available (they define the struct layouts the
  drop-in must match).
"""
from __future__ import annotations

import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "t3ns_b200")
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

ENGINE_SOURCES = ["capi.cu", "heff.cu", "davidson.cu", "precond_noalloc.cu", "rops_update.cu",
                  "dense.cu", "server.cu"]


def _run(cmd, cwd=None):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=cwd)


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build_engine(force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, "libt3ns_b200.so")
    srcs = [os.path.join(CSRC, s) for s in ENGINE_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(INCLUDE, "t3ns_b200.h"))
    if force or _stale(out, deps):
        from concurrent.futures import ThreadPoolExecutor
        objs = [os.path.join(LIBDIR, os.path.basename(s) + ".o") for s in srcs]
        headers = [d for d in deps if d not in srcs]
        # an object is rebuilt when its source or any header is newer
        cmds = [[NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                 "-Xptxas", "-warn-spills", "-I", INCLUDE, "-I", CSRC, "-c", s, "-o", o]
                for s, o in zip(srcs, objs) if force or _stale(o, [s, *headers])]
        # the translation units compile independently (heff.cu dominates)
        with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
            list(ex.map(_run, cmds))
        _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-lcudart_static", "-lrt", "-ldl",
              "-lpthread"])
    return out


SHIM_INCLUDE = os.path.join(ROOT, "oracle", "shim")
DROPIN_SOURCES = ["heff_dropin.c", "pupdate_dropin.c", "bupdate_dropin.c", "sum_dropin.c",
                  "dense_dropin.c"]


def reference_checkout(reference: str | None = None) -> str:
    """The reference T3NS checkout whose headers the drop-in is compiled
    against: the argument, else $T3NS_REFERENCE.  Raises when neither names
    a checkout."""
    ref = reference or os.environ.get("T3NS_REFERENCE")
    if not ref or not os.path.isdir(os.path.join(ref, "include")):
        raise RuntimeError("the reference checkout is not known: set T3NS_REFERENCE to the "
                           "T3NS source tree (its include/ defines the drop-in's struct layouts)")
    return ref


def build_dropin(force: bool = False, reference: str | None = None):
    """libt3ns_dropin.so: the reference entry points on top of the engine.
    Compiled against the reference headers, whose struct layouts it must
    match (reference_checkout())."""
    ref_include = os.path.join(reference_checkout(reference), "include")
    engine = build_engine()
    out = os.path.join(LIBDIR, "libt3ns_dropin.so")
    srcs = [os.path.join(CSRC, "dropin", f) for f in DROPIN_SOURCES]
    hdrs = [os.path.join(CSRC, "dropin", f) for f in os.listdir(os.path.join(CSRC, "dropin"))
            if f.endswith(".h")]
    if force or _stale(out, srcs + hdrs + [engine, os.path.join(INCLUDE, "t3ns_b200.h")]):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu11", "-w", "-DMAX_SYMMETRIES=5",
              "-DNDEBUG", "-I", ref_include, "-I", SHIM_INCLUDE, "-I", INCLUDE,
              "-o", out, *srcs, "-L", LIBDIR, "-l:libt3ns_b200.so", "-Wl,-rpath,$ORIGIN",
              "-lpthread"])
    return out


def build_all(force: bool = False, reference: str | None = None):
    """The engine, and the drop-in when the reference checkout is known
    (argument or $T3NS_REFERENCE); without it the drop-in is not rebuilt
    and a message says so."""
    out = {"engine": build_engine(force), "dropin": None}
    try:
        ref = reference_checkout(reference)
    except RuntimeError as e:
        print(f"drop-in not rebuilt: {e}", flush=True)
        return out
    out["dropin"] = build_dropin(force, ref)
    return out


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv))
