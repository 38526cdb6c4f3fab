"""The C-ABI libraries load without a GPU and export every entry point the
headers in include/ declare."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(t3ns_\w+|[a-z_A-Z]\w*)\s*\(", txt, flags=re.M)
    return sorted({n for n in names if not n.startswith("T3NS")})


def test_engine_exports_all_declared_symbols():
    p = os.path.join(ROOT, "t3ns_b200", "_lib", "libt3ns_b200.so")
    if not os.path.exists(p):
        pytest.fail("engine library not built")
    lib = C.CDLL(p)
    names = declared("t3ns_b200.h")
    assert "t3ns_heff_create" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    lib.t3ns_version.restype = C.c_char_p
    assert b"sm_100a" in lib.t3ns_version()


def test_dropin_exports_all_declared_symbols():
    p = os.path.join(ROOT, "t3ns_b200", "_lib", "libt3ns_dropin.so")
    if not os.path.exists(p):
        pytest.skip("drop-in not built (needs the reference headers)")
    out = subprocess.run(["nm", "-D", "--defined-only", p], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    names = declared("t3ns_dropin.h")
    assert {"init_Heffdata", "matvecT3NS", "make_diagonal", "destroy_Heffdata", "davidson",
            "sparse_eigensolve", "davidson_diagonal_preconditioner"} <= set(names)
    missing = [n for n in names if n not in exported]
    assert not missing, missing
