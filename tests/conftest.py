import glob
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_steps():
    return sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.t3c")))


def captured_steps(max_bytes=400 << 20):
    """Step files captured at build time (oracle/_ref/captures), small ones."""
    out = []
    for p in sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "captures", "*", "step_*.t3c"))):
        if os.path.getsize(p) <= max_bytes:
            out.append(p)
    return out


def pupdate_captures(kind="pupdate"):
    """Renormalised-operator update captures with their compiled schedules:
    kind "pupdate" (physical) or "bupdate" (branching)."""
    out = []
    for p in sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "captures", "pupdate_*",
                                           f"{kind}_*.t3c"))):
        if os.path.exists(p.replace(".t3c", ".sched")):
            out.append(p)
    return out
