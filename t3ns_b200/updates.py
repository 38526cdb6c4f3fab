"""ctypes bindings of the engine's renormalised-operator update entry points
(``t3ns_pupdate_host``, ``t3ns_bupdate_host``) over compiled schedules in
the step-file record layout ("pu.*" / "bu.*" records, as the drop-in's
``t3ns_dropin_pupdate_write`` / ``t3ns_dropin_bupdate_write`` write them),
and the algorithmic FLOPs of a schedule."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native


class PupdateDesc(C.Structure):
    _fields_ = [("is_left", C.c_int), ("nunits", C.c_int), ("unit_ptr", C.c_void_p),
                ("nentries", C.c_int), ("dims", C.c_void_p), ("t_off", C.c_void_p),
                ("ta_off", C.c_void_p), ("pref", C.c_void_p), ("op_ptr", C.c_void_p),
                ("old_off", C.c_void_p), ("new_off", C.c_void_p), ("t_elems", C.c_int64),
                ("old_elems", C.c_int64), ("new_elems", C.c_int64)]


class BupdateDesc(C.Structure):
    _fields_ = [("ax", C.c_int * 3), ("nunits", C.c_int), ("unit_ptr", C.c_void_p),
                ("nentries", C.c_int), ("dims", C.c_void_p), ("t_off", C.c_void_p),
                ("ta_off", C.c_void_p), ("pref", C.c_void_p), ("op_ptr", C.c_void_p),
                ("o1_off", C.c_void_p), ("o2_off", C.c_void_p), ("new_off", C.c_void_p),
                ("t_elems", C.c_int64), ("o1_elems", C.c_int64), ("o2_elems", C.c_int64),
                ("new_elems", C.c_int64)]


def pupdate_host(sch: dict, T: np.ndarray, old: np.ndarray) -> np.ndarray:
    """Physical update: the updated set's elements (before zero-block
    removal) in the schedule's layout."""
    lib = native.load()
    lib.t3ns_pupdate_host.argtypes = [C.POINTER(PupdateDesc), C.c_void_p, C.c_void_p, C.c_void_p]
    keep = {k: np.ascontiguousarray(sch[k]) for k in sch}
    d = PupdateDesc()
    d.is_left = int(sch["pu.is_left"][0])
    d.nunits = len(keep["pu.unit_ptr"]) - 1
    d.unit_ptr = keep["pu.unit_ptr"].ctypes.data
    d.nentries = len(keep["pu.pref"])
    for f in ("dims", "t_off", "ta_off", "pref", "op_ptr", "old_off", "new_off"):
        setattr(d, f, keep["pu." + f].ctypes.data)
    T = np.ascontiguousarray(T)
    old = np.ascontiguousarray(old)
    d.t_elems, d.old_elems = T.size, old.size
    d.new_elems = int(keep["pu.new_base"][-1])
    new = np.empty(max(d.new_elems, 1))
    native.check(lib.t3ns_pupdate_host(C.byref(d), T.ctypes.data, old.ctypes.data,
                                       new.ctypes.data), "pupdate_host")
    return new[:d.new_elems]


def bupdate_host(sch: dict, T: np.ndarray, o1: np.ndarray, o2: np.ndarray) -> np.ndarray:
    """Branching update: the unique operators' elements in the schedule's
    layout."""
    lib = native.load()
    lib.t3ns_bupdate_host.argtypes = [C.POINTER(BupdateDesc), C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
    keep = {k: np.ascontiguousarray(sch[k]) for k in sch}
    d = BupdateDesc()
    for i in range(3):
        d.ax[i] = int(keep["bu.ax"][i])
    d.nunits = len(keep["bu.unit_ptr"]) - 1
    d.unit_ptr = keep["bu.unit_ptr"].ctypes.data
    d.nentries = len(keep["bu.pref"])
    for f in ("dims", "t_off", "ta_off", "pref", "op_ptr", "o1_off", "o2_off", "new_off"):
        setattr(d, f, keep["bu." + f].ctypes.data)
    T, o1, o2 = (np.ascontiguousarray(a) for a in (T, o1, o2))
    d.t_elems, d.o1_elems, d.o2_elems = T.size, o1.size, o2.size
    d.new_elems = int(keep["bu.unique_base"][-1])
    new = np.empty(max(d.new_elems, 1))
    native.check(lib.t3ns_bupdate_host(C.byref(d), T.ctypes.data, o1.ctypes.data,
                                       o2.ctypes.data, new.ctypes.data), "bupdate_host")
    return new[:d.new_elems]


def pupdate_flops(sch: dict) -> float:
    """2*M0*M1*N1 + 2*N0*M0*N1 per (entry, operator) term."""
    dims = sch["pu.dims"].reshape(-1, 4).astype(np.float64)
    terms = np.diff(sch["pu.op_ptr"]).astype(np.float64)
    m0, m1, n0, n1 = dims.T
    return float(np.sum(terms * (2 * m0 * m1 * n1 + 2 * n0 * m0 * n1)))


def bupdate_flops(sch: dict) -> float:
    """Per (entry, instruction) term: both operator applications in the
    cheaper order, then the contraction with the bra block."""
    a, b, g = (int(v) for v in sch["bu.ax"])
    dims = sch["bu.dims"].reshape(-1, 6).astype(np.float64)
    terms = np.diff(sch["bu.op_ptr"]).astype(np.float64)
    kd, bd = dims[:, :3], dims[:, 3:]
    a_first = kd[:, b] * bd[:, a] * (kd[:, a] + bd[:, b])
    b_first = kd[:, a] * bd[:, b] * (kd[:, b] + bd[:, a])
    apply_ops = 2 * kd[:, g] * np.minimum(a_first, b_first)
    contract = 2 * bd[:, g] * kd[:, g] * bd[:, a] * bd[:, b]
    return float(np.sum(terms * (apply_ops + contract)))
