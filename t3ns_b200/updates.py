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


class SumUniqueDesc(C.Structure):
    _fields_ = [("nnew", C.c_int), ("begin_ptr", C.c_void_p), ("begin", C.c_void_p),
                ("new_base", C.c_void_p), ("instr_ptr", C.c_void_p), ("instr_src", C.c_void_p),
                ("instr_pref", C.c_void_p), ("unique_elems", C.c_int64)]


def sum_desc(unique_hss, unique_begin, unique_base, nblocks_of_hss, hss_of_new, instr_new,
             instr_unique, instr_pref):
    """Descriptor of t3ns_sum_unique_host: unique operator u has MPO sector
    unique_hss[u], block begin offsets unique_begin[u] and element base
    unique_base[u]; new operator k has sector hss_of_new[k] and takes the
    layout of the first unique operator of that sector; instruction i adds
    instr_pref[i] times unique operator instr_unique[i] into new operator
    instr_new[i] (in instruction order).  Returns (desc, arrays kept alive)."""
    nnew = len(hss_of_new)
    begins, bases, ptr = [], [0], [0]
    for k in range(nnew):
        u0 = int(np.flatnonzero(np.asarray(unique_hss) == hss_of_new[k])[0])
        bb = np.asarray(unique_begin[u0], np.int32)
        assert len(bb) == nblocks_of_hss(int(hss_of_new[k])) + 1
        begins.append(bb)
        ptr.append(ptr[-1] + len(bb))
        bases.append(bases[-1] + int(bb[-1]))
    order = np.argsort(np.asarray(instr_new), kind="stable")
    counts = np.bincount(np.asarray(instr_new), minlength=nnew)
    keep = {
        "begin_ptr": np.asarray(ptr, np.int64),
        "begin": np.concatenate(begins).astype(np.int32) if begins else np.zeros(1, np.int32),
        "new_base": np.asarray(bases, np.int64),
        "instr_ptr": np.concatenate([[0], np.cumsum(counts)]).astype(np.int32),
        "instr_src": np.asarray(unique_base, np.int64)[np.asarray(instr_unique)[order]],
        "instr_pref": np.asarray(instr_pref, np.float64)[order],
    }
    d = SumUniqueDesc()
    d.nnew = nnew
    for f in ("begin_ptr", "begin", "new_base", "instr_ptr", "instr_src", "instr_pref"):
        keep[f] = np.ascontiguousarray(keep[f])
        setattr(d, f, keep[f].ctypes.data)
    d.unique_elems = int(unique_base[-1])
    return d, keep


def _sum_outputs(keep):
    nnew = len(keep["new_base"]) - 1
    new_tel = np.empty(max(int(keep["new_base"][-1]), 1))
    new_begin = np.empty_like(keep["begin"])
    out_base = np.empty(nnew + 1, np.int64)
    return new_tel, new_begin, out_base


def _split_sum(keep, new_tel, new_begin, out_base):
    """[(begin offsets after zero-block removal, elements)] per new operator."""
    out = []
    bp = keep["begin_ptr"]
    for k in range(len(bp) - 1):
        out.append((new_begin[bp[k]:bp[k + 1]].astype(np.int64),
                    new_tel[out_base[k]:out_base[k + 1]].copy()))
    return out


def sum_unique_host(d, keep, unique: np.ndarray):
    """t3ns_sum_unique_host on the unique operators' concatenated elements."""
    lib = native.load()
    lib.t3ns_sum_unique_host.argtypes = [C.POINTER(SumUniqueDesc)] + [C.c_void_p] * 4
    unique = np.ascontiguousarray(unique, dtype=np.float64)
    new_tel, new_begin, out_base = _sum_outputs(keep)
    native.check(lib.t3ns_sum_unique_host(C.byref(d), unique.ctypes.data, new_tel.ctypes.data,
                                          new_begin.ctypes.data, out_base.ctypes.data),
                 "sum_unique_host")
    return _split_sum(keep, new_tel, new_begin, out_base)


def bupdate_sum_desc(rec: dict, sch: dict):
    """The sum descriptor of a captured branching update ("bu.*" schedule
    records; block counts per MPO sector from the captured result, ops2)."""
    uhss = sch["bu.unique_hss"]
    ubb = sch["bu.unique_beginblock"].astype(np.int64)
    bbh = rec["ops2.begin_blocks_of_hss"]

    def nbl(h):
        return int(bbh[h + 1] - bbh[h])
    ubegin, off = [], 0
    for u in range(len(uhss)):
        n = nbl(int(uhss[u]))
        ubegin.append(ubb[off:off + n + 1])
        off += n + 1
    instr = sch["bu.instr"].reshape(-1, 3)
    return sum_desc(uhss, ubegin, sch["bu.unique_base"], nbl, sch["bu.hss_of_new"], instr[:, 2],
                    sch["bu.instr_unique"], sch["bu.instr_pref"])


def bupdate_sum_host(rec: dict, sch: dict):
    """t3ns_bupdate_sum_host on a captured branching update: the new set after
    the device sum and zero-block removal, [(begin, elements)] per operator."""
    lib = native.load()
    lib.t3ns_bupdate_sum_host.argtypes = [C.POINTER(BupdateDesc), C.POINTER(SumUniqueDesc)] + \
        [C.c_void_p] * 6
    keep = {k: np.ascontiguousarray(sch[k]) for k in sch}
    d = BupdateDesc()
    for i in range(3):
        d.ax[i] = int(keep["bu.ax"][i])
    d.nunits = len(keep["bu.unit_ptr"]) - 1
    d.unit_ptr = keep["bu.unit_ptr"].ctypes.data
    d.nentries = len(keep["bu.pref"])
    for f in ("dims", "t_off", "ta_off", "pref", "op_ptr", "o1_off", "o2_off", "new_off"):
        setattr(d, f, keep["bu." + f].ctypes.data)
    T, o1, o2 = (np.ascontiguousarray(rec[k]) for k in ("T.tel", "ops0.tel", "ops1.tel"))
    d.t_elems, d.o1_elems, d.o2_elems = T.size, o1.size, o2.size
    d.new_elems = int(keep["bu.unique_base"][-1])
    sd, skeep = bupdate_sum_desc(rec, sch)
    new_tel, new_begin, out_base = _sum_outputs(skeep)
    native.check(lib.t3ns_bupdate_sum_host(C.byref(d), C.byref(sd), T.ctypes.data, o1.ctypes.data,
                                           o2.ctypes.data, new_tel.ctypes.data,
                                           new_begin.ctypes.data, out_base.ctypes.data),
                 "bupdate_sum_host")
    return _split_sum(skeep, new_tel, new_begin, out_base)
