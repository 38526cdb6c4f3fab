"""Helpers to replay captured renormalised-operator updates: build the
engine descriptor from a compiled schedule ("pu.*" records), emulate it on
the CPU (numpy) or run it through the C ABI, apply the reference's zero-block
removal (kick_zero_blocks, src/sparseblocks.c:73-107) and compare with the
reference's output captured in the same file ("ops1.*" records)."""
import ctypes as C

import numpy as np

from t3ns_b200 import native


class PupdateDesc(C.Structure):
    _fields_ = [("is_left", C.c_int), ("nunits", C.c_int), ("unit_ptr", C.c_void_p),
                ("nentries", C.c_int), ("dims", C.c_void_p), ("t_off", C.c_void_p),
                ("ta_off", C.c_void_p), ("pref", C.c_void_p), ("op_ptr", C.c_void_p),
                ("old_off", C.c_void_p), ("new_off", C.c_void_p), ("t_elems", C.c_int64),
                ("old_elems", C.c_int64), ("new_elems", C.c_int64)]


def ops_structure(rec, i):
    """(begin arrays per operator, concatenated elements) of operator set i."""
    nrops = int(rec[f"ops{i}.nrops"][0])
    hss = rec[f"ops{i}.hss_of_ops"]
    bbh = rec[f"ops{i}.begin_blocks_of_hss"]
    bb = rec[f"ops{i}.beginblock"]
    out, off = [], 0
    for k in range(nrops):
        n = int(bbh[hss[k] + 1] - bbh[hss[k]])
        out.append(bb[off:off + n + 1].astype(np.int64))
        off += n + 1
    return out, rec[f"ops{i}.tel"]


def emulate_pupdate(rec, sch):
    """numpy replay of the compiled schedule: the updated elements before
    zero-block removal, in the updated set's concatenation."""
    T = rec["T.tel"]
    old = rec["ops0.tel"]
    new = np.zeros(int(sch["pu.new_base"][-1]))
    il = int(sch["pu.is_left"][0])
    dims = sch["pu.dims"].reshape(-1, 4)
    for e in range(len(sch["pu.pref"])):
        M0, M1, N0, N1 = (int(v) for v in dims[e])
        t0, ta0 = int(sch["pu.t_off"][e]), int(sch["pu.ta_off"][e])
        if il:
            Tb = T[t0:t0 + M1 * N1].reshape(N1, M1).T          # M1 x N1
            Ta = T[ta0:ta0 + M0 * N0].reshape(N0, M0).T.T      # (M0 x N0)^T -> N0 x M0
        else:
            Tb = T[t0:t0 + N1 * M1].reshape(M1, N1)            # (N1 x M1)^T -> M1 x N1
            Ta = T[ta0:ta0 + N0 * M0].reshape(M0, N0).T        # N0 x M0
        for p in range(sch["pu.op_ptr"][e], sch["pu.op_ptr"][e + 1]):
            o, n = int(sch["pu.old_off"][p]), int(sch["pu.new_off"][p])
            O = old[o:o + M0 * M1].reshape(M1, M0).T
            U = sch["pu.pref"][e] * (Ta @ O @ Tb)
            new[n:n + N0 * N1] += U.T.reshape(-1)
    return new


def run_pupdate_gpu(rec, sch):
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
    T = np.ascontiguousarray(rec["T.tel"])
    old = np.ascontiguousarray(rec["ops0.tel"])
    d.t_elems, d.old_elems = T.size, old.size
    d.new_elems = int(keep["pu.new_base"][-1])
    new = np.empty(max(d.new_elems, 1))
    native.check(lib.t3ns_pupdate_host(C.byref(d), T.ctypes.data, old.ctypes.data,
                                       new.ctypes.data), "pupdate_host")
    return new[:d.new_elems]


def kick_and_compare(rec, sch, new):
    """Apply zero-block removal (a block whose elements are all below 1e-20
    in magnitude is dropped) to `new` operator by operator and compare with
    the reference output: same surviving blocks, elements equal to the given
    relative tolerance.  Returns the largest element difference relative to
    the largest reference element."""
    begins, ref = ops_structure(rec, 1)
    pre = sch["pu.new_beginblock"].astype(np.int64)
    base = sch["pu.new_base"].astype(np.int64)
    scale = max(np.abs(ref).max() if ref.size else 0.0, 1e-300)
    worst, roff, poff = 0.0, 0, 0
    for k, bb in enumerate(begins):
        nb = len(bb) - 1
        pbb = pre[poff:poff + nb + 1]
        poff += nb + 1
        seg = new[int(base[k]):int(base[k + 1])]
        rseg = ref[roff:roff + int(bb[-1])]
        roff += int(bb[-1])
        for b in range(nb):
            blk = seg[pbb[b]:pbb[b + 1]]
            keep = blk.size and np.any(np.abs(blk) >= 1e-20)
            rsz = int(bb[b + 1] - bb[b])
            assert (blk.size if keep else 0) == rsz, (k, b, blk.size, rsz)
            if rsz:
                worst = max(worst, float(np.abs(blk - rseg[bb[b]:bb[b + 1]]).max()) / scale)
    return worst
