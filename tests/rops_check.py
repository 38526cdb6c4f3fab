"""Helpers to replay captured renormalised-operator updates: build the
engine descriptor from a compiled schedule ("pu.*" records for the physical
update, "bu.*" for the branching one), emulate it on the CPU (numpy) or run
it through the C ABI, sum unique operators as the reference does, apply the
reference's zero-block removal (kick_zero_blocks, src/sparseblocks.c:73-107)
and compare with the reference's output captured in the same file ("ops1.*"
records for the physical update, "ops2.*" for the branching one)."""
import numpy as np

from t3ns_b200 import updates


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
    return updates.pupdate_host(sch, rec["T.tel"], rec["ops0.tel"])


def kick_compare(rec, idx, pre):
    """Apply zero-block removal (a block whose elements are all below 1e-20
    in magnitude is dropped) to the operators `pre` -- a list of (begin array
    before removal, elements) per operator -- and compare with the
    reference's operator set `idx` of the capture: same surviving blocks,
    elements compared relative to the largest reference element.  Returns
    that largest relative difference."""
    begins, ref = ops_structure(rec, idx)
    assert len(begins) == len(pre)
    scale = max(np.abs(ref).max() if ref.size else 0.0, 1e-300)
    worst, roff = 0.0, 0
    for k, bb in enumerate(begins):
        nb = len(bb) - 1
        pbb, seg = pre[k]
        assert len(pbb) == nb + 1, (k, len(pbb), nb)
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


def _nblocks(rec, idx, hss):
    bbh = rec[f"ops{idx}.begin_blocks_of_hss"]
    return int(bbh[hss + 1] - bbh[hss])


def kick_and_compare(rec, sch, new):
    """kick_compare for a physical update: `new` is the updated set's
    concatenated elements in the schedule's layout."""
    pre = sch["pu.new_beginblock"].astype(np.int64)
    base = sch["pu.new_base"].astype(np.int64)
    out, poff = [], 0
    for k, h in enumerate(rec["ops1.hss_of_ops"]):
        n = _nblocks(rec, 1, int(h))
        out.append((pre[poff:poff + n + 1], new[int(base[k]):int(base[k + 1])]))
        poff += n + 1
    return kick_compare(rec, 1, out)


def _block3(arr, off, d):
    """Column-major block of dims d as an array indexed [i0, i1, i2]."""
    n = d[0] * d[1] * d[2]
    return arr[off:off + n].reshape(d[2], d[1], d[0]).transpose(2, 1, 0)


def _block2(arr, off, r, c):
    return arr[off:off + r * c].reshape(c, r).T


def emulate_bupdate(rec, sch):
    """numpy replay of a compiled branching-update schedule: the unique
    operators' concatenated elements."""
    T, O1, O2 = rec["T.tel"], rec["ops0.tel"], rec["ops1.tel"]
    a, b, g = (int(v) for v in sch["bu.ax"])
    new = np.zeros(int(sch["bu.unique_base"][-1]))
    dims = sch["bu.dims"].reshape(-1, 6)
    bra, ket = "abc", "xyz"
    spec = (f"{bra},{ket},{bra[a]}{ket[a]},{bra[b]}{ket[b]}->{bra[g]}{ket[g]}")
    for e in range(len(sch["bu.pref"])):
        kd, bd = [int(v) for v in dims[e, :3]], [int(v) for v in dims[e, 3:]]
        Tk = _block3(T, int(sch["bu.t_off"][e]), kd)
        Tb = _block3(T, int(sch["bu.ta_off"][e]), bd)
        for p in range(sch["bu.op_ptr"][e], sch["bu.op_ptr"][e + 1]):
            A = _block2(O1, int(sch["bu.o1_off"][p]), bd[a], kd[a])
            B = _block2(O2, int(sch["bu.o2_off"][p]), bd[b], kd[b])
            U = sch["bu.pref"][e] * np.einsum(spec, Tb, Tk, A, B, optimize=True)
            n = int(sch["bu.new_off"][p])
            new[n:n + U.size] += U.T.reshape(-1)
    return new


def run_bupdate_gpu(rec, sch):
    return updates.bupdate_host(sch, rec["T.tel"], rec["ops0.tel"], rec["ops1.tel"])


def sum_unique(rec, sch, unique):
    """The reference's sum_unique_rOperators (src/rOperators_init.c:228-265)
    on the unique operators: new operator k = sum of instr.pref times the
    unique operator of every instruction that writes k.  Returns the
    (begin array, elements) of every new operator before zero-block removal;
    the block counts per MPO sector come from the captured result (ops2)."""
    ubase = sch["bu.unique_base"].astype(np.int64)
    uhss = sch["bu.unique_hss"]
    ubb = sch["bu.unique_beginblock"].astype(np.int64)
    begins, off = [], 0
    for u in range(len(uhss)):
        n = _nblocks(rec, 2, int(uhss[u]))
        begins.append(ubb[off:off + n + 1])
        off += n + 1
    hss_new = sch["bu.hss_of_new"]
    instr = sch["bu.instr"].reshape(-1, 3)
    out = []
    for k in range(len(hss_new)):
        # layout of any unique operator of the same MPO sector
        u0 = int(np.flatnonzero(uhss == hss_new[k])[0])
        acc = np.zeros(int(begins[u0][-1]))
        for i in np.flatnonzero(instr[:, 2] == k):
            u = int(sch["bu.instr_unique"][i])
            acc += sch["bu.instr_pref"][i] * unique[int(ubase[u]):int(ubase[u + 1])]
        out.append((begins[u0], acc))
    return out


def compare_summed(rec, idx, got):
    """Compares a new set after the sum and zero-block removal -- a list of
    (begin array, elements) per operator -- with the reference's operator set
    `idx` of the capture: identical surviving blocks, elements relative to
    the largest reference element.  Returns that largest relative
    difference."""
    begins, ref = ops_structure(rec, idx)
    assert len(begins) == len(got)
    scale = max(np.abs(ref).max() if ref.size else 0.0, 1e-300)
    worst, roff = 0.0, 0
    for k, bb in enumerate(begins):
        gbb, gel = got[k]
        assert np.array_equal(np.asarray(gbb, np.int64), bb), k
        rseg = ref[roff:roff + int(bb[-1])]
        roff += int(bb[-1])
        if rseg.size:
            worst = max(worst, float(np.abs(gel - rseg).max()) / scale)
    return worst
