"""Step-file maintenance for the captured workloads (test infrastructure).

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


def structure_only(path, out):
    """Writes the step's structure without operator values or vectors: each
    ops{i}.tel record becomes ops{i}.tel_len, and the loaders fill the
    operator elements from a fixed seed (the matvec's cost and schedule depend
    only on the structure).  Used for benchmark workloads too large to ship
    with their values."""
    s = read_step(path)
    rec = {}
    for k, v in s.items():
        if k.startswith(("x", "y", "diag", "eig.")):
            continue
        if k.endswith(".tel"):
            rec[k + "_len"] = np.array([v.size], np.int64)
            continue
        rec[k] = v
    write_step(out, rec)


if __name__ == "__main__":
    if sys.argv[1] == "structure":
        structure_only(sys.argv[2], sys.argv[3])
        print(sys.argv[3], os.path.getsize(sys.argv[3]) >> 20, "MiB")
    else:
        for p in sys.argv[1:]:
            before = os.path.getsize(p)
            trim(p)
            print(p, before >> 20, "MiB ->", os.path.getsize(p) >> 20, "MiB")
