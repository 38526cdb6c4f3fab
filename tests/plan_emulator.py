"""Host-side emulation of the matvec work plan (numpy), used to check the
plan's tiling, pair splitting, contraction sequences and operator row
offsets without a GPU.

For selected output blocks it recomputes every work unit of the block the
way the kernel organises it -- the unit's pairs, term by term, contracting
the memory axes in the pair's sequence with tiled axes restricted to the
tile's rows -- adds the units into the block (split units add partial sums)
and returns the blocks for comparison with the reference's matvec output."""
import ctypes as C
import os
import tempfile

import numpy as np

from t3ns_b200 import native
from t3ns_b200.stepfile import read_step

UNIT_FIELDS = 10   # nb, b0, bt, c0, ct, a0, at, p0, p1, split


def dump_plan(desc, config=0):
    lib = native.load()
    lib.t3ns_heff_plan_dump_config.argtypes = [C.POINTER(native.HeffDesc), C.c_int, C.c_char_p]
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "plan.t3c")
        native.check(lib.t3ns_heff_plan_dump_config(C.byref(desc.desc), config, p.encode()),
                     "plan_dump")
        return read_step(p)


def units_of(plan):
    return plan["plan.units"].reshape(-1, UNIT_FIELDS)


def emulate_blocks(s, plan, x, blocks):
    nops = 2 if int(s["isdmrg"][0]) else 3
    ops = np.concatenate([s[f"ops{i}.tel"] for i in range(nops)])
    units = units_of(plan)
    pairs = plan["plan.pairs"].reshape(-1, 4)
    edims = plan["plan.edims"].reshape(-1, 3)
    offs = plan["plan.op_off"].reshape(-1, 3)
    pref = plan["plan.pref"]
    boff = s["beginblock"].astype(np.int64)
    out = {}
    for nb in blocks:
        dn = [int(v) for v in edims[nb]]
        blk = np.zeros((dn[2], dn[1], dn[0]))
        for u in np.nonzero(units[:, 0] == nb)[0]:
            _, b0, bt, c0, ct, a0, at, p0, p1, _split = (int(v) for v in units[u])
            ext = [at, bt, ct]
            row0 = [a0, b0, c0]
            tile = np.zeros((ct, bt, at))
            for p in range(p0, p1):
                old, axes, t0, t1 = (int(v) for v in pairs[p])
                nst = (axes >> 6) & 3
                seq = [(axes >> (2 * k)) & 3 for k in range(nst)]
                do = [int(v) for v in edims[old]]
                psi = x[boff[old]:boff[old + 1]].reshape(do[2], do[1], do[0])   # [c][b][a]
                for t in range(t0, t1):
                    T = psi
                    for a in seq:
                        op = ops[offs[t, a]: offs[t, a] + dn[a] * do[a]].reshape(do[a], dn[a]).T
                        op = op[row0[a]:row0[a] + ext[a]]
                        ax_np = 2 - a
                        T = np.moveaxis(np.tensordot(op, T, axes=([1], [ax_np])), 0, ax_np)
                    tile += pref[t] * T
            blk[c0:c0 + ct, b0:b0 + bt, a0:a0 + at] += tile
        out[nb] = blk.reshape(-1)
    return out


def shared_flops_lower_bound(plan):
    """Smallest FLOP count any contraction sequence can execute for the
    plan's terms when the terms of a pair that apply the same first-stage
    operator share that stage's result (the kernel's grouping, untiled):
    per pair, the minimum over the sequences of (first stage x distinct
    first-stage operators + the other stages x terms)."""
    import itertools
    pairs = plan["plan.pairs"].reshape(-1, 4)
    edims = plan["plan.edims"].reshape(-1, 3).astype(np.float64)
    offs = plan["plan.op_off"].reshape(-1, 3)
    ptr = plan["plan.pair_ptr"]
    total = 0.0
    for nb in range(len(ptr) - 1):
        dn = edims[nb]
        for p in range(ptr[nb], ptr[nb + 1]):
            old, axes, t0, t1 = (int(v) for v in pairs[p])
            nst = (axes >> 6) & 3
            do = edims[old]
            best = None
            for seq in itertools.permutations(range(3), nst):
                w = do.copy()
                cost = 0.0
                for k, a in enumerate(seq):
                    f = 2.0 * dn[a] * np.prod(w)
                    w[a] = dn[a]
                    n = len(np.unique(offs[t0:t1, a])) if (k == 0 and nst == 3) else t1 - t0
                    cost += f * n
                best = cost if best is None else min(best, cost)
            total += best
    return total


def reference_block(s, y, nb):
    boff = s["beginblock"].astype(np.int64)
    return y[boff[nb]:boff[nb + 1]]
