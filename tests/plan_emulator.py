"""Host-side emulation of the matvec work plan (numpy), used to check the
plan's tiling, contraction sequences and operator row offsets without a GPU.

For selected work units it recomputes the unit's output tile exactly the way
the kernel organises it -- pair by pair, term by term, contracting the memory
axes in the pair's sequence, with tiled axes restricted to the tile's rows --
and returns the tiles for comparison with the reference's matvec output."""
import ctypes as C
import os
import tempfile

import numpy as np

from t3ns_b200 import native
from t3ns_b200.stepfile import read_step


def dump_plan(desc):
    lib = native.load()
    lib.t3ns_heff_plan_dump.argtypes = [C.POINTER(native.HeffDesc), C.c_char_p]
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "plan.t3c")
        native.check(lib.t3ns_heff_plan_dump(C.byref(desc.desc), p.encode()), "plan_dump")
        return read_step(p)


def op_buffer(s, nops):
    return np.concatenate([s[f"ops{i}.tel"] for i in range(nops)])


def emulate_units(s, plan, x, unit_ids):
    nops = 2 if int(s["isdmrg"][0]) else 3
    ops = op_buffer(s, nops)
    units = plan["plan.units"].reshape(-1, 5)
    pairs = plan["plan.pairs"].reshape(-1, 4)
    pptr = plan["plan.pair_ptr"]
    edims = plan["plan.edims"].reshape(-1, 3)
    offs = plan["plan.op_off"].reshape(-1, 3)
    pref = plan["plan.pref"]
    boff = s["beginblock"].astype(np.int64)
    out = []
    for u in unit_ids:
        nb, b0, bt, c0, ct = (int(v) for v in units[u])
        dn = edims[nb]
        ext = [int(dn[0]), bt, ct]
        row0 = [0, b0, c0]
        tile = np.zeros(ext[0] * ext[1] * ext[2])
        for p in range(pptr[nb], pptr[nb + 1]):
            old, axes, t0, t1 = (int(v) for v in pairs[p])
            nst = (axes >> 6) & 3
            seq = [(axes >> (2 * k)) & 3 for k in range(nst)]
            do = edims[old]
            psi = x[boff[old]:boff[old + 1]].reshape(do[2], do[1], do[0])   # [c][b][a]
            for t in range(t0, t1):
                T = psi
                for a in seq:
                    r = ext[a]
                    op = ops[offs[t, a]: offs[t, a] + dn[a] * do[a]].reshape(do[a], dn[a]).T
                    op = op[row0[a]:row0[a] + r]                                # (r x do)
                    ax_np = 2 - a                                              # numpy axis
                    T = np.moveaxis(np.tensordot(op, T, axes=([1], [ax_np])), 0, ax_np)
                tile += pref[t] * T.reshape(-1)
        out.append(tile.reshape(ext[2], ext[1], ext[0]))
    return out


def reference_tile(s, plan, y, u):
    units = plan["plan.units"].reshape(-1, 5)
    edims = plan["plan.edims"].reshape(-1, 3)
    nb, b0, bt, c0, ct = (int(v) for v in units[u])
    dn = edims[nb]
    boff = s["beginblock"].astype(np.int64)
    blk = y[boff[nb]:boff[nb + 1]].reshape(dn[2], dn[1], dn[0])
    return blk[c0:c0 + ct, b0:b0 + bt, :]
