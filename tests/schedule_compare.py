"""Compares a compiled schedule ("my.*" records) with the reference's replay
schedule ("sr.*" records) of the same step: same (new, old) pairs, same
contraction order, and per pair the same multiset of (MPO combination,
operator blocks, prefactor), prefactors bit-identical."""
import numpy as np


def entries(rec, prefix):
    pp = rec[prefix + "pair_ptr"]
    po = rec[prefix + "pair_old"]
    por = rec[prefix + "pair_order"]
    cp = rec[prefix + "combo_ptr"]
    cm = rec[prefix + "combo_mpo"]
    cs = rec[prefix + "combo_sbops"].reshape(-1, 3)
    cf = rec[prefix + "combo_pref"]
    out = {}
    nb = len(pp) - 1
    for n in range(nb):
        for p in range(pp[n], pp[n + 1]):
            key = (n, int(po[p]))
            combos = sorted((int(cm[c]), tuple(int(v) for v in cs[c]), float(cf[c]).hex())
                            for c in range(cp[p], cp[p + 1]))
            assert key not in out, f"duplicate pair {key}"
            out[key] = (int(por[p]), combos)
    return out


def compare(ref, mine, isdmrg):
    a = entries(ref, "sr.")
    b = entries(mine, "my.")
    if isdmrg:
        # the third operator block is meaningless for two-operator steps
        def strip(d):
            return {k: (o, sorted((m, s[:2], f) for m, s, f in c)) for k, (o, c) in d.items()}
        a, b = strip(a), strip(b)
    missing = sorted(set(a) - set(b))
    extra = sorted(set(b) - set(a))
    diff = [k for k in a if k in b and a[k] != b[k]]
    return missing, extra, diff
