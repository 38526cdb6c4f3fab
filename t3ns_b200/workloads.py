"""Seeded synthetic Hamiltonians for the benchmark and serving workloads.

The quantum-chemistry workloads use a synthetic, seeded integral set instead
of a molecule (no dataset is involved):

* ``h`` is symmetric; its diagonal is N(-2.0, 0.5) and its off-diagonal is
  N(0, 0.05 * exp(-|p-q|/4));
* ``(pq|rs) = sum_L B^L_pq B^L_rs`` with ``B^L`` symmetric, entries
  N(0, 0.1 * exp(-|p-q|/6)), which makes the electron-repulsion supermatrix
  positive semidefinite and 8-fold symmetric;
* the core energy is 0.

Draw order (pinned so every component sees the same integrals), from
``numpy.random.default_rng(seed)``:

1. one full n x n N(0,1) matrix, scaled element-wise by 0.05 exp(-|p-q|/4);
   its strict upper triangle, symmetrised, is the off-diagonal of ``h``;
2. ``normal(-2.0, 0.5, n)`` for the diagonal of ``h``;
3. for L = 0 .. nfactors-1: one full n x n N(0,1) matrix scaled by
   0.1 exp(-|p-q|/6); its upper triangle including the diagonal, symmetrised,
   is ``B^L``.

The FCIDUMP written follows what the reference reader expects
(reference ``src/hamiltonian_qc.c:828-901`` and the symmetric fill of
``:933-950``): chemist notation, one line per unique ``i >= j``, ``k >= l``,
``(ij) >= (kl)`` (triangular pair index), then the one-body ``i >= j`` lines
with ``k = l = 0``, then the core energy line.
"""
from __future__ import annotations

import os

import numpy as np


def synthetic_qc_integrals(n: int, seed: int = 0, nfactors: int = 72):
    """Return ``(h, eri)``: ``h`` (n, n) and ``eri`` (n, n, n, n), chemist order."""
    rng = np.random.default_rng(seed)
    p = np.arange(n)
    dist = np.abs(p[:, None] - p[None, :])
    off = rng.normal(0.0, 1.0, (n, n)) * 0.05 * np.exp(-dist / 4.0)
    off = np.triu(off, 1)
    h = off + off.T
    h[p, p] = rng.normal(-2.0, 0.5, n)
    B = np.empty((nfactors, n, n))
    for L in range(nfactors):
        b = rng.normal(0.0, 1.0, (n, n)) * 0.1 * np.exp(-dist / 6.0)
        up = np.triu(b)
        B[L] = up + np.triu(b, 1).T
    eri = np.einsum("Lpq,Lrs->pqrs", B, B)
    return h, eri


def write_fcidump(path, h, eri, nelec: int, ms2: int = 0, core: float = 0.0) -> None:
    """Write integrals in the FCIDUMP layout the reference reader accepts."""
    n = h.shape[0]
    ii, jj = np.tril_indices(n)          # i >= j, row-major over i
    tri = ii * (ii + 1) // 2 + jj
    lines = [" &FCI NORB=%d,NELEC=%d,MS2=%d,\n" % (n, nelec, ms2),
             "  ORBSYM=%s,\n" % ",".join(["1"] * n),
             "  ISYM=1,\n", " /\n"]
    for a in range(len(ii)):
        i, j = int(ii[a]), int(jj[a])
        for b in range(len(ii)):
            if tri[b] > tri[a]:
                continue
            k, l = int(ii[b]), int(jj[b])
            v = eri[i, j, k, l]
            if abs(v) > 1e-20:
                lines.append("%23.16E %3d %3d %3d %3d\n" % (v, i + 1, j + 1, k + 1, l + 1))
    for a in range(len(ii)):
        i, j = int(ii[a]), int(jj[a])
        if abs(h[i, j]) > 1e-20:
            lines.append("%23.16E %3d %3d %3d %3d\n" % (h[i, j], i + 1, j + 1, 0, 0))
    lines.append("%23.16E %3d %3d %3d %3d\n" % (core, 0, 0, 0, 0))
    tmp = str(path) + ".tmp%d" % os.getpid()
    with open(tmp, "w") as f:
        f.writelines(lines)
    os.replace(tmp, path)


def synthetic_qc_fcidump(path, n: int, nelec: int, seed: int = 0, nfactors: int = 72) -> str:
    """Generate (once) the seeded synthetic FCIDUMP at ``path`` and return it."""
    path = str(path)
    if not os.path.exists(path):
        h, eri = synthetic_qc_integrals(n, seed, nfactors)
        write_fcidump(path, h, eri, nelec)
    return path
