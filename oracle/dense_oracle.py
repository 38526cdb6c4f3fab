"""CPU restatement of the dense factorisations the reference's site-tensor
decomposition takes from LAPACK.  TEST INFRASTRUCTURE ONLY: the tests use it
as the checker; the product never imports it.

The reference calls LAPACKE_dgesdd, LAPACKE_dgeqrf and LAPACKE_dorgqr
(src/siteTensor_decompose.c:1060, :565, :285, :295) from the BLAS/LAPACK it
is linked with, here the OpenBLAS 0.3.15 that bundles reference LAPACK.  For
the block sizes T3NS produces (at most 128 columns) LAPACK's dgeqrf and
dorgqr run their unblocked forms, restated here from the published LAPACK
algorithms:

* dlarfg: for alpha and the vector x below it, beta = -sign(alpha) *
  hypot(alpha, |x|), tau = (beta - alpha) / beta, v = x / (alpha - beta);
  tau = 0 (H = I) when x = 0;
* dgeqr2: reflector j from column j, applied to the trailing columns;
* dorg2r: Q = H_0 ... H_{k-1} applied to the first n unit columns,
  accumulated from the last reflector backwards.

The SVD is checked through invariants (singular values, reconstruction,
orthonormality, singular subspaces), since singular vectors are defined up
to sign and rotation within degenerate singular values; the restatement is
one-sided Jacobi (Hestenes 1958), which the GPU code also uses.

Pinned: tests/test_dense.py compares every function here with the reference
LAPACK's own outputs captured by oracle/t3ns_run.c --capture-dense.
"""
import numpy as np


def geqr2(a):
    """Householder QR of a (m x n) with LAPACK's conventions: returns the
    overwritten matrix (R on and above the diagonal, reflectors below) and
    tau."""
    a = np.array(a, dtype=np.float64, order="F", copy=True)
    m, n = a.shape
    k = min(m, n)
    tau = np.zeros(k)
    for j in range(k):
        alpha = a[j, j]
        xnorm = np.linalg.norm(a[j + 1:, j])
        if xnorm == 0.0:
            tau[j] = 0.0
            continue
        beta = -np.copysign(np.hypot(alpha, xnorm), alpha)
        tau[j] = (beta - alpha) / beta
        a[j + 1:, j] /= (alpha - beta)
        a[j, j] = beta
        if j + 1 < n:
            v = np.concatenate(([1.0], a[j + 1:, j]))
            w = v @ a[j:, j + 1:]
            a[j:, j + 1:] -= tau[j] * np.outer(v, w)
    return a, tau


def org2r(a, tau, n, k):
    """The first n columns of H_0 ... H_{k-1} from the reflectors stored below
    the diagonal of a (m x >= n) and tau[k]."""
    a = np.array(a[:, :n], dtype=np.float64, order="F", copy=True)
    m = a.shape[0]
    for j in range(k, n):
        a[:, j] = 0.0
        a[j, j] = 1.0
    for i in range(k - 1, -1, -1):
        if i < n - 1:
            a[i, i] = 1.0
            v = a[i:, i].copy()
            w = v @ a[i:, i + 1:]
            a[i:, i + 1:] -= tau[i] * np.outer(v, w)
        if i < m - 1:
            a[i + 1:, i] *= -tau[i]
        a[i, i] = 1.0 - tau[i]
        a[:i, i] = 0.0
    return a


def jacobi_svd(a, tol=None, max_sweeps=60):
    """Thin SVD by one-sided Jacobi: (u, s, vt) with s descending."""
    a = np.asarray(a, dtype=np.float64)
    m, n = a.shape
    trans = m < n
    w = (a.T if trans else a).copy(order="F")
    mm, nn = w.shape
    v = np.eye(nn)
    tol = tol if tol is not None else 4.0 * np.finfo(float).eps * np.sqrt(mm)
    for _ in range(max_sweeps):
        rotated = False
        for p in range(nn - 1):
            for q in range(p + 1, nn):
                x, y = w[:, p], w[:, q]
                al, be, ga = x @ x, y @ y, x @ y
                den = np.sqrt(al) * np.sqrt(be)
                if not den > 0.0 or not abs(ga) > tol * den:
                    continue
                zeta = (be - al) / (2.0 * ga)
                t = np.copysign(1.0, zeta) / (abs(zeta) + np.sqrt(1.0 + zeta * zeta))
                c = 1.0 / np.sqrt(1.0 + t * t)
                s = c * t
                w[:, [p, q]] = np.column_stack((c * x - s * y, s * x + c * y))
                v[:, [p, q]] = np.column_stack((c * v[:, p] - s * v[:, q],
                                                s * v[:, p] + c * v[:, q]))
                rotated = True
        if not rotated:
            break
    else:
        raise RuntimeError("Jacobi sweeps did not converge")
    s = np.linalg.norm(w, axis=0)
    order = sorted(range(nn), key=lambda j: (-s[j], j))
    s = s[order]
    uw = w[:, order] / np.where(s > 1e-300, s, 1.0)
    vs = v[:, order]
    if trans:
        return vs, s, uw.T
    return uw, s, vs.T
