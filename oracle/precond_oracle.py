"""CPU restatement of the reference Davidson diagonal preconditioner.

TEST INFRASTRUCTURE (the oracle): only the tests load it, as the checker of
the engine's preconditioner entry points (t3ns_precondition_host,
t3ns_precondition_device_noalloc) and of the drop-in's
davidson_diagonal_preconditioner.  The product never imports it.

Follows reference src/davidson.c:223-257 (davidson_diagonal_preconditioner)
step by step, in numpy float64:
  - K = diag(diagonal - theta), each diagonal difference of magnitude at or
    below DIAG_CUTOFF = 1e-12 (src/davidson.c:21) replaced by +-1e-12 with the
    sign of the difference (a zero difference counts as positive);
  - Olsen correction: uK = K^-1 u (u = result), alpha = -(uK . t) / (uK . u);
  - t <- t + alpha u (cblas_daxpy), then t <- -K^-1 t.
The reference sums uKr and uKu in an OpenMP reduction, whose order depends on
the thread count; numpy's pairwise sums differ from it only by rounding.
"""
import numpy as np

DIAG_CUTOFF = 1e-12


def _k(diagonal, theta):
    diff = np.asarray(diagonal, dtype=np.float64) - theta
    return np.where(np.abs(diff) > DIAG_CUTOFF, diff, np.where(diff < 0, -DIAG_CUTOFF, DIAG_CUTOFF))


def precondition(result, theta, diagonal, vec_t):
    """Returns the preconditioned correction vector (vec_t is not modified)."""
    u = np.asarray(result, dtype=np.float64)
    t = np.array(vec_t, dtype=np.float64)
    k = _k(diagonal, theta)
    uk = u / k
    alpha = -np.dot(uk, t) / np.dot(uk, u)
    t = t + alpha * u
    return -t / k
