"""Dense factorisations of the site-tensor decomposition (the reference's
LAPACKE_dgesdd / dgeqrf / dorgqr calls, src/siteTensor_decompose.c:285, :295,
:565, :1060) against the reference LAPACK's own outputs.

Captures (oracle/t3ns_run.c --capture-dense) hold each call's input and the
outputs of the LAPACK the reference is linked with.  CPU: the oracle's
restatement (oracle/dense_oracle.py) reproduces them, which pins it.  GPU:
the engine's kernels, through the C ABI, reproduce them -- QR factors and Q
elementwise to 1e-13 (scaled by the column norms), singular values to 1e-13
of the largest, and singular vectors through the invariants that define
them (reconstruction, orthonormality, the projector of every singular
value separated from its neighbours by a relative gap of 1e-6) -- plus
edge cases the sweeps produce: rank-deficient blocks (zero singular values,
whose vectors must still be orthonormal), single rows and columns, zero
matrices and wide matrices."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from conftest import ROOT
from t3ns_b200.stepfile import read_step

import sys
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import dense_oracle as do  # noqa: E402

CAPDIRS = [os.path.join(ROOT, "oracle", "_ref", "captures", d) for d in ("dense_hub10", "dense_qc12")]


def _caps(kind):
    out = []
    for d in CAPDIRS:
        out += sorted(glob.glob(os.path.join(d, f"{kind}_*.t3c")))
    return out


GESDD, GEQRF, ORGQR = _caps("gesdd"), _caps("geqrf"), _caps("orgqr")
IDS = lambda p: "/".join(p.split("/")[-2:])  # noqa: E731


def _mat(rec, name, m, n):
    return rec[name].reshape(n, m).T if m * n else np.zeros((m, n))


def _gesdd_rec(p):
    r = read_step(p)
    m, n = int(r["gesdd.m"][0]), int(r["gesdd.n"][0])
    jobz = chr(int(r["gesdd.jobz"][0]))
    a = _mat(r, "gesdd.a", m, n)
    k = min(m, n)
    u = _mat(r, "gesdd.u", m, k) if jobz == "S" else None
    vt = _mat(r, "gesdd.vt", k, n) if jobz == "S" else None
    return a, jobz, r["gesdd.s"], u, vt


def check_svd(a, s, u, vt, s_ref, tol=1e-13):
    """Singular values against s_ref; u, vt (if given) through the invariants
    of a thin SVD of a."""
    m, n = a.shape
    k = min(m, n)
    smax = max(float(s_ref.max()) if s_ref.size else 0.0, 1e-300)
    assert np.all(np.diff(s) <= 0), "not descending"
    assert np.abs(s - s_ref).max() <= tol * smax
    if u is None:
        return
    anorm = max(np.linalg.norm(a), 1e-300)
    assert np.linalg.norm(u * s @ vt - a) <= tol * anorm * 10
    assert np.abs(u.T @ u - np.eye(k)).max() <= tol * 10
    assert np.abs(vt @ vt.T - np.eye(k)).max() <= tol * 10


def check_subspaces(s, u, vt, s_ref, u_ref, vt_ref, gap=1e-6, tol=1e-9):
    """Projectors onto the singular subspace of every cluster of singular
    values (relative gap `gap` to the neighbours) agree."""
    k = len(s_ref)
    smax = max(float(s_ref.max()), 1e-300)
    start = 0
    for i in range(1, k + 1):
        if i == k or (s_ref[i - 1] - s_ref[i]) > gap * smax:
            if s_ref[start] > 1e-8 * smax:
                sl = slice(start, i)
                pu, pr = u[:, sl] @ u[:, sl].T, u_ref[:, sl] @ u_ref[:, sl].T
                assert np.abs(pu - pr).max() <= tol, (start, i)
                pv, qv = vt[sl].T @ vt[sl], vt_ref[sl].T @ vt_ref[sl]
                assert np.abs(pv - qv).max() <= tol, (start, i)
            start = i


# ---------------------------------------------------------------- CPU: oracle pins

@pytest.mark.skipif(not GEQRF, reason="no dense captures")
@pytest.mark.parametrize("path", GEQRF[::3], ids=IDS)
def test_oracle_geqr2_pinned(path):
    r = read_step(path)
    m, n = int(r["geqrf.m"][0]), int(r["geqrf.n"][0])
    qr, tau = do.geqr2(_mat(r, "geqrf.a", m, n))
    ref = _mat(r, "geqrf.qr", m, n)
    scale = np.maximum(np.linalg.norm(ref, axis=0), 1e-300)
    assert (np.abs(qr - ref) / scale).max() <= 1e-13
    assert np.abs(tau - r["geqrf.tau"]).max() <= 1e-13


@pytest.mark.skipif(not ORGQR, reason="no dense captures")
@pytest.mark.parametrize("path", ORGQR[::3], ids=IDS)
def test_oracle_org2r_pinned(path):
    r = read_step(path)
    m, n, k = (int(r[f"orgqr.{x}"][0]) for x in "mnk")
    q = do.org2r(_mat(r, "orgqr.a", m, n), r["orgqr.tau"], n, k)
    assert np.abs(q - _mat(r, "orgqr.q", m, n)).max() <= 1e-13


@pytest.mark.skipif(not GESDD, reason="no dense captures")
@pytest.mark.parametrize("path", GESDD[::4], ids=IDS)
def test_oracle_jacobi_svd_pinned(path):
    a, jobz, s_ref, u_ref, vt_ref = _gesdd_rec(path)
    u, s, vt = do.jacobi_svd(a)
    check_svd(a, s, u, vt, s_ref)
    if jobz == "S":
        check_subspaces(s, u, vt, s_ref, u_ref, vt_ref)


# ---------------------------------------------------------------- GPU: engine

def _lib():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from t3ns_b200 import native
    lib = native.load()
    lib.t3ns_gesdd_host.argtypes = [C.c_char, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    lib.t3ns_geqrf_host.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    lib.t3ns_orgqr_host.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    return lib, native


def gpu_gesdd(a, jobz="S", pad=3):
    """The engine's SVD with leading dimensions larger than the matrix."""
    lib, native = _lib()
    m, n = a.shape
    k = min(m, n)
    lda, ldu, ldvt = m + pad, m + pad, k + pad
    abuf = np.zeros((n, lda))
    abuf[:, :m] = a.T
    s = np.zeros(max(k, 1))
    ubuf = np.zeros((max(k, 1), ldu))
    vbuf = np.zeros((max(n, 1), ldvt))
    native.check(lib.t3ns_gesdd_host(jobz.encode(), m, n, abuf.ctypes.data, lda, s.ctypes.data,
                                     ubuf.ctypes.data, ldu, vbuf.ctypes.data, ldvt), "gesdd")
    if jobz == "N":
        return None, s[:k], None
    return ubuf[:k, :m].T.copy(), s[:k], vbuf[:n, :k].T.copy()


def gpu_geqrf(a):
    lib, native = _lib()
    m, n = a.shape
    buf = np.asfortranarray(a.copy())
    tau = np.zeros(max(min(m, n), 1))
    native.check(lib.t3ns_geqrf_host(m, n, buf.ctypes.data, m, tau.ctypes.data), "geqrf")
    return buf, tau[:min(m, n)]


def gpu_orgqr(a, tau, n, k):
    lib, native = _lib()
    m = a.shape[0]
    buf = np.asfortranarray(a[:, :n].copy())
    t = np.ascontiguousarray(tau[:k]) if k else np.zeros(1)
    native.check(lib.t3ns_orgqr_host(m, n, k, buf.ctypes.data, m, t.ctypes.data), "orgqr")
    return buf


@pytest.mark.gpu
@pytest.mark.parametrize("path", GESDD, ids=IDS)
def test_gesdd_gpu_matches_reference(path):
    a, jobz, s_ref, u_ref, vt_ref = _gesdd_rec(path)
    u, s, vt = gpu_gesdd(a, jobz)
    check_svd(a, s, u, vt, s_ref)
    if jobz == "S":
        check_subspaces(s, u, vt, s_ref, u_ref, vt_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("path", GEQRF, ids=IDS)
def test_geqrf_gpu_matches_reference(path):
    r = read_step(path)
    m, n = int(r["geqrf.m"][0]), int(r["geqrf.n"][0])
    qr, tau = gpu_geqrf(_mat(r, "geqrf.a", m, n))
    ref = _mat(r, "geqrf.qr", m, n)
    scale = np.maximum(np.linalg.norm(ref, axis=0), 1e-300)
    assert (np.abs(qr - ref) / scale).max() <= 1e-13
    assert np.abs(tau - r["geqrf.tau"]).max() <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("path", ORGQR, ids=IDS)
def test_orgqr_gpu_matches_reference(path):
    r = read_step(path)
    m, n, k = (int(r[f"orgqr.{x}"][0]) for x in "mnk")
    q = gpu_orgqr(_mat(r, "orgqr.a", m, n), r["orgqr.tau"], n, k)
    assert np.abs(q - _mat(r, "orgqr.q", m, n)).max() <= 1e-13


def _edge_cases():
    rng = np.random.default_rng(7)
    low = rng.standard_normal((40, 3)) @ rng.standard_normal((3, 12))   # rank 3 of 12
    q, _ = np.linalg.qr(rng.standard_normal((30, 30)))
    return {
        "tall": rng.standard_normal((300, 17)),
        "wide": rng.standard_normal((9, 250)),
        "square": rng.standard_normal((64, 64)),
        "rank3_tall": low,
        "rank3_wide": low.T.copy(),
        "zero_cols": np.hstack([rng.standard_normal((20, 4)), np.zeros((20, 5))]),
        "zeros": np.zeros((7, 5)),
        "one_row": rng.standard_normal((1, 33)),
        "one_col": rng.standard_normal((33, 1)),
        "one": np.array([[-2.5]]),
        "orthogonal": q,                                                 # all sigma = 1
        "graded": rng.standard_normal((50, 20)) * np.logspace(0, -12, 20),
        "large_smem_overflow": rng.standard_normal((700, 60)),
    }


EDGE = _edge_cases()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(EDGE))
def test_gesdd_gpu_edge_cases(name):
    a = EDGE[name]
    s_np = np.linalg.svd(a, compute_uv=False)
    u, s, vt = gpu_gesdd(a, "S")
    check_svd(a, s, u, vt, s_np, tol=1e-13)
    _, s_n, _ = gpu_gesdd(a, "N")
    assert np.array_equal(s_n, s)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(EDGE))
def test_qr_gpu_edge_cases(name):
    a = EDGE[name]
    m, n = a.shape
    qr, tau = gpu_geqrf(a)
    qr_o, tau_o = do.geqr2(a)
    scale = np.maximum(np.linalg.norm(a, axis=0), 1e-300)
    assert (np.abs(np.triu(qr) - np.triu(qr_o)) / scale).max() <= 1e-12
    k = min(m, n)
    q = gpu_orgqr(qr, tau, k, k)
    assert np.abs(q.T @ q - np.eye(k)).max() <= 1e-13
    assert np.linalg.norm(q @ np.triu(qr)[:k] - a) <= 1e-13 * max(np.linalg.norm(a), 1e-300) * 10


@pytest.mark.gpu
def test_dense_workspace_reuse_across_sizes_and_threads():
    """Each host thread keeps its device workspace and pinned staging buffer
    between calls and grows them on demand: results of a call do not depend
    on the sizes that ran before it on the thread, nor on other threads
    calling at the same time (bit-identical to one call at a time)."""
    import threading
    names = sorted(EDGE)
    order = names + names[::-1]        # sizes grow and shrink on one thread

    def run(name):
        a = EDGE[name]
        u, s, vt = gpu_gesdd(a, "S")
        qr, tau = gpu_geqrf(a)
        k = min(a.shape)
        return u, s, vt, qr, tau, gpu_orgqr(qr, tau, k, k)

    alone = {name: run(name) for name in names}
    for name in order:
        for x, y in zip(run(name), alone[name]):
            assert np.array_equal(x, y), name
    errors = []

    def worker(seed):
        try:
            for name in np.random.default_rng(seed).permutation(order):
                for x, y in zip(run(name), alone[name]):
                    assert np.array_equal(x, y), name
        except Exception as e:          # reported on the main thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors


def test_engine_declares_dense_entry_points():
    hdr = open(os.path.join(ROOT, "include", "t3ns_b200.h")).read()
    for name in ("t3ns_gesdd_host", "t3ns_geqrf_host", "t3ns_orgqr_host"):
        assert name + "(" in hdr
