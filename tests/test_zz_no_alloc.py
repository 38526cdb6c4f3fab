"""The allocation-free preconditioner entry point.

Callers that cannot allocate device memory when they precondition (a pool
that owns the whole GPU, code that must not trigger the implicit device
synchronisation of cudaMalloc/cudaFree) call
t3ns_precondition_device_noalloc with their own device buffers; its only
scratch is a fixed array inside the library.  This test calls it through the
C ABI twice in a row, on different inputs, and checks each result against
the allocating entry point t3ns_precondition_host and against the CPU
restatement of the reference's preconditioner (oracle/precond_oracle.py,
reference src/davidson.c:223-257, cutoff branch included), within the
1e-12 relative tolerance of the other parity tests; the second, smaller call
also shows that nothing of the first call's scratch leaks into it.  It also
checks the size limit is enforced.  It lives in its own file, collected last, and passes alone in a
fresh process as well as after the other tests.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from conftest import ROOT
from t3ns_b200 import native

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import precond_oracle  # noqa: E402

pytestmark = pytest.mark.gpu

RTOL = 1e-12
T3NS_E_LIMIT = -4


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _inputs(seed, n):
    rng = np.random.default_rng(seed)
    result = rng.standard_normal(n)
    result /= np.linalg.norm(result)
    diag = rng.uniform(-3.0, 5.0, n)
    diag[::977] = 0.7            # exercises the 1e-12 cutoff at theta = 0.7
    vec_t = rng.standard_normal(n) * 1e-3
    return result, diag, vec_t


def _host_reference(lib, result, theta, diag, vec_t):
    out = vec_t.copy()
    f64p = C.POINTER(C.c_double)
    native.check(lib.t3ns_precondition_host(result.size, result.ctypes.data_as(f64p), theta,
                                            diag.ctypes.data_as(f64p), out.ctypes.data_as(f64p)),
                 "precondition_host")
    return out


def test_noalloc_matches_allocating_entry_point(torch_cuda):
    torch = torch_cuda
    lib = native.load()
    stream = torch.cuda.current_stream()
    for call, (seed, n, theta) in enumerate([(1, 1_000_003, 0.7), (2, 257, -1.25)]):
        result, diag, vec_t = _inputs(seed, n)
        ref = _host_reference(lib, result, theta, diag, vec_t)
        d_r = torch.from_numpy(result).cuda()
        d_d = torch.from_numpy(diag).cuda()
        d_t = torch.from_numpy(vec_t).cuda()
        torch.cuda.synchronize()
        rc = lib.t3ns_precondition_device_noalloc(n, C.c_void_p(d_r.data_ptr()), theta,
                                                  C.c_void_p(d_d.data_ptr()),
                                                  C.c_void_p(d_t.data_ptr()),
                                                  C.c_void_p(stream.cuda_stream))
        native.check(rc, "precondition_device_noalloc")
        got = d_t.cpu().numpy()
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= RTOL, (call, err)
        want = precond_oracle.precondition(result, theta, diag, vec_t)
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= RTOL, (call, err)


def test_noalloc_rejects_sizes_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    lib = native.load()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    rc = lib.t3ns_precondition_device_noalloc(16777217, p, 0.0, p,
                                              p, None)
    assert rc == T3NS_E_LIMIT
    assert b"scratch limit" in lib.t3ns_last_error()
    torch.cuda.synchronize()
    assert float(buf.abs().sum()) == 0.0   # nothing was launched
