"""The allocation-free relative-error entry point agrees with the regular one.

h2dev_solve_rel_err_device_noalloc serves callers that may not allocate
device memory (a serving loop whose HBM is all handed out by its own budgeted
pool, or a latency-critical path that cannot afford the device-wide
synchronisation cudaMalloc / cudaFree can cause).  It keeps its partial sums
in a fixed array inside the library instead of a per-call buffer.  This file
sorts last so that a run stopping at the first failure has run every other
test before it; it also passes on its own in a fresh process.

The device arrays below are allocated by the test (torch), not by the entry
point; the entry point itself only reads dX/dRef and writes dErr.
"""
import ctypes as C

import numpy as np
import pytest

import mxc_b200 as m
from mxc_b200 import _lib

pytestmark = pytest.mark.gpu

SCRATCH_DOUBLES = 16384  # the library's fixed limit: 2 * ceil(n / 16384) * nrhs


def _noalloc(handle, dX, dR, n, nrhs, ld, dErr):
    return _lib.lib().h2dev_solve_rel_err_device_noalloc(handle.h, n, nrhs, C.c_void_p(dX.data_ptr()),
                                                         C.c_void_p(dR.data_ptr()), ld, C.c_void_p(dErr.data_ptr()))


def _case(seed, nrhs, n):
    rng = np.random.default_rng(seed)
    X = rng.random((nrhs, n))
    R = X + 1e-6 * rng.standard_normal((nrhs, n))
    return X, R


def test_noalloc_matches_regular_entry_two_calls_in_a_row(handle):
    import torch

    # Two consecutive calls with different shapes: the second uses more
    # scratch than the first and must not see the first call's leftovers.
    for seed, nrhs, n in ((11, 3, 70001), (12, 2, 400003)):
        X, R = _case(seed, nrhs, n)
        dX = torch.from_numpy(X).cuda()
        dR = torch.from_numpy(R).cuda()
        dErr = torch.full((nrhs,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert _noalloc(handle, dX, dR, n, nrhs, n, dErr) == _lib.H2DEV_OK
        handle.synchronize()
        got = dErr.cpu().numpy()
        exp = m.rel_err_device(handle, dX.data_ptr(), dR.data_ptr(), n, nrhs, n)
        np.testing.assert_allclose(got, exp, rtol=1e-12, atol=0)
        for c in range(nrhs):
            host = m.H2MatrixSolver.solveRelErr(X[c], R[c])
            assert abs(got[c] - host) <= 1e-12 * host


def test_noalloc_uses_whole_scratch_and_rejects_larger(handle):
    import torch

    # n = 1 with nrhs = 8192 needs exactly the 16384-double limit; one more
    # column is refused before any device work.
    nrhs = SCRATCH_DOUBLES // 2
    X, R = _case(13, nrhs + 1, 1)
    dX = torch.from_numpy(X).cuda()
    dR = torch.from_numpy(R).cuda()
    dErr = torch.zeros(nrhs + 1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert _noalloc(handle, dX, dR, 1, nrhs, 1, dErr) == _lib.H2DEV_OK
    handle.synchronize()
    exp = m.rel_err_device(handle, dX.data_ptr(), dR.data_ptr(), 1, nrhs, 1)
    np.testing.assert_allclose(dErr.cpu().numpy()[:nrhs], exp, rtol=1e-12, atol=0)
    rc = _noalloc(handle, dX, dR, 1, nrhs + 1, 1, dErr)
    assert rc == _lib.H2DEV_ERR_ARG
    assert b"limit" in _lib.lib().h2dev_last_error_message()
