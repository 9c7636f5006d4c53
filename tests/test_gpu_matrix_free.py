"""Matrix-free operator (H2DEV_OPT_MATRIX_FREE): in interpolative mode the
leaf near blocks and the couplings are kernel evaluations on point sets
(h2matrix.cpp:184-188, 239-240), so the matvec (h2matrix.cpp:251-344)
evaluates them on the fly.  Same bases as the stored operator, so the
products agree to rounding (the on-the-fly kernel uses one rsqrt where the
stored near blocks use the reference's std::hypot form: a few ulp per
entry); the dense residual of a full solve meets the same 1e-10 bar; the
solver holds a small fraction of the stored operator's memory."""
import numpy as np
import pytest

import mxc_b200 as m

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def operator(handle, k, t, b, mf, eps=1e-10, samples=2000):
    handle.set_option(m._lib.OPT_MATRIX_FREE, 1 if mf else 0)
    try:
        return m.H2MatrixSolver(handle, k, eps, 100, 0, t, 2.0, b, samples=samples)
    finally:
        handle.set_option(m._lib.OPT_MATRIX_FREE, 0)


@pytest.fixture(scope="module")
def pair(handle):
    N = 8192
    L = m.levels_for(N, 256)
    b = m.uniform_unit_cube_rnd(N, 21)
    t = m.build_tree(b, L)
    k = m.Laplace3D(1e-2)
    h1 = m.Handle(0)
    h2 = m.Handle(0)
    A = operator(h1, k, t, b, False)
    Amf = operator(h2, k, t, b, True)
    yield A, Amf, h1, h2, k, t, b
    A.close()
    Amf.close()
    h1.close()
    h2.close()


@pytest.mark.parametrize("nrhs", [1, 2, 3, 5, 16])
def test_matrix_free_matvec_equals_stored(pair, nrhs):
    A, Amf, h1, h2, k, t, b = pair
    N = b.shape[0]
    X = np.asfortranarray(np.random.default_rng(nrhs).random((N, nrhs)))
    Y1 = X.copy(order="F")
    Y2 = X.copy(order="F")
    A.matVecMul(Y1 if nrhs > 1 else Y1[:, 0])
    Amf.matVecMul(Y2 if nrhs > 1 else Y2[:, 0])
    if nrhs == 1:
        Y1, Y2 = Y1[:, :1], Y2[:, :1]
    for c in range(nrhs):
        assert rel(Y2[:, c], Y1[:, c]) < 1e-13, c


def test_matrix_free_matvec_vs_dense(pair, handle):
    A, Amf, h1, h2, k, t, b = pair
    x = np.random.default_rng(7).random(b.shape[0])
    y = x.copy()
    Amf.matVecMul(y)
    assert rel(y, m.dense_matvec(handle, k, b, x)) < 1e-10


def test_matrix_free_holds_far_less_memory(pair):
    A, Amf, h1, h2, k, t, b = pair
    h1.trim()
    h2.trim()
    live_stored, _ = h1.memory()
    live_mf, _ = h2.memory()
    assert live_mf * 5 < live_stored, (live_mf, live_stored)


def test_matrix_free_operator_cannot_be_factorized(pair):
    A, Amf, h1, h2, k, t, b = pair
    with pytest.raises(m.H2DevError) as e:
        Amf.factorizeM()
    assert e.value.code == m._lib.H2DEV_ERR_STATE


def test_matrix_free_gmres_meets_dense_tolerance(pair, handle):
    A, Amf, h1, h2, k, t, b = pair
    N = b.shape[0]
    M = m.H2MatrixSolver(h2, k, 0.0, 100, 0, t, 2.0, b, samples=2000, precision=m.FP32)
    M.factorizeM()
    Xt = np.asfortranarray(np.random.default_rng(9).random((N, 4)))
    B = m.dense_matvec(handle, k, b, Xt)
    X = np.zeros((N, 4), order="F")
    rc = Amf.solveGMRES(1e-10, M, X, B, 10, 50, early_exit=True)
    M.close()
    assert rc == 0
    R = B - m.dense_matvec(handle, k, b, X)
    for c in range(4):
        assert np.linalg.norm(R[:, c]) / np.linalg.norm(B[:, c]) < 1e-10
