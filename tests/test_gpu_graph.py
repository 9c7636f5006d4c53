"""GMRES with its control flow on the device, and the whole solve as one
CUDA graph (H2DEV_OPT_GRAPH_SOLVE: a WHILE node over restart cycles, an IF
node around each Arnoldi step).  The graph launches the same kernels in the
same order as the step-by-step path, so solutions, residual histories and
cycle counts are identical; both follow solver.cpp:144-201 per column."""
import numpy as np
import pytest

import mxc_b200 as m

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sys8k():
    h = m.Handle(0)
    N = 8192
    L = m.levels_for(N, 256)
    b = m.uniform_unit_cube_rnd(N, 41)
    t = m.build_tree(b, L)
    k = m.Laplace3D(1e-3)
    A = m.H2MatrixSolver(h, k, 1e-11, 100, 0, t, 2.0, b, samples=4000)
    M = m.H2MatrixSolver(h, k, 0.0, 100, 0, t, 2.0, b, samples=2000, precision=m.FP32)
    M.factorizeM()
    Xt = np.asfortranarray(np.random.default_rng(3).random((N, 5)))
    B = m.dense_matvec(h, k, b, Xt)
    yield h, A, M, B, k, b
    A.close()
    M.close()
    h.close()


def solve(h, A, M, B, graph, early, tol=1e-10, outer=50):
    h.set_option(m._lib.OPT_GRAPH_SOLVE, 1 if graph else 0)
    try:
        X = np.zeros_like(B, order="F")
        rc = A.solveGMRES(tol, M, X, B, 10, outer, early_exit=early)
        return X, rc, np.array(A.resid, copy=True), np.array(A.iters, copy=True)
    finally:
        h.set_option(m._lib.OPT_GRAPH_SOLVE, 0)


@pytest.mark.parametrize("early", [True, False])
def test_graph_solve_equals_step_by_step(sys8k, early):
    h, A, M, B, k, b = sys8k
    X1, rc1, r1, i1 = solve(h, A, M, B, False, early)
    X2, rc2, r2, i2 = solve(h, A, M, B, True, early)
    assert rc1 == rc2 == 0
    assert np.array_equal(i1, i2)
    assert np.array_equal(r1, r2)
    assert np.array_equal(X1, X2)
    R = B - m.dense_matvec(h, k, b, X2)
    assert max(np.linalg.norm(R[:, c]) / np.linalg.norm(B[:, c]) for c in range(B.shape[1])) < 1e-10


def test_graph_solve_stops_at_outer_limit(sys8k):
    h, A, M, B, k, b = sys8k
    X, rc, r, it = solve(h, A, M, B, True, True, tol=1e-30, outer=2)
    assert rc == m._lib.H2DEV_ERR_NOCONV
    assert np.all(it == 2)
    X1, rc1, r1, it1 = solve(h, A, M, B, False, True, tol=1e-30, outer=2)
    assert np.array_equal(X, X1) and np.array_equal(r, r1)


def test_graph_solve_with_zero_outer_does_nothing(sys8k):
    h, A, M, B, k, b = sys8k
    X, rc, r, it = solve(h, A, M, B, True, True, outer=0)
    assert np.all(it == 0) and not X.any()


def test_graph_replay_with_new_right_hand_sides(sys8k):
    """The captured solve is kept on the operator and replayed by later calls
    with the same preconditioner and shape; new right-hand sides give their
    own (step-by-step-identical) solutions."""
    h, A, M, B, k, b = sys8k
    X0, *_ = solve(h, A, M, B, True, True)
    B2 = np.asfortranarray(B[:, ::-1] * 0.5)
    X2g, rc, r2g, i2g = solve(h, A, M, B2, True, True)   # replay
    X2s, rc_s, r2s, i2s = solve(h, A, M, B2, False, True)
    assert rc == rc_s == 0
    assert np.array_equal(X2g, X2s) and np.array_equal(r2g, r2s) and np.array_equal(i2g, i2s)
    np.testing.assert_allclose(X2g, X0[:, ::-1] * 0.5, rtol=1e-8, atol=1e-12)
