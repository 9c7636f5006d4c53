"""BF16 substitution (H2DEV_OPT_PRECOND_BF16): the ULV solve of an FP32
preconditioner (h2matrix.cpp:448-537) applied from BF16 copies of its blocks
with FP32 arithmetic.  Against the FP32 apply of the same factorization: the
same result to BF16 precision (8 significand bits: 2^-9 per entry, a few
times that after the level sweeps); and GMRES with the FP64 operator still
reaches the 1e-10 dense residual, possibly in more steps."""
import numpy as np
import pytest

import mxc_b200 as m

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def sys8k(handle):
    N = 8192
    L = m.levels_for(N, 256)
    b = m.uniform_unit_cube_rnd(N, 31)
    t = m.build_tree(b, L)
    k = m.Laplace3D(1e-3)
    A = m.H2MatrixSolver(handle, k, 1e-11, 100, 0, t, 2.0, b, samples=4000)
    M32 = m.H2MatrixSolver(handle, k, 0.0, 100, 0, t, 2.0, b, samples=2000, precision=m.FP32)
    handle.set_option(m._lib.OPT_PRECOND_BF16, 1)
    try:
        Mbf = m.H2MatrixSolver(handle, k, 0.0, 100, 0, t, 2.0, b, samples=2000, precision=m.FP32)
    finally:
        handle.set_option(m._lib.OPT_PRECOND_BF16, 0)
    M32.factorizeM()
    Mbf.factorizeM()
    yield A, M32, Mbf, k, b
    for s in (A, M32, Mbf):
        s.close()


@pytest.mark.parametrize("nrhs", [1, 3, 16])
def test_bf16_apply_matches_fp32_apply(sys8k, nrhs):
    A, M32, Mbf, k, b = sys8k
    X = np.asfortranarray(np.random.default_rng(nrhs).random((b.shape[0], nrhs)))
    Y1 = X.copy(order="F")
    Y2 = X.copy(order="F")
    M32.solvePrecondition(Y1 if nrhs > 1 else Y1[:, 0])
    Mbf.solvePrecondition(Y2 if nrhs > 1 else Y2[:, 0])
    for c in range(nrhs):
        e = rel(Y2[:, c], Y1[:, c])
        assert 1e-6 < e < 3e-2, (c, e)  # BF16-level agreement (and not FP32-level: the BF16 path ran)


def test_bf16_preconditioned_gmres_reaches_dense_tolerance(sys8k, handle):
    A, M32, Mbf, k, b = sys8k
    N = b.shape[0]
    Xt = np.asfortranarray(np.random.default_rng(5).random((N, 4)))
    B = m.dense_matvec(handle, k, b, Xt)
    X32 = np.zeros((N, 4), order="F")
    A.solveGMRES(1e-10, M32, X32, B, 10, 50, early_exit=True)
    it32 = np.asarray(A.iters).copy()
    X = np.zeros((N, 4), order="F")
    rc = A.solveGMRES(1e-10, Mbf, X, B, 10, 50, early_exit=True)
    assert rc == 0
    assert np.all(np.asarray(A.iters) >= it32)
    R = B - m.dense_matvec(handle, k, b, X)
    for c in range(4):
        assert np.linalg.norm(R[:, c]) / np.linalg.norm(B[:, c]) < 1e-10
        assert rel(X[:, c], X32[:, c]) < 1e-8
