"""Project autotuner (H2DEV_OPT_AUTOTUNE): per plan shape bucket, the
launch variants of the block applies (row tilings of the streaming applies,
rows per thread of the matrix-free apply with at most 4 right-hand sides)
are timed once and the fastest is kept.  The variants tile rows differently but sum every row in the same
order, so results with and without the tuner are identical bit for bit."""
import numpy as np
import pytest

import mxc_b200 as m

pytestmark = pytest.mark.gpu


def build(h, mf, tune):
    h.set_option(m._lib.OPT_AUTOTUNE, 1 if tune else 0)
    h.set_option(m._lib.OPT_MATRIX_FREE, 1 if mf else 0)
    N = 8192
    L = m.levels_for(N, 256)
    b = m.uniform_unit_cube_rnd(N, 51)
    t = m.build_tree(b, L)
    k = m.Laplace3D(1e-3)
    A = m.H2MatrixSolver(h, k, 1e-10, 100, 0, t, 2.0, b, samples=2000)
    h.set_option(m._lib.OPT_MATRIX_FREE, 0)
    M = m.H2MatrixSolver(h, k, 0.0, 100, 0, t, 2.0, b, samples=2000, precision=m.FP32)
    M.factorizeM()
    return A, M, N


@pytest.mark.parametrize("mf", [False, True])
def test_autotuned_applies_equal_default_applies(mf):
    h1, h2 = m.Handle(0), m.Handle(0)
    A1, M1, N = build(h1, mf, False)
    A2, M2, _ = build(h2, mf, True)
    X = np.asfortranarray(np.random.default_rng(4).random((N, 16)))
    Y1, Y2 = X.copy(order="F"), X.copy(order="F")
    A1.matVecMul(Y1)
    A2.matVecMul(Y2)
    assert np.array_equal(Y1, Y2)
    Z1, Z2 = X.copy(order="F"), X.copy(order="F")
    M1.solvePrecondition(Z1)
    M2.solvePrecondition(Z2)
    assert np.array_equal(Z1, Z2)
    rep = h2.autotune_report()
    assert rep and not h1.autotune_report()
    for key, choice, ms in rep:
        assert 0 <= choice < max(1, len(ms)) and all(v >= 0 for v in ms)
    if mf:
        # Matrix-free plans with more than 4 right-hand sides have one kernel
        # (tensor-core fragments); with at most 4 the rows-per-thread choice
        # is tuned, again without changing a bit.
        X4 = np.asfortranarray(X[:, :4])
        Y1, Y2 = X4.copy(order="F"), X4.copy(order="F")
        A1.matVecMul(Y1)
        A2.matVecMul(Y2)
        assert np.array_equal(Y1, Y2)
        assert any(k.startswith("mf_matvec") for k, _, _ in h2.autotune_report())
    for s in (A1, M1, A2, M2):
        s.close()
    h1.close()
    h2.close()
