"""GPU parity of the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances: kernel blocks are bit-exact (Laplace) or within 4 ulp (Yukawa);
everything downstream of a QR is compared in relative 2-norm with bounds
stated per test.  The preconditioned system is ill-conditioned (the dense
matrix has condition ~1e5-1e6 at these sizes), which is what the looser
substitution bounds reflect.
"""
import numpy as np
import pytest

import h2_oracle as O
import mxc_b200 as m
from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def problem(N, leaf=256, seed=999):
    L = m.levels_for(N, leaf)
    b = m.uniform_unit_cube_rnd(N, seed)
    t = m.build_tree(b, L)
    bo = O.uniform_unit_cube_rnd(N, seed)
    cells = O.build_binary_tree(bo, L)
    assert np.array_equal(b, bo)
    return b, t, cells, L


# ---------------------------------------------------------------- kernels

def test_gen_block_bitexact_vs_reference(handle):
    g = load_golden(golden_cases()[0])
    b = gold_b = g["bodies"]
    ij = g["probe_ij"]
    lap = m.Laplace3D(1.0)
    full = m.gen_block(handle, lap, b[:64], b)
    vals = np.array([full[i, j] for i, j in ij])
    assert np.array_equal(vals, g["probe_laplace"])
    yuk = m.Yukawa3D(1.0, 1.0)
    fy = m.gen_block(handle, yuk, b[:64], gold_b)
    vy = np.array([fy[i, j] for i, j in ij])
    np.testing.assert_allclose(vy, g["probe_yukawa"], rtol=1e-15, atol=0)


def test_gen_block_matches_oracle_ragged(handle):
    rng = np.random.default_rng(1)
    bi = rng.random((313, 3))
    bj = np.vstack([rng.random((17, 3)), bi[:5]])  # coincident bodies hit the diagonal value
    for k, ok in ((m.Laplace3D(2.0), O.Kernel(O.LAPLACE, 2.0)), (m.Yukawa3D(1.0, 0.7), O.Kernel(O.YUKAWA, 1.0, 0.7))):
        got = m.gen_block(handle, k, bi, bj)
        exp = O.gen_matrix(ok, bi, bj)
        if k.kind == m.KERNEL_LAPLACE:
            assert np.array_equal(got, exp)
        else:
            np.testing.assert_allclose(got, exp, rtol=1e-15)
    assert m.gen_block(handle, m.Laplace3D(), bi[:0], bj).shape == (0, 22)


def test_dense_matvec_vs_oracle(handle):
    N = 3000
    b = m.uniform_unit_cube_rnd(N, 5)
    X = np.asfortranarray(np.random.default_rng(2).random((N, 3)))
    got = m.dense_matvec(handle, m.Laplace3D(), b, X)
    exp = O.dense_matvec(O.Kernel(), b, X)
    assert rel(got, exp) < 1e-13
    x1 = X[:, 0].copy()
    assert rel(m.dense_matvec(handle, m.Laplace3D(), b, x1), exp[:, 0]) < 1e-13


# ---------------------------------------------------------------- H^2 operator

@pytest.fixture(scope="module")
def op2048(handle):
    N = 2048
    b, t, cells, L = problem(N)
    k = m.Laplace3D()
    A = m.H2MatrixSolver(handle, k, 1e-10, 100, 0, t, 2.0, b, samples=2000)
    Ao = O.H2MatrixSolver(O.Kernel(), 1e-10, 100, 0, cells, 2.0, O.uniform_unit_cube_rnd(N, 999) if False else b.copy(), L, 2000)
    return A, Ao, b, t, cells, L


def test_operator_ranks_match_oracle(op2048):
    A, Ao, b, t, cells, L = op2048
    for lvl in range(L + 1):
        d, r = A.level_dims(lvl)
        assert np.array_equal(d, Ao.A[lvl].Dims), lvl
        diff = np.abs(r - Ao.A[lvl].DimsLr)
        assert diff.max() <= 1 and (diff > 0).sum() <= max(1, len(r) // 8), (lvl, r, Ao.A[lvl].DimsLr)


def test_operator_matvec_vs_oracle_and_dense(op2048, handle):
    A, Ao, b, t, cells, L = op2048
    x = m.uniform_rhs(b.shape[0])
    y = x.copy()
    A.matVecMul(y)
    yo = Ao.matvec(x)
    yd = m.dense_matvec(handle, m.Laplace3D(), b, x)
    assert rel(y, yo) < 1e-10
    assert rel(y, yd) < 1e-10


def test_operator_matvec_multi_rhs(op2048):
    A, Ao, b, t, cells, L = op2048
    N = b.shape[0]
    X = np.asfortranarray(np.random.default_rng(3).random((N, 5)))
    Y = X.copy(order="F")
    A.matVecMul(Y)
    for c in range(5):
        y1 = X[:, c].copy()
        A.matVecMul(y1)
        assert rel(Y[:, c], y1) < 1e-14


def test_operator_matvec_overlap_is_bitwise_serial(op2048, handle):
    """The near field runs on a side stream, overlapping the upward / far /
    downward passes; with per-launch profiling on, the same plans run one
    after another on the main stream.  Same plans, same summation order:
    the results are identical bit for bit (16 right-hand sides, the
    tensor-core streaming path)."""
    A, Ao, b, t, cells, L = op2048
    N = b.shape[0]
    X = np.asfortranarray(np.random.default_rng(5).random((N, 16)))
    Y1 = X.copy(order="F")
    A.matVecMul(Y1)
    handle.profile(True)
    try:
        Y2 = X.copy(order="F")
        A.matVecMul(Y2)
    finally:
        handle.profile(False)
    assert np.array_equal(Y1, Y2)
    assert rel(Y1[:, 0], m.dense_matvec(handle, m.Laplace3D(), b, X[:, 0].copy())) < 1e-10


# ---------------------------------------------------------------- preconditioner

@pytest.fixture(scope="module")
def pre2048(handle):
    """Preconditioner built with the reference's own sequence (Householder
    sample QR + Eigen-rule column-pivoted QR)."""
    N = 2048
    b, t, cells, L = problem(N)
    handle.set_basis_mode(m._lib.BASIS_HOUSEHOLDER)
    try:
        M = m.H2MatrixSolver(handle, m.Laplace3D(), 0.0, 100, 0, t, 2.0, b, samples=2000)
    finally:
        handle.set_basis_mode(m._lib.BASIS_GRAM)
    Mo = O.H2MatrixSolver(O.Kernel(), 0.0, 100, 0, cells, 2.0, b.copy(), L, 2000)
    return M, Mo, b, t, cells, L


def test_precond_basis_matches_oracle(pre2048):
    M, Mo, b, t, cells, L = pre2048
    lvl = L
    S = M.export(lvl, m._lib.EXPORT_S).reshape(-1, 3)
    dims, ranks = M.level_dims(lvl)
    off = 0
    for i, (d, r) in enumerate(zip(dims, ranks)):
        So = Mo.A[lvl].S[i]
        # Skeletons (the first `rank` pivots) in the same order; the
        # fixed-rank CPQR stops after `rank` pivots, so the redundant bodies
        # only have to be the same set (no computation reads their order).
        assert np.array_equal(S[off:off + r], So[:r]), ("skeleton order differs", i)
        a = S[off + r:off + d]
        bb = So[r:]
        assert np.array_equal(a[np.lexsort(a.T)], bb[np.lexsort(bb.T)]), ("redundant set differs", i)
        off += d
    Q = M.export(lvl, m._lib.EXPORT_Q)
    Qo = np.concatenate([q.ravel(order="F") for q in Mo.A[lvl].Q])
    # Columns of the orthogonal completion are unique up to rounding (same
    # Householder convention on both sides).
    assert rel(Q, Qo) < 1e-9
    C = M.export(lvl, m._lib.EXPORT_C)
    Co = np.concatenate([c.ravel(order="F") for c in Mo.A[lvl].C]) if Mo.A[lvl].C else np.zeros(0)
    assert rel(C, Co) < 1e-9


def test_precond_factor_and_substitution(pre2048):
    M, Mo, b, t, cells, L = pre2048
    info = M.factorizeM()
    info_o = Mo.factorize()
    assert info == info_o
    N = b.shape[0]
    x = m.uniform_rhs(N)
    z = x.copy()
    M.solvePrecondition(z)
    zo = Mo.solve_precondition(x)
    assert rel(z, zo) < 1e-10


def test_leveled_rank_matches_oracle(handle):
    """leveled_rank > 0: rank (levels - l) * leveled_rank + rank at level l
    (solver.cpp:29), the reference's own basis sequence; ranks per level,
    skeletons, the factorization's info and the substitution agree with the
    oracle."""
    N = 4096
    b, t, cells, L = problem(N)
    rank, lrank = 48, 24
    handle.set_basis_mode(m._lib.BASIS_HOUSEHOLDER)
    try:
        M = m.H2MatrixSolver(handle, m.Laplace3D(), 0.0, rank, lrank, t, 2.0, b, samples=2000)
    finally:
        handle.set_basis_mode(m._lib.BASIS_GRAM)
    Mo = O.H2MatrixSolver(O.Kernel(), 0.0, rank, lrank, cells, 2.0, b.copy(), L, 2000)
    for lvl in range(L + 1):
        d, r = M.level_dims(lvl)
        assert np.array_equal(d, Mo.A[lvl].Dims), lvl
        assert np.array_equal(r, Mo.A[lvl].DimsLr), lvl
        if lvl >= 1:
            assert r.max() <= (L - lvl) * lrank + rank
    assert int(M.level_dims(L)[1].max()) == rank and int(M.level_dims(L - 1)[1].max()) == rank + lrank
    S = M.export(L, m._lib.EXPORT_S).reshape(-1, 3)
    dims, ranks = M.level_dims(L)
    off = 0
    for i, (dd, rr) in enumerate(zip(dims, ranks)):
        assert np.array_equal(S[off:off + rr], Mo.A[L].S[i][:rr]), i
        off += dd
    assert M.factorizeM() == Mo.factorize()
    x = m.uniform_rhs(N)
    z = x.copy()
    M.solvePrecondition(z)
    assert rel(z, Mo.solve_precondition(x)) < 1e-7


def test_precond_before_factorize_is_an_error(handle):
    b, t, cells, L = problem(1024, leaf=128)
    M = m.H2MatrixSolver(handle, m.Laplace3D(), 0.0, 64, 0, t, 2.0, b, samples=500)
    with pytest.raises(m.H2DevError) as e:
        M.solvePrecondition(np.ones(1024))
    assert e.value.code == m._lib.H2DEV_ERR_STATE


# ---------------------------------------------------------------- GMRES

def test_gmres_fp64_matches_oracle_and_dense(op2048, pre2048, handle):
    A, Ao, b, t, cells, L = op2048
    M, Mo, *_ = pre2048
    if M.info is None:
        M.factorizeM()
        Mo.factorize()
    N = b.shape[0]
    xt = m.uniform_rhs(N)
    B = m.dense_matvec(handle, m.Laplace3D(), b, xt)
    X = np.zeros(N)
    rc = A.solveGMRES(1e-10, M, X, B, 10, 50)
    assert rc == 0
    xo, reso, ito = Ao.solve_gmres(1e-10, Mo, np.zeros(N), B, 10, 50)
    assert A.iters == ito
    assert A.resid[A.iters] < 1e-10
    np.testing.assert_allclose(A.resid[:ito + 1], reso, rtol=1e-3, atol=1e-13)
    assert rel(X, xo) < 1e-8
    r = B - m.dense_matvec(handle, m.Laplace3D(), b, X)
    assert np.linalg.norm(r) / np.linalg.norm(B) < 1e-10


def test_gmres_multi_rhs_equals_single(op2048, pre2048, handle):
    A, Ao, b, t, cells, L = op2048
    M = pre2048[0]
    if M.info is None:
        M.factorizeM()
    N = b.shape[0]
    rng = np.random.default_rng(4)
    Xt = np.asfortranarray(rng.random((N, 3)))
    B = m.dense_matvec(handle, m.Laplace3D(), b, Xt)
    X = np.zeros((N, 3), order="F")
    A.solveGMRES(1e-10, M, X, B, 10, 50)
    for c in range(3):
        x1 = np.zeros(N)
        A2 = A  # same operator object, single column
        A2.solveGMRES(1e-10, M, x1, B[:, c].copy(), 10, 50)
        assert rel(X[:, c], x1) < 1e-12


def test_gmres_fp32_preconditioner_reaches_fp64_tolerance(op2048, handle):
    A, Ao, b, t, cells, L = op2048
    M32 = m.H2MatrixSolver(handle, m.Laplace3D(), 0.0, 100, 0, t, 2.0, b, samples=2000, precision=m.FP32)
    M32.factorizeM()
    N = b.shape[0]
    xt = m.uniform_rhs(N)
    B = m.dense_matvec(handle, m.Laplace3D(), b, xt)
    X = np.zeros(N)
    rc = A.solveGMRES(1e-10, M32, X, B, 10, 50)
    assert rc == 0
    r = B - m.dense_matvec(handle, m.Laplace3D(), b, X)
    assert np.linalg.norm(r) / np.linalg.norm(B) < 1e-10


# ---------------------------------------------------------------- edge cases

def test_single_box_tree(handle):
    """N < leaf: one box, no far field; the preconditioner is a dense LU."""
    g = load_golden([c for c in golden_cases() if "n300" in c][0])
    N = int(g["N"])
    b = m.uniform_unit_cube_rnd(N, int(g["seed"]))
    t = m.build_tree(b, 0)
    A = m.H2MatrixSolver(handle, m.Laplace3D(), 1e-10, 50, 0, t, 2.0, b)
    M = m.H2MatrixSolver(handle, m.Laplace3D(), 0.0, 50, 0, t, 2.0, b)
    M.factorizeM()
    xt = m.uniform_rhs(N)
    B = m.dense_matvec(handle, m.Laplace3D(), b, xt)
    y = xt.copy()
    A.matVecMul(y)
    assert rel(y, B) < 1e-14
    z = B.copy()
    M.solvePrecondition(z)
    assert rel(z, xt) < 1e-8
    X = np.zeros(N)
    assert A.solveGMRES(1e-10, M, X, B, 10, 5) == 0
    assert A.iters == 1


def test_hss_mode_ulv_is_exact_inverse(handle):
    """theta = 0 (mode "hss", main.cpp:139-140): the ULV inverts its own H^2 matrix."""
    b, t, cells, L = problem(2048)
    M = m.H2MatrixSolver(handle, m.Laplace3D(), 0.0, 100, 0, t, 0.0, b, samples=2000)
    x = m.uniform_rhs(2048)
    y = x.copy()
    M.matVecMul(y)
    M.factorizeM()
    M.solvePrecondition(y)
    assert rel(y, x) < 1e-7


def test_ragged_leaves_and_full_far_lists(handle):
    """N = 2000 (leaves of 250), every far body used (samples <= 0)."""
    N = 2000
    b, t, cells, L = problem(N)
    A = m.H2MatrixSolver(handle, m.Laplace3D(), 1e-9, 100, 0, t, 2.0, b, samples=0)
    Ao = O.H2MatrixSolver(O.Kernel(), 1e-9, 100, 0, cells, 2.0, b.copy(), L, 0)
    x = m.uniform_rhs(N)
    y = x.copy()
    A.matVecMul(y)
    assert rel(y, Ao.matvec(x)) < 1e-9


def test_ulv_exact_inverse_low_rank_kernel_multilevel(handle):
    """K = d^2 + 1 (exactly low-rank off-diagonal blocks): the device ULV is an
    exact inverse through every level under strong admissibility, in FP64."""
    N, leaf, theta, rank = 4096, 128, 2.0, 16
    b, t, cells, L = problem(N, leaf)
    k = m.Quadratic(1.0 / 50.0, 1.0)
    # The reference's own sequence (Householder sample QR + column-pivoted QR)
    # resolves the rank-6 range to rounding; the Gram path (checked below)
    # only to sqrt(eps).
    handle.set_basis_mode(m._lib.BASIS_HOUSEHOLDER)
    try:
        M = m.H2MatrixSolver(handle, k, 0.0, rank, 0, t, theta, b)
    finally:
        handle.set_basis_mode(m._lib.BASIS_GRAM)
    xt = m.uniform_rhs(N)
    A = O.gen_matrix(O.Kernel(O.QUADRATIC, 1.0 / 50.0, 1.0), b, b)
    B = A @ xt
    y = xt.copy()
    M.matVecMul(y)
    assert rel(y, B) < 1e-12
    M.factorizeM()
    z = B.copy()
    M.solvePrecondition(z)
    assert rel(z, xt) < 1e-9
    # Default Gram + pivoted-Cholesky bases: rank 16 exceeds the numerical
    # rank 6, the floored pivots keep the basis finite and the ULV accurate.
    Mg = m.H2MatrixSolver(handle, k, 0.0, rank, 0, t, theta, b)
    y = xt.copy()
    Mg.matVecMul(y)
    assert rel(y, B) < 1e-7
    Mg.factorizeM()
    z = B.copy()
    Mg.solvePrecondition(z)
    assert np.all(np.isfinite(z)) and rel(z, xt) < 1e-5
    # FP32 storage: exact up to single precision
    M32 = m.H2MatrixSolver(handle, k, 0.0, rank, 0, t, theta, b, precision=m.FP32)
    M32.factorizeM()
    z = B.copy()
    M32.solvePrecondition(z)
    assert rel(z, xt) < 5e-3



def test_gram_basis_matches_householder_basis_and_oracle(handle, pre2048):
    """Default fixed-rank path (Gram + pivoted Cholesky) selects the same
    skeletons as the column-pivoted QR and gives the same preconditioner."""
    Mh, Mo, b, t, cells, L = pre2048
    Mg = m.H2MatrixSolver(handle, m.Laplace3D(), 0.0, 100, 0, t, 2.0, b, samples=2000)
    for lvl in range(L + 1):
        dg, rg = Mg.level_dims(lvl)
        assert np.array_equal(dg, Mo.A[lvl].Dims) and np.array_equal(rg, Mo.A[lvl].DimsLr)
    Sg = Mg.export(L, m._lib.EXPORT_S).reshape(-1, 3)
    dims, ranks = Mg.level_dims(L)
    off, same = 0, 0
    for i, (d, r) in enumerate(zip(dims, ranks)):
        same += np.array_equal(Sg[off:off + r], Mo.A[L].S[i][:r])
        off += d
    assert same >= len(dims) - 1
    Qg = Mg.export(L, m._lib.EXPORT_Q)
    Qo = np.concatenate([q.ravel(order="F") for q in Mo.A[L].Q])
    assert rel(Qg, Qo) < 1e-7
    Mg.factorizeM()
    if Mh.info is None:
        Mh.factorizeM()
        Mo.factorize()
    x = m.uniform_rhs(b.shape[0])
    zg, zh = x.copy(), x.copy()
    Mg.solvePrecondition(zg)
    Mh.solvePrecondition(zh)
    assert rel(zg, zh) < 1e-5


def test_rel_err_device_matches_host(handle):
    import torch

    rng = np.random.default_rng(9)
    n, nrhs = 70001, 3
    X = rng.random((nrhs, n))
    R = X + 1e-6 * rng.standard_normal((nrhs, n))
    dX = torch.from_numpy(X).cuda()
    dR = torch.from_numpy(R).cuda()
    torch.cuda.synchronize()
    got = m.rel_err_device(handle, dX.data_ptr(), dR.data_ptr(), n, nrhs, n)
    for c in range(nrhs):
        exp = m.H2MatrixSolver.solveRelErr(X[c], R[c])
        assert abs(got[c] - exp) <= 1e-12 * exp


def test_register_streaming_apply_matches_tiled_apply(handle, op2048):
    """The multi-RHS apply kernel (A streamed into registers) and the tiled
    segmented GEMM give the same H^2 matvec and ULV substitution."""
    A, Ao, b, t, cells, L = op2048
    N = b.shape[0]
    X = np.asfortranarray(np.random.default_rng(5).random((N, 16)))
    outs = []
    for tiled in (0, 1):
        handle.set_option(m._lib.OPT_SKINNY_TILED, tiled)
        try:
            A2 = m.H2MatrixSolver(handle, m.Laplace3D(), 1e-10, 100, 0, t, 2.0, b, samples=2000)
            M2 = m.H2MatrixSolver(handle, m.Laplace3D(), 0.0, 100, 0, t, 2.0, b, samples=2000, precision=m.FP32)
            M2.factorizeM()
            Y = X.copy(order="F")
            A2.matVecMul(Y)
            Z = X.copy(order="F")
            M2.solvePrecondition(Z)
            y1 = X[:, 3].copy()
            A2.matVecMul(y1)
            outs.append((Y, Z, y1))
        finally:
            handle.set_option(m._lib.OPT_SKINNY_TILED, 0)
    assert rel(outs[0][0], outs[1][0]) < 1e-13
    assert rel(outs[0][2], outs[1][2]) < 1e-13
    assert rel(outs[0][1], outs[1][1]) < 1e-3  # FP32 preconditioner, different summation order


def test_geometric_sampling_matches_oracle(handle):
    """Level-geometric far-list cap: same ranks and the same operator as the oracle."""
    N = 4096
    b, t, cells, L = problem(N)
    handle.set_option(m._lib.OPT_SAMPLING, 1)
    try:
        A = m.H2MatrixSolver(handle, m.Laplace3D(), 1e-10, 100, 0, t, 2.0, b, samples=1000)
    finally:
        handle.set_option(m._lib.OPT_SAMPLING, 0)
    Ao = O.H2MatrixSolver(O.Kernel(), 1e-10, 100, 0, cells, 2.0, b.copy(), L, 1000, sampling=1)
    for lvl in range(L + 1):
        d, r = A.level_dims(lvl)
        assert np.abs(r - Ao.A[lvl].DimsLr).max() <= 1, lvl
    x = m.uniform_rhs(N)
    y = x.copy()
    A.matVecMul(y)
    assert rel(y, Ao.matvec(x)) < 1e-9


# ---------------------------------------------------------------- reference configuration C1

def test_c1_configuration_matches_oracle_fixture(handle):
    """The reference's CPU-runnable case (N = 20000, Laplace diagonal 1,
    theta 2, leaf 256, operator eps 1e-10 / 2000 samples, preconditioner rank
    100 / 2000 samples, one RHS) against the oracle fixture from
    tests/golden/make_c1_fixture.py: ranks per level, the H^2 matvec of
    x_true, the factorization's singular-block counts and its substitution
    M^-1 x_true, and three GMRES(10) restarts, in which the reference method
    stagnates on this system in both implementations."""
    import os
    from conftest import GOLDEN
    g = np.load(os.path.join(GOLDEN, "oracle_c1_n20000.npz"))
    N = 20000
    L = int(g["levels"])
    assert L == m.levels_for(N, 256)
    b = m.uniform_unit_cube_rnd(N, 999)
    t = m.build_tree(b, L)
    k = m.Laplace3D()
    A = m.H2MatrixSolver(handle, k, 1e-10, 100, 0, t, 2.0, b, samples=2000)
    handle.set_basis_mode(m._lib.BASIS_HOUSEHOLDER)
    try:
        M = m.H2MatrixSolver(handle, k, 0.0, 100, 0, t, 2.0, b, samples=2000)
    finally:
        handle.set_basis_mode(m._lib.BASIS_GRAM)
    for lvl in range(L + 1):
        d, r = A.level_dims(lvl)
        assert np.array_equal(d, g["op_dims_%d" % lvl]), lvl
        diff = np.abs(r - g["op_ranks_%d" % lvl])
        assert diff.max() <= 1 and (diff > 0).sum() <= max(1, len(r) // 8), lvl
        _, rp = M.level_dims(lvl)
        assert np.array_equal(rp, g["pc_ranks_%d" % lvl]), lvl
    xt = m.uniform_rhs(N)
    y = xt.copy()
    A.matVecMul(y)
    assert rel(y, g["y_op"]) < 1e-10
    info = M.factorizeM()
    assert list(np.atleast_1d(info)) == list(g["info"])
    z = xt.copy()
    M.solvePrecondition(z)
    # Both sides solve with A_rr by a partial-pivot LU and triangular solves
    # (h2matrix.cpp:377-379).  The C1 redundant blocks are so ill-conditioned
    # that rounding alone moves M^-1 x_true by several percent (the oracle's
    # own result moves by 12% when its LU solve is swapped for an explicit
    # inverse of the same matrix); the device result agrees to 9.3%, at the
    # level that conditioning allows (N = 2048 agrees to 1e-10, see
    # test_precond_factor_and_substitution).
    assert rel(z, g["z_pc"]) < 0.15
    B = m.dense_matvec(handle, k, b, xt)
    X = np.zeros(N)
    A.solveGMRES(1e-10, M, X, B, 10, 3)
    assert A.iters == int(g["iters"])
    # Both stagnate: the restart residuals stay within 1% of 1 (they differ
    # in the third digit, rounding amplified by the weak preconditioner).
    assert np.max(np.abs(np.asarray(A.resid[:A.iters + 1]) - 1.0)) < 1e-2
    assert np.max(np.abs(g["resid"] - 1.0)) < 1e-2


def test_yukawa_system_matches_oracle(handle):
    """Yukawa e^{-alpha r} / r (kernel.hpp:40-50) through the whole path at
    N = 2048: operator ranks, matvec, factorization, substitution and GMRES
    against the oracle."""
    N = 2048
    b, t, cells, L = problem(N)
    k = m.Yukawa3D(1.0, 1.0)
    ko = O.Kernel(O.YUKAWA, 1.0, 1.0)
    A = m.H2MatrixSolver(handle, k, 1e-10, 100, 0, t, 2.0, b, samples=2000)
    Ao = O.H2MatrixSolver(ko, 1e-10, 100, 0, cells, 2.0, b.copy(), L, 2000)
    handle.set_basis_mode(m._lib.BASIS_HOUSEHOLDER)
    try:
        M = m.H2MatrixSolver(handle, k, 0.0, 100, 0, t, 2.0, b, samples=2000)
    finally:
        handle.set_basis_mode(m._lib.BASIS_GRAM)
    Mo = O.H2MatrixSolver(ko, 0.0, 100, 0, cells, 2.0, b.copy(), L, 2000)
    for lvl in range(L + 1):
        d, r = A.level_dims(lvl)
        assert np.array_equal(d, Ao.A[lvl].Dims)
        assert np.abs(r - Ao.A[lvl].DimsLr).max() <= 1
    x = m.uniform_rhs(N)
    y = x.copy()
    A.matVecMul(y)
    assert rel(y, Ao.matvec(x)) < 1e-10
    assert rel(y, m.dense_matvec(handle, k, b, x)) < 1e-9
    assert M.factorizeM() == Mo.factorize()
    z = x.copy()
    M.solvePrecondition(z)
    assert rel(z, Mo.solve_precondition(x)) < 1e-7
    B = m.dense_matvec(handle, k, b, x)
    X = np.zeros(N)
    A.solveGMRES(1e-10, M, X, B, 10, 50)
    xo, reso, ito = Ao.solve_gmres(1e-10, Mo, np.zeros(N), B, 10, 50)
    assert A.iters == ito
    np.testing.assert_allclose(A.resid[:ito + 1], reso, rtol=1e-3, atol=1e-13)
    assert rel(X, xo) < 1e-8
