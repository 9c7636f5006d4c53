"""Invariants of the oracle's restatement that do not depend on a GPU.

The reference's dense algebra (Eigen) cannot be built here, so beyond the
pinned tree/list/kernel fixtures the oracle is checked against mathematics:
the ULV factorization must be an exact inverse whenever the reference's
dropped fill is exactly zero, and the pivoted QR must follow Eigen's rules.
"""
import numpy as np
import pytest
import scipy.linalg as sla

import h2_oracle as O


def test_ulv_exact_two_boxes_synthetic():
    """Off-diagonal block in the skeleton spans: the reference ULV is exact."""
    rng = np.random.default_rng(0)
    n, k = 20, 6
    U = [np.linalg.qr(rng.standard_normal((n, n)))[0] for _ in range(2)]
    S12 = rng.standard_normal((k, k))
    A11 = rng.standard_normal((n, n)); A11 = A11 + A11.T + 8 * np.eye(n)
    A22 = rng.standard_normal((n, n)); A22 = A22 + A22.T + 8 * np.eye(n)
    A12 = U[0][:, :k] @ S12 @ U[1][:, :k].T
    Ad = np.block([[A11, A12], [A12.T, A22]])

    def lvl(l, nodes, ar, ac):
        return O.Level(l, (1 << l) - 1, nodes, np.array(ar), np.array(ac), np.zeros(nodes + 1, dtype=np.int64),
                       np.array([], dtype=np.int64))

    s = O.H2MatrixSolver.__new__(O.H2MatrixSolver)
    s.levels = 1
    leaf = lvl(1, 2, [0, 2, 4], [0, 1, 0, 1])
    root = lvl(0, 1, [0, 1], [0])
    leaf.Dims = np.array([n, n]); leaf.DimsLr = np.array([k, k])
    leaf.Q = [U[0].copy(), U[1].copy()]; leaf.R = [np.zeros((n, n)), np.zeros((n, n))]
    leaf.A = [A11.copy(), A12.copy(), A12.T.copy(), A22.copy()]
    leaf.NA = [(0, 0, 0), (0, 0, k), (0, k, 0), (0, k, k)]
    root.Dims = np.array([2 * k]); root.DimsLr = np.array([0])
    root.Q = [np.eye(2 * k)]; root.R = [np.zeros((2 * k, 2 * k))]; root.A = [np.zeros((2 * k, 2 * k))]
    s.A = [root, leaf]
    s.lenX = 2 * n
    s.factorize()
    b = rng.standard_normal(2 * n)
    x = s.solve_precondition(b)
    xe = np.linalg.solve(Ad, b)
    assert np.linalg.norm(x - xe) / np.linalg.norm(xe) < 1e-12


@pytest.mark.parametrize("N,leaf,theta,rank", [(2000, 64, 2.0, 10), (4096, 128, 1.0, 12)])
def test_ulv_exact_multilevel_low_rank_kernel(N, leaf, theta, rank):
    """K = d^2 + 1 has rank <= 6 off-diagonal blocks: no fill is dropped at any level."""
    L = O.levels_for(N, leaf)
    b = O.uniform_unit_cube_rnd(N, 999)
    cells = O.build_binary_tree(b, L)
    k = O.Kernel(O.QUADRATIC, 1.0 / 50.0, 1.0)
    A = O.gen_matrix(k, b, b)
    xt = O.xbody_uniform(N)
    B = A @ xt
    M = O.H2MatrixSolver(k, 0.0, rank, 0, cells, theta, b, L, 0)
    assert O.solve_rel_err(M.matvec(xt), B) < 1e-13
    assert len(M.A[L].CCols) > 0 and len(M.A[L].ACols) > (1 << L)  # strong admissibility, real far field
    M.factorize()
    z = M.solve_precondition(B)
    assert O.solve_rel_err(z, xt) < 1e-10


def test_hss_mode_is_exact_inverse_of_its_h2_matrix():
    N = 2048
    L = O.levels_for(N, 256)
    b = O.uniform_unit_cube_rnd(N, 999)
    cells = O.build_binary_tree(b, L)
    M = O.H2MatrixSolver(O.Kernel(), 0.0, 100, 0, cells, 0.0, b, L, 2000)
    x = O.xbody_uniform(N)
    y = M.matvec(x)
    M.factorize()
    assert O.solve_rel_err(M.solve_precondition(y), x) < 1e-7


def test_colpiv_qr_matches_lapack_pivots_on_separated_columns():
    rng = np.random.default_rng(3)
    X = rng.standard_normal((60, 40)) * np.logspace(0, -8, 40)[None, :]
    X = X[:, rng.permutation(40)]
    qr, perm, maxpiv, nz = O.colpiv_qr(X)
    _, R, P = sla.qr(X, pivoting=True, mode="economic")
    assert np.array_equal(perm, P)
    np.testing.assert_allclose(np.abs(np.diag(qr)), np.abs(np.diag(R)), rtol=1e-8)
    assert O.colpiv_rank(qr, maxpiv, nz, 1e-5) == int(np.sum(np.abs(np.diag(R)) > abs(R[0, 0]) * 1e-5))


def test_colpiv_rank_zero_matrix_and_threshold_rules():
    # Eigen's nonzero-pivot test is strict (0 < 0 is false), so an all-zero
    # matrix keeps nonzero_pivots = size; the threshold rank is still 0.
    qr, perm, maxpiv, nz = O.colpiv_qr(np.zeros((5, 4)))
    assert nz == 4 and maxpiv == 0.0 and O.colpiv_rank(qr, maxpiv, nz, 1e-10) == 0


def test_compute_basis_identity_when_full_rank():
    """rank == M: Q = I, R = upper(Q_in) (h2matrix.cpp:57-60)."""
    rng = np.random.default_rng(5)
    X = rng.random((8, 3))
    F = rng.random((40, 3)) + 3.0
    a = np.eye(8)
    r, c = O.compute_basis(O.Kernel(), 8.0, X, F, a, True)
    assert r == 8 and np.array_equal(a, np.eye(8)) and np.array_equal(c, np.eye(8))


def test_small_gmres_converges_and_matches_dense():
    N = 2048
    L = O.levels_for(N, 256)
    b = O.uniform_unit_cube_rnd(N, 999)
    cells = O.build_binary_tree(b, L)
    k = O.Kernel()
    xt = O.xbody_uniform(N)
    B = O.dense_matvec(k, b, xt)
    A = O.H2MatrixSolver(k, 1e-10, 100, 0, cells, 2.0, b, L, 2000)
    M = O.H2MatrixSolver(k, 0.0, 100, 0, cells, 2.0, b, L, 2000)
    M.factorize()
    x, res, it = A.solve_gmres(1e-10, M, np.zeros(N), B, 10, 50)
    assert res[it] < 1e-10 and it <= 5
    r = B - O.dense_matvec(k, b, x)
    assert np.linalg.norm(r) / np.linalg.norm(B) < 1e-10


def test_ulv_exact_two_boxes_synthetic_complex():
    """Complex symmetric version (Helmholtz arithmetic): left transforms by
    U^H, right ones by conj(U) (h2matrix.cpp:373-396, 532); with the
    off-diagonal block U0[:, :k] S U1[:, :k]^T in the skeleton spans the ULV is
    exact."""
    rng = np.random.default_rng(1)
    n, k = 20, 6

    def cplx(*shape):
        return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)

    U = [np.linalg.qr(cplx(n, n))[0] for _ in range(2)]
    S12 = cplx(k, k)
    G1, G2 = cplx(n, n), cplx(n, n)
    A11 = G1 + G1.T + 8 * np.eye(n)
    A22 = G2 + G2.T + 8 * np.eye(n)
    A12 = U[0][:, :k] @ S12 @ U[1][:, :k].T
    Ad = np.block([[A11, A12], [A12.T, A22]])
    assert np.allclose(Ad, Ad.T)

    def lvl(l, nodes, ar, ac):
        return O.Level(l, (1 << l) - 1, nodes, np.array(ar), np.array(ac), np.zeros(nodes + 1, dtype=np.int64),
                       np.array([], dtype=np.int64))

    s = O.H2MatrixSolver.__new__(O.H2MatrixSolver)
    s.dt = np.complex128
    s.levels = 1
    leaf = lvl(1, 2, [0, 2, 4], [0, 1, 0, 1])
    root = lvl(0, 1, [0, 1], [0])
    z = lambda m: np.zeros((m, m), dtype=np.complex128)
    leaf.Dims = np.array([n, n]); leaf.DimsLr = np.array([k, k])
    leaf.Q = [U[0].copy(), U[1].copy()]; leaf.R = [z(n), z(n)]
    leaf.A = [A11.copy(), A12.copy(), A12.T.copy(), A22.copy()]
    leaf.NA = [(0, 0, 0), (0, 0, k), (0, k, 0), (0, k, k)]
    root.Dims = np.array([2 * k]); root.DimsLr = np.array([0])
    root.Q = [np.eye(2 * k, dtype=np.complex128)]; root.R = [z(2 * k)]; root.A = [z(2 * k)]
    s.A = [root, leaf]
    s.lenX = 2 * n
    s.factorize()
    b = cplx(2 * n)
    x = s.solve_precondition(b)
    xe = np.linalg.solve(Ad, b)
    assert np.linalg.norm(x - xe) / np.linalg.norm(xe) < 1e-12


def test_hss_mode_is_exact_inverse_of_its_h2_matrix_complex():
    """Helmholtz3D(1, 0.1) on the reference's sphere: in HSS mode (theta 0)
    the complex ULV of the fixed-rank H^2 matrix inverts that matrix, and the
    operator (ID, eps 1e-10) reproduces the dense complex product."""
    import math

    N = 1024
    L = O.levels_for(N, 128)
    g = math.pi * (3.0 - math.sqrt(5.0))
    i = np.arange(N)
    r = math.sqrt(N / (4 * math.pi))
    y = r - 2.0 * r * (i / (N - 1))
    ring = np.sqrt(r * r - y * y)
    b = np.ascontiguousarray(np.stack([ring * np.cos(g * i), y, ring * np.sin(g * i)], 1))
    cells = O.build_binary_tree(b, L)
    k = O.Kernel(O.HELMHOLTZ, 0.1, 1.0)
    x = O.xbody_uniform(N).astype(np.complex128) * (1 + 0.5j)
    A = O.H2MatrixSolver(k, 1e-10, 50, 0, cells, 1.0, b.copy(), L)
    assert O.solve_rel_err(A.matvec(x), O.dense_matvec(k, b, x)) < 1e-9
    M = O.H2MatrixSolver(k, 0.0, 40, 0, cells, 0.0, b.copy(), L)
    yv = M.matvec(x)
    M.factorize()
    z = M.solve_precondition(yv)
    assert np.linalg.norm(z - x) / np.linalg.norm(x) < 1e-9


def test_complex_gmres_reaches_dense_solution():
    """The reference's default run at N = 1024 (Helmholtz3D(1, 0.1) on the
    sphere, theta 1, rank 50): complex GMRES with the complex ULV
    preconditioner reaches 1e-10 and the dense solution."""
    import math

    N = 1024
    L = O.levels_for(N, 256)
    g = math.pi * (3.0 - math.sqrt(5.0))
    i = np.arange(N)
    r = math.sqrt(N / (4 * math.pi))
    y = r - 2.0 * r * (i / (N - 1))
    ring = np.sqrt(r * r - y * y)
    b = np.ascontiguousarray(np.stack([ring * np.cos(g * i), y, ring * np.sin(g * i)], 1))
    cells = O.build_binary_tree(b, L)
    k = O.Kernel(O.HELMHOLTZ, 0.1, 1.0)
    A = O.H2MatrixSolver(k, 1e-10, 50, 0, cells, 1.0, b.copy(), L)
    M = O.H2MatrixSolver(k, 0.0, 50, 0, cells, 1.0, b.copy(), L)
    M.factorize()
    x = O.xbody_uniform(N).astype(np.complex128)
    Kd = O.gen_matrix(k, b, b)
    B = Kd @ x
    X, res, it = A.solve_gmres(1e-10, M, np.zeros(N, np.complex128), B, 10, 50)
    assert res[it] < 1e-10 and it <= 5
    assert np.linalg.norm(Kd @ X - B) / np.linalg.norm(B) < 1e-9
    assert np.linalg.norm(X - np.linalg.solve(Kd, B)) / np.linalg.norm(x) < 1e-8
