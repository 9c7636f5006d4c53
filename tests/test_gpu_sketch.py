"""Operator bases from the sketch of every far body (sampling mode 2).

The reference factors each box's whole far block (h2matrix.cpp:13-63,
h-matrix.cpp:97,122-127).  Mode 2 keeps every far body and runs the
column-pivoted QR on the random-sign sketch Omega XF (k_sketch.cu); the
oracle forms the same Omega (oracle/h2_oracle.py sketch_signs), so ranks and
skeletons agree up to rounding near the threshold, and the operator's
accuracy is that of the whole far field rather than of a strided sample.
"""
import numpy as np
import pytest

import h2_oracle as O
import mxc_b200 as m

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def sketch_solver(handle, k, eps, t, b, theta=2.0, samples=0):
    handle.set_option(m._lib.OPT_SAMPLING, m._lib.SAMPLING_SKETCH)
    try:
        return m.H2MatrixSolver(handle, k, eps, 100, 0, t, theta, b, samples=samples)
    finally:
        handle.set_option(m._lib.OPT_SAMPLING, m._lib.SAMPLING_STRIDED)


def test_sketch_signs_oracle_rule():
    """The sign matrix depends only on (row, body index); rows are balanced."""
    f = np.array([5, 17, 4096, 123456], dtype=np.int64)
    S = O.sketch_signs(130, f)
    assert S.shape == (130, 4) and set(np.unique(S)) <= {-1.0, 1.0}
    np.testing.assert_array_equal(O.sketch_signs(130, f[::-1]), S[:, ::-1])
    big = O.sketch_signs(256, np.arange(20000))
    assert abs(big.mean()) < 0.01


@pytest.fixture(scope="module")
def sk4096(handle):
    N = 4096
    L = m.levels_for(N, 256)
    b = m.uniform_unit_cube_rnd(N, 999)
    t = m.build_tree(b, L)
    cells = O.build_binary_tree(O.uniform_unit_cube_rnd(N, 999), L)
    A = sketch_solver(handle, m.Laplace3D(), 1e-10, t, b)
    Ao = O.H2MatrixSolver(O.Kernel(), 1e-10, 100, 0, cells, 2.0, b.copy(), L, 0, 2)
    return A, Ao, b, L


def test_sketch_ranks_and_skeletons_match_oracle(sk4096):
    A, Ao, b, L = sk4096
    for lvl in range(L + 1):
        d, r = A.level_dims(lvl)
        assert np.array_equal(d, Ao.A[lvl].Dims), lvl
        diff = np.abs(r - Ao.A[lvl].DimsLr)
        assert diff.max() <= 1 and (diff > 0).sum() <= max(1, len(r) // 8), (lvl, r, Ao.A[lvl].DimsLr)
    # leaf skeletons: the first rank bodies of each box, as sets
    S = A.export(L, m._lib.EXPORT_S).reshape(-1, 3)
    dims, ranks = A.level_dims(L)
    off = 0
    same = 0
    for i in range(len(dims)):
        ro = int(Ao.A[L].DimsLr[i])
        if ranks[i] == ro:
            got = {tuple(x) for x in S[off:off + ranks[i]]}
            exp = {tuple(x) for x in Ao.A[L].S[i][:ro]}
            same += got == exp
        off += dims[i]
    assert same >= len(dims) - 2


def test_sketch_matvec_vs_oracle_and_dense(sk4096, handle):
    A, Ao, b, L = sk4096
    x = m.uniform_rhs(b.shape[0])
    y = x.copy()
    A.matVecMul(y)
    yd = m.dense_matvec(handle, m.Laplace3D(), b, x)
    assert rel(y, Ao.matvec(x)) < 1e-10
    assert rel(y, yd) < 1e-10


def test_sketch_beats_strided_sampling(handle):
    """At 32,768 bodies a leaf's far list has ~30,000 bodies; 1,000 strided
    samples leave the operator far less accurate than the sketch of all of
    them at the same threshold."""
    N = 32768
    L = m.levels_for(N, 256)
    b = m.uniform_unit_cube_rnd(N, 7)
    t = m.build_tree(b, L)
    k = m.Laplace3D(1e-4)
    x = np.random.default_rng(11).random(N)
    yd = m.dense_matvec(handle, k, b, x)
    A1 = m.H2MatrixSolver(handle, k, 1e-11, 100, 0, t, 2.0, b, samples=1000)
    y1 = x.copy()
    A1.matVecMul(y1)
    A1.close()
    A2 = sketch_solver(handle, k, 1e-11, t, b)
    y2 = x.copy()
    A2.matVecMul(y2)
    A2.close()
    e1, e2 = rel(y1, yd), rel(y2, yd)
    assert e2 < 1e-11 and e2 < e1 / 10, (e1, e2)


def test_sketch_near_levels_plus_samples_matches_oracle(handle):
    """samples > 0 in sketch mode: the far boxes of the box's level and the
    two above in full, plus strided samples of the farther list; same set of
    bodies and signs as the oracle, so the same ranks (to rounding), and the
    operator as accurate as with every far body."""
    N = 16384
    L = m.levels_for(N, 256)
    b = m.uniform_unit_cube_rnd(N, 999)
    t = m.build_tree(b, L)
    cells = O.build_binary_tree(O.uniform_unit_cube_rnd(N, 999), L)
    k = m.Laplace3D(1e-4)
    A = sketch_solver(handle, k, 1e-11, t, b, samples=1000)
    Afull = sketch_solver(handle, k, 1e-11, t, b, samples=0)
    Ao = O.H2MatrixSolver(O.Kernel(O.LAPLACE, 1e-4), 1e-11, 100, 0, cells, 2.0, b.copy(), L, 1000, 2)
    for lvl in range(L + 1):
        d, r = A.level_dims(lvl)
        assert np.array_equal(d, Ao.A[lvl].Dims), lvl
        diff = np.abs(r - Ao.A[lvl].DimsLr)
        assert diff.max() <= 1 and (diff > 0).sum() <= max(1, len(r) // 8), (lvl, r, Ao.A[lvl].DimsLr)
    x = np.random.default_rng(2).random(N)
    yd = m.dense_matvec(handle, k, b, x)
    y = x.copy()
    A.matVecMul(y)
    yf = x.copy()
    Afull.matVecMul(yf)
    assert rel(y, Ao.matvec(x)) < 1e-11
    # Cheaper than the whole far field, and less accurate (at 16,384 bodies
    # about 7x the full sketch's error, still well inside the threshold).
    assert rel(yf, yd) < 1e-12 and rel(y, yd) < 1e-11
