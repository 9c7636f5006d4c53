"""Pin the oracle and the library's host plan to the reference's own outputs.

The fixtures come from the reference's build_tree.cpp / test_funcs.hpp /
kernel.hpp compiled under oracle/_ref (tests/golden/make_fixtures.py).
Everything here is bit-exact except Yukawa, whose exp() may differ by an ulp
between numpy and glibc.
"""
import math

import numpy as np
import pytest

import h2_oracle as O
import mxc_b200 as m
from conftest import golden_cases, load_golden

CASES = golden_cases()


@pytest.fixture(params=CASES, ids=[c.split("/")[-1][:-4] for c in CASES])
def gold(request):
    return load_golden(request.param)


def test_fixtures_present():
    assert len(CASES) >= 3


def test_oracle_points_and_rhs(gold):
    N, seed = int(gold["N"]), int(gold["seed"])
    b = O.uniform_unit_cube_rnd(N, seed)
    L = int(gold["levels"])
    O.build_binary_tree(b, L)
    assert np.array_equal(b, gold["bodies"])
    assert np.array_equal(O.xbody_uniform(N), gold["xbody"])


def test_oracle_tree_and_lists(gold):
    N, seed, L = int(gold["N"]), int(gold["seed"]), int(gold["levels"])
    assert O.levels_for(N, int(gold["leaf"])) == L
    b = O.uniform_unit_cube_rnd(N, seed)
    cells = O.build_binary_tree(b, L)
    for key, arr in (("child", cells.child), ("body", cells.body), ("R", cells.R), ("C", cells.C)):
        assert np.array_equal(arr, gold[key]), key
    for name, kind, th in (("near", "N", float(gold["theta"])), ("far", "F", float(gold["theta"])), ("far0", "F", 0.0)):
        csr = O.build_csr(kind, cells, th)
        assert np.array_equal(csr.RowIndex, gold[name + "_row"]), name
        assert np.array_equal(csr.ColIndex, gold[name + "_col"]), name


def test_oracle_kernel_values(gold):
    b = gold["bodies"]
    ij = gold["probe_ij"]
    lap = O.Kernel(O.LAPLACE, 1.0)
    yuk = O.Kernel(O.YUKAWA, 1.0, 1.0)
    vl = np.array([O.gen_matrix(lap, b[i:i + 1], b[j:j + 1])[0, 0] for i, j in ij])
    vy = np.array([O.gen_matrix(yuk, b[i:i + 1], b[j:j + 1])[0, 0] for i, j in ij])
    assert np.array_equal(vl, gold["probe_laplace"])
    np.testing.assert_allclose(vy, gold["probe_yukawa"], rtol=4e-16, atol=0)
    # Helmholtz3D(1, 0.1), the reference's default kernel (complex): numpy's
    # complex exp against glibc's, within an ulp or so of the magnitude
    helm = O.Kernel(O.HELMHOLTZ, 0.1, 1.0)
    vh = np.array([O.gen_matrix(helm, b[i:i + 1], b[j:j + 1])[0, 0] for i, j in ij])
    assert np.max(np.abs(vh - gold["probe_helmholtz"]) / np.abs(gold["probe_helmholtz"])) < 6e-16


def test_mesh_sphere(gold):
    """mesh_sphere(N, sqrt(N / 4 pi)) of the reference (main.cpp:68) against
    the Python API's restatement (cos/sin of numpy vs glibc: within an ulp)."""
    import mxc_b200 as m

    ref = gold["mesh_sphere"]
    n = ref.shape[0]
    got = m.mesh_sphere(n, math.sqrt(n / (4 * math.pi)))
    assert np.array_equal(got[:, 1], ref[:, 1])
    np.testing.assert_allclose(got, ref, rtol=0, atol=4e-16 * math.sqrt(n))


def test_library_host_plan(gold):
    """The library's C++ host plan (points, rhs, tree, CSR lists) matches the reference bit for bit."""
    N, seed, L = int(gold["N"]), int(gold["seed"]), int(gold["levels"])
    assert m.levels_for(N, int(gold["leaf"])) == L
    b = m.uniform_unit_cube_rnd(N, seed)
    t = m.build_tree(b, L)
    assert np.array_equal(b, gold["bodies"])
    assert np.array_equal(m.uniform_rhs(N), gold["xbody"])
    for key, arr in (("child", t.child), ("body", t.body), ("R", t.R), ("C", t.C)):
        assert np.array_equal(arr, gold[key]), key
    for name, kind, th in (("near", "N", float(gold["theta"])), ("far", "F", float(gold["theta"])), ("far0", "F", 0.0)):
        row, col = m.pair_csr(kind, t, th)
        assert np.array_equal(row, gold[name + "_row"]), name
        assert np.array_equal(col, gold[name + "_col"]), name


def test_sampling_rule_matches_oracle():
    """Far-list sampling (build extension) picks the same rows in both."""
    ranges = [(0, 100), (250, 260), (1000, 1733)]
    idx = np.concatenate([np.arange(a, b) for a, b in ranges])
    for s in (0, 1, 7, 500, 843, 844, 5000):
        keep = O.sample_indices(len(idx), s)
        exp = idx[keep]
        assert len(exp) == (len(idx) if s <= 0 or s >= len(idx) else s)
