"""Geometric, leaf-capped tree split (h2_build_tree_capped, a build
extension: the reference's median split gives equal leaves,
build_tree.cpp:67-99).  Host-only: the library's tree equals the oracle's
restatement bit for bit, every leaf holds leaf_min..leaf_max bodies, and on
clustered bodies the cuts follow the geometry (unequal leaves)."""
import numpy as np
import pytest

import h2_oracle as O
import mxc_b200 as m
from mxc_b200 import serving as S


@pytest.mark.parametrize("n,levels,lmin,lmax", [(20000, 6, 128, 512), (4096, 5, 32, 256), (3000, 4, 100, 300)])
def test_capped_tree_matches_oracle_and_respects_caps(n, levels, lmin, lmax):
    pts = S.gaussian_mixture_points(n, 32, seed=5)
    b = pts.copy()
    t = m.build_tree(b, levels, leaf_min=lmin, leaf_max=lmax)
    bo = pts.copy()
    c = O.build_binary_tree_capped(bo, levels, lmin, lmax)
    assert np.array_equal(b, bo)
    assert np.array_equal(t.child, c.child) and np.array_equal(t.body, c.body)
    assert np.array_equal(t.R, c.R) and np.array_equal(t.C, c.C)
    leaves = t.body[(1 << levels) - 1:]
    sizes = leaves[:, 1] - leaves[:, 0]
    assert sizes.min() >= lmin and sizes.max() <= lmax and sizes.sum() == n
    assert sizes.max() > sizes.min()  # clustered bodies: the cuts are not medians
    # near / far lists over the uneven tree are still a partition of all leaf pairs
    near = m.pair_csr("N", t, 2.0)
    assert near[0][-1] > 0


def test_capped_tree_rejects_infeasible_caps():
    b = np.random.default_rng(1).random((1000, 3))
    with pytest.raises(m.H2DevError):
        m.build_tree(b, 3, leaf_min=200, leaf_max=300)
