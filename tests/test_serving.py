"""Serving loop: continuous batching, HBM-budget admission, results alone
versus in the mix.

The scheduler tests (no GPU) run the Server over a host-side stand-in for a
resident system whose solve is X = B / 2 (optionally slow), so that column
packing, request splitting, eviction and re-admission are checked exactly.
The GPU test runs two real systems and checks that a right-hand side solved
alone and solved while batched with other requests (of both systems, in
flight together) give the same solution within 1e-10 relative, both
meeting the tolerance by dense residual.
"""
import threading
import time

import numpy as np
import pytest

import mxc_b200 as m
from mxc_b200 import serving as S


class FakeSystem:
    built = []

    def __init__(self, spec, max_batch, footprint=10, delay=0.0):
        self.n = spec.points.shape[0]
        self.footprint = footprint
        self.delay = delay
        self.widths = []
        self.closed = False
        FakeSystem.built.append(self)

    def solve(self, B, tol, inner, outer):
        self.widths.append(B.shape[1])
        if self.delay:
            time.sleep(self.delay)
        k = B.shape[1]
        return B / 2.0, 0, np.zeros((outer + 1, k)), np.zeros(k, dtype=np.int64)

    def close(self):
        self.closed = True


def spec(n=50, seed=0):
    return S.SystemSpec(points=np.random.default_rng(seed).random((n, 3)))


def test_requests_are_packed_split_and_returned_in_order():
    FakeSystem.built = []
    srv = S.Server(hbm_budget_bytes=100, max_batch=16, workers=1, build_system=lambda s, mb: FakeSystem(s, mb))
    try:
        sid = srv.add_system(spec())
        rng = np.random.default_rng(1)
        Bs = [rng.random((50, k)) for k in (3, 20, 5, 1, 16)]
        futs = [srv.submit(sid, B) for B in Bs]
        for B, f in zip(Bs, futs):
            X, resid, lat = f.result(timeout=10)
            np.testing.assert_array_equal(X, B / 2.0)
            assert X.shape == B.shape and lat >= 0
        st = srv.stats()
        assert st["requests"] == 5 and st["columns"] == 45
        # every batch runs at the full width (padding), and 45 columns need >= 3 batches
        assert all(w == 16 for w in FakeSystem.built[0].widths)
        assert st["batches"] >= 3
    finally:
        srv.close()


def test_requests_arriving_during_a_batch_join_the_next_one():
    FakeSystem.built = []
    srv = S.Server(hbm_budget_bytes=100, max_batch=16, workers=1,
                   build_system=lambda s, mb: FakeSystem(s, mb, delay=0.3))
    try:
        sid = srv.add_system(spec())
        f0 = srv.submit(sid, np.ones((50, 2)))
        time.sleep(0.1)  # the first batch is running now
        later = [srv.submit(sid, np.full((50, 3), float(i))) for i in range(4)]
        for f in [f0] + later:
            f.result(timeout=10)
        # the four late requests (12 columns) were packed into one batch
        assert srv.stats()["batches"] == 2
    finally:
        srv.close()


def test_admission_evicts_least_recently_used_idle_system_and_readmits():
    FakeSystem.built = []
    srv = S.Server(hbm_budget_bytes=25, max_batch=4, workers=1, build_system=lambda s, mb: FakeSystem(s, mb))
    try:
        a = srv.add_system(spec(seed=1))
        b = srv.add_system(spec(seed=2))
        srv.submit(a, np.ones(50)).result(timeout=10)  # a used after b: b is LRU
        c = srv.add_system(spec(seed=3))  # 3 x 10 > 25: evicts b
        assert srv.is_resident(a) and srv.is_resident(c) and not srv.is_resident(b)
        assert FakeSystem.built[1].closed
        X, _, _ = srv.submit(b, np.full(50, 4.0)).result(timeout=10)  # b rebuilt, LRU (a) evicted
        np.testing.assert_array_equal(X[:, 0], np.full(50, 2.0))
        assert srv.is_resident(b) and srv.resident_bytes() <= 25
    finally:
        srv.close()


def test_admission_makes_room_before_building():
    """With an estimate, idle systems are evicted before the new one is
    built, so the build never runs on top of a full budget."""
    FakeSystem.built = []
    seen = []
    holder = {}

    def build(s, mb):
        srv_ = holder["srv"]
        seen.append(sum(x.footprint for x in srv_._sys.values()))
        return FakeSystem(s, mb, footprint=40)

    srv = S.Server(hbm_budget_bytes=100, max_batch=4, workers=1, build_system=build,
                   estimate_footprint=lambda sp: 40)
    holder["srv"] = srv
    try:
        for i in range(3):
            srv.add_system(spec(seed=i))
        # the third build saw at most 60 bytes resident (one system evicted first)
        assert seen == [0, 40, 40] and srv.resident_bytes() <= 100
    finally:
        srv.close()


class FailingSystem(FakeSystem):
    def solve(self, B, tol, inner, outer):
        if len(self.widths) == 0:
            self.widths.append(B.shape[1])
            raise RuntimeError("injected device failure")
        return super().solve(B, tol, inner, outer)


def test_failed_batch_drops_the_rest_of_its_requests():
    """A request split over batches fails with its first batch; its queued
    columns are dropped and later batches complete the other requests."""
    FakeSystem.built = []
    srv = S.Server(hbm_budget_bytes=100, max_batch=4, workers=1,
                   build_system=lambda s, mb: FailingSystem(s, mb, delay=0.05))
    try:
        sid = srv.add_system(spec())
        big = srv.submit(sid, np.ones((50, 10)))  # 3 batches; the first fails
        others = [srv.submit(sid, np.full((50, 2), float(i))) for i in range(3)]
        with pytest.raises(RuntimeError):
            big.result(timeout=10)
        for i, f in enumerate(others):
            X, _, _ = f.result(timeout=10)
            np.testing.assert_array_equal(X, np.full((50, 2), i / 2.0))
    finally:
        srv.close()


def test_system_larger_than_budget_is_refused():
    srv = S.Server(hbm_budget_bytes=5, max_batch=4, workers=1, build_system=lambda s, mb: FakeSystem(s, mb))
    try:
        with pytest.raises(MemoryError):
            srv.add_system(spec())
    finally:
        srv.close()


def test_gaussian_mixture_points_are_seeded_and_in_the_cube():
    p = S.gaussian_mixture_points(5000, seed=4)
    q = S.gaussian_mixture_points(5000, seed=4)
    assert np.array_equal(p, q) and p.min() >= 0.0 and p.max() <= 1.0
    assert not np.array_equal(p, S.gaussian_mixture_points(5000, seed=5))


@pytest.mark.gpu
def test_result_alone_equals_result_in_the_mix(handle):
    k = m.Laplace3D(1e-3)
    specs = [S.SystemSpec(points=m.uniform_unit_cube_rnd(4096, 11), kernel=k, op_eps=1e-10, rank=64, samples=1000),
             S.SystemSpec(points=S.gaussian_mixture_points(4096, seed=12), kernel=k, op_eps=1e-10, rank=64,
                          samples=1000)]
    srv = S.Server(hbm_budget_bytes=40 << 30, max_batch=16, workers=2)
    try:
        sids = [srv.add_system(sp) for sp in specs]
        rng = np.random.default_rng(13)
        probe = rng.random(4096)
        X_alone, res_alone, _ = srv.submit(sids[0], probe).result(timeout=300)
        # The same right-hand side in the mix: requests of both systems, of
        # several widths, submitted together from two threads.
        futs = []

        def load(sid, count):
            for i in range(count):
                futs.append(srv.submit(sid, rng.random((4096, 1 + (i * 7) % 12))))

        th = [threading.Thread(target=load, args=(sids[1], 6)), threading.Thread(target=load, args=(sids[0], 3))]
        for t in th:
            t.start()
        mid = srv.submit(sids[0], np.column_stack([rng.random(4096), probe, rng.random(4096)]))
        for t in th:
            t.join()
        X_mix, res_mix, _ = mid.result(timeout=300)
        for f in futs:
            f.result(timeout=300)
        x0, x1 = X_alone[:, 0], X_mix[:, 1]
        assert np.linalg.norm(x1 - x0) / np.linalg.norm(x0) < 1e-10
        assert res_alone[0] < 1e-10 and res_mix[1] < 1e-10
        # dense check of the probe's solution (tree-ordered bodies of system 0)
        sys0 = srv._sys[sids[0]]
        r = probe - m.dense_matvec(handle, k, sys0.bodies, x0)
        assert np.linalg.norm(r) / np.linalg.norm(probe) < 1e-8
        st = srv.stats()
        assert st["requests"] == 11 and st["p99_s"] >= st["p50_s"] > 0
    finally:
        srv.close()
