"""Serving loop: resident factored H^2 systems answering solve requests.

A `Server` keeps factored systems (H^2 operator A plus its ULV
preconditioner M) resident on the device, admits them against an HBM
budget, and answers `submit(system, B, tol)` requests with
ULV-preconditioned GMRES.  Batching is continuous: whenever a system is
idle, the right-hand sides queued for it (from any number of requests,
arrived at any time) are packed into one batch of up to `max_batch`
columns and solved by one batched GMRES call; requests that arrive while a
batch runs join the next one, and a request larger than the batch width is
spread over consecutive batches.  Each system has its own device handle
(stream), and `workers` host threads serve different systems at once, so
their kernels overlap on the GPU.  Every batch runs at the full batch width
(padding columns repeat the first right-hand side and are discarded), so a
system's launch plans are built once.

Admission: a system's footprint is the device memory its handle holds
after build, factorization and a warm-up solve (`Handle.memory`).  Before a
system is built, room for it is made under the budget: its footprint is
taken from an earlier build of the same system, else from a conservative
per-body estimate, and idle systems are evicted in least-recently-used order
(their solvers and handle are freed) until that much is free; the room stays
reserved while the build runs, so concurrent admissions cannot overcommit,
and the measured footprint replaces the reservation afterwards (evicting
more if the build came out larger).  A request for an evicted system
rebuilds it under the same rule.  Latency is measured per request from
`submit` to the completion of its last column.

Each column's GMRES is independent of the others in its batch (the batched
GMRES keeps one Krylov basis, Hessenberg matrix and convergence test per
column), so a result does not depend on what it was batched with beyond
rounding; `tests/test_serving.py` checks alone-versus-in-the-mix agreement.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from . import _lib as L
from .solver import H2MatrixSolver, Handle, Kernel, Laplace3D, build_tree, levels_for


def gaussian_mixture_points(n: int, ncomp: int = 32, seed: int = 0, sigma=(0.01, 0.2)) -> np.ndarray:
    """n points from a seeded mixture of ncomp isotropic Gaussians with means
    uniform in the unit cube and standard deviations uniform in `sigma`,
    folded back into the cube by reflection at its faces (the uneven-density
    inputs of the batching and serving configurations; reflection, unlike
    clipping, creates no coincident points)."""
    rng = np.random.default_rng(seed)
    means = rng.random((ncomp, 3))
    sig = rng.uniform(sigma[0], sigma[1], ncomp)
    comp = rng.integers(0, ncomp, n)
    pts = means[comp] + sig[comp, None] * rng.standard_normal((n, 3))
    pts = np.mod(pts, 2.0)
    pts = np.where(pts > 1.0, 2.0 - pts, pts)
    return np.ascontiguousarray(pts)


def unit_sphere_points(n: int, seed: int = 0) -> np.ndarray:
    """n points uniform on the unit sphere's surface (seeded): normalised
    standard-normal 3-vectors (the scale-up configuration's inputs)."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return np.ascontiguousarray(v)


@dataclass
class SystemSpec:
    """What a resident system is built from (kept so an evicted system can
    be rebuilt)."""
    points: np.ndarray  # N x 3, any order (the tree sorts them)
    kernel: Kernel = field(default_factory=Laplace3D)
    op_eps: float = 1e-8
    rank: int = 100
    samples: int = 4000
    op_samples: int = 0  # 0: same as samples
    theta: float = 2.0
    leaf: int = 256
    precision: int = L.FP32  # preconditioner precision; the operator is FP64
    device: int = 0
    # Operator near blocks and couplings stored in HBM, or evaluated inside
    # each matvec (H2DEV_OPT_MATRIX_FREE): a fraction of the memory, slower
    # matvecs; lets more large systems stay resident under one budget.
    matrix_free: bool = False
    # Each batched solve as one CUDA graph (H2DEV_OPT_GRAPH_SOLVE), captured
    # at the warm-up and replayed: no host round trip per Arnoldi step, so
    # systems served by concurrent workers do not wait on each other's syncs.
    graph_solve: bool = True


class ResidentSystem:
    """A built, factored system on its own device handle."""

    # Device bytes per body of a built system (operator at eps 1e-8 and an
    # FP32 rank-100 preconditioner held about 190 KB per body at 8,192 to
    # 262,144 bodies; with a matrix-free operator the preconditioner is most
    # of it): the admission estimate before a first build.
    BYTES_PER_BODY_ESTIMATE = 256 * 1024
    BYTES_PER_BODY_ESTIMATE_MATRIX_FREE = 128 * 1024

    @classmethod
    def estimate_footprint(cls, spec: SystemSpec) -> int:
        per = cls.BYTES_PER_BODY_ESTIMATE_MATRIX_FREE if spec.matrix_free else cls.BYTES_PER_BODY_ESTIMATE
        return int(per * spec.points.shape[0])

    def __init__(self, spec: SystemSpec, max_batch: int, warm: bool = True, inner: int = 10, outer: int = 50,
                 tol: float = 1e-10):
        self.spec = spec
        self.handle = Handle(spec.device)
        n = spec.points.shape[0]
        levels = levels_for(n, spec.leaf)
        # build_tree sorts the points in place (tree order); requests' vectors
        # are in that order, as in the reference.
        self.bodies = np.ascontiguousarray(spec.points, dtype=np.float64).copy()
        self.tree = build_tree(self.bodies, levels)
        ops = spec.op_samples or spec.samples
        self.handle.set_option(L.OPT_MATRIX_FREE, 1 if spec.matrix_free else 0)
        try:
            self.A = H2MatrixSolver(self.handle, spec.kernel, spec.op_eps, spec.rank, 0, self.tree, spec.theta,
                                    self.bodies, samples=ops, precision=L.FP64)
        finally:
            self.handle.set_option(L.OPT_MATRIX_FREE, 0)
        self.M = H2MatrixSolver(self.handle, spec.kernel, 0.0, spec.rank, 0, self.tree, spec.theta, self.bodies,
                                samples=spec.samples, precision=spec.precision)
        self.M.factorizeM()
        # Construction temporaries go back to the driver; the cache then
        # keeps only what a solve reuses, which the footprint includes.
        self.handle.trim()
        self.n = n
        self.max_batch = max_batch
        self.handle.set_option(L.OPT_GRAPH_SOLVE, 1 if spec.graph_solve else 0)
        if warm:
            # Builds the batch-width plans once, and with graph solves captures
            # the solve at the serving shape and tolerance (all measured in the
            # footprint).
            B = np.ones((n, max_batch), order="F")
            X = np.zeros((n, max_batch), order="F")
            self.A.solveGMRES(tol, self.M, X, B, inner, outer, early_exit=True)
        self.handle.synchronize()
        live, cached = self.handle.memory()
        self.footprint = live + cached

    def solve(self, B: np.ndarray, tol: float, inner: int, outer: int):
        X = np.zeros_like(B, order="F")
        rc = self.A.solveGMRES(tol, self.M, X, B, inner, outer, early_exit=True)
        resid = np.asarray(self.A.resid)
        iters = np.asarray(self.A.iters)
        return X, rc, resid, iters

    def close(self):
        self.A.close()
        self.M.close()
        self.handle.close()


@dataclass
class _Request:
    sid: int
    B: np.ndarray  # n x k, Fortran order
    tol: float
    t_submit: float
    future: cf.Future
    X: np.ndarray = None
    resid: np.ndarray = None  # final relative residual per column
    next_col: int = 0  # first column not yet handed to a batch
    done_cols: int = 0


class Server:
    """Continuous-batching solve server over resident systems."""

    def __init__(self, hbm_budget_bytes: int, max_batch: int = 16, workers: int = 2, inner: int = 10,
                 outer: int = 50, build_system: Optional[Callable[[SystemSpec, int], "ResidentSystem"]] = None,
                 estimate_footprint: Optional[Callable[[SystemSpec], int]] = None):
        self.budget = int(hbm_budget_bytes)
        self.max_batch = max_batch
        self.inner, self.outer = inner, outer
        self._specs: Dict[int, SystemSpec] = {}
        self._sys: Dict[int, ResidentSystem] = {}
        self._queue: Dict[int, collections.deque] = {}
        self._busy: set = set()
        self._last_use: Dict[int, float] = {}
        self._lock = threading.Condition()
        self._stop = False
        self._latency: List[float] = []
        self._columns_done = 0
        self._batches = 0
        self._t0 = time.perf_counter()
        # build_system(spec, max_batch) -> an object with n, footprint, solve(B, tol, inner, outer) and
        # close(); ResidentSystem by default (other builders serve host-side tests of the scheduler).
        if build_system is None:
            self._builder: Callable[[SystemSpec], ResidentSystem] = lambda s: ResidentSystem(
                s, self.max_batch, inner=self.inner, outer=self.outer)
        else:
            self._builder = lambda s: build_system(s, self.max_batch)
        # Footprint assumed for a system never built before: ResidentSystem's
        # per-body estimate by default; with another builder, the given
        # estimate or none (then room is made once the build is measured).
        if estimate_footprint is None:
            estimate_footprint = ResidentSystem.estimate_footprint if build_system is None else (lambda spec: 0)
        self._estimate: Callable[[SystemSpec], int] = estimate_footprint
        self._footprint_seen: Dict[int, int] = {}  # sid -> measured footprint of its last build
        self._reserved: Dict[int, int] = {}  # sid -> bytes held for a build in progress
        self._workers = [threading.Thread(target=self._work, daemon=True) for _ in range(workers)]
        for w in self._workers:
            w.start()

    # ------------------------------------------------------------ admission
    def resident_bytes(self) -> int:
        """Footprints of the resident systems plus room reserved for builds in progress."""
        return sum(s.footprint for s in self._sys.values()) + sum(self._reserved.values())

    def _evict_for(self, need: int, keep: int) -> None:
        """Evicts idle systems, least recently used first, until `need` more
        bytes fit (called with the lock held)."""
        while self.resident_bytes() + need > self.budget:
            idle = [sid for sid in self._sys if sid != keep and sid not in self._busy and not self._queue[sid]]
            if not idle:
                raise MemoryError("system does not fit in the HBM budget and no idle system can be evicted")
            victim = min(idle, key=lambda sid: self._last_use.get(sid, 0.0))
            self._sys.pop(victim).close()

    def _admit(self, sid: int) -> ResidentSystem:
        spec = self._specs[sid]
        with self._lock:
            # Make room before building: the build allocates all of its
            # device memory, so evicting afterwards would overshoot the budget.
            need = self._footprint_seen.get(sid) or self._estimate(spec)
            self._evict_for(need, keep=sid)
            self._reserved[sid] = need
        try:
            system = self._builder(spec)
        except BaseException:
            with self._lock:
                self._reserved.pop(sid, None)
            raise
        with self._lock:
            self._reserved.pop(sid, None)
            self._footprint_seen[sid] = system.footprint
            try:
                self._evict_for(system.footprint, keep=sid)
            except MemoryError:
                system.close()
                raise
            self._sys[sid] = system
            self._last_use[sid] = time.perf_counter()
        return system

    def add_system(self, spec: SystemSpec) -> int:
        """Builds, factors and admits a system; returns its id."""
        with self._lock:
            sid = len(self._specs)
            self._specs[sid] = spec
            self._queue[sid] = collections.deque()
        self._admit(sid)
        return sid

    def is_resident(self, sid: int) -> bool:
        with self._lock:
            return sid in self._sys

    # ------------------------------------------------------------ requests
    def submit(self, sid: int, B: np.ndarray, tol: float = 1e-10) -> cf.Future:
        """Queues B (n or n x k right-hand sides) for system `sid`; the future
        resolves to (X, per-column final relative residuals, latency s)."""
        B = np.asarray(B, dtype=np.float64)
        if B.ndim == 1:
            B = B[:, None]
        B = np.asfortranarray(B)
        fut: cf.Future = cf.Future()
        req = _Request(sid, B, tol, time.perf_counter(), fut, X=np.zeros_like(B, order="F"),
                       resid=np.zeros(B.shape[1]))
        with self._lock:
            if sid not in self._specs:
                raise KeyError(sid)
            self._queue[sid].append(req)
            self._lock.notify_all()
        return fut

    def _pick(self) -> Optional[int]:
        """System with the oldest waiting request among idle ones (lock held)."""
        best, t_best = None, None
        for sid, q in self._queue.items():
            if q and sid not in self._busy:
                t = q[0].t_submit
                if t_best is None or t < t_best:
                    best, t_best = sid, t
        return best

    def _work(self) -> None:
        while True:
            with self._lock:
                while not self._stop and self._pick() is None:
                    self._lock.wait()
                if self._stop:
                    return
                sid = self._pick()
                self._busy.add(sid)
                # Pack up to max_batch columns from the queue, oldest first.
                parts = []  # (request, first column, count)
                width = 0
                tol = None
                for req in list(self._queue[sid]):
                    if req.future.done():  # failed earlier: drop its remaining columns
                        self._queue[sid].remove(req)
                        continue
                    if width >= self.max_batch:
                        break
                    if tol is not None and req.tol != tol:
                        break
                    tol = req.tol
                    take = min(req.B.shape[1] - req.next_col, self.max_batch - width)
                    parts.append((req, req.next_col, take))
                    req.next_col += take
                    width += take
                    if req.next_col == req.B.shape[1]:
                        self._queue[sid].popleft()
                system = self._sys.get(sid)
            try:
                if system is None:
                    system = self._admit(sid)
                n = system.n
                Bb = np.empty((n, self.max_batch), order="F")
                c = 0
                for req, c0, k in parts:
                    Bb[:, c:c + k] = req.B[:, c0:c0 + k]
                    c += k
                Bb[:, c:] = Bb[:, :1]  # padding columns, discarded
                X, rc, resid, iters = system.solve(Bb, tol, self.inner, self.outer)
                t_done = time.perf_counter()
                finished = []
                with self._lock:
                    self._batches += 1
                    c = 0
                    for req, c0, k in parts:
                        if req.future.done():  # failed in another batch; its columns here are discarded
                            c += k
                            continue
                        req.X[:, c0:c0 + k] = X[:, c:c + k]
                        for j in range(k):
                            req.resid[c0 + j] = resid[int(iters[c + j]), c + j]
                        req.done_cols += k
                        c += k
                        if req.done_cols == req.B.shape[1]:
                            lat = t_done - req.t_submit
                            self._latency.append(lat)
                            self._columns_done += req.B.shape[1]
                            finished.append((req, lat))
                    self._last_use[sid] = t_done
                for req, lat in finished:
                    if not req.future.done():
                        req.future.set_result((req.X, req.resid, lat))
            except BaseException as e:  # propagate to every request in the batch
                with self._lock:
                    for req, _, _ in parts:
                        if not req.future.done():
                            req.future.set_exception(e)
                        # a failed request's columns still queued go nowhere
                        if req in self._queue[sid]:
                            self._queue[sid].remove(req)
            finally:
                with self._lock:
                    self._busy.discard(sid)
                    self._lock.notify_all()

    # ------------------------------------------------------------ reporting
    def stats(self) -> dict:
        with self._lock:
            lat = np.array(self._latency)
            elapsed = time.perf_counter() - self._t0
            return {"requests": int(lat.size), "columns": int(self._columns_done), "batches": int(self._batches),
                    "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
                    "p99_s": float(np.percentile(lat, 99)) if lat.size else None,
                    "elapsed_s": elapsed}

    def reset_stats(self) -> None:
        with self._lock:
            self._latency = []
            self._columns_done = 0
            self._batches = 0
            self._t0 = time.perf_counter()

    def close(self) -> None:
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        for w in self._workers:
            w.join()
        for s in self._sys.values():
            s.close()
        self._sys.clear()
