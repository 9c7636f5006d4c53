"""FP64 CPU restatement of delta-leader/mxc's H^2 solver path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``mxc_b200``) imports this
module; only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline / reference arm use it, and only as the checker.

Every matrix of the reference is ``std::complex<double>``.  For the real
kernels on this path (Laplace3D, Yukawa3D) every imaginary part stays zero,
so ``adjoint`` reduces to ``transpose`` and ``conjugate`` to the identity and
this restatement works in real FP64.  For Helmholtz3D (kernel.hpp:63-74, the
reference's default) it works in complex128 with the reference's own
``adjoint`` / ``transpose`` / ``conjugate`` placements (h2matrix.cpp:266,
373-396, 532), Eigen's complex Householder rules and GMRES with adjoint inner
products (solver.cpp:151-197).

Pinning: the point generator, tree, Near/Far lists and kernel values are
checked bit-for-bit against the reference's own build_tree.cpp /
test_funcs.hpp / kernel.hpp compiled under ``oracle/_ref`` (fixtures in
``tests/golden``).  The dense algebra (Eigen 3.4 HouseholderQR,
ColPivHouseholderQR, PartialPivLU) cannot be built here (no Eigen, no MPI),
so that part of the restatement is *parity unpinned* against the reference
binary; it is checked against its own mathematical invariants (dense matvec
residuals, exact-solution recovery) instead.

Sampling (``samples``): the reference code uses every far body of a box
(h-matrix.cpp:97,122-127).  ``samples > 0`` caps that list at ``samples``
rows, chosen with the deterministic stride rule of ``sample_indices``; this is
a build extension named by the benchmark configurations, and ``samples <= 0``
reproduces the reference exactly.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla

# --------------------------------------------------------------------------
# Random inputs (test_funcs.hpp:31-41, main.cpp:73-76)
# --------------------------------------------------------------------------


def uniform_unit_cube_rnd(n: int, seed: int, diameter: float = 1.0, dim: int = 3) -> np.ndarray:
    """std::mt19937(seed) + uniform_real_distribution(0, diameter), test_funcs.hpp:31-41.

    libstdc++'s generate_canonical<double, 53> takes two 32-bit draws per
    double: (g0 + g1 * 2^32) / 2^64, rounded once in double.
    """
    bg = np.random.MT19937()
    bg._legacy_seeding(seed)
    draws = 2 * 3 * n
    raw = bg.random_raw(draws).astype(np.uint64)
    g0 = raw[0::2].astype(np.float64)
    g1 = raw[1::2].astype(np.float64)
    u = (g0 + g1 * 4294967296.0) / 18446744073709551616.0
    u = np.where(u >= 1.0, np.nextafter(1.0, 0.0), u)
    vals = u * diameter + 0.0
    out = vals.reshape(n, 3).copy()
    if dim < 3:
        # test_funcs.hpp:39 draws only for the first ``dim`` coordinates.
        raise NotImplementedError("only dim == 3 is on the solver path")
    return out


class _MT19937_64:
    """std::mt19937_64 with the default seed 5489 (used by main.cpp:73)."""

    N, M = 312, 156
    A = np.uint64(0xB5026F5AA96619E9)
    UM = np.uint64(0xFFFFFFFF80000000)
    LM = np.uint64(0x7FFFFFFF)

    def __init__(self, seed: int = 5489):
        mt = [0] * self.N
        mt[0] = seed & 0xFFFFFFFFFFFFFFFF
        for i in range(1, self.N):
            prev = mt[i - 1]
            mt[i] = (6364136223846793005 * (prev ^ (prev >> 62)) + i) & 0xFFFFFFFFFFFFFFFF
        self.mt = np.array(mt, dtype=np.uint64)

    def _twist(self):
        mt = self.mt
        n, m = self.N, self.M
        one = np.uint64(1)
        # i in [0, n-m): reads old mt[i+1], old mt[i+m]
        y = (mt[0:n - m] & self.UM) | (mt[1:n - m + 1] & self.LM)
        mt[0:n - m] = mt[m:n] ^ (y >> one) ^ np.where((y & one) == one, self.A, np.uint64(0))
        # i in [n-m, n-1): reads old mt[i+1], new mt[i+m-n]
        y = (mt[n - m:n - 1] & self.UM) | (mt[n - m + 1:n] & self.LM)
        mt[n - m:n - 1] = mt[0:m - 1] ^ (y >> one) ^ np.where((y & one) == one, self.A, np.uint64(0))
        y = (mt[n - 1] & self.UM) | (mt[0] & self.LM)
        mt[n - 1] = mt[m - 1] ^ (y >> one) ^ (self.A if (int(y) & 1) else np.uint64(0))

    def draws(self, count: int) -> np.ndarray:
        out = np.empty(count, dtype=np.uint64)
        got = 0
        while got < count:
            self._twist()
            y = self.mt.copy()
            y ^= (y >> np.uint64(29)) & np.uint64(0x5555555555555555)
            y ^= (y << np.uint64(17)) & np.uint64(0x71D67FFFEDA60000)
            y ^= (y << np.uint64(37)) & np.uint64(0xFFF7EEE000000000)
            y ^= y >> np.uint64(43)
            take = min(self.N, count - got)
            out[got:got + take] = y[:take]
            got += take
        return out


def xbody_uniform(n: int) -> np.ndarray:
    """Default-seeded mt19937_64 + uniform_real_distribution(0,1): main.cpp:73-76."""
    g = _MT19937_64().draws(n)
    u = g.astype(np.float64) / 18446744073709551616.0
    return np.where(u >= 1.0, np.nextafter(1.0, 0.0), u)


# --------------------------------------------------------------------------
# Kernels (kernel.hpp:28-50, kernel.cpp:71-85)
# --------------------------------------------------------------------------

LAPLACE, YUKAWA, QUADRATIC, HELMHOLTZ = 0, 1, 2, 3


@dataclass
class Kernel:
    kind: int = LAPLACE
    singularity: float = 1.0  # ctor argument s; the diagonal value is 1/s
    alpha: float = 1.0        # Yukawa decay, Helmholtz wave number

    @property
    def dtype(self):
        """complex128 for Helmholtz3D (kernel.hpp:63-74), float64 otherwise."""
        return np.complex128 if self.kind == HELMHOLTZ else np.float64

    def eval_d(self, d: np.ndarray) -> np.ndarray:
        with np.errstate(divide="ignore", invalid="ignore"):
            if self.kind == HELMHOLTZ:
                v = np.exp(-1j * self.alpha * d) / d
            elif self.kind == LAPLACE:
                v = 1.0 / d
            elif self.kind == YUKAWA:
                v = np.exp(-self.alpha * d) / d
            elif self.kind == QUADRATIC:
                # not a reference kernel: exactly low-rank off-diagonal blocks
                v = d * d + self.alpha
            else:
                raise ValueError("kernel kind")
        return np.where(d == 0.0, 1.0 / self.singularity, v)


def hypot3(dx: np.ndarray, dy: np.ndarray, dz: np.ndarray) -> np.ndarray:
    """libstdc++ std::hypot(x, y, z): a * sqrt((x/a)^2 + (y/a)^2 + (z/a)^2), a = max |.|."""
    dx = np.abs(dx)
    dy = np.abs(dy)
    dz = np.abs(dz)
    a = np.maximum(np.maximum(dx, dy), dz)
    with np.errstate(divide="ignore", invalid="ignore"):
        sx = dx / a
        sy = dy / a
        sz = dz / a
        r = a * np.sqrt(sx * sx + sy * sy + sz * sz)
    return np.where(a == 0.0, 0.0, r)


def gen_matrix(kern: Kernel, bi: np.ndarray, bj: np.ndarray) -> np.ndarray:
    """kernel.cpp:71-85: A[iy, ix] = K(hypot(bi[iy] - bj[ix])), returned as an (m, n) array."""
    bi = np.asarray(bi, dtype=np.float64).reshape(-1, 3)
    bj = np.asarray(bj, dtype=np.float64).reshape(-1, 3)
    d = hypot3(bi[:, None, 0] - bj[None, :, 0], bi[:, None, 1] - bj[None, :, 1],
               bi[:, None, 2] - bj[None, :, 2])
    return kern.eval_d(d)


def dense_matvec(kern: Kernel, bodies: np.ndarray, x: np.ndarray, chunk: int = 2048) -> np.ndarray:
    """y = A_dense x with A generated block-row by block-row (never stored whole)."""
    n = bodies.shape[0]
    x2 = x.reshape(n, -1)
    y = np.zeros(x2.shape, dtype=np.result_type(x2, kern.dtype))
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        y[s:e] = gen_matrix(kern, bodies[s:e], bodies) @ x2
    return y.reshape(x.shape)


# --------------------------------------------------------------------------
# Tree and admissibility (build_tree.cpp:8-99)
# --------------------------------------------------------------------------


@dataclass
class Cells:
    child: np.ndarray  # (ncells, 2) int64
    body: np.ndarray   # (ncells, 2) int64
    R: np.ndarray      # (ncells, 3)
    C: np.ndarray      # (ncells, 3)

    @property
    def ncells(self) -> int:
        return self.child.shape[0]


def get_bounds(b: np.ndarray):
    """build_tree.cpp:8-22."""
    mn = b.min(axis=0)
    mx = b.max(axis=0)
    C = (mn + mx) * 0.5
    R = np.where((mn == mx) & (mn == 0.0), 0.0, (mx - mn) * 0.5 + 1.0e-8)
    return R, C


def build_binary_tree(bodies: np.ndarray, levels: int) -> Cells:
    """build_tree.cpp:67-99: median split along the longest dimension; sorts ``bodies`` in place.

    std::sort is not stable; for points with distinct coordinates (the random
    inputs on this path) any correct sort gives the same order.
    """
    nb = bodies.shape[0]
    nleaf = 1 << levels
    ncells = 2 * nleaf - 1
    child = np.full((ncells, 2), -1, dtype=np.int64)
    body = np.full((ncells, 2), -1, dtype=np.int64)
    R = np.zeros((ncells, 3))
    C = np.zeros((ncells, 3))
    body[0] = (0, nb)
    R[0], C[0] = get_bounds(bodies)
    for i in range(nleaf - 1):
        sdim = int(np.argmax(R[i]))  # std::max_element: first maximum
        b0, b1 = body[i]
        seg = bodies[b0:b1]
        order = np.argsort(seg[:, sdim], kind="stable")
        bodies[b0:b1] = seg[order]
        c0 = 2 * i + 1
        child[i] = (c0, c0 + 2)
        loc = b0 + (b1 - b0) // 2
        body[c0] = (b0, loc)
        body[c0 + 1] = (loc, b1)
        R[c0], C[c0] = get_bounds(bodies[b0:loc])
        R[c0 + 1], C[c0 + 1] = get_bounds(bodies[loc:b1])
    return Cells(child, body, R, C)


def build_binary_tree_capped(bodies: np.ndarray, levels: int, leaf_min: int, leaf_max: int) -> Cells:
    """Geometric, leaf-capped split (build extension; the reference only has
    the median split of build_tree.cpp:67-99): each cell is sorted along its
    longest extent as in build_binary_tree, cut at the first body at or past
    its bounding-box centre, the cut clamped so each child can still give its
    h = 2^(levels - l - 1) leaves leaf_min..leaf_max bodies."""
    nb = bodies.shape[0]
    nleaf = 1 << levels
    ncells = 2 * nleaf - 1
    child = np.full((ncells, 2), -1, dtype=np.int64)
    body = np.full((ncells, 2), -1, dtype=np.int64)
    R = np.zeros((ncells, 3))
    C = np.zeros((ncells, 3))
    body[0] = (0, nb)
    R[0], C[0] = get_bounds(bodies)
    for i in range(nleaf - 1):
        level = int(math.floor(math.log2(i + 1)))
        sdim = int(np.argmax(R[i]))
        b0, b1 = body[i]
        seg = bodies[b0:b1]
        order = np.argsort(seg[:, sdim], kind="stable")
        bodies[b0:b1] = seg[order]
        n = int(b1 - b0)
        left = int(np.searchsorted(bodies[b0:b1, sdim], C[i, sdim], side="left"))
        h = 1 << (levels - level - 1)
        lo, hi = max(leaf_min * h, n - leaf_max * h), min(leaf_max * h, n - leaf_min * h)
        left = min(max(left, lo), hi) if lo <= hi else n // 2
        c0 = 2 * i + 1
        child[i] = (c0, c0 + 2)
        mid = b0 + left
        body[c0] = (b0, mid)
        body[c0 + 1] = (mid, b1)
        R[c0], C[c0] = get_bounds(bodies[b0:mid])
        R[c0 + 1], C[c0 + 1] = get_bounds(bodies[mid:b1])
    return Cells(child, body, R, C)


@dataclass
class CSR:
    RowIndex: np.ndarray
    ColIndex: np.ndarray

    def lookup(self, i: int, j: int) -> int:
        if i < 0 or i + 1 >= len(self.RowIndex):
            return -1
        s, e = self.RowIndex[i], self.RowIndex[i + 1]
        hits = np.nonzero(self.ColIndex[s:e] == j)[0]
        return int(s + hits[0]) if len(hits) else -1


def build_csr(kind: str, cells: Cells, theta: float) -> CSR:
    """build_tree.cpp:24-58: dual-tree recursion from (0, 0), emitted level by level.

    Admissible iff |c_i - c_j|^2 > theta * (|r_i|^2 + |r_j|^2), each sum taken
    left to right as std::transform_reduce does for three terms.
    """
    pairs_i = [np.array([0], dtype=np.int64)]
    pairs_j = [np.array([0], dtype=np.int64)]
    out_i, out_j = [], []
    cur_i, cur_j = pairs_i[0], pairs_j[0]
    while len(cur_i):
        d = cells.C[cur_i] - cells.C[cur_j]
        dC = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        ri, rj = cells.R[cur_i], cells.R[cur_j]
        dR1 = (ri[:, 0] * ri[:, 0] + ri[:, 1] * ri[:, 1]) + ri[:, 2] * ri[:, 2]
        dR2 = (rj[:, 0] * rj[:, 0] + rj[:, 1] * rj[:, 1]) + rj[:, 2] * rj[:, 2]
        admis = dC > theta * (dR1 + dR2)
        emit = admis if kind == "F" else ~admis
        out_i.append(cur_i[emit])
        out_j.append(cur_j[emit])
        rec = (~admis) & (cells.child[cur_i, 0] >= 0) & (cells.child[cur_j, 0] >= 0)
        ci, cj = cur_i[rec], cur_j[rec]
        if len(ci) == 0:
            break
        # children are (c0, c0+1) for each; all four combinations
        a0 = cells.child[ci, 0]
        b0 = cells.child[cj, 0]
        cur_i = np.concatenate([a0, a0, a0 + 1, a0 + 1])
        cur_j = np.concatenate([b0, b0 + 1, b0, b0 + 1])
    I = np.concatenate(out_i)
    J = np.concatenate(out_j)
    order = np.lexsort((J, I))
    I, J = I[order], J[order]
    row = np.zeros(cells.ncells + 1, dtype=np.int64)
    np.add.at(row, I + 1, 1)
    row = np.cumsum(row)
    return CSR(row, J.astype(np.int64))


# --------------------------------------------------------------------------
# Far-body lists (h-matrix.cpp:72-137, far lists only) and sampling
# --------------------------------------------------------------------------


def far_body_lists(cells: Cells, far: CSR, levels: int):
    """Per box: the list of far body *ranges* (parent's list, then own far boxes).

    Returned as {cell: [(b0, b1), ...]} for every cell at levels 1..L; the
    root (level 0) has none (its Hmatrix is never constructed, solver.cpp:31).
    """
    lists = {0: []}
    for l in range(1, levels + 1):
        for c in range((1 << l) - 1, (1 << (l + 1)) - 1):
            parent = (c - 1) // 2
            rng = list(lists[parent])
            for k in range(far.RowIndex[c], far.RowIndex[c + 1]):
                x = far.ColIndex[k]
                rng.append((int(cells.body[x, 0]), int(cells.body[x, 1])))
            lists[c] = rng
    lists[0] = []
    return lists


def sample_indices(total: int, samples: int) -> np.ndarray:
    """Rows kept from a far list of ``total`` bodies: all of them when
    ``samples <= 0`` or ``samples >= total``, else floor(j * total / samples)."""
    if samples <= 0 or samples >= total:
        return np.arange(total, dtype=np.int64)
    j = np.arange(samples, dtype=np.int64)
    return (j * total) // samples


def far_body_groups(cells: Cells, far: CSR, levels: int):
    """{cell: [first range index of each tree-level group]} matching far_body_lists."""
    lists = far_body_lists(cells, far, levels)
    groups = {0: []}
    for l in range(1, levels + 1):
        for c in range((1 << l) - 1, (1 << (l + 1)) - 1):
            parent = (c - 1) // 2
            groups[c] = list(groups[parent]) + [len(lists[parent]) if parent else 0]
    return groups


def geometric_allocation(gsize, samples: int):
    """Level-geometric split of ``samples`` over groups (last = nearest)."""
    G = len(gsize)
    alloc = [0] * G
    rem = samples
    for g in range(G - 1, -1, -1):
        share = rem if g == 0 else (rem + 1) // 2
        alloc[g] = min(gsize[g], share)
        rem -= alloc[g]
    for g in range(G - 1, -1, -1):
        if rem <= 0:
            break
        extra = min(gsize[g] - alloc[g], rem)
        alloc[g] += extra
        rem -= extra
    return alloc


SKETCH_MUL_F = np.uint64(0x9E3779B97F4A7C15)
SKETCH_MUL_W = np.uint64(0xD1B54A32D192ED03)
SKETCH_ADD = np.uint64(0x2545F4914F6CDD1D)


def _mix64(z: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser (Steele, Lea and Flood 2014), uint64 wrap-around."""
    z = z ^ (z >> np.uint64(30))
    z = z * np.uint64(0xBF58476D1CE4E5B9)
    z = z ^ (z >> np.uint64(27))
    z = z * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def sketch_signs(p: int, fidx: np.ndarray) -> np.ndarray:
    """(p, len(fidx)) random-sign matrix of the full-far-field sketch.

    Entry (a, f) is -1 when bit (a mod 64) of the 64-bit word
    mix64(body_f * MUL_F + (a div 64) * MUL_W + ADD) is set, else +1; it
    depends only on the row and the body's index in the tree-sorted body
    array, so the library's kernel forms the same matrix in any order.
    """
    fidx = np.asarray(fidx, dtype=np.int64).astype(np.uint64)
    words = (p + 63) // 64
    with np.errstate(over="ignore"):
        z = (fidx[None, :] * SKETCH_MUL_F + np.arange(words, dtype=np.uint64)[:, None] * SKETCH_MUL_W
             + SKETCH_ADD)
        z = _mix64(z)
    a = np.arange(p)
    bits = (z[a >> 6, :] >> (a & 63).astype(np.uint64)[:, None]) & np.uint64(1)
    return np.where(bits == 1, -1.0, 1.0)


def far_indices(ranges, samples: int = 0, gstart=None) -> np.ndarray:
    """Tree-sorted body indices of the far list the sketch mode uses: every
    far body when ``samples <= 0``; otherwise the far boxes of the box's own
    level and the two above it in full, then ``samples`` strided bodies
    (sample_indices) of the farther part of the list."""
    if not ranges:
        return np.zeros(0, dtype=np.int64)
    cut = gstart[-3] if (samples > 0 and gstart is not None and len(gstart) >= 3) else 0
    near = [np.arange(b0, b1, dtype=np.int64) for b0, b1 in ranges[cut:]]
    parts = near
    if cut > 0:
        farther = np.concatenate([np.arange(b0, b1, dtype=np.int64) for b0, b1 in ranges[:cut]])
        parts = near + [farther[sample_indices(len(farther), samples)]]
    return np.concatenate(parts) if parts else np.zeros(0, dtype=np.int64)


def far_bodies(bodies: np.ndarray, ranges, samples: int, gstart=None, mode: int = 0) -> np.ndarray:
    """Rows of a box's far list kept under ``samples``: mode 0 strided over the
    whole list, mode 1 level-geometric (build extensions; samples <= 0 keeps all).
    Mode 2 (sketch) keeps every far body."""
    if not ranges:
        return np.zeros((0, 3))
    idx = np.concatenate([np.arange(b0, b1, dtype=np.int64) for b0, b1 in ranges])
    total = len(idx)
    if mode == 2:
        return bodies[far_indices(ranges, samples, gstart)]
    if mode == 0 or samples <= 0 or samples >= total:
        keep = sample_indices(total, samples)
        return bodies[idx[keep]]
    bounds = list(gstart) + [len(ranges)]
    parts = []
    gidx = []
    for g in range(len(gstart)):
        sub = ranges[bounds[g]:bounds[g + 1]]
        gidx.append(np.concatenate([np.arange(b0, b1, dtype=np.int64) for b0, b1 in sub]) if sub
                    else np.zeros(0, dtype=np.int64))
    alloc = geometric_allocation([len(x) for x in gidx], samples)
    for g, x in enumerate(gidx):
        if alloc[g] == 0:
            continue
        keep = sample_indices(len(x), 0 if alloc[g] == len(x) else alloc[g])
        parts.append(x[keep])
    return bodies[np.concatenate(parts)]


# --------------------------------------------------------------------------
# Dense algebra restated from Eigen 3.4 (the reference's third-party boundary)
# --------------------------------------------------------------------------

DBL_EPS = np.finfo(np.float64).eps
DBL_MIN = np.finfo(np.float64).tiny


def householder_r(X: np.ndarray) -> np.ndarray:
    """R of a Householder QR (HouseholderQR::matrixQR upper part)."""
    if X.shape[0] == 0 or X.shape[1] == 0:
        return np.zeros((min(X.shape), X.shape[1]), dtype=X.dtype)
    return sla.qr(X, mode="r", check_finite=False)[0]


def colpiv_qr(Xin: np.ndarray):
    """Eigen 3.4 ColPivHouseholderQR::computeInPlace restated.

    Returns (qr, perm, maxpivot, nonzero_pivots).  ``qr`` holds R in its
    upper triangle; ``perm[k]`` is the original index of pivoted column k
    (A P = Q R, (A P)[:, k] = A[:, perm[k]]).  Complex input follows
    makeHouseholderInPlace's complex rules: beta real with the sign opposite
    to Re c0, tau = conj((beta - c0) / beta), H = I - tau v v^* applied on
    the left (H maps the pivot column to beta e1).
    """
    cplx = np.iscomplexobj(Xin)
    qr = np.array(Xin, dtype=np.complex128 if cplx else np.float64, copy=True)
    rows, cols = qr.shape
    size = min(rows, cols)
    perm = np.arange(cols)
    norms_upd = np.linalg.norm(qr, axis=0) if rows else np.zeros(cols)
    norms_dir = norms_upd.copy()
    max_norm = norms_upd.max() if cols else 0.0
    threshold_helper = (max_norm * DBL_EPS) ** 2 / rows if rows else 0.0
    downdate_thr = math.sqrt(DBL_EPS)
    nonzero = size
    maxpivot = 0.0
    for k in range(size):
        tail = norms_upd[k:]
        bi = int(np.argmax(tail)) + k
        big_sq = norms_upd[bi] ** 2
        if nonzero == size and big_sq < threshold_helper * (rows - k):
            nonzero = k
        if bi != k:
            qr[:, [k, bi]] = qr[:, [bi, k]]
            norms_upd[[k, bi]] = norms_upd[[bi, k]]
            norms_dir[[k, bi]] = norms_dir[[bi, k]]
            perm[[k, bi]] = perm[[bi, k]]
        # makeHouseholderInPlace on qr[k:, k]
        c0 = qr[k, k]
        tail_v = qr[k + 1:, k]
        if cplx:
            tsq = float(np.vdot(tail_v, tail_v).real)
            if tsq <= DBL_MIN and c0.imag * c0.imag <= DBL_MIN:
                tau = 0.0
                beta = c0.real
                ess = np.zeros_like(tail_v)
            else:
                beta = math.sqrt(c0.real * c0.real + c0.imag * c0.imag + tsq)
                if c0.real >= 0:
                    beta = -beta
                ess = tail_v / (c0 - beta)
                tau = np.conj((beta - c0) / beta)
        else:
            tsq = float(tail_v @ tail_v)
            if tsq <= DBL_MIN:
                tau = 0.0
                beta = c0
                ess = np.zeros_like(tail_v)
            else:
                beta = math.sqrt(c0 * c0 + tsq)
                if c0 >= 0:
                    beta = -beta
                ess = tail_v / (c0 - beta)
                tau = (beta - c0) / beta
        qr[k + 1:, k] = ess
        qr[k, k] = beta
        if abs(beta) > maxpivot:
            maxpivot = abs(beta)
        # applyHouseholderOnTheLeft to qr[k:, k+1:]
        if tau != 0.0 and k + 1 < cols:
            blk = qr[k:, k + 1:]
            w = blk[0] + (np.conj(ess) if cplx else ess) @ blk[1:]
            blk[0] -= tau * w
            blk[1:] -= tau * np.outer(ess, w)
        # norm downdate
        for j in range(k + 1, cols):
            if norms_upd[j] != 0.0:
                t = abs(qr[k, j]) / norms_upd[j]
                t = (1.0 + t) * (1.0 - t)
                if t < 0.0:
                    t = 0.0
                t2 = t * (norms_upd[j] / norms_dir[j]) ** 2
                if t2 <= downdate_thr:
                    norms_dir[j] = float(np.linalg.norm(qr[k + 1:, j]))
                    norms_upd[j] = norms_dir[j]
                else:
                    norms_upd[j] *= math.sqrt(t)
    return qr, perm, maxpivot, nonzero


def colpiv_rank(qr: np.ndarray, maxpivot: float, nonzero: int, threshold: float) -> int:
    """ColPivHouseholderQR::rank() with a prescribed relative threshold."""
    thr = abs(maxpivot) * threshold
    d = np.abs(np.diag(qr)[:nonzero])
    return int(np.count_nonzero(d > thr))


def compute_basis(kern: Kernel, epi: float, Xbodies: np.ndarray, Fbodies: np.ndarray,
                  a: np.ndarray, orth: bool, sketch_idx: np.ndarray | None = None):
    """h2matrix.cpp:13-63.

    ``Xbodies`` (M, 3) is permuted in place (skeletons first).  ``a`` is the
    incoming M x M Q (identity at a leaf, children's R blocks above) and is
    replaced by the basis; returns (rank, c) with c the M x M R matrix.

    ``sketch_idx`` (build extension, sampling mode 2): the body indices of
    ``Fbodies``; when the far list is longer than M, the column-pivoted QR
    runs on the M x M sketch S XF (S the random-sign matrix of
    ``sketch_signs``) instead of on R of QR(XF).  Both have the column
    geometry of XF up to the sketch's distortion, so the ID keeps the
    whole far field's accuracy (Halko, Martinsson and Tropp 2011, randomized
    interpolative decomposition) at the cost of one GEMM.
    """
    M = Xbodies.shape[0]
    N = Fbodies.shape[0]
    K = min(M, N)
    rank = 0
    dt = kern.dtype
    c = np.zeros((M, M), dtype=dt)
    if K > 0:
        XF = gen_matrix(kern, Fbodies, Xbodies)  # N x M
        if K < N and sketch_idx is not None:
            RX = sketch_signs(M, sketch_idx) @ XF
        elif K < N:
            RX = np.triu(householder_r(XF)[:K])
        else:
            RX = XF
        qr, perm, maxpivot, nonzero = colpiv_qr(RX)
        rank = min(K, int(math.floor(epi)))
        if epi < 1.0:
            rank = colpiv_rank(qr, maxpivot, nonzero, epi)
        if 0 < rank < M:
            R11 = np.triu(qr[:rank, :rank])
            T = sla.solve_triangular(R11, qr[:rank, rank:], lower=False, check_finite=False)
            top = np.hstack([np.eye(rank), T])       # rank x M, pivoted order
            Xbodies[:] = Xbodies[perm]
            PCt = np.zeros((M, rank), dtype=dt)
            PCt[perm, :] = top.T
            if orth:
                RX2 = np.triu(a) @ PCt
                Qf, Rf = sla.qr(RX2, mode="full", check_finite=False)
                a[:] = Qf
                c[:rank, :rank] = np.triu(Rf[:rank, :rank])
            else:
                a[:] = 0.0
                a[:, :rank] = PCt
                c[:rank, :rank] = np.eye(rank)
        else:
            c = np.triu(a)
            a[:] = np.eye(M)
    return rank, c


# --------------------------------------------------------------------------
# H^2 matrix per level (h2matrix.cpp) and the solver (solver.cpp)
# --------------------------------------------------------------------------


@dataclass
class Level:
    l: int
    gbegin: int
    nodes: int
    ARows: np.ndarray
    ACols: np.ndarray
    CRows: np.ndarray
    CCols: np.ndarray
    Dims: np.ndarray = None
    DimsLr: np.ndarray = None
    Q: list = field(default_factory=list)
    R: list = field(default_factory=list)
    S: list = field(default_factory=list)
    A: list = field(default_factory=list)
    C: list = field(default_factory=list)
    NA: list = field(default_factory=list)  # child near block -> (parent ij, row off, col off)
    X: list = field(default_factory=list)
    Y: list = field(default_factory=list)
    Z: list = field(default_factory=list)
    W: list = field(default_factory=list)
    info: int = 0

    def diag(self, i: int) -> int:
        s, e = self.ARows[i], self.ARows[i + 1]
        hits = np.nonzero(self.ACols[s:e] == i)[0]
        return int(s + hits[0]) if len(hits) else -1

    def lookupA(self, i: int, j: int) -> int:
        s, e = self.ARows[i], self.ARows[i + 1]
        hits = np.nonzero(self.ACols[s:e] == j)[0]
        return int(s + hits[0]) if len(hits) else -1

    def lookupC(self, i: int, j: int) -> int:
        s, e = self.CRows[i], self.CRows[i + 1]
        hits = np.nonzero(self.CCols[s:e] == j)[0]
        return int(s + hits[0]) if len(hits) else -1


def _level_csr(csr: CSR, l: int):
    g0 = (1 << l) - 1
    g1 = (1 << (l + 1)) - 1
    rows = csr.RowIndex[g0:g1 + 1] - csr.RowIndex[g0]
    cols = csr.ColIndex[csr.RowIndex[g0]:csr.RowIndex[g1]] - g0
    return rows.astype(np.int64), cols.astype(np.int64)


class H2MatrixSolver:
    """solver.hpp:11-47 / solver.cpp restated for one process.

    ``eps`` follows the reference: eps == 0 selects the fixed-rank,
    orthogonal-basis preconditioner mode (solver.cpp:28-36) with far lists
    from weak admissibility; eps > 0 selects the ID operator mode.
    """

    dt = np.float64  # element type of every block and vector; complex128 for Helmholtz3D

    def __init__(self, kern: Kernel, epi: float, rank: int, leveled_rank: int, cells: Cells,
                 theta: float, bodies: np.ndarray, levels: int, samples: int = 0, sampling: int = 0):
        self.kern = kern
        self.dt = kern.dtype  # complex128 for Helmholtz3D: the reference's complex arithmetic
        self.levels = levels
        self.cells = cells
        self.bodies = bodies
        near = build_csr("N", cells, theta)
        far = build_csr("F", cells, theta)
        fix_rank = epi == 0.0
        far_list_csr = build_csr("F", cells, 0.0) if fix_rank else far
        self.near, self.far = near, far
        ranges = far_body_lists(cells, far_list_csr, levels)
        self.gstart = far_body_groups(cells, far_list_csr, levels)
        self.sampling = sampling
        self.A: list[Level] = []
        for l in range(levels + 1):
            ar, ac = _level_csr(near, l)
            cr, cc = _level_csr(far, l)
            self.A.append(Level(l, (1 << l) - 1, 1 << l, ar, ac, cr, cc))

        def rank_func(l):
            return (levels - l) * leveled_rank + rank

        for l in range(levels, -1, -1):
            e = float(rank_func(l)) if fix_rank else epi
            self._construct(l, e, ranges, samples)
        self.lenX = int(cells.body[0, 1] - cells.body[0, 0])

    # h2matrix.cpp:72-249
    def _construct(self, l, epi, ranges, samples):
        kern = self.kern
        cells = self.cells
        bodies = self.bodies
        lev = self.A[l]
        nodes = lev.nodes
        g0 = lev.gbegin
        low = self.A[l + 1] if l < self.levels else None
        if low is None:
            Dims = np.array([cells.body[g0 + i, 1] - cells.body[g0 + i, 0] for i in range(nodes)], dtype=np.int64)
        else:
            Dims = np.array([low.DimsLr[2 * i] + low.DimsLr[2 * i + 1] for i in range(nodes)], dtype=np.int64)
        lev.Dims = Dims
        lev.DimsLr = np.zeros(nodes, dtype=np.int64)
        dt = self.dt
        lev.Q = [np.zeros((d, d), dtype=dt) for d in Dims]
        lev.R = [np.zeros((d, d), dtype=dt) for d in Dims]
        lev.S = [np.zeros((d, 3)) for d in Dims]
        nA = int(lev.ARows[-1])
        lev.A = [None] * nA
        for i in range(nodes):
            for ij in range(lev.ARows[i], lev.ARows[i + 1]):
                lev.A[ij] = np.zeros((Dims[i], Dims[lev.ACols[ij]]), dtype=dt)
        lev.X = [np.zeros(d, dtype=dt) for d in Dims]
        lev.Y = [np.zeros(d, dtype=dt) for d in Dims]

        if Dims.sum():
            for i in range(nodes):
                M = Dims[i]
                if low is not None:
                    off = 0
                    for y in (2 * i, 2 * i + 1):
                        ny = int(low.DimsLr[y])
                        lev.S[i][off:off + ny] = low.S[y][:ny]
                        lev.Q[i][off:off + ny, off:off + ny] = low.R[y][:ny, :ny]
                        if M > 0:
                            for ij in range(lev.ARows[i], lev.ARows[i + 1]):
                                j = int(lev.ACols[ij])
                                offx = 0
                                for x in (2 * j, 2 * j + 1):
                                    nx = int(low.DimsLr[x])
                                    lowN = low.lookupA(y, x)
                                    lowC = low.lookupC(y, x)
                                    if lowN >= 0:
                                        low.NA[lowN] = (ij, off, offx)
                                    elif lowC >= 0:
                                        lev.A[ij][off:off + ny, offx:offx + nx] = low.C[lowC]
                                    offx += nx
                        off += ny
                else:
                    ci = g0 + i
                    b0, b1 = cells.body[ci]
                    lev.S[i][:] = bodies[b0:b1]
                    lev.Q[i][:] = np.eye(M)
                    for ij in range(lev.ARows[i], lev.ARows[i + 1]):
                        cj = g0 + int(lev.ACols[ij])
                        lev.A[ij][:] = gen_matrix(kern, bodies[b0:b1], bodies[cells.body[cj, 0]:cells.body[cj, 1]])

            for i in range(nodes):
                fb = far_bodies(bodies, ranges.get(g0 + i, []), samples, self.gstart.get(g0 + i, []),
                                self.sampling)
                sk = (far_indices(ranges.get(g0 + i, []), samples, self.gstart.get(g0 + i, []))
                      if self.sampling == 2 else None)
                rank, c = compute_basis(kern, epi, lev.S[i], fb, lev.Q[i], 1.0 <= epi, sk)
                lev.R[i] = c
                lev.DimsLr[i] = rank

        nC = int(lev.CRows[-1])
        lev.C = [None] * nC
        lev.NA = [None] * nA
        lev.Z = [np.zeros(r, dtype=self.dt) for r in lev.DimsLr]
        lev.W = [np.zeros(r, dtype=self.dt) for r in lev.DimsLr]
        if lev.DimsLr.sum():
            for i in range(nodes):
                My = int(lev.DimsLr[i])
                Ry = np.triu(lev.R[i][:My, :My])
                for ij in range(lev.CRows[i], lev.CRows[i + 1]):
                    x = int(lev.CCols[ij])
                    Nx = int(lev.DimsLr[x])
                    Rx = np.triu(lev.R[x][:Nx, :Nx])
                    Ayx = gen_matrix(kern, lev.S[i][:My], lev.S[x][:Nx])
                    if 1.0 <= epi:
                        lev.C[ij] = Ry @ Ayx @ Rx.T
                    else:
                        lev.C[ij] = Ayx

    # ---- matvec (h2matrix.cpp:251-344, solver.cpp:76-88) ----
    def _split(self, lev: Level, vec: np.ndarray, sizes):
        out, o = [], 0
        for d in sizes:
            out.append(vec[o:o + d].copy())
            o += d
        return out

    def matvec(self, x: np.ndarray) -> np.ndarray:
        L = self.levels
        A = self.A
        xin = np.asarray(x, dtype=self.dt)
        for l in range(L, -1, -1):
            lev = A[l]
            src = xin if l == L else np.concatenate(A[l + 1].Z) if len(A[l + 1].Z) else np.zeros(0, dtype=self.dt)
            lev.X = self._split(lev, src, lev.Dims)
            # h2matrix.cpp:266: z = q^T x (transpose, no conjugate)
            lev.Z = [lev.Q[i][:, :lev.DimsLr[i]].T @ lev.X[i] if lev.DimsLr[i] > 0 else np.zeros(0, dtype=self.dt)
                     for i in range(lev.nodes)]
        for l in range(0, L):
            lev = A[l]
            for i in range(lev.nodes):
                K = lev.DimsLr[i]
                if K > 0:
                    w = lev.W[i]
                    for ij in range(lev.CRows[i], lev.CRows[i + 1]):
                        w = w + lev.C[ij] @ lev.Z[lev.CCols[ij]]
                    lev.W[i] = w
                    lev.Y[i] = lev.Q[i][:, :K] @ w
            nxt = np.concatenate(lev.Y) if lev.nodes else np.zeros(0, dtype=self.dt)
            A[l + 1].W = self._split(A[l + 1], nxt, A[l + 1].DimsLr)
        lev = A[L]
        lev.X = self._split(lev, xin, lev.Dims)
        y = []
        for i in range(lev.nodes):
            M = lev.Dims[i]
            K = lev.DimsLr[i]
            yi = np.zeros(M, dtype=self.dt)
            if K > 0:
                w = lev.W[i]
                for ij in range(lev.CRows[i], lev.CRows[i + 1]):
                    w = w + lev.C[ij] @ lev.Z[lev.CCols[ij]]
                lev.W[i] = w
                yi += lev.Q[i][:, :K] @ w
            for ij in range(lev.ARows[i], lev.ARows[i + 1]):
                yi += lev.A[ij] @ lev.X[lev.ACols[ij]]
            y.append(yi)
        return np.concatenate(y)

    # ---- factorization (h2matrix.cpp:346-446, solver.cpp:90-100) ----
    def factorize(self):
        L = self.levels
        for l in range(L, -1, -1):
            self._factorize_level(self.A[l])
            if l > 0:
                self._copy_next(self.A[l - 1], self.A[l])
        return [lev.info for lev in self.A]

    def _factorize_level(self, lev: Level):
        nodes = lev.nodes
        lev.info = 0
        B = [None] * nodes
        for i in range(nodes):
            d = lev.diag(i)
            M = int(lev.Dims[i])
            Ms = int(lev.DimsLr[i])
            Mr = M - Ms
            U = lev.Q[i]
            Uh = U.conj().T  # Ui.adjoint() (h2matrix.cpp:373-379); U^T for real kernels
            Aii = lev.A[d]
            b = Uh @ Aii.T
            Aii[:] = Uh @ b.T
            V = np.zeros((M, M), dtype=self.dt)
            V[:Ms] = Uh[:Ms]
            if Mr > 0:
                lu, piv = sla.lu_factor(Aii[Ms:, Ms:], check_finite=False)
                V[Ms:] = sla.lu_solve((lu, piv), Uh[Ms:], check_finite=False)
                if Ms > 0:
                    Aii[Ms:, :Ms] = V[Ms:] @ b[:Ms].T
                    Aii[:Ms, :Ms] -= Aii[:Ms, Ms:] @ Aii[Ms:, :Ms]
                with np.errstate(over="ignore", under="ignore"):
                    det = np.prod(np.diag(lu))  # may overflow or underflow, as Eigen's product does
                lev.info += int(abs(det) <= DBL_MIN)
            lev.R[i] = V
            for ij in range(lev.ARows[i], lev.ARows[i + 1]):
                if ij != d:
                    j = int(lev.ACols[ij])
                    Uj = lev.Q[j]
                    Aij = lev.A[ij]
                    bj = Uj.conj().T @ Aij.T
                    Aij[:] = V @ bj.T
            Bi = np.zeros((Mr, M), dtype=self.dt)
            Bi[:, :Ms] = Aii[Ms:, :Ms]
            Bi[:, Ms:] = V[Ms:] @ U[:, Ms:]
            B[i] = Bi
        for i in range(nodes):
            d = lev.diag(i)
            M = int(lev.Dims[i])
            Ms = int(lev.DimsLr[i])
            Mr = M - Ms
            Aii = lev.A[d]
            for ij in range(lev.ARows[i], lev.ARows[i + 1]):
                if ij != d:
                    j = int(lev.ACols[ij])
                    N = int(lev.Dims[j])
                    Ns = int(lev.DimsLr[j])
                    Nr = N - Ns
                    Aij = lev.A[ij]
                    Bj = B[j]
                    upd = Aii[:Ms, Ms:] @ Aij[Ms:, :Ns] + Aij[:Ms, Ns:] @ Bj[:Nr, :Ns]
                    Aij[:Ms, :Ns] -= upd
                    Aii[:Ms, :Ms] -= Aij[:Ms, Ns:] @ Bj[:Nr, Ns:N] @ Aij[:Ms, Ns:].T

    def _copy_next(self, up: Level, low: Level):
        for i in range(low.nodes):
            Ms = int(low.DimsLr[i])
            for ij in range(low.ARows[i], low.ARows[i + 1]):
                j = int(low.ACols[ij])
                Ns = int(low.DimsLr[j])
                if Ms > 0 and Ns > 0:
                    pij, ro, co = low.NA[ij]
                    up.A[pij][ro:ro + Ms, co:co + Ns] = low.A[ij][:Ms, :Ns]

    # ---- ULV substitution (h2matrix.cpp:448-537, solver.cpp:121-132) ----
    def solve_precondition(self, x: np.ndarray) -> np.ndarray:
        L = self.levels
        A = self.A
        for l in range(L, -1, -1):
            lev = A[l]
            src = np.asarray(x, dtype=self.dt) if l == L else np.concatenate(A[l + 1].Z)
            lev.Y = self._split(lev, src, lev.Dims)
            lev.X = [lev.R[i] @ lev.Y[i] if lev.Dims[i] > 0 else np.zeros(0, dtype=self.dt) for i in range(lev.nodes)]
            Z = []
            for i in range(lev.nodes):
                Ms = int(lev.DimsLr[i])
                z = lev.X[i][:Ms].copy()
                if Ms > 0:
                    for ij in range(lev.ARows[i], lev.ARows[i + 1]):
                        j = int(lev.ACols[ij])
                        Ns = int(lev.DimsLr[j])
                        Nr = int(lev.Dims[j]) - Ns
                        if Nr > 0:
                            z -= lev.A[ij][:Ms, Ns:] @ lev.X[j][Ns:]
                Z.append(z)
            lev.Z = Z
        for l in range(0, L + 1):
            lev = A[l]
            if l == 0:
                W = [np.zeros(int(r), dtype=self.dt) for r in lev.DimsLr]
            else:
                W = self._split(lev, np.concatenate(A[l - 1].Y), lev.DimsLr)
            lev.W = W
            Xn = []
            for i in range(lev.nodes):
                M = int(lev.Dims[i])
                Ms = int(lev.DimsLr[i])
                Mr = M - Ms
                xi = lev.X[i].copy()
                xi[:Ms] = W[i]
                if Mr > 0:
                    for ij in range(lev.ARows[i], lev.ARows[i + 1]):
                        j = int(lev.ACols[ij])
                        Ns = int(lev.DimsLr[j])
                        if Ns > 0:
                            xi[Ms:] -= lev.A[ij][Ms:, :Ns] @ W[j]
                Xn.append(xi)
            lev.X = Xn
            # h2matrix.cpp:532: y = conj(q) x
            lev.Y = [lev.Q[i].conj() @ lev.X[i] if lev.Dims[i] > 0 else np.zeros(0, dtype=self.dt)
                     for i in range(lev.nodes)]
        return np.concatenate(A[L].Y)

    # ---- GMRES (solver.cpp:144-201) ----
    def solve_gmres(self, tol: float, Msolver: "H2MatrixSolver", x: np.ndarray, b: np.ndarray,
                    inner: int, outer: int, early_exit: bool = False):
        N = self.lenX
        ld = inner + 1
        dt = self.dt
        B = np.asarray(b, dtype=dt)
        X = np.array(x, dtype=dt, copy=True)
        normb = math.sqrt(float(np.vdot(B, B).real))
        if normb == 0.0:
            normb = 1.0
        Rv = B.copy()
        resid = [1.0]
        iters = 0
        while iters < outer and tol <= resid[iters]:
            Rv = Msolver.solve_precondition(Rv)
            beta = math.sqrt(float(np.vdot(Rv, Rv).real))
            H = np.zeros((ld, inner), dtype=dt)
            v = np.zeros((N, ld), dtype=dt)
            v[:, 0] = Rv * (1.0 / beta)
            for i in range(inner):
                Rv = self.matvec(v[:, i])
                Rv = Msolver.solve_precondition(Rv)
                H[:i + 1, i] = v[:, :i + 1].conj().T @ Rv
                Rv = Rv - v[:, :i + 1] @ H[:i + 1, i]
                H[i + 1, i] = math.sqrt(float(np.vdot(Rv, Rv).real))
                v[:, i + 1] = Rv * (1.0 / H[i + 1, i])
            s = np.zeros(ld, dtype=dt)
            s[0] = beta
            y = np.linalg.lstsq(H, s, rcond=None)[0]
            X = X + v[:, :inner] @ y
            Rv = -X
            Rv = self.matvec(Rv)
            Rv = Rv + B
            iters += 1
            resid.append(math.sqrt(float(np.vdot(Rv, Rv).real)) / normb)
        return X, np.array(resid), iters


def solve_rel_err(x: np.ndarray, ref: np.ndarray) -> float:
    """solver.cpp:229-238 (real parts only, also for complex vectors)."""
    d = np.real(x - ref)
    r = np.real(ref)
    return math.sqrt(float(d @ d) / float(r @ r))


def levels_for(N: int, leaf: int) -> int:
    """main.cpp:54-55."""
    leaf = N if N < leaf else leaf
    return int(math.log2(N / leaf))
