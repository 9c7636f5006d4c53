"""Python mirror of the reference's solver interface (solver.hpp:11-47).

``H2MatrixSolver`` keeps the reference's method names and argument meaning:
``matVecMul``, ``factorizeM``, ``solvePrecondition``, ``solveGMRES`` and the
static ``solveRelErr``; every vector is in tree-sorted body order and the
operations work in place.  All numerical work runs in libmxcb200.so on the
GPU; this module only moves arrays across the C ABI.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Tree:
    """Cells of buildBinaryTree (build_tree.cpp:67-99) as flat arrays."""

    def __init__(self, levels: int, child: np.ndarray, body: np.ndarray, R: np.ndarray, Cc: np.ndarray):
        self.levels = levels
        self.child = child
        self.body = body
        self.R = R
        self.C = Cc

    @property
    def ncells(self) -> int:
        return self.child.shape[0]


def uniform_unit_cube_rnd(n: int, seed: int, diameter: float = 1.0, dim: int = 3) -> np.ndarray:
    """test_funcs.hpp:31-41 (std::mt19937, run in the library's host code)."""
    b = np.empty((n, 3), dtype=np.float64)
    L.check(L.lib().h2_uniform_unit_cube_rnd(_ptr(b), n, diameter, dim, seed), "h2_uniform_unit_cube_rnd")
    return b


def mesh_sphere(n: int, r: float) -> np.ndarray:
    """test_funcs.hpp:43-61 mesh_sphere, the reference's default geometry:
    golden-angle spiral of n bodies on a sphere of radius r (the reference
    uses r = sqrt(n / 4 pi), one body per unit area); the same formula as the
    C++ API's mesh_sphere."""
    golden = math.pi * (3.0 - math.sqrt(5.0))
    i = np.arange(n, dtype=np.float64)
    t = i / (n - 1) if n > 1 else np.zeros(n)
    y = r - 2.0 * r * t
    ring = np.sqrt(r * r - y * y)
    a = golden * i
    return np.ascontiguousarray(np.stack([ring * np.cos(a), y, ring * np.sin(a)], axis=1))


def uniform_rhs(n: int) -> np.ndarray:
    """main.cpp:73-76 (default-seeded std::mt19937_64, uniform[0,1))."""
    x = np.empty(n, dtype=np.float64)
    L.check(L.lib().h2_uniform_rhs(_ptr(x), n), "h2_uniform_rhs")
    return x


def levels_for(n: int, leaf: int) -> int:
    return int(L.lib().h2_levels_for(n, leaf))


def build_tree(bodies: np.ndarray, levels: int, leaf_min: int = 0, leaf_max: int = 0) -> Tree:
    """buildBinaryTree: sorts ``bodies`` (n x 3, C-contiguous float64) in place.

    With leaf_min / leaf_max (extension): geometric cuts clamped so every leaf
    holds leaf_min..leaf_max bodies (h2_build_tree_capped), for clustered
    bodies; the default is the reference's median split."""
    assert bodies.dtype == np.float64 and bodies.flags.c_contiguous and bodies.shape[1] == 3
    nc = (2 << levels) - 1
    child = np.empty((nc, 2), dtype=np.int64)
    body = np.empty((nc, 2), dtype=np.int64)
    R = np.empty((nc, 3))
    Cc = np.empty((nc, 3))
    if leaf_min or leaf_max:
        L.check(L.lib().h2_build_tree_capped(_ptr(bodies), bodies.shape[0], levels, leaf_min, leaf_max, _ptr(child),
                                             _ptr(body), _ptr(R), _ptr(Cc)), "h2_build_tree_capped")
    else:
        L.check(L.lib().h2_build_tree(_ptr(bodies), bodies.shape[0], levels, _ptr(child), _ptr(body), _ptr(R),
                                      _ptr(Cc)), "h2_build_tree")
    return Tree(levels, child, body, R, Cc)


def pair_csr(kind: str, tree: Tree, theta: float):
    """CSR::CSR (build_tree.cpp:41-58): (RowIndex, ColIndex) of the near or far pairs."""
    row = np.zeros(tree.ncells + 1, dtype=np.int64)
    nnz = C.c_int64()
    args = (kind.encode(), tree.ncells, _ptr(tree.child), _ptr(tree.body), _ptr(tree.R), _ptr(tree.C), theta)
    L.check(L.lib().h2_pair_csr(*args, _ptr(row), None, 0, C.byref(nnz)), "h2_pair_csr")
    col = np.zeros(nnz.value, dtype=np.int64)
    L.check(L.lib().h2_pair_csr(*args, _ptr(row), _ptr(col), nnz.value, C.byref(nnz)), "h2_pair_csr")
    return row, col


class Handle:
    """deviceHandle (gpu_handles.cuh:10-15): one stream on one device."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        L.check(L.lib().h2dev_handle_create(device, C.byref(h)), "h2dev_handle_create")
        self.h = h

    def synchronize(self):
        L.check(L.lib().h2dev_handle_synchronize(self.h), "h2dev_handle_synchronize")

    def set_option(self, option: int, value: int):
        L.check(L.lib().h2dev_set_option(self.h, option, value), "h2dev_set_option")

    def set_basis_mode(self, mode: int):
        """BASIS_GRAM (default) or BASIS_HOUSEHOLDER for fixed-rank bases of solvers created next."""
        L.check(L.lib().h2dev_set_option(self.h, L.OPT_BASIS, mode), "h2dev_set_option")

    def profile(self, on: bool = True):
        L.check(L.lib().h2dev_profile_enable(self.h, 1 if on else 0), "h2dev_profile_enable")

    def profile_report(self) -> dict:
        """{kernel: (launches, device ms, algorithmic flops, algorithmic bytes)}."""
        cnt = C.c_int64()
        L.check(L.lib().h2dev_profile_report(self.h, 0, None, None, None, None, None, C.byref(cnt)),
                "h2dev_profile_report")
        n = cnt.value
        names = C.create_string_buffer(48 * max(n, 1))
        nl = np.zeros(max(n, 1), dtype=np.int64)
        ms = np.zeros(max(n, 1))
        fl = np.zeros(max(n, 1))
        by = np.zeros(max(n, 1))
        L.check(L.lib().h2dev_profile_report(self.h, n, names, _ptr(nl), _ptr(ms), _ptr(fl), _ptr(by), C.byref(cnt)),
                "h2dev_profile_report")
        out = {}
        for k in range(n):
            nm = names.raw[48 * k:48 * k + 48].split(b"\0", 1)[0].decode()
            out[nm] = (int(nl[k]), float(ms[k]), float(fl[k]), float(by[k]))
        return out

    def profile_timeline(self) -> list:
        """[(kernel, start ms, device ms)] for every profiled launch, in order."""
        cnt = C.c_int64()
        L.check(L.lib().h2dev_profile_timeline(self.h, 0, None, None, None, C.byref(cnt)), "h2dev_profile_timeline")
        n = cnt.value
        names = C.create_string_buffer(48 * max(n, 1))
        t0 = np.zeros(max(n, 1))
        dt = np.zeros(max(n, 1))
        L.check(L.lib().h2dev_profile_timeline(self.h, n, names, _ptr(t0), _ptr(dt), C.byref(cnt)),
                "h2dev_profile_timeline")
        return [(names.raw[48 * k:48 * k + 48].split(b"\0", 1)[0].decode(), float(t0[k]), float(dt[k]))
                for k in range(n)]

    def memory(self) -> tuple:
        """(live bytes, cached free bytes) of this handle's device memory."""
        live, cached = C.c_int64(), C.c_int64()
        L.check(L.lib().h2dev_handle_memory(self.h, C.byref(live), C.byref(cached)), "h2dev_handle_memory")
        return live.value, cached.value

    def memory_peak(self, reset: bool = False) -> int:
        """High-water mark of the live bytes since creation or the last reset."""
        v = C.c_int64()
        L.check(L.lib().h2dev_handle_memory_peak(self.h, C.byref(v), 1 if reset else 0), "h2dev_handle_memory_peak")
        return v.value

    def trim(self) -> None:
        """Return the handle's cached device blocks to the driver."""
        L.check(L.lib().h2dev_handle_trim(self.h), "h2dev_handle_trim")

    @staticmethod
    def launch_count() -> int:
        """Kernels launched by the library in this process so far."""
        v = C.c_int64()
        L.check(L.lib().h2dev_launch_count(C.byref(v)), "h2dev_launch_count")
        return v.value

    def autotune_report(self) -> list:
        """Autotuner decisions of this handle: (bucket key, chosen variant, [ms per variant])."""
        n = C.c_int64()
        L.check(L.lib().h2dev_autotune_report(self.h, 0, None, None, None, C.byref(n)), "h2dev_autotune_report")
        cnt = n.value
        if cnt == 0:
            return []
        keys = C.create_string_buffer(64 * cnt)
        choice = np.zeros(cnt, dtype=np.int32)
        ms = np.zeros(3 * cnt)
        L.check(L.lib().h2dev_autotune_report(self.h, cnt, keys, _ptr(choice), _ptr(ms), C.byref(n)),
                "h2dev_autotune_report")
        raw = keys.raw
        return [(raw[64 * i:64 * (i + 1)].split(b"\0", 1)[0].decode(), int(choice[i]),
                 [float(v) for v in ms[3 * i:3 * i + 3] if v >= 0]) for i in range(cnt)]

    def fma_peak_tflops(self, precision: int = L.FP64) -> float:
        v = C.c_double()
        L.check(L.lib().h2dev_probe_fma_peak(self.h, precision, C.byref(v)), "h2dev_probe_fma_peak")
        return v.value

    def timer_start(self):
        L.check(L.lib().h2dev_timer_start(self.h), "h2dev_timer_start")

    def timer_stop(self) -> float:
        ms = C.c_double()
        L.check(L.lib().h2dev_timer_stop(self.h, C.byref(ms)), "h2dev_timer_stop")
        return ms.value

    def close(self):
        if self.h:
            L.lib().h2dev_handle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Kernel:
    """Laplace3D(s) / Yukawa3D(s, alpha) / Helmholtz3D(k, s) of kernel.hpp:28-74."""

    def __init__(self, kind: int = L.KERNEL_LAPLACE, singularity: float = 1.0, alpha: float = 1.0):
        self.kind = kind
        self.singularity = singularity
        self.alpha = alpha


def Laplace3D(s: float = 1.0) -> Kernel:
    return Kernel(L.KERNEL_LAPLACE, s, 0.0)


def Yukawa3D(s: float = 1.0, a: float = 1.0) -> Kernel:
    return Kernel(L.KERNEL_YUKAWA, s, a)


def Helmholtz3D(wave_number: float = 1.0, s: float = 1.0) -> Kernel:
    """exp(-i k d) / d, 1/s at d == 0 (kernel.hpp:63-74): complex matrices and vectors.

    The device holds the real symmetric form of the complex matrix (two real
    unknowns per body); vectors passed to a Helmholtz solver are complex128
    arrays, and level dims / ranks count real unknowns."""
    return Kernel(L.KERNEL_HELMHOLTZ, s, wave_number)


def Quadratic(s: float = 1.0, a: float = 1.0) -> Kernel:
    """d^2 + a off the diagonal: exactly low-rank off-diagonal blocks (ULV exactness checks)."""
    return Kernel(L.KERNEL_QUADRATIC, s, a)


def _as_cols(X: np.ndarray, cplx: bool = False):
    """(n,) or (n, nrhs) float64 -> Fortran-ordered 2-D view + nrhs + ld.

    cplx: complex128 arrays, whose columns the library reads as 2n doubles
    (interleaved real and imaginary parts); ld then counts doubles."""
    if cplx and X.dtype != np.complex128:
        raise TypeError("a Helmholtz solver takes complex128 vectors, got %s" % X.dtype)
    if not cplx and X.dtype != np.float64:
        raise TypeError("a real-kernel solver takes float64 vectors, got %s" % X.dtype)
    w = 2 if cplx else 1
    if X.ndim == 1:
        if not X.flags.c_contiguous:
            raise ValueError("vectors must be contiguous")
        return X.reshape(-1, 1, order="F"), 1, w * X.shape[0]
    if not X.flags.f_contiguous:
        raise ValueError("multi-RHS arrays must be column-major (order='F')")
    return X, X.shape[1], w * X.shape[0]


class H2MatrixSolver:
    """H2MatrixSolver (solver.hpp:11-47) on one B200.

    eps > 0: operator (ID basis, relative threshold eps); eps == 0:
    fixed-rank orthogonal-basis preconditioner.  ``samples`` caps each box's
    far list (<= 0: every far body, as the reference).  ``precision``:
    FP64 or FP32 storage and arithmetic of this matrix.
    """

    def __init__(self, handle: Handle, kernel: Kernel, eps: float, rank: int, leveled_rank: int, tree: Tree,
                 theta: float, bodies: np.ndarray, samples: int = 0, precision: int = L.FP64):
        s = C.c_void_p()
        self.handle = handle
        self.levels = tree.levels
        n = bodies.shape[0]
        L.check(L.lib().h2dev_solver_create(handle.h, kernel.kind, kernel.singularity, kernel.alpha, eps, rank,
                                            leveled_rank, tree.ncells, _ptr(tree.child), _ptr(tree.body),
                                            _ptr(tree.R), _ptr(tree.C), theta, _ptr(bodies), n, tree.levels,
                                            samples, precision, C.byref(s)), "h2dev_solver_create")
        self.s = s
        self.complex = kernel.kind == L.KERNEL_HELMHOLTZ
        self.local_bodies = (0, n)
        self.resid = None
        self.iters = 0
        self.info = None

    # ------------------------------------------------------------ reference API
    def matVecMul(self, X: np.ndarray) -> None:
        A, nrhs, ld = _as_cols(X, self.complex)
        L.check(L.lib().h2dev_matvec(self.s, nrhs, _ptr(A), ld), "h2dev_matvec")

    def factorizeM(self) -> list:
        info = np.zeros(self.levels + 1, dtype=np.int32)
        rc = L.lib().h2dev_factorize(self.s, _ptr(info))
        L.check(rc, "h2dev_factorize", allow=(L.H2DEV_ERR_SINGULAR,))
        self.info = [int(v) for v in info]
        for lvl in range(self.levels, -1, -1):
            if self.info[lvl]:
                print("singularity detected at level %d." % lvl)
        return self.info

    def solvePrecondition(self, X: np.ndarray) -> None:
        A, nrhs, ld = _as_cols(X, self.complex)
        L.check(L.lib().h2dev_solve_precondition(self.s, nrhs, _ptr(A), ld), "h2dev_solve_precondition")

    def solveGMRES(self, tol: float, M: "H2MatrixSolver", X: np.ndarray, B: np.ndarray, inner_iters: int,
                   outer_iters: int, early_exit: bool = False) -> int:
        dt = np.complex128 if self.complex else np.float64
        Xa, nrhs, ld = _as_cols(X, self.complex)
        Ba, nb, ldb = _as_cols(np.asarray(B, dtype=dt, order="F"), self.complex)
        assert nb == nrhs and ldb == ld
        resid = np.zeros((outer_iters + 1, nrhs), order="F")
        iters = np.zeros(nrhs, dtype=np.int64)
        rc = L.lib().h2dev_solve_gmres(self.s, M.s, tol, nrhs, _ptr(Xa), _ptr(Ba), ld, inner_iters, outer_iters,
                                       1 if early_exit else 0, _ptr(resid), _ptr(iters))
        L.check(rc, "h2dev_solve_gmres", allow=(L.H2DEV_ERR_NOCONV,))
        self.resid = resid if nrhs > 1 else resid[:, 0]
        self.iters = iters if nrhs > 1 else int(iters[0])
        return rc

    @staticmethod
    def solveRelErr(X: np.ndarray, ref: np.ndarray) -> float:
        """solver.cpp:229-238 (host-side reduction of two vectors; of complex
        vectors only the real parts enter, as in the reference)."""
        d = np.real(np.asarray(X) - np.asarray(ref))
        r = np.real(np.asarray(ref))
        return math.sqrt(float(np.sum(d * d)) / float(np.sum(r * r)))

    # ------------------------------------------------------------ device-pointer API
    def matvec_device(self, ptr: int, nrhs: int, ld: int) -> None:
        L.check(L.lib().h2dev_matvec_device(self.s, nrhs, C.c_void_p(ptr), ld), "h2dev_matvec_device")

    def precondition_device(self, ptr: int, nrhs: int, ld: int) -> None:
        L.check(L.lib().h2dev_solve_precondition_device(self.s, nrhs, C.c_void_p(ptr), ld),
                "h2dev_solve_precondition_device")

    def gmres_device(self, M: "H2MatrixSolver", tol: float, xptr: int, bptr: int, nrhs: int, ld: int, inner: int,
                     outer: int, early_exit: bool = False):
        resid = np.zeros((outer + 1, nrhs), order="F")
        iters = np.zeros(nrhs, dtype=np.int64)
        rc = L.lib().h2dev_solve_gmres_device(self.s, M.s, tol, nrhs, C.c_void_p(xptr), C.c_void_p(bptr), ld,
                                              inner, outer, 1 if early_exit else 0, _ptr(resid), _ptr(iters))
        L.check(rc, "h2dev_solve_gmres_device", allow=(L.H2DEV_ERR_NOCONV,))
        return rc, resid, iters

    # ------------------------------------------------------------ inspection
    def shape(self):
        lv = C.c_int64()
        n = C.c_int64()
        L.check(L.lib().h2dev_solver_shape(self.s, C.byref(lv), C.byref(n)), "h2dev_solver_shape")
        return lv.value, n.value

    def level_dims(self, level: int):
        nodes = 1 << level
        d = np.zeros(nodes, dtype=np.int64)
        r = np.zeros(nodes, dtype=np.int64)
        L.check(L.lib().h2dev_solver_level_dims(self.s, level, _ptr(d), _ptr(r)), "h2dev_solver_level_dims")
        return d, r

    def export(self, level: int, what: int) -> np.ndarray:
        cnt = C.c_int64()
        L.check(L.lib().h2dev_solver_export_size(self.s, level, what, C.byref(cnt)), "export_size")
        out = np.zeros(cnt.value)
        if cnt.value:
            L.check(L.lib().h2dev_solver_export(self.s, level, what, _ptr(out)), "export")
        return out

    def close(self):
        if getattr(self, "s", None):
            L.lib().h2dev_solver_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rel_err_device(handle: Handle, xptr: int, refptr: int, n: int, nrhs: int, ld: int) -> np.ndarray:
    """solveRelErr (solver.cpp:229-238) of nrhs device columns; returns host values."""
    out = np.zeros(nrhs)
    L.check(L.lib().h2dev_solve_rel_err_device(handle.h, n, nrhs, C.c_void_p(xptr), C.c_void_p(refptr), ld, _ptr(out)),
            "h2dev_solve_rel_err_device")
    return out


def gen_block(handle: Handle, kernel: Kernel, bi: np.ndarray, bj: np.ndarray) -> np.ndarray:
    """gen_matrix (kernel.cpp:71-85) on the device; returns an (m, n) array
    (complex128 for Helmholtz3D)."""
    bi = np.ascontiguousarray(bi, dtype=np.float64)
    bj = np.ascontiguousarray(bj, dtype=np.float64)
    m, n = bi.shape[0], bj.shape[0]
    cplx = kernel.kind == L.KERNEL_HELMHOLTZ
    out = np.zeros((m, n), dtype=np.complex128 if cplx else np.float64, order="F")
    L.check(L.lib().h2dev_gen_block(handle.h, kernel.kind, kernel.singularity, kernel.alpha, _ptr(bi), m, _ptr(bj),
                                    n, _ptr(out)), "h2dev_gen_block")
    return out


def dense_matvec(handle: Handle, kernel: Kernel, bodies: np.ndarray, X: np.ndarray) -> np.ndarray:
    """Y = A_dense X (FP64, matrix-free on the device; complex for Helmholtz3D)."""
    bodies = np.ascontiguousarray(bodies, dtype=np.float64)
    cplx = kernel.kind == L.KERNEL_HELMHOLTZ
    Xa, nrhs, ld = _as_cols(np.asarray(X, dtype=np.complex128 if cplx else np.float64, order="F"), cplx)
    Y = np.zeros_like(Xa, order="F")
    L.check(L.lib().h2dev_dense_matvec(handle.h, kernel.kind, kernel.singularity, kernel.alpha, _ptr(bodies),
                                       bodies.shape[0], nrhs, _ptr(Xa), _ptr(Y), ld), "h2dev_dense_matvec")
    return Y.reshape(X.shape) if np.asarray(X).ndim == 1 else Y
