"""ctypes binding of libmxcb200.so (the C ABI declared in include/h2dev.h).

Loading fails loudly when the library has not been built: there is no
Python or CPU fallback for any device entry point.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmxcb200.so")

H2DEV_OK = 0
H2DEV_ERR_ARG = 1
H2DEV_ERR_CUDA = 2
H2DEV_ERR_OOM = 3
H2DEV_ERR_STATE = 4
H2DEV_ERR_SINGULAR = 5
H2DEV_ERR_NOCONV = 6

KERNEL_LAPLACE = 0
KERNEL_YUKAWA = 1
KERNEL_QUADRATIC = 2
KERNEL_HELMHOLTZ = 3
FP64 = 0
FP32 = 1

OPT_BASIS = 0
OPT_SKINNY_TILED = 1
OPT_SAMPLING = 2
OPT_TENSOR_CORES = 3
OPT_MATRIX_FREE = 4
OPT_PRECOND_BF16 = 5
OPT_GRAPH_SOLVE = 6
OPT_AUTOTUNE = 7
BASIS_GRAM, BASIS_HOUSEHOLDER = 0, 1
# H2DEV_OPT_SAMPLING values: strided cap, level-geometric cap, sketch of every far body
SAMPLING_STRIDED, SAMPLING_GEOMETRIC, SAMPLING_SKETCH = 0, 1, 2

EXPORT_S, EXPORT_Q, EXPORT_R, EXPORT_A, EXPORT_C = range(5)

_i64 = C.c_int64
_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_vp = C.c_void_p

# name -> (restype, argtypes); every symbol include/h2dev.h declares.
SIGNATURES = {
    "h2_uniform_unit_cube_rnd": (C.c_int, [_vp, _i64, C.c_double, _i64, C.c_uint]),
    "h2_uniform_rhs": (C.c_int, [_vp, _i64]),
    "h2_build_tree": (C.c_int, [_vp, _i64, _i64, _vp, _vp, _vp, _vp]),
    "h2_levels_for": (_i64, [_i64, _i64]),
    "h2_build_tree_capped": (C.c_int, [_vp, _i64, _i64, _i64, _i64, _vp, _vp, _vp, _vp]),
    "h2_pair_csr": (C.c_int, [C.c_char, _i64, _vp, _vp, _vp, _vp, C.c_double, _vp, _vp, _i64, _i64p]),
    "h2dev_handle_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "h2dev_handle_destroy": (C.c_int, [_vp]),
    "h2dev_handle_synchronize": (C.c_int, [_vp]),
    "h2dev_set_option": (C.c_int, [_vp, C.c_int, _i64]),
    "h2dev_solver_create": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_double, _i64, _i64, _i64,
                                      _vp, _vp, _vp, _vp, C.c_double, _vp, _i64, _i64, _i64, C.c_int,
                                      C.POINTER(_vp)]),
    "h2dev_solver_destroy": (C.c_int, [_vp]),
    "h2dev_solver_shape": (C.c_int, [_vp, _i64p, _i64p]),
    "h2dev_solver_level_dims": (C.c_int, [_vp, _i64, _vp, _vp]),
    "h2dev_matvec": (C.c_int, [_vp, _i64, _vp, _i64]),
    "h2dev_matvec_device": (C.c_int, [_vp, _i64, _vp, _i64]),
    "h2dev_factorize": (C.c_int, [_vp, _vp]),
    "h2dev_solve_precondition": (C.c_int, [_vp, _i64, _vp, _i64]),
    "h2dev_solve_precondition_device": (C.c_int, [_vp, _i64, _vp, _i64]),
    "h2dev_solve_gmres": (C.c_int, [_vp, _vp, C.c_double, _i64, _vp, _vp, _i64, _i64, _i64, C.c_int, _vp,
                                    _vp]),
    "h2dev_solve_gmres_device": (C.c_int, [_vp, _vp, C.c_double, _i64, _vp, _vp, _i64, _i64, _i64, C.c_int,
                                           _vp, _vp]),
    "h2dev_solve_rel_err_device": (C.c_int, [_vp, _i64, _i64, _vp, _vp, _i64, _vp]),
    "h2dev_solve_rel_err_device_noalloc": (C.c_int, [_vp, _i64, _i64, _vp, _vp, _i64, _vp]),
    "h2dev_gen_block": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, _vp, _i64, _vp, _i64, _vp]),
    "h2dev_dense_matvec": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, _vp, _i64, _i64, _vp, _vp, _i64]),
    "h2dev_dense_matvec_device": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, _vp, _i64, _i64, _vp, _vp,
                                            _i64]),
    "h2dev_solver_export_size": (C.c_int, [_vp, _i64, C.c_int, _i64p]),
    "h2dev_solver_export": (C.c_int, [_vp, _i64, C.c_int, _vp]),
    "h2dev_profile_enable": (C.c_int, [_vp, C.c_int]),
    "h2dev_profile_report": (C.c_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _i64p]),
    "h2dev_profile_timeline": (C.c_int, [_vp, _i64, _vp, _vp, _vp, _i64p]),
    "h2dev_launch_count": (C.c_int, [_i64p]),
    "h2dev_autotune_report": (C.c_int, [_vp, _i64, _vp, _vp, _vp, _i64p]),
    "h2dev_handle_memory": (C.c_int, [_vp, _i64p, _i64p]),
    "h2dev_handle_trim": (C.c_int, [_vp]),
    "h2dev_handle_memory_peak": (C.c_int, [_vp, _i64p, C.c_int]),
    "h2dev_batched_gemm_device": (C.c_int, [_vp, C.c_int, _i64, _i64, _i64, _i64, _i64, C.c_int, C.c_int, C.c_double,
                                            _vp, _i64, _i64, _vp, _i64, _i64, C.c_double, _vp, _i64, _i64]),
    "h2dev_probe_fma_peak": (C.c_int, [_vp, C.c_int, _dp]),
    "h2dev_timer_start": (C.c_int, [_vp]),
    "h2dev_timer_stop": (C.c_int, [_vp, _dp]),
    "h2dev_last_error_message": (C.c_char_p, []),
}

_lib = None


class H2DevError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__("%s failed with status %d: %s" % (where, code, msg))
        self.code = code


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libmxcb200.so is not built (run: python -m mxc_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code: int, where: str, allow=()) -> int:
    if code != H2DEV_OK and code not in allow:
        msg = lib().h2dev_last_error_message()
        raise H2DevError(code, where, msg.decode() if msg else "")
    return code
