"""The C ABI library loads (no GPU needed) and exports every declared symbol."""
import ctypes
import os
import re

import mxc_b200 as m
from mxc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "h2dev.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(h2(?:dev)?_[a-z0-9_]+)\s*\(", txt)))


def test_header_lists_functions():
    names = declared_functions()
    assert "h2dev_solver_create" in names and "h2dev_solve_gmres" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_host_entry_points_validate_arguments():
    import numpy as np

    b = np.zeros((4, 3))
    with __import__("pytest").raises(m.H2DevError):
        m.build_tree(b, 5)  # more leaves than bodies
    assert m.levels_for(20000, 256) == 6
    assert m.levels_for(100, 256) == 0


def test_vector_argument_validation():
    """The Python mirror rejects vectors of the wrong element type or layout
    before any device call: complex128 for a Helmholtz solver, float64 for
    the real kernels, column-major multi-RHS arrays."""
    import numpy as np
    import pytest
    from mxc_b200 import solver as S

    x = np.zeros(8)
    Xf = np.zeros((8, 3), order="F")
    assert S._as_cols(x)[1:] == (1, 8)
    assert S._as_cols(Xf)[1:] == (3, 8)
    assert S._as_cols(np.zeros((8, 3), dtype=np.complex128, order="F"), True)[1:] == (3, 16)
    with pytest.raises(TypeError):
        S._as_cols(np.zeros(8, dtype=np.complex128))
    with pytest.raises(TypeError):
        S._as_cols(x, True)
    with pytest.raises(ValueError):
        S._as_cols(np.zeros((8, 3)))  # row-major
