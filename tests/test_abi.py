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
