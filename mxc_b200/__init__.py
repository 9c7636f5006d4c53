"""B200-native H^2-matrix ULV-preconditioned GMRES solver (sm_100a).

A drop-in for delta-leader/mxc's solver path: the C ABI in include/h2dev.h
(libmxcb200.so) plus this Python mirror of solver.hpp's H2MatrixSolver.
"""
from ._lib import (FP32, FP64, KERNEL_HELMHOLTZ, KERNEL_LAPLACE, KERNEL_QUADRATIC, KERNEL_YUKAWA, H2DevError,  # noqa: F401
                   LIB_PATH, lib)
from .solver import (H2MatrixSolver, Handle, Helmholtz3D, Kernel, Laplace3D, Quadratic, Tree, Yukawa3D, build_tree,  # noqa: F401
                     dense_matvec, gen_block, levels_for, mesh_sphere, pair_csr, rel_err_device, uniform_rhs, uniform_unit_cube_rnd)
