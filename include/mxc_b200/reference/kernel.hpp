// kernel.hpp under the reference's own file name, so code written against the
// reference (#include <kernel.hpp>) compiles unchanged with this directory on its
// include path.  Replaces kernel.hpp:1-78 Accessor, DenseZMat, MatrixAccessor, Laplace3D, Yukawa3D, Helmholtz3D, gen_matrix;
// everything is declared in mxc_b200/h2_solver.hpp (one process, one GPU).
#pragma once

#include "../h2_solver.hpp"
