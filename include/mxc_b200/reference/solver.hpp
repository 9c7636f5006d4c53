// solver.hpp under the reference's own file name, so code written against the
// reference (#include <solver.hpp>) compiles unchanged with this directory on its
// include path.  Replaces solver.hpp:11-47 H2MatrixSolver;
// everything is declared in mxc_b200/h2_solver.hpp (one process, one GPU).
#pragma once

#include "../h2_solver.hpp"
