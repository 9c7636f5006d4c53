// build_tree.hpp under the reference's own file name, so code written against the
// reference (#include <build_tree.hpp>) compiles unchanged with this directory on its
// include path.  Replaces build_tree.hpp:1-26 Cell, CSR-level lists, buildBinaryTree;
// everything is declared in mxc_b200/h2_solver.hpp (one process, one GPU).
#pragma once

#include "../h2_solver.hpp"
