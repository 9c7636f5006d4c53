// h2matrix.hpp under the reference's own file name, so code written against the
// reference (#include <h2matrix.hpp>) compiles unchanged with this directory on its
// include path.  Replaces h2matrix.hpp:11-57 H2Matrix (per-level metadata);
// everything is declared in mxc_b200/h2_solver.hpp (one process, one GPU).
#pragma once

#include "../h2_solver.hpp"
