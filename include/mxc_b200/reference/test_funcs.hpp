// test_funcs.hpp under the reference's own file name, so code written against the
// reference (#include <test_funcs.hpp>) compiles unchanged with this directory on its
// include path.  Replaces test_funcs.hpp:31-111 uniform_unit_cube_rnd, mesh_sphere, write_to_csv;
// everything is declared in mxc_b200/h2_solver.hpp (one process, one GPU).
#pragma once

#include "../h2_solver.hpp"
