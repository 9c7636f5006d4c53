// comm-mpi.hpp under the reference's own file name, so code written against the
// reference (#include <comm-mpi.hpp>) compiles unchanged with this directory on its
// include path.  Replaces comm-mpi.hpp:1-53 MPI and ColCommMPI (single-process stand-in);
// everything is declared in mxc_b200/h2_solver.hpp (one process, one GPU).
#pragma once

#include "../h2_solver.hpp"
