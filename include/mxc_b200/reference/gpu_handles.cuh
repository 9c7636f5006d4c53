// gpu_handles.cuh under the reference's own file name, so code written against the
// reference (#include <gpu_handles.cuh>) compiles unchanged with this directory on its
// include path.  Replaces gpu_handles.cuh:10-18 deviceHandle_t, ncclComms, initGpuEnvs, finalizeGpuEnvs;
// everything is declared in mxc_b200/h2_solver.hpp (one process, one GPU).
#pragma once

#include "../h2_solver.hpp"
