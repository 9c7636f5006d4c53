// mpi_single.hpp — the single-process stand-in for the MPI layer the
// reference's host code is written against (comm-mpi.hpp:1-53 and the MPI
// calls of main.cpp / solver.cpp).  This library runs one process on one
// GPU: every box of every level is local, so each collective of the
// reference's ColCommMPI (comm-mpi.cpp:198-245: level_merge, level_sum,
// neighbor_bcast) is the identity and the communicator is a plain tag.
//
// The names and signatures below are the subset of MPI the reference's
// callers use (MPI_Init / MPI_Finalize / MPI_Comm_rank / MPI_Comm_size /
// MPI_Barrier / MPI_Wtime / MPI_Allreduce / MPI_Comm_free), with the
// semantics of a one-rank MPI_COMM_WORLD.  Do not include a real <mpi.h> in
// the same translation unit: the two define the same names.
#pragma once

#include <chrono>
#include <cstddef>
#include <cstring>

#if defined(MPI_VERSION) || defined(OMPI_MPI_H) || defined(MPI_INCLUDED)
#error "mxc_b200/mpi_single.hpp replaces MPI for a single process; do not include <mpi.h> with it"
#endif

typedef int MPI_Comm;
// A datatype is its size in bytes, which is all a one-rank reduction needs.
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_COMM_NULL ((MPI_Comm)-1)
#define MPI_IN_PLACE ((void*)1)
#define MPI_SUCCESS 0
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_LONG_LONG ((MPI_Datatype)8)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_C_DOUBLE_COMPLEX ((MPI_Datatype)16)
#define MPI_SUM ((MPI_Op)0)
#define MPI_MAX ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
inline int MPI_Comm_size(MPI_Comm, int* size) {
  *size = 1;
  return MPI_SUCCESS;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Comm_free(MPI_Comm* comm) {
  *comm = MPI_COMM_NULL;
  return MPI_SUCCESS;
}
inline double MPI_Wtime() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
// One rank: the reduction of one contribution is that contribution.
inline int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype datatype, MPI_Op, MPI_Comm) {
  if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf && count > 0)
    std::memcpy(recvbuf, sendbuf, (size_t)count * (size_t)datatype);
  return MPI_SUCCESS;
}

// comm-mpi.hpp:9-52 ColCommMPI, reduced to what callers outside the solver
// touch: the communication stopwatch (comm-mpi.cpp:247-262), which reads 0
// because nothing is communicated.
class ColCommMPI {
public:
  static double get_comm_time() { return 0.; }
  static void record_mpi() {}
};
