// h2_solver.hpp — C++ host API of the B200 H^2 solver, with the names and
// argument order of the reference's solver.hpp / build_tree.hpp /
// kernel.hpp / test_funcs.hpp (one process, one GPU, no MPI), on top of the
// C ABI in h2dev.h.  The headers under include/mxc_b200/reference/ carry the
// reference's own file names, so a caller written against the reference
// compiles unchanged with that directory on its include path.
//
// Differences a caller of the reference sees:
//  * MPI is the single-process stand-in of mpi_single.hpp (MPI_Comm is a
//    tag, every collective the identity); the constructor's MPI_Comm is
//    accepted and must describe one process.
//  * The dense-matrix Accessor argument of the constructor is accepted and
//    not read (in the reference it only fed the randomized SVD of
//    Hmatrix::construct, h-matrix.cpp:103-116, whose result is never used).
//  * Kernels run on the device, so the solver accepts Laplace3D, Yukawa3D
//    and Helmholtz3D (a MatrixAccessor subclass of the caller's own works on
//    the host, for gen_matrix, but the solver rejects it).  With a real
//    kernel the std::complex<double> vector overloads take and return zero
//    imaginary parts and throw if an input has a nonzero one.  With
//    Helmholtz3D the vectors are complex and only the std::complex<double>
//    overloads are accepted; the device holds the real symmetric form of the
//    complex matrix (two real unknowns per body), so A[l].Dims / DimsLr count
//    real unknowns, twice the reference's complex box dimensions.
//  * The *Device methods (factorizeDeviceM, solvePreconditionDevice,
//    solveGMRESDevice, matVecMulSp) are the same device computations as the
//    plain ones: every method here runs on the GPU.
//  * Failures throw std::runtime_error with the library's message instead of
//    printing `info`; a GMRES that stops above tol is not a failure (resid
//    and iters tell).
//  * Extensions: `samples` (far-list cap of the basis construction), the
//    storage precision of a matrix, and multi-right-hand-side solves.
#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <utility>
#include <vector>

#include "../h2dev.h"
#include "mpi_single.hpp"

// Cell of the binary tree (build_tree.hpp:6-15).
class Cell {
public:
  std::array<long long, 2> Child;
  std::array<long long, 2> Body;
  std::array<double, 3> R;
  std::array<double, 3> C;
  Cell() : Child{-1, -1}, Body{-1, -1}, R{0., 0., 0.}, C{0., 0., 0.} {}
};

// buildBinaryTree (build_tree.cpp:67-99): sorts bodies (nbodies x 3,
// row-major) in place and fills the 2^(levels+1) - 1 cells.
void buildBinaryTree(Cell* cells, double* bodies, long long nbodies, long long levels);

// Kernel of the matrix (kernel.hpp:23-50): K(d) of the distance d between
// two bodies, the value 1/s at d == 0.  The device evaluates the kernels it
// knows (kind); operator() is the same function on the host, virtual as in
// the reference so a caller may derive its own (kind -1: host only).
class MatrixAccessor {
public:
  int kind = -1;
  double s = 1., alpha = 0.;
  MatrixAccessor() = default;
  MatrixAccessor(int kind, double s, double alpha) : kind(kind), s(s), alpha(alpha) {}
  virtual ~MatrixAccessor() = default;
  virtual std::complex<double> operator()(double d) const;
};

class Laplace3D : public MatrixAccessor {
public:
  double singularity;  // the diagonal value 1/s, as the reference's member
  explicit Laplace3D(double s) : MatrixAccessor(H2DEV_KERNEL_LAPLACE, s, 0.), singularity(1. / s) {}
};

class Yukawa3D : public MatrixAccessor {
public:
  double singularity;
  Yukawa3D(double s, double a) : MatrixAccessor(H2DEV_KERNEL_YUKAWA, s, a), singularity(1. / s) {}
};

// Helmholtz3D (kernel.hpp:63-74): exp(-i k d) / d, 1/s at d == 0.
class Helmholtz3D : public MatrixAccessor {
public:
  double k;
  double singularity;
  Helmholtz3D(double wave_number, double s)
      : MatrixAccessor(H2DEV_KERNEL_HELMHOLTZ, s, wave_number), k(wave_number), singularity(1. / s) {}
};

// gen_matrix (kernel.cpp:71-85): Aij (m x n, column-major) = K(|bi_y - bj_x|)
// with the distance of the 3-argument std::hypot.  Laplace3D / Yukawa3D /
// Helmholtz3D blocks are generated on the device (Laplace bit for bit as the
// reference's host loop); other MatrixAccessor kinds by the host loop.
void gen_matrix(const MatrixAccessor& eval, long long m, long long n, const double* bi, const double* bj,
                std::complex<double> Aij[]);

// Dense operator access (kernel.hpp:6-19): C = op(A(iA:, jA:)) B.  The
// reference's constructor takes one and only feeds it to a randomized SVD
// whose output is never read; here it is accepted and not read.  DenseZMat
// holds the whole M x N complex matrix on the host (zero-initialised, filled
// by gen_matrix) and multiplies with it on the host, as the reference's
// dense check does (main.cpp:83-84, 114).
class Accessor {
public:
  long long M, N;
  Accessor(long long M, long long N) : M(M), N(N) {}
  virtual ~Accessor() = default;
  virtual void op_Aij_mulB(char opA, long long mC, long long nC, long long k, long long iA, long long jA,
                           const std::complex<double>* B_in, long long strideB, std::complex<double>* C_out,
                           long long strideC) const = 0;
};

class DenseZMat : public Accessor {
public:
  std::complex<double>* A;
  DenseZMat(long long M, long long N);
  ~DenseZMat() override;
  DenseZMat(const DenseZMat&) = delete;
  DenseZMat& operator=(const DenseZMat&) = delete;
  void op_Aij_mulB(char opA, long long mC, long long nC, long long k, long long iA, long long jA,
                   const std::complex<double>* B_in, long long strideB, std::complex<double>* C_out,
                   long long strideC) const override;
};

// Device environment of the reference's *Device methods (gpu_handles.cuh:
// 10-18, gpu_handles.cu:54-71): here the library's device handle; NCCL
// communicators do not exist in one process (ncclComms is an unused tag).
typedef h2dev_handle_t deviceHandle_t;
typedef void* ncclComms;
void initGpuEnvs(deviceHandle_t* handle);
void finalizeGpuEnvs(deviceHandle_t handle);

// Per-level metadata of the reference's H2Matrix (h2matrix.hpp:11-57):
// box dimensions and ranks, the near-pair CSR of the level (level-local
// column indices) and the singular-block count of the last factorization.
// The matrix containers (Q, R, A, C, U, X, Y, Z, W) stay in device memory;
// h2dev_solver_export copies one level's container out.
class H2Matrix {
public:
  long long lenX = 0;
  long long LowerZ = 0;
  std::vector<long long> Dims;
  std::vector<long long> DimsLr;
  std::vector<long long> ARows;
  std::vector<long long> ACols;
  int info = 0;
};

// Point sets of the reference's test_funcs.hpp: uniform_unit_cube_rnd
// (std::mt19937(seed)) and mesh_sphere (golden-angle spiral on a sphere of
// radius r).
void uniform_unit_cube_rnd(double* bodies, long long nbodies, double diameter, long long dim, unsigned seed);
void mesh_sphere(double* bodies, long long nbodies, double r);
// test_funcs.hpp:94-111: appends the 25-column result row (plus the residual
// history) the reference's plot scripts read.
void write_to_csv(const char* fname, int mpi_size, long long N, double theta, long long leaf_size, long long rank,
                  double epi, const char* mode, double h2cerr, double h2ctime, double h2ctime_comm, double h2mvtime,
                  double h2mvtime_comm, double dense_mvtime, double mctime, double mctime_comm, double mcerr,
                  double factor_time, double factor_time_comm, double sub_time, double sub_time_comm, double sub_err,
                  double gmres_err, double gmres_iters, double gmres_time, double gmres_time_comm,
                  const double* iter_err);

// H2MatrixSolver (solver.hpp:11-47).  epi > 0: operator with an
// interpolative basis of relative threshold epi; epi == 0: fixed-rank
// orthogonal-basis preconditioner.  Vectors are host arrays in the tree
// order left by buildBinaryTree, length local_bodies.second -
// local_bodies.first (= N).
class H2MatrixSolver {
public:
  long long levels = 0;
  std::vector<H2Matrix> A;    // per-level metadata, levels + 1 entries
  std::vector<MPI_Comm> allocedComm;  // always empty: one process allocates no communicators
  std::pair<long long, long long> local_bodies{0, 0};
  std::vector<double> resid;  // GMRES relative residual history (outer + 1 per right-hand side)
  long long iters = 0;        // GMRES restart cycles (first right-hand side)
  std::vector<int> info;      // singular redundant blocks per level after factorizeM

  H2MatrixSolver() = default;
  // The reference's constructor (solver.hpp:28, solver.cpp:12-41): every far
  // body enters the bases, as in the reference.  eval_d is not read; world
  // must be a one-process communicator.
  H2MatrixSolver(const Accessor& eval_d, const MatrixAccessor& eval, double epi, long long rank,
                 long long leveled_rank, const std::vector<Cell>& cells, double theta, const double bodies[],
                 long long levels, MPI_Comm world = MPI_COMM_WORLD);
  H2MatrixSolver(const MatrixAccessor& eval, double epi, long long rank, long long leveled_rank,
                 const std::vector<Cell>& cells, double theta, const double bodies[], long long levels,
                 long long samples = 0, int precision = H2DEV_FP64, h2dev_handle_t handle = nullptr);
  H2MatrixSolver(const H2MatrixSolver&) = delete;
  H2MatrixSolver& operator=(const H2MatrixSolver&) = delete;
  H2MatrixSolver(H2MatrixSolver&& o) noexcept;
  H2MatrixSolver& operator=(H2MatrixSolver&& o) noexcept;
  ~H2MatrixSolver();

  void matVecMul(double X[]);
  void matVecMul(std::complex<double> X[]);
  void factorizeM();
  void solvePrecondition(double X[]);
  void solvePrecondition(std::complex<double> X[]);
  void solveGMRES(double tol, H2MatrixSolver& M, double X[], const double B[], long long inner_iters,
                  long long outer_iters);
  void solveGMRES(double tol, H2MatrixSolver& M, std::complex<double> X[], const std::complex<double> B[],
                  long long inner_iters, long long outer_iters);
  // nrhs columns of length N with leading dimension ld; resid holds
  // (outer_iters + 1) entries per column.
  void solveGMRES(double tol, H2MatrixSolver& M, double X[], const double B[], long long nrhs, long long ld,
                  long long inner_iters, long long outer_iters, bool early_exit = false);

  // The reference's device-side methods (solver.hpp:29-45).  Every
  // computation of this class already runs on the device, so these are the
  // plain methods above; init / alloc / free calls have nothing to do.
  void init_gpu_handles(const ncclComms nccl_comms);
  void move_data_gpu();
  void allocSparseMV(deviceHandle_t handle, const ncclComms nccl_comms);
  void matVecMulSp(deviceHandle_t handle, std::complex<double> X[]);
  void factorizeDeviceM(deviceHandle_t handle);
  void solvePreconditionDevice(deviceHandle_t handle, std::complex<double> X[]);
  void solveGMRESDevice(deviceHandle_t handle, double tol, H2MatrixSolver& M, std::complex<double> X[],
                        const std::complex<double> B[], long long inner_iters, long long outer_iters,
                        const ncclComms nccl_comms);
  void free_all_comms();
  void freeSparseMV();
  void free_gpu_handles();

  // solveRelErr (solver.cpp:229-238): sqrt(sum (x - ref)^2 / sum ref^2) over
  // the real parts (the reference's complex overload ignores imaginary parts).
  static double solveRelErr(long long lenX, const double X[], const double ref[]);
  static double solveRelErr(long long lenX, const std::complex<double> X[], const std::complex<double> ref[],
                            MPI_Comm world = MPI_COMM_WORLD);

  h2dev_solver_t handle_solver() const { return s_; }
  // The device handle used when none is given: device 0, created on first use.
  static h2dev_handle_t default_handle();

private:
  void create(const MatrixAccessor& eval, double epi, long long rank, long long leveled_rank,
              const std::vector<Cell>& cells, double theta, const double bodies[], long long samples, int precision);
  void fill_levels(const std::vector<Cell>& cells, double theta);
  h2dev_solver_t s_ = nullptr;
  h2dev_handle_t h_ = nullptr;
  bool complex_ = false;  // Helmholtz3D: complex vectors
};

// Y = A_dense X (matrix-free on the GPU, FP64) for nrhs columns.  With
// Helmholtz3D, X and Y hold complex columns as interleaved real/imaginary
// parts (2n doubles each, ld >= 2n).
void dense_matvec(const MatrixAccessor& eval, const double bodies[], long long n, long long nrhs, const double X[],
                  double Y[], long long ld, h2dev_handle_t handle = nullptr);
