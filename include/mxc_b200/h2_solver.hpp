// h2_solver.hpp — C++ host API of the B200 H^2 solver, with the names and
// argument order of the reference's solver.hpp / build_tree.hpp /
// kernel.hpp (one process, one GPU, no MPI), on top of the C ABI in h2dev.h.
//
// Differences a caller of the reference sees:
//  * The dense-matrix Accessor argument of the constructor is gone (it only
//    fed the reference's randomized SVD, whose result is never read).
//  * Kernels are the real Laplace3D and Yukawa3D (the complex Helmholtz3D is
//    not implemented); std::complex<double> vector overloads take and return
//    zero imaginary parts and throw if an input has a nonzero one.
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

// Cell of the binary tree (build_tree.hpp:6-15).
class Cell {
public:
  std::array<long long, 2> Child;
  std::array<long long, 2> Body;
  std::array<double, 3> R;
  std::array<double, 3> C;
  Cell() : Child{-1, -1}, Body{-1, -1}, R{0., 0., 0.}, C{0., 0., 0.} {}
};

// buildBinaryTree (build_tree.cpp:93-125): sorts bodies (nbodies x 3,
// row-major) in place and fills the 2^(levels+1) - 1 cells.
void buildBinaryTree(Cell* cells, double* bodies, long long nbodies, long long levels);

// Kernels (kernel.hpp:28-50): value 1/s at distance 0.
class MatrixAccessor {
public:
  int kind;
  double s, alpha;
  MatrixAccessor(int kind, double s, double alpha) : kind(kind), s(s), alpha(alpha) {}
  virtual ~MatrixAccessor() = default;
  double operator()(double d) const;  // host evaluation, as the device kernels
};

class Laplace3D : public MatrixAccessor {
public:
  explicit Laplace3D(double s) : MatrixAccessor(H2DEV_KERNEL_LAPLACE, s, 0.) {}
};

class Yukawa3D : public MatrixAccessor {
public:
  Yukawa3D(double s, double a) : MatrixAccessor(H2DEV_KERNEL_YUKAWA, s, a) {}
};

// Point sets of the reference's test_funcs.hpp: uniform_unit_cube_rnd
// (std::mt19937(seed)) and mesh_sphere (golden-angle spiral on a sphere of
// radius r).
void uniform_unit_cube_rnd(double* bodies, long long nbodies, double diameter, long long dim, unsigned seed);
void mesh_sphere(double* bodies, long long nbodies, double r);

// H2MatrixSolver (solver.hpp:11-47).  epi > 0: operator with an
// interpolative basis of relative threshold epi; epi == 0: fixed-rank
// orthogonal-basis preconditioner.  Vectors are host arrays in the tree
// order left by buildBinaryTree, length local_bodies.second -
// local_bodies.first (= N).
class H2MatrixSolver {
public:
  long long levels = 0;
  std::pair<long long, long long> local_bodies{0, 0};
  std::vector<double> resid;  // GMRES relative residual history (outer + 1 per right-hand side)
  long long iters = 0;        // GMRES restart cycles (first right-hand side)
  std::vector<int> info;      // singular redundant blocks per level after factorizeM

  H2MatrixSolver() = default;
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

  // solveRelErr (solver.cpp:276-285): sqrt(sum |x - ref|^2 / sum |ref|^2).
  static double solveRelErr(long long lenX, const double X[], const double ref[]);
  static double solveRelErr(long long lenX, const std::complex<double> X[], const std::complex<double> ref[]);

  h2dev_solver_t handle_solver() const { return s_; }
  // The device handle used when none is given: device 0, created on first use.
  static h2dev_handle_t default_handle();

private:
  h2dev_solver_t s_ = nullptr;
  h2dev_handle_t h_ = nullptr;
};

// Y = A_dense X (matrix-free on the GPU, FP64) for nrhs columns.
void dense_matvec(const MatrixAccessor& eval, const double bodies[], long long n, long long nrhs, const double X[],
                  double Y[], long long ld, h2dev_handle_t handle = nullptr);
