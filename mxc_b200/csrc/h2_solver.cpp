// C++ host API (include/mxc_b200/h2_solver.hpp) over the C ABI of h2dev.h:
// the reference's class and function names, backed by the device solver.
#include "mxc_b200/h2_solver.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <mutex>
#include <stdexcept>
#include <string>

namespace {

void check(int rc, const char* what) {
  if (rc != H2DEV_OK) {
    const char* msg = h2dev_last_error_message();
    throw std::runtime_error(std::string(what) + " failed (status " + std::to_string(rc) +
                             "): " + (msg ? msg : ""));
  }
}

// Real parts of n complex values; throws when an imaginary part is nonzero
// (the kernels here are real, so every vector of a solve is real).
std::vector<double> real_parts(const std::complex<double>* X, long long n) {
  std::vector<double> r((size_t)n);
  for (long long i = 0; i < n; i++) {
    if (X[i].imag() != 0.) throw std::runtime_error("complex vector with a nonzero imaginary part (real kernels only)");
    r[(size_t)i] = X[i].real();
  }
  return r;
}

void put_real(std::complex<double>* X, const std::vector<double>& r) {
  for (size_t i = 0; i < r.size(); i++) X[i] = std::complex<double>(r[i], 0.);
}

}  // namespace

void buildBinaryTree(Cell* cells, double* bodies, long long nbodies, long long levels) {
  const long long nc = (2LL << levels) - 1;
  std::vector<int64_t> child((size_t)nc * 2), body((size_t)nc * 2);
  std::vector<double> R((size_t)nc * 3), Cc((size_t)nc * 3);
  check(h2_build_tree(bodies, nbodies, levels, child.data(), body.data(), R.data(), Cc.data()), "h2_build_tree");
  for (long long i = 0; i < nc; i++) {
    for (int k = 0; k < 2; k++) {
      cells[i].Child[k] = child[(size_t)(2 * i + k)];
      cells[i].Body[k] = body[(size_t)(2 * i + k)];
    }
    for (int k = 0; k < 3; k++) {
      cells[i].R[k] = R[(size_t)(3 * i + k)];
      cells[i].C[k] = Cc[(size_t)(3 * i + k)];
    }
  }
}

std::complex<double> MatrixAccessor::operator()(double d) const {
  if (kind < 0) throw std::logic_error("MatrixAccessor: a kernel of the caller's own must override operator()");
  if (d == 0.) return 1. / s;
  if (kind == H2DEV_KERNEL_YUKAWA) return std::exp(-alpha * d) / d;
  if (kind == H2DEV_KERNEL_QUADRATIC) return d * d + alpha;
  if (kind == H2DEV_KERNEL_HELMHOLTZ) return std::exp(std::complex<double>(0., -alpha * d)) / d;
  return 1. / d;
}

void gen_matrix(const MatrixAccessor& eval, long long m, long long n, const double* bi, const double* bj,
                std::complex<double> Aij[]) {
  if (m <= 0 || n <= 0) return;
  const bool device =
      eval.kind == H2DEV_KERNEL_LAPLACE || eval.kind == H2DEV_KERNEL_YUKAWA || eval.kind == H2DEV_KERNEL_HELMHOLTZ;
  if (!device) {
    for (long long x = 0; x < n; x++)
      for (long long y = 0; y < m; y++) {
        const double d = std::hypot(bi[3 * y] - bj[3 * x], bi[3 * y + 1] - bj[3 * x + 1], bi[3 * y + 2] - bj[3 * x + 2]);
        Aij[y + x * m] = eval(d);
      }
    return;
  }
  // Column panels of at most 2^26 doubles through the device generator (a
  // Helmholtz panel holds interleaved real and imaginary parts).
  const long long w = eval.kind == H2DEV_KERNEL_HELMHOLTZ ? 2 : 1;
  const long long cols = std::max<long long>(1, ((long long)1 << 26) / (w * m));
  std::vector<double> buf((size_t)(w * m * std::min(cols, n)));
  for (long long x0 = 0; x0 < n; x0 += cols) {
    const long long nc = std::min(cols, n - x0);
    check(h2dev_gen_block(H2MatrixSolver::default_handle(), eval.kind, eval.s, eval.alpha, bi, m, bj + 3 * x0, nc,
                          buf.data()),
          "h2dev_gen_block");
    for (long long e = 0; e < m * nc; e++)
      Aij[x0 * m + e] = w == 2 ? std::complex<double>(buf[(size_t)(2 * e)], buf[(size_t)(2 * e + 1)])
                               : std::complex<double>(buf[(size_t)e], 0.);
  }
}

DenseZMat::DenseZMat(long long M, long long N) : Accessor(M, N), A(nullptr) {
  if (0 < M && 0 < N) A = new std::complex<double>[(size_t)(M * N)]();
}

DenseZMat::~DenseZMat() { delete[] A; }

void DenseZMat::op_Aij_mulB(char opA, long long mC, long long nC, long long k, long long iA, long long jA,
                            const std::complex<double>* B_in, long long strideB, std::complex<double>* C_out,
                            long long strideC) const {
  // C (mC x nC) = op(A_sub) B (k x nC); A_sub starts at (iA, jA) with leading
  // dimension M: mC x k as stored ('N'), k x mC transposed ('T') or
  // conjugate-transposed ('C').
  const std::complex<double>* As = A + iA + jA * M;
  const bool t = opA == 'T' || opA == 't', c = opA == 'C' || opA == 'c';
  for (long long j = 0; j < nC; j++) {
    std::complex<double>* cj = C_out + j * strideC;
    const std::complex<double>* bj = B_in + j * strideB;
    for (long long i = 0; i < mC; i++) cj[i] = 0.;
    if (t || c) {
      for (long long i = 0; i < mC; i++) {
        std::complex<double> acc = 0.;
        for (long long q = 0; q < k; q++) acc += (c ? std::conj(As[q + i * M]) : As[q + i * M]) * bj[q];
        cj[i] = acc;
      }
    } else {
      for (long long q = 0; q < k; q++) {
        const std::complex<double> b = bj[q];
        const std::complex<double>* aq = As + q * M;
        for (long long i = 0; i < mC; i++) cj[i] += aq[i] * b;
      }
    }
  }
}

void initGpuEnvs(deviceHandle_t* handle) { check(h2dev_handle_create(0, handle), "h2dev_handle_create"); }

void finalizeGpuEnvs(deviceHandle_t handle) {
  if (handle) check(h2dev_handle_destroy(handle), "h2dev_handle_destroy");
}

void write_to_csv(const char* fname, int mpi_size, long long N, double theta, long long leaf_size, long long rank,
                  double epi, const char* mode, double h2cerr, double h2ctime, double h2ctime_comm, double h2mvtime,
                  double h2mvtime_comm, double dense_mvtime, double mctime, double mctime_comm, double mcerr,
                  double factor_time, double factor_time_comm, double sub_time, double sub_time_comm, double sub_err,
                  double gmres_err, double gmres_iters, double gmres_time, double gmres_time_comm,
                  const double* iter_err) {
  std::ofstream f(fname, std::ios_base::app);
  if (!f) return;
  f << mpi_size << ',' << N << ',' << theta << ',' << leaf_size << ',' << rank << ',' << epi << ',' << mode << ',';
  f << h2cerr << ',' << h2ctime << ',' << h2ctime_comm << ',' << h2mvtime << ',' << h2mvtime_comm << ','
    << dense_mvtime << ',';
  f << mctime << ',' << mctime_comm << ',' << mcerr << ',' << factor_time << ',' << factor_time_comm << ',' << sub_time
    << ',' << sub_time_comm << ',' << sub_err << ',';
  f << gmres_err << ',' << gmres_iters << ',' << gmres_time << ',' << gmres_time_comm;
  for (long long i = 0; i <= (long long)gmres_iters; i++) f << ',' << iter_err[i];
  f << std::endl;
}

void uniform_unit_cube_rnd(double* bodies, long long nbodies, double diameter, long long dim, unsigned seed) {
  check(h2_uniform_unit_cube_rnd(bodies, nbodies, diameter, dim, seed), "h2_uniform_unit_cube_rnd");
}

void mesh_sphere(double* bodies, long long nbodies, double r) {
  // Golden-angle (Fibonacci) spiral: point i at height y_i running from r to
  // -r in equal steps, turned by i times the golden angle about the y axis.
  const double golden = M_PI * (3. - std::sqrt(5.));
  for (long long i = 0; i < nbodies; i++) {
    const double t = nbodies > 1 ? (double)i / (double)(nbodies - 1) : 0.;
    const double y = r - 2. * r * t;
    const double ring = std::sqrt(r * r - y * y);
    const double a = golden * (double)i;
    bodies[3 * i] = ring * std::cos(a);
    bodies[3 * i + 1] = y;
    bodies[3 * i + 2] = ring * std::sin(a);
  }
}

h2dev_handle_t H2MatrixSolver::default_handle() {
  static std::once_flag once;
  static h2dev_handle_t h = nullptr;
  std::call_once(once, [] { check(h2dev_handle_create(0, &h), "h2dev_handle_create"); });
  return h;
}

H2MatrixSolver::H2MatrixSolver(const Accessor&, const MatrixAccessor& eval, double epi, long long rank,
                               long long leveled_rank, const std::vector<Cell>& cells, double theta,
                               const double bodies[], long long levels, MPI_Comm world)
    : levels(levels), h_(default_handle()) {
  int size = 1;
  MPI_Comm_size(world, &size);
  if (size != 1) throw std::invalid_argument("H2MatrixSolver: one process only (MPI_Comm of size 1)");
  create(eval, epi, rank, leveled_rank, cells, theta, bodies, 0, H2DEV_FP64);
}

H2MatrixSolver::H2MatrixSolver(const MatrixAccessor& eval, double epi, long long rank, long long leveled_rank,
                               const std::vector<Cell>& cells, double theta, const double bodies[], long long levels,
                               long long samples, int precision, h2dev_handle_t handle)
    : levels(levels), h_(handle ? handle : default_handle()) {
  create(eval, epi, rank, leveled_rank, cells, theta, bodies, samples, precision);
}

void H2MatrixSolver::create(const MatrixAccessor& eval, double epi, long long rank, long long leveled_rank,
                            const std::vector<Cell>& cells, double theta, const double bodies[], long long samples,
                            int precision) {
  if (eval.kind != H2DEV_KERNEL_LAPLACE && eval.kind != H2DEV_KERNEL_YUKAWA && eval.kind != H2DEV_KERNEL_QUADRATIC &&
      eval.kind != H2DEV_KERNEL_HELMHOLTZ)
    throw std::invalid_argument("H2MatrixSolver: the device evaluates Laplace3D, Yukawa3D and Helmholtz3D kernels only");
  complex_ = eval.kind == H2DEV_KERNEL_HELMHOLTZ;
  const long long nc = (long long)cells.size();
  if (nc < (2LL << levels) - 1) throw std::invalid_argument("cells: fewer than 2^(levels+1) - 1 cells");
  std::vector<int64_t> child((size_t)nc * 2), body((size_t)nc * 2);
  std::vector<double> R((size_t)nc * 3), Cc((size_t)nc * 3);
  for (long long i = 0; i < nc; i++) {
    for (int k = 0; k < 2; k++) {
      child[(size_t)(2 * i + k)] = cells[(size_t)i].Child[k];
      body[(size_t)(2 * i + k)] = cells[(size_t)i].Body[k];
    }
    for (int k = 0; k < 3; k++) {
      R[(size_t)(3 * i + k)] = cells[(size_t)i].R[k];
      Cc[(size_t)(3 * i + k)] = cells[(size_t)i].C[k];
    }
  }
  const long long n = cells[0].Body[1] - cells[0].Body[0];
  check(h2dev_solver_create(h_, eval.kind, eval.s, eval.alpha, epi, rank, leveled_rank, nc, child.data(), body.data(),
                            R.data(), Cc.data(), theta, bodies, n, levels, samples, precision, &s_),
        "h2dev_solver_create");
  local_bodies = {0, n};
  fill_levels(cells, theta);
}

// H2Matrix metadata per level: Dims / DimsLr from the device solver, the
// near-pair CSR of the level from the tree (build_tree.cpp:41-58) with
// level-local columns, lenX = sum of Dims, LowerZ = 0 (one process holds
// every box, so a level's vector starts at the lower level's first rank).
void H2MatrixSolver::fill_levels(const std::vector<Cell>& cells, double theta) {
  const long long nc = (2LL << levels) - 1;
  std::vector<int64_t> child((size_t)nc * 2), body((size_t)nc * 2);
  std::vector<double> R((size_t)nc * 3), Cc((size_t)nc * 3);
  for (long long i = 0; i < nc; i++) {
    for (int k = 0; k < 2; k++) {
      child[(size_t)(2 * i + k)] = cells[(size_t)i].Child[k];
      body[(size_t)(2 * i + k)] = cells[(size_t)i].Body[k];
    }
    for (int k = 0; k < 3; k++) {
      R[(size_t)(3 * i + k)] = cells[(size_t)i].R[k];
      Cc[(size_t)(3 * i + k)] = cells[(size_t)i].C[k];
    }
  }
  std::vector<int64_t> row((size_t)nc + 1);
  int64_t nnz = 0;
  check(h2_pair_csr('N', nc, child.data(), body.data(), R.data(), Cc.data(), theta, row.data(), nullptr, 0, &nnz),
        "h2_pair_csr");
  std::vector<int64_t> col((size_t)std::max<int64_t>(1, nnz));
  check(h2_pair_csr('N', nc, child.data(), body.data(), R.data(), Cc.data(), theta, row.data(), col.data(), nnz, &nnz),
        "h2_pair_csr");
  A.assign((size_t)levels + 1, H2Matrix());
  for (long long l = 0; l <= levels; l++) {
    H2Matrix& m = A[(size_t)l];
    const long long nodes = 1LL << l, g0 = nodes - 1;
    m.Dims.assign((size_t)nodes, 0);
    m.DimsLr.assign((size_t)nodes, 0);
    std::vector<int64_t> d((size_t)nodes), r((size_t)nodes);
    check(h2dev_solver_level_dims(s_, l, d.data(), r.data()), "h2dev_solver_level_dims");
    m.lenX = 0;
    for (long long i = 0; i < nodes; i++) {
      m.Dims[(size_t)i] = d[(size_t)i];
      m.DimsLr[(size_t)i] = r[(size_t)i];
      m.lenX += d[(size_t)i];
    }
    m.ARows.assign(1, 0);
    for (long long i = 0; i < nodes; i++) {
      for (int64_t k = row[(size_t)(g0 + i)]; k < row[(size_t)(g0 + i + 1)]; k++) m.ACols.push_back(col[(size_t)k] - g0);
      m.ARows.push_back((long long)m.ACols.size());
    }
  }
}

H2MatrixSolver::H2MatrixSolver(H2MatrixSolver&& o) noexcept { *this = std::move(o); }

H2MatrixSolver& H2MatrixSolver::operator=(H2MatrixSolver&& o) noexcept {
  if (this != &o) {
    if (s_) h2dev_solver_destroy(s_);
    levels = o.levels;
    A = std::move(o.A);
    local_bodies = o.local_bodies;
    resid = std::move(o.resid);
    iters = o.iters;
    info = std::move(o.info);
    s_ = o.s_;
    h_ = o.h_;
    complex_ = o.complex_;
    o.s_ = nullptr;
  }
  return *this;
}

H2MatrixSolver::~H2MatrixSolver() {
  if (s_) h2dev_solver_destroy(s_);
}

void H2MatrixSolver::matVecMul(double X[]) {
  if (complex_) throw std::invalid_argument("matVecMul: Helmholtz3D takes complex vectors");
  const long long n = local_bodies.second - local_bodies.first;
  check(h2dev_matvec(s_, 1, X, n), "h2dev_matvec");
}

// Complex vectors of a Helmholtz3D solver go to the device as interleaved
// real/imaginary parts (the std::complex<double> layout).
void H2MatrixSolver::matVecMul(std::complex<double> X[]) {
  if (complex_) {
    const long long n = local_bodies.second - local_bodies.first;
    check(h2dev_matvec(s_, 1, reinterpret_cast<double*>(X), 2 * n), "h2dev_matvec");
    return;
  }
  std::vector<double> r = real_parts(X, local_bodies.second - local_bodies.first);
  matVecMul(r.data());
  put_real(X, r);
}

void H2MatrixSolver::factorizeM() {
  info.assign((size_t)levels + 1, 0);
  const int rc = h2dev_factorize(s_, info.data());
  if (rc != H2DEV_ERR_SINGULAR) check(rc, "h2dev_factorize");
  for (long long l = 0; l <= levels && l < (long long)A.size(); l++) A[(size_t)l].info = info[(size_t)l];
  // solver.cpp:97-99
  for (long long l = levels; l >= 0; l--)
    if (info[(size_t)l]) std::printf("singularity detected at level %lld.\n", l);
}

void H2MatrixSolver::solvePrecondition(double X[]) {
  if (complex_) throw std::invalid_argument("solvePrecondition: Helmholtz3D takes complex vectors");
  const long long n = local_bodies.second - local_bodies.first;
  check(h2dev_solve_precondition(s_, 1, X, n), "h2dev_solve_precondition");
}

void H2MatrixSolver::solvePrecondition(std::complex<double> X[]) {
  if (complex_) {
    const long long n = local_bodies.second - local_bodies.first;
    check(h2dev_solve_precondition(s_, 1, reinterpret_cast<double*>(X), 2 * n), "h2dev_solve_precondition");
    return;
  }
  std::vector<double> r = real_parts(X, local_bodies.second - local_bodies.first);
  solvePrecondition(r.data());
  put_real(X, r);
}

void H2MatrixSolver::solveGMRES(double tol, H2MatrixSolver& M, double X[], const double B[], long long nrhs,
                                long long ld, long long inner_iters, long long outer_iters, bool early_exit) {
  if (complex_) throw std::invalid_argument("solveGMRES: Helmholtz3D takes complex vectors");
  resid.assign((size_t)((outer_iters + 1) * nrhs), 0.);
  std::vector<int64_t> it((size_t)nrhs, 0);
  const int rc = h2dev_solve_gmres(s_, M.s_, tol, nrhs, X, B, ld, inner_iters, outer_iters, early_exit ? 1 : 0,
                                   resid.data(), it.data());
  if (rc != H2DEV_ERR_NOCONV) check(rc, "h2dev_solve_gmres");
  iters = nrhs > 0 ? it[0] : 0;
}

void H2MatrixSolver::solveGMRES(double tol, H2MatrixSolver& M, double X[], const double B[], long long inner_iters,
                                long long outer_iters) {
  const long long n = local_bodies.second - local_bodies.first;
  solveGMRES(tol, M, X, B, 1, n, inner_iters, outer_iters, false);
}

void H2MatrixSolver::solveGMRES(double tol, H2MatrixSolver& M, std::complex<double> X[],
                                const std::complex<double> B[], long long inner_iters, long long outer_iters) {
  const long long n = local_bodies.second - local_bodies.first;
  if (complex_) {
    if (!M.complex_) throw std::invalid_argument("solveGMRES: operator and preconditioner kernels differ");
    resid.assign((size_t)(outer_iters + 1), 0.);
    int64_t it = 0;
    const int rc = h2dev_solve_gmres(s_, M.s_, tol, 1, reinterpret_cast<double*>(X), reinterpret_cast<const double*>(B),
                                     2 * n, inner_iters, outer_iters, 0, resid.data(), &it);
    if (rc != H2DEV_ERR_NOCONV) check(rc, "h2dev_solve_gmres");
    iters = it;
    return;
  }
  std::vector<double> x = real_parts(X, n), b = real_parts(B, n);
  solveGMRES(tol, M, x.data(), b.data(), 1, n, inner_iters, outer_iters, false);
  put_real(X, x);
}

double H2MatrixSolver::solveRelErr(long long lenX, const double X[], const double ref[]) {
  double num = 0., den = 0.;
  for (long long i = 0; i < lenX; i++) {
    const double d = X[i] - ref[i];
    num += d * d;
    den += ref[i] * ref[i];
  }
  return std::sqrt(num / den);
}

// solver.cpp:229-238 sums the squares of the real parts only (of the
// difference and of ref); imaginary parts do not enter the error.
double H2MatrixSolver::solveRelErr(long long lenX, const std::complex<double> X[], const std::complex<double> ref[],
                                   MPI_Comm) {
  double num = 0., den = 0.;
  for (long long i = 0; i < lenX; i++) {
    const double d = X[i].real() - ref[i].real();
    num += d * d;
    den += ref[i].real() * ref[i].real();
  }
  return std::sqrt(num / den);
}

void dense_matvec(const MatrixAccessor& eval, const double bodies[], long long n, long long nrhs, const double X[],
                  double Y[], long long ld, h2dev_handle_t handle) {
  h2dev_handle_t h = handle ? handle : H2MatrixSolver::default_handle();
  check(h2dev_dense_matvec(h, eval.kind, eval.s, eval.alpha, bodies, n, nrhs, X, Y, ld), "h2dev_dense_matvec");
}

// The reference's device-side methods: the same device computations.
void H2MatrixSolver::init_gpu_handles(const ncclComms) {}
void H2MatrixSolver::move_data_gpu() {}
void H2MatrixSolver::allocSparseMV(deviceHandle_t, const ncclComms) {}
void H2MatrixSolver::matVecMulSp(deviceHandle_t, std::complex<double> X[]) { matVecMul(X); }
void H2MatrixSolver::factorizeDeviceM(deviceHandle_t) { factorizeM(); }
void H2MatrixSolver::solvePreconditionDevice(deviceHandle_t, std::complex<double> X[]) { solvePrecondition(X); }
void H2MatrixSolver::solveGMRESDevice(deviceHandle_t, double tol, H2MatrixSolver& M, std::complex<double> X[],
                                      const std::complex<double> B[], long long inner_iters, long long outer_iters,
                                      const ncclComms) {
  solveGMRES(tol, M, X, B, inner_iters, outer_iters);
}
void H2MatrixSolver::free_all_comms() { allocedComm.clear(); }
void H2MatrixSolver::freeSparseMV() {}
void H2MatrixSolver::free_gpu_handles() {}
