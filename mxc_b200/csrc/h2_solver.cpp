// C++ host API (include/mxc_b200/h2_solver.hpp) over the C ABI of h2dev.h:
// the reference's class and function names, backed by the device solver.
#include "mxc_b200/h2_solver.hpp"

#include <cmath>
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

double MatrixAccessor::operator()(double d) const {
  if (d == 0.) return 1. / s;
  if (kind == H2DEV_KERNEL_YUKAWA) return std::exp(-alpha * d) / d;
  if (kind == H2DEV_KERNEL_QUADRATIC) return d * d + alpha;
  return 1. / d;
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

H2MatrixSolver::H2MatrixSolver(const MatrixAccessor& eval, double epi, long long rank, long long leveled_rank,
                               const std::vector<Cell>& cells, double theta, const double bodies[], long long levels,
                               long long samples, int precision, h2dev_handle_t handle)
    : levels(levels), h_(handle ? handle : default_handle()) {
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
}

H2MatrixSolver::H2MatrixSolver(H2MatrixSolver&& o) noexcept { *this = std::move(o); }

H2MatrixSolver& H2MatrixSolver::operator=(H2MatrixSolver&& o) noexcept {
  if (this != &o) {
    if (s_) h2dev_solver_destroy(s_);
    levels = o.levels;
    local_bodies = o.local_bodies;
    resid = std::move(o.resid);
    iters = o.iters;
    info = std::move(o.info);
    s_ = o.s_;
    h_ = o.h_;
    o.s_ = nullptr;
  }
  return *this;
}

H2MatrixSolver::~H2MatrixSolver() {
  if (s_) h2dev_solver_destroy(s_);
}

void H2MatrixSolver::matVecMul(double X[]) {
  const long long n = local_bodies.second - local_bodies.first;
  check(h2dev_matvec(s_, 1, X, n), "h2dev_matvec");
}

void H2MatrixSolver::matVecMul(std::complex<double> X[]) {
  std::vector<double> r = real_parts(X, local_bodies.second - local_bodies.first);
  matVecMul(r.data());
  put_real(X, r);
}

void H2MatrixSolver::factorizeM() {
  info.assign((size_t)levels + 1, 0);
  const int rc = h2dev_factorize(s_, info.data());
  if (rc != H2DEV_ERR_SINGULAR) check(rc, "h2dev_factorize");
}

void H2MatrixSolver::solvePrecondition(double X[]) {
  const long long n = local_bodies.second - local_bodies.first;
  check(h2dev_solve_precondition(s_, 1, X, n), "h2dev_solve_precondition");
}

void H2MatrixSolver::solvePrecondition(std::complex<double> X[]) {
  std::vector<double> r = real_parts(X, local_bodies.second - local_bodies.first);
  solvePrecondition(r.data());
  put_real(X, r);
}

void H2MatrixSolver::solveGMRES(double tol, H2MatrixSolver& M, double X[], const double B[], long long nrhs,
                                long long ld, long long inner_iters, long long outer_iters, bool early_exit) {
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

double H2MatrixSolver::solveRelErr(long long lenX, const std::complex<double> X[], const std::complex<double> ref[]) {
  double num = 0., den = 0.;
  for (long long i = 0; i < lenX; i++) {
    num += std::norm(X[i] - ref[i]);
    den += std::norm(ref[i]);
  }
  return std::sqrt(num / den);
}

void dense_matvec(const MatrixAccessor& eval, const double bodies[], long long n, long long nrhs, const double X[],
                  double Y[], long long ld, h2dev_handle_t handle) {
  h2dev_handle_t h = handle ? handle : H2MatrixSolver::default_handle();
  check(h2dev_dense_matvec(h, eval.kind, eval.s, eval.alpha, bodies, n, nrhs, X, Y, ld), "h2dev_dense_matvec");
}
