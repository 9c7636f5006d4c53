// lorasp: the reference's command-line driver (main.cpp:37-216) on the B200
// solver.  Same positional arguments, defaults, printed lines and CSV row:
//
//   lorasp [N [theta [leaf [rank [leveled_rank [epi [mode [csv]]]]]]]] [options]
//
//   N 2048, theta 1, leaf 256, rank 50, leveled_rank 0, epi 1e-10, mode h2
//   (hss: the preconditioner with theta 0); csv: append one result row.
//
// The reference fixes its kernel and geometry in the source; here they are
// options (the default geometry is the reference's: mesh_sphere of radius
// sqrt(N / 4 pi)) and its kernel (Helmholtz3D with wave number 1 and
// s = 0.1, main.cpp:62), on complex vectors as the reference's.
//   --kernel helmholtz|laplace|yukawa   --singularity S
//   --alpha A (Helmholtz wave number or Yukawa decay, 1)
//   --geometry sphere|cube    --seed K (cube: std::mt19937 seed, 999)
//   --samples S   far-list cap of the basis construction (0: every far body)
//   --precision fp64|fp32     storage of the preconditioner
// The reference's dense N x N matrix and its host matvec are replaced by the
// matrix-free FP64 device matvec (same products, no N^2 memory).
#include <algorithm>
#include <chrono>
#include <complex>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mxc_b200/h2_solver.hpp"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void usage() {
  std::printf(
      "usage: lorasp [N [theta [leaf [rank [leveled_rank [epi [mode [csv]]]]]]]]\n"
      "              [--kernel helmholtz|laplace|yukawa] [--singularity S] [--alpha A]\n"
      "              [--geometry sphere|cube] [--seed K] [--samples S] [--precision fp64|fp32]\n");
}

typedef std::complex<double> cplx;

// Y = K X with the matrix-free FP64 device matvec (main.cpp:83-84 multiplies
// by the dense matrix): complex columns as interleaved parts for
// Helmholtz3D, real parts for the real kernels.
void dense_apply(const MatrixAccessor& eval, const double* body, long long n, const std::vector<cplx>& X,
                 std::vector<cplx>& Y) {
  if (eval.kind == H2DEV_KERNEL_HELMHOLTZ) {
    dense_matvec(eval, body, n, 1, reinterpret_cast<const double*>(X.data()), reinterpret_cast<double*>(Y.data()),
                 2 * n);
    return;
  }
  std::vector<double> x((size_t)n), y((size_t)n);
  for (long long i = 0; i < n; i++) x[(size_t)i] = X[(size_t)i].real();
  dense_matvec(eval, body, n, 1, x.data(), y.data(), n);
  for (long long i = 0; i < n; i++) Y[(size_t)i] = cplx(y[(size_t)i], 0.);
}

}  // namespace

int main(int argc, char* argv[]) {
  std::vector<std::string> pos;
  std::string kernel = "helmholtz", geometry = "sphere", precision = "fp64";
  double singularity = 0.1, alpha = 1.;
  unsigned seed = 999;
  long long samples = 0;
  for (int i = 1; i < argc; i++) {
    const std::string a = argv[i];
    auto value = [&](const char* name) -> std::string {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "lorasp: %s needs a value\n", name);
        std::exit(2);
      }
      return argv[++i];
    };
    if (a == "-h" || a == "--help") {
      usage();
      return 0;
    } else if (a == "--kernel") {
      kernel = value("--kernel");
    } else if (a == "--singularity") {
      singularity = std::atof(value("--singularity").c_str());
    } else if (a == "--alpha") {
      alpha = std::atof(value("--alpha").c_str());
    } else if (a == "--geometry") {
      geometry = value("--geometry");
    } else if (a == "--seed") {
      seed = (unsigned)std::atoll(value("--seed").c_str());
    } else if (a == "--samples") {
      samples = std::atoll(value("--samples").c_str());
    } else if (a == "--precision") {
      precision = value("--precision");
    } else if (a.size() > 1 && a[0] == '-' && a[1] == '-') {
      std::fprintf(stderr, "lorasp: unknown option %s\n", a.c_str());
      usage();
      return 2;
    } else {
      pos.push_back(a);
    }
  }
  auto arg = [&](size_t k) -> const char* { return k < pos.size() ? pos[k].c_str() : nullptr; };
  long long Nbody = arg(0) ? std::atoll(arg(0)) : 2048;
  const double theta = arg(1) ? std::atof(arg(1)) : 1e0;
  long long leaf_size = arg(2) ? std::atoll(arg(2)) : 256;
  const long long rank = arg(3) ? std::atoll(arg(3)) : 50;
  const long long leveled_rank = arg(4) ? std::atoll(arg(4)) : 0;
  const double epi = arg(5) ? std::atof(arg(5)) : 1e-10;
  const std::string mode = arg(6) ? std::string(arg(6)) : "h2";
  const char* csv = arg(7);
  if (Nbody < 2 || leaf_size < 1 || (mode != "h2" && mode != "hss") || (kernel != "helmholtz" && kernel != "laplace" && kernel != "yukawa") ||
      (geometry != "sphere" && geometry != "cube") || (precision != "fp64" && precision != "fp32")) {
    usage();
    return 2;
  }

  try {
    leaf_size = Nbody < leaf_size ? Nbody : leaf_size;
    const long long levels = h2_levels_for(Nbody, leaf_size);
    const long long ncells = (2LL << levels) - 1;
    const MatrixAccessor eval = kernel == "yukawa"    ? (MatrixAccessor)Yukawa3D(singularity, alpha)
                                : kernel == "laplace" ? (MatrixAccessor)Laplace3D(singularity)
                                                      : (MatrixAccessor)Helmholtz3D(alpha, singularity);
    const int pc_precision = precision == "fp32" ? H2DEV_FP32 : H2DEV_FP64;

    std::vector<double> body((size_t)Nbody * 3);
    std::vector<cplx> Xbody((size_t)Nbody);
    std::vector<Cell> cell((size_t)ncells);
    if (geometry == "sphere")
      mesh_sphere(body.data(), Nbody, std::sqrt((double)Nbody / (4. * M_PI)));
    else
      uniform_unit_cube_rnd(body.data(), Nbody, 1., 3, seed);
    buildBinaryTree(cell.data(), body.data(), Nbody, levels);
    {  // main.cpp:73-76: real parts from the default-seeded std::mt19937_64
      std::vector<double> xr((size_t)Nbody);
      if (h2_uniform_rhs(xr.data(), Nbody) != H2DEV_OK) throw std::runtime_error("h2_uniform_rhs failed");
      for (long long i = 0; i < Nbody; i++) Xbody[(size_t)i] = cplx(xr[(size_t)i], 0.);
    }

    double h2_construct_time = now_s();
    H2MatrixSolver matA(eval, epi, rank, leveled_rank, cell, theta, body.data(), levels, samples, H2DEV_FP64);
    h2_construct_time = now_s() - h2_construct_time;

    const long long lenX = matA.local_bodies.second - matA.local_bodies.first;
    std::vector<cplx> X1(Xbody), X2((size_t)lenX, 0.);
    double matvec_time = now_s();
    matA.matVecMul(X1.data());
    matvec_time = now_s() - matvec_time;

    double refmatvec_time = now_s();
    dense_apply(eval, body.data(), Nbody, Xbody, X2);
    refmatvec_time = now_s() - refmatvec_time;
    const double cerr = H2MatrixSolver::solveRelErr(lenX, X1.data(), X2.data());

    std::cout << "Construct Err: " << cerr << std::endl;
    std::cout << "H^2-Matrix Construct Time: " << h2_construct_time << ", " << 0. << std::endl;
    std::cout << "H^2-Matvec Time: " << matvec_time << ", " << 0. << std::endl;
    std::cout << "Dense Matvec Time: " << refmatvec_time << std::endl;

    double m_construct_time = now_s();
    H2MatrixSolver matM(eval, 0., rank, leveled_rank, cell, mode == "h2" ? theta : 0., body.data(), levels, samples,
                        pc_precision);
    m_construct_time = now_s() - m_construct_time;

    X1 = Xbody;
    matM.matVecMul(X1.data());
    const double cerr_m = H2MatrixSolver::solveRelErr(lenX, X1.data(), X2.data());

    double h2_factor_time = now_s();
    matM.factorizeM();
    h2_factor_time = now_s() - h2_factor_time;
    X1 = X2;

    double h2_sub_time = now_s();
    matM.solvePrecondition(X1.data());
    h2_sub_time = now_s() - h2_sub_time;
    const double serr = H2MatrixSolver::solveRelErr(lenX, X1.data(), Xbody.data());
    std::fill(X1.begin(), X1.end(), cplx(0., 0.));

    std::cout << "H^2-Preconditioner Construct Time: " << m_construct_time << ", " << 0. << std::endl;
    std::cout << "H^2-Preconditioner Construct Err: " << cerr_m << std::endl;
    std::cout << "H^2-Matrix Factorization Time: " << h2_factor_time << ", " << 0. << std::endl;
    std::cout << "H^2-Matrix Substitution Time: " << h2_sub_time << ", " << 0. << std::endl;
    std::cout << "H^2-Matrix Substitution Err: " << serr << std::endl;

    double gmres_time = now_s();
    matA.solveGMRES(epi, matM, X1.data(), X2.data(), 10, 50);
    gmres_time = now_s() - gmres_time;

    std::cout << "GMRES Residual: " << matA.resid[(size_t)matA.iters] << ", Iters: " << matA.iters << std::endl;
    std::cout << "GMRES Time: " << gmres_time << ", Comm: " << 0. << std::endl;
    for (long long i = 0; i <= matA.iters; i++) std::cout << "iter " << i << ": " << matA.resid[(size_t)i] << std::endl;

    if (csv != nullptr)  // one process: mpi_size 1, comm times 0
      write_to_csv(csv, 1, Nbody, theta, leaf_size, rank, epi, mode.data(), cerr, h2_construct_time, 0., matvec_time,
                   0., refmatvec_time, m_construct_time, 0., cerr_m, h2_factor_time, 0., h2_sub_time, 0., serr,
                   matA.resid[(size_t)matA.iters], (double)matA.iters, gmres_time, 0., matA.resid.data());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "lorasp: %s\n", e.what());
    return 1;
  }
  return 0;
}
