// Test infrastructure only: a driver linked against the reference's own
// build_tree.cpp (compiled from its source tree, never copied) plus the
// header-only test_funcs.hpp and kernel.hpp.  It writes the reference's
// points, tree, Near/Far lists and kernel values to a binary dump that the
// fixture generator (tests/golden/make_fixtures.py) turns into golden files.
//
// Output layout (little-endian, all int64 unless noted):
//   N, levels, ncells
//   bodies    (N*3 f64, tree-sorted, as buildBinaryTree leaves them)
//   xbody     (N f64, mt19937_64 default seed, uniform[0,1), main.cpp:73-76)
//   cells     ncells x (child0, child1, body0, body1) int64, R (3 f64), C (3 f64)
//   for each list in (Near theta, Far theta, Far 0):
//     nrow = ncells+1, RowIndex[nrow], nnz, ColIndex[nnz]
//   kernel probe: npairs, then for each pair (i, j, laplace f64, yukawa f64)
//   Helmholtz probe (the same pairs): npairs, then for each pair the real
//   and imaginary part (f64) of Helmholtz3D(1, 0.1), main.cpp:62
//   sphere: N, then mesh_sphere(N, sqrt(N / 4 pi)) (N*3 f64), main.cpp:68
#include <build_tree.hpp>
#include <kernel.hpp>
#include <test_funcs.hpp>

#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

static void put_i(FILE* f, long long v) { fwrite(&v, sizeof(v), 1, f); }
static void put_d(FILE* f, double v) { fwrite(&v, sizeof(v), 1, f); }

static void put_csr(FILE* f, const CSR& c) {
  put_i(f, (long long)c.RowIndex.size());
  fwrite(c.RowIndex.data(), sizeof(long long), c.RowIndex.size(), f);
  put_i(f, (long long)c.ColIndex.size());
  fwrite(c.ColIndex.data(), sizeof(long long), c.ColIndex.size(), f);
}

int main(int argc, char** argv) {
  if (argc < 6) {
    fprintf(stderr, "usage: ref_driver N leaf theta seed out.bin\n");
    return 2;
  }
  long long N = atoll(argv[1]);
  long long leaf = atoll(argv[2]);
  double theta = atof(argv[3]);
  unsigned seed = (unsigned)atoll(argv[4]);
  const char* out = argv[5];

  leaf = N < leaf ? N : leaf;
  long long levels = (long long)std::log2((double)N / leaf);
  long long nleaf = 1ll << levels;
  long long ncells = nleaf + nleaf - 1;

  std::vector<double> body(N * 3);
  std::vector<double> xbody(N);
  std::vector<Cell> cell(ncells);
  uniform_unit_cube_rnd(&body[0], N, 1, 3, seed);
  buildBinaryTree(&cell[0], &body[0], N, levels);

  std::mt19937_64 gen;
  std::uniform_real_distribution<double> ud(0., 1.);
  for (long long i = 0; i < N; i++) xbody[i] = ud(gen);

  CSR nearL('N', cell, cell, theta);
  CSR farL('F', cell, cell, theta);
  CSR hssL('F', cell, cell, 0.);

  FILE* f = fopen(out, "wb");
  if (!f) return 1;
  put_i(f, N); put_i(f, levels); put_i(f, ncells);
  fwrite(body.data(), sizeof(double), body.size(), f);
  fwrite(xbody.data(), sizeof(double), xbody.size(), f);
  for (const Cell& c : cell) {
    put_i(f, c.Child[0]); put_i(f, c.Child[1]); put_i(f, c.Body[0]); put_i(f, c.Body[1]);
    for (int k = 0; k < 3; k++) put_d(f, c.R[k]);
    for (int k = 0; k < 3; k++) put_d(f, c.C[k]);
  }
  put_csr(f, nearL); put_csr(f, farL); put_csr(f, hssL);

  // Kernel probe: the first 64 bodies against bodies spread over the set,
  // with the distance taken the way gen_matrix takes it (3-argument hypot).
  Laplace3D lap(1.);
  Yukawa3D yuk(1., 1.);
  long long np = 64 * 64;
  put_i(f, np);
  for (long long a = 0; a < 64; a++)
    for (long long b = 0; b < 64; b++) {
      long long i = a % N, j = (b * 7919) % N;
      const double* bi = &body[3 * i];
      const double* bj = &body[3 * j];
      double d = std::hypot(bi[0] - bj[0], bi[1] - bj[1], bi[2] - bj[2]);
      put_i(f, i); put_i(f, j);
      put_d(f, lap(d).real()); put_d(f, yuk(d).real());
    }
  Helmholtz3D helm(1., 1e-1);
  put_i(f, np);
  for (long long a = 0; a < 64; a++)
    for (long long b = 0; b < 64; b++) {
      long long i = a % N, j = (b * 7919) % N;
      const double* bi = &body[3 * i];
      const double* bj = &body[3 * j];
      std::complex<double> v = helm(std::hypot(bi[0] - bj[0], bi[1] - bj[1], bi[2] - bj[2]));
      put_d(f, v.real()); put_d(f, v.imag());
    }
  std::vector<double> sphere(N * 3);
  mesh_sphere(&sphere[0], N, std::sqrt(N / (4 * M_PI)));
  put_i(f, N);
  fwrite(sphere.data(), sizeof(double), sphere.size(), f);
  fclose(f);
  return 0;
}
