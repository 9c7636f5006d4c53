"""C++ host API (include/mxc_b200/h2_solver.hpp) and the lorasp command-line
driver.

Without a GPU: a small program compiled against the header builds the tree
and the reference's point sets through the C++ names (Cell,
buildBinaryTree, uniform_unit_cube_rnd, mesh_sphere), and must agree
exactly with the C ABI used by the Python mirror; lorasp answers --help and
rejects bad arguments.  With a GPU: lorasp runs the reference's main.cpp
flow (construct, matvec check, preconditioner, factorization, substitution,
GMRES, CSV row) and its construction and substitution errors equal the
Python API's on the same points, kernel and parameters.
"""
import math
import os
import re
import subprocess

import numpy as np
import pytest

import mxc_b200 as m

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "mxc_b200")
LORASP = os.path.join(LIBDIR, "lorasp")

PROGRAM = r"""
#include <cstdio>
#include <vector>
#include "mxc_b200/h2_solver.hpp"
int main() {
  const long long n = 1000, levels = 2, nc = (2 << levels) - 1;
  std::vector<double> b(3 * n), s(3 * n);
  uniform_unit_cube_rnd(b.data(), n, 1., 3, 999);
  std::vector<Cell> cells(nc);
  buildBinaryTree(cells.data(), b.data(), n, levels);
  for (long long i = 0; i < nc; i++)
    std::printf("%lld %lld %lld %lld %.17g %.17g %.17g %.17g %.17g %.17g\n", cells[i].Child[0], cells[i].Child[1],
                cells[i].Body[0], cells[i].Body[1], cells[i].R[0], cells[i].R[1], cells[i].R[2], cells[i].C[0],
                cells[i].C[1], cells[i].C[2]);
  for (long long i = 0; i < 3 * n; i++) std::printf("%.17g\n", b[i]);
  mesh_sphere(s.data(), 7, 2.0);
  for (int i = 0; i < 21; i++) std::printf("%.17g\n", s[i]);
  std::printf("%.17g %.17g\n", Laplace3D(0.5)(0.).real(), Yukawa3D(1., 2.)(0.5).real());
  return 0;
}
"""


def _compile(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    subprocess.run(["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L" + LIBDIR, "-lmxcb200", "-Wl,-rpath," + LIBDIR], check=True, capture_output=True)
    return exe


def test_cpp_header_tree_and_points_match_the_c_abi(tmp_path):
    out = subprocess.run([str(_compile(tmp_path))], check=True, capture_output=True, text=True).stdout.split("\n")
    levels, n = 2, 1000
    nc = (2 << levels) - 1
    b = m.uniform_unit_cube_rnd(n, 999)
    t = m.build_tree(b, levels)
    for i in range(nc):
        f = out[i].split()
        assert [int(v) for v in f[:4]] == [*t.child[i], *t.body[i]]
        assert np.array_equal(np.array([float(v) for v in f[4:10]]), np.concatenate([t.R[i], t.C[i]]))
    cpp_bodies = np.array([float(v) for v in out[nc:nc + 3 * n]]).reshape(n, 3)
    assert np.array_equal(cpp_bodies, b)
    sphere = np.array([float(v) for v in out[nc + 3 * n:nc + 3 * n + 21]]).reshape(7, 3)
    golden = math.pi * (3.0 - math.sqrt(5.0))
    y = 2.0 - 4.0 * np.arange(7) / 6.0
    ring = np.sqrt(4.0 - y * y)
    exp = np.column_stack([ring * np.cos(golden * np.arange(7)), y, ring * np.sin(golden * np.arange(7))])
    np.testing.assert_allclose(sphere, exp, rtol=0, atol=1e-14)
    np.testing.assert_allclose(np.linalg.norm(sphere, axis=1), 2.0, rtol=1e-14)
    lap0, yuk = (float(v) for v in out[nc + 3 * n + 21].split())
    assert lap0 == 2.0 and abs(yuk - math.exp(-1.0) / 0.5) < 1e-15


def test_lorasp_help_and_bad_arguments():
    r = subprocess.run([LORASP, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage: lorasp" in r.stdout
    assert subprocess.run([LORASP, "1000", "2", "256", "50", "0", "1e-10", "bogus"], capture_output=True).returncode == 2
    assert subprocess.run([LORASP, "--kernel", "gaussian"], capture_output=True).returncode == 2
    assert subprocess.run([LORASP, "--no-such-option"], capture_output=True).returncode == 2


def _value(text, label):
    return float(re.search(re.escape(label) + r" ([-+0-9.eE]+)", text).group(1))


@pytest.mark.gpu
def test_lorasp_runs_the_reference_flow_and_matches_the_python_api(tmp_path, handle):
    n, theta, leaf, rank, eps, samples = 4096, 2.0, 256, 100, 1e-10, 2000
    csv = tmp_path / "run.csv"
    r = subprocess.run([LORASP, str(n), str(theta), str(leaf), str(rank), "0", str(eps), "h2", str(csv),
                        "--kernel", "laplace", "--geometry", "cube", "--singularity", "0.1", "--samples", str(samples)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    cerr = _value(out, "Construct Err:")
    serr = _value(out, "H^2-Matrix Substitution Err:")
    res = _value(out, "GMRES Residual:")
    iters = int(re.search(r"Iters: (\d+)", out).group(1))
    hist = [float(v) for v in re.findall(r"iter \d+: ([-+0-9.eE]+)", out)]
    assert cerr < 1e-8 and math.isfinite(serr)
    assert len(hist) == iters + 1 and hist[0] == 1.0 and res == hist[-1] and all(map(math.isfinite, hist))
    row = csv.read_text().strip().split(",")
    assert len(row) == 25 + iters + 1 and row[6] == "h2" and int(row[1]) == n
    # The same construction, factorization and substitution through the
    # Python API: same points, tree, kernel and parameters give the same
    # operator and preconditioner, so the same errors.  (How well this
    # preconditioner reproduces x depends on the system -- Laplace with a
    # diagonal of 10 on the unit cube is ill-conditioned -- so the check is
    # agreement between the two front ends, not a bound.)
    b = m.uniform_unit_cube_rnd(n, 999)
    L = m.levels_for(n, leaf)
    t = m.build_tree(b, L)
    k = m.Laplace3D(0.1)
    A = m.H2MatrixSolver(handle, k, eps, rank, 0, t, theta, b, samples=samples)
    x = m.uniform_rhs(n)
    y = x.copy()
    A.matVecMul(y)
    yd = m.dense_matvec(handle, k, b, x)
    cerr_py = np.linalg.norm(y - yd) / np.linalg.norm(yd)
    A.close()
    M = m.H2MatrixSolver(handle, k, 0.0, rank, 0, t, theta, b, samples=samples)
    M.factorizeM()
    z = yd.copy()
    M.solvePrecondition(z)
    serr_py = np.linalg.norm(z - x) / np.linalg.norm(x)
    M.close()
    assert abs(cerr - cerr_py) <= 1e-3 * cerr_py, (cerr, cerr_py)
    assert abs(serr - serr_py) <= 1e-4 * serr_py, (serr, serr_py)


# The reference's main.cpp call sequence, written only against the
# reference's own header names and signatures (solver.hpp, test_funcs.hpp,
# kernel.hpp, comm-mpi.hpp): MPI_Init, a DenseZMat filled by gen_matrix,
# H2MatrixSolver(denseA, eval, epi, rank, leveled_rank, cell, theta, body,
# levels), matVecMul against op_Aij_mulB, the preconditioner by copy-style
# assignment, factorizeM, solvePrecondition, solveGMRES, solveRelErr,
# ColCommMPI::get_comm_time, write_to_csv, free_all_comms, MPI_Finalize.
REF_PROGRAM = r"""
#include <solver.hpp>
#include <test_funcs.hpp>
#include <cmath>
#include <complex>
#include <iostream>
#include <random>
#include <string>
#include <vector>
int main(int argc, char* argv[]) {
  MPI_Init(&argc, &argv);
  long long Nbody = 2048, leaf_size = 256, rank = 100, leveled_rank = 0;
  double theta = 2., epi = 1e-10;
  std::string mode = "h2";
  const char* csv = argc > 1 ? argv[1] : nullptr;
  long long levels = (long long)std::log2((double)Nbody / leaf_size);
  long long Nleaf = (long long)1 << levels, ncells = Nleaf + Nleaf - 1;
  Laplace3D eval(1e-4);
  std::vector<double> body(Nbody * 3);
  std::vector<std::complex<double>> Xbody(Nbody);
  std::vector<Cell> cell(ncells);
  uniform_unit_cube_rnd(&body[0], Nbody, 1, 3, 999);
  buildBinaryTree(&cell[0], &body[0], Nbody, levels);
  std::mt19937_64 gen;
  std::uniform_real_distribution<double> uniform_dist(0., 1.);
  for (auto& x : Xbody) x = std::complex<double>(uniform_dist(gen), 0.);
  DenseZMat denseA(Nbody, Nbody);
  gen_matrix(eval, Nbody, Nbody, &body[0], &body[0], denseA.A);
  MPI_Barrier(MPI_COMM_WORLD);
  double t0 = MPI_Wtime();
  H2MatrixSolver matA(denseA, eval, epi, rank, leveled_rank, cell, theta, &body[0], levels);
  double h2_construct_time = MPI_Wtime() - t0;
  long long lenX = matA.local_bodies.second - matA.local_bodies.first;
  std::vector<std::complex<double>> X1(lenX, std::complex<double>(0., 0.)), X2(lenX, std::complex<double>(0., 0.));
  std::copy(&Xbody[matA.local_bodies.first], &Xbody[matA.local_bodies.second], &X1[0]);
  matA.matVecMul(&X1[0]);
  denseA.op_Aij_mulB('N', lenX, 1, Nbody, matA.local_bodies.first, 0, &Xbody[0], Nbody, &X2[0], lenX);
  double cerr = H2MatrixSolver::solveRelErr(lenX, &X1[0], &X2[0]);
  int mpi_rank = 0, mpi_size = 1;
  MPI_Comm_rank(MPI_COMM_WORLD, &mpi_rank);
  MPI_Comm_size(MPI_COMM_WORLD, &mpi_size);
  std::cout << "Construct Err: " << cerr << std::endl;
  H2MatrixSolver matM;
  if (mode.compare("h2") == 0)
    matM = H2MatrixSolver(denseA, eval, 0., rank, leveled_rank, cell, theta, &body[0], levels);
  std::copy(&Xbody[matM.local_bodies.first], &Xbody[matM.local_bodies.second], &X1[0]);
  matM.matVecMul(&X1[0]);
  double cerr_m = H2MatrixSolver::solveRelErr(lenX, &X1[0], &X2[0]);
  matM.factorizeM();
  std::copy(X2.begin(), X2.end(), X1.begin());
  matM.solvePrecondition(&X1[0]);
  double serr = H2MatrixSolver::solveRelErr(lenX, &X1[0], &Xbody[matM.local_bodies.first]);
  std::fill(X1.begin(), X1.end(), std::complex<double>(0., 0.));
  std::cout << "H^2-Preconditioner Construct Err: " << cerr_m << std::endl;
  std::cout << "H^2-Matrix Substitution Err: " << serr << std::endl;
  matA.solveGMRES(epi, matM, &X1[0], &X2[0], 10, 50);
  double xerr = H2MatrixSolver::solveRelErr(lenX, &X1[0], &Xbody[0]);
  std::cout << "GMRES Residual: " << matA.resid[matA.iters] << ", Iters: " << matA.iters << std::endl;
  std::cout << "Solution Err: " << xerr << std::endl;
  std::cout << "Levels: " << matA.A.size() << " " << matA.A[levels].Dims.size() << " " << matA.A[levels].ARows.back()
            << " " << ColCommMPI::get_comm_time() << std::endl;
  if (csv != nullptr)
    write_to_csv(csv, mpi_size, Nbody, theta, leaf_size, rank, epi, mode.data(), cerr, h2_construct_time, 0., 0., 0.,
                 0., 0., 0., cerr_m, 0., 0., 0., 0., serr, matA.resid[matA.iters], matA.iters, 0., 0.,
                 matA.resid.data());
  matA.free_all_comms();
  matM.free_all_comms();
  MPI_Finalize();
  return 0;
}
"""


def _compile_ref(tmp_path):
    src = tmp_path / "ref_main.cpp"
    src.write_text(REF_PROGRAM)
    exe = tmp_path / "ref_main"
    r = subprocess.run(["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include", "mxc_b200", "reference"),
                        str(src), "-o", str(exe), "-L" + LIBDIR, "-lmxcb200", "-Wl,-rpath," + LIBDIR],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_reference_signature_program_compiles(tmp_path):
    """main.cpp's calls, with only the reference's header names on the
    include path, compile and link against the library."""
    _compile_ref(tmp_path)


@pytest.mark.gpu
def test_reference_signature_program_runs(tmp_path):
    exe = _compile_ref(tmp_path)
    csv = tmp_path / "ref.csv"
    r = subprocess.run([str(exe), str(csv)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    assert _value(out, "Construct Err:") < 1e-9
    assert _value(out, "GMRES Residual:") < 1e-10
    assert _value(out, "Solution Err:") < 1e-8
    lv = re.search(r"Levels: (\d+) (\d+) (\d+) (\S+)", out)
    assert int(lv.group(1)) == 4 and int(lv.group(2)) == 8 and int(lv.group(3)) > 8 and float(lv.group(4)) == 0.0
    row = csv.read_text().strip().split(",")
    iters = int(re.search(r"Iters: (\d+)", out).group(1))
    assert len(row) == 25 + iters + 1 and row[0] == "1" and row[6] == "h2"
