// Host-side plan of the H^2 solver: tree, admissibility lists, per-level box
// structure and the block layouts the device kernels index.  All of it is
// cheap integer / small-float work done once per matrix on the host.
#pragma once

#include <cstdint>
#include <vector>

namespace h2b {

typedef int64_t i64;

// One tree cell (build_tree.hpp:7-15): children range, body range, half
// extent R and centre C.
struct Cell {
  i64 child[2] = {-1, -1};
  i64 body[2] = {-1, -1};
  double R[3] = {0., 0., 0.};
  double C[3] = {0., 0., 0.};
};

// Pair list in CSR form over all cells (build_tree.hpp:17-24).
struct PairCSR {
  std::vector<i64> row;  // ncells + 1
  std::vector<i64> col;
  i64 lookup(i64 i, i64 j) const;
};

// std::mt19937 + uniform_real_distribution(0, diameter), test_funcs.hpp:31-41.
void uniform_unit_cube_rnd(double* bodies, i64 n, double diameter, i64 dim, unsigned seed);
// Default-seeded std::mt19937_64 + uniform_real_distribution(0,1), main.cpp:73-76.
void uniform_rhs(double* x, i64 n);

// buildBinaryTree (build_tree.cpp:67-99): sorts bodies in place.
void build_binary_tree(Cell* cells, double* bodies, i64 nbodies, i64 levels);

// Geometric split clamped so every leaf holds leaf_min..leaf_max bodies
// (requires leaf_min 2^levels <= nbodies <= leaf_max 2^levels).
void build_binary_tree_capped(Cell* cells, double* bodies, i64 nbodies, i64 levels, i64 leaf_min, i64 leaf_max);

// CSR lists (build_tree.cpp:24-58); kind 'N' near, 'F' far.
PairCSR build_pair_csr(char kind, const std::vector<Cell>& cells, double theta);

// Deterministic cap of a far-body list to ``samples`` rows (samples <= 0:
// keep all, the reference behaviour): row j of the sample is entry
// floor(j * total / samples) of the concatenated list.
void sample_far_list(const std::vector<std::pair<i64, i64>>& ranges, i64 samples, std::vector<int>& out_idx);
// Level-geometric cap: gstart[g] is the first range appended at tree level
// g+1 (g = 0 farthest, last = the box's own level).  The own-level group gets
// half of the budget, each level further out half of what is left, the
// farthest the rest; each group is then strided as in sample_far_list.
void sample_far_list_geometric(const std::vector<std::pair<i64, i64>>& ranges, const std::vector<i64>& gstart,
                               i64 samples, std::vector<int>& out_idx);

// Per-level box structure of one H^2 matrix (the single-process view of
// ColCommMPI: every box of a level is local, comm-mpi.cpp:49-150).
struct LevelPlan {
  int level = 0;
  i64 gbegin = 0;  // first cell index of the level
  i64 nodes = 0;
  std::vector<i64> arow, acol;  // near pairs, level-local CSR
  std::vector<i64> crow, ccol;  // far pairs (couplings), level-local CSR
  std::vector<i64> diag;        // index of (i,i) in acol per row
};

}  // namespace h2b
