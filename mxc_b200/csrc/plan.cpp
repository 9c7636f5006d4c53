// Host plan layer: the reference's geometry / tree / list rules restated.
#include "plan.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <random>

namespace h2b {

i64 PairCSR::lookup(i64 i, i64 j) const {
  if (i < 0 || (i64)row.size() <= i + 1) return -1;
  for (i64 k = row[i]; k < row[i + 1]; k++)
    if (col[k] == j) return k;
  return -1;
}

void uniform_unit_cube_rnd(double* bodies, i64 n, double diameter, i64 dim, unsigned seed) {
  // test_funcs.hpp:31-41: one generator, coordinates drawn in body order.
  std::mt19937 gen(seed);
  std::uniform_real_distribution<double> dist(0., diameter);
  for (i64 i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) bodies[3 * i + k] = k < dim ? dist(gen) : 0.;
}

void uniform_rhs(double* x, i64 n) {
  std::mt19937_64 gen;
  std::uniform_real_distribution<double> dist(0., 1.);
  for (i64 i = 0; i < n; i++) x[i] = dist(gen);
}

// Centre and half-extent of a body range, build_tree.cpp:8-22.
static void bounds(const double* b, i64 n, double R[3], double C[3]) {
  for (int k = 0; k < 3; k++) {
    double lo = b[k], hi = b[k];
    for (i64 i = 1; i < n; i++) {
      double v = b[3 * i + k];
      lo = v < lo ? v : lo;
      hi = hi < v ? v : hi;
    }
    C[k] = (lo + hi) * 0.5;
    R[k] = (lo == hi && lo == 0.) ? 0. : ((hi - lo) * 0.5 + 1.e-8);
  }
}

void build_binary_tree(Cell* cells, double* bodies, i64 nbodies, i64 levels) {
  cells[0].body[0] = 0;
  cells[0].body[1] = nbodies;
  bounds(bodies, nbodies, cells[0].R, cells[0].C);
  i64 nleaf = (i64)1 << levels;
  typedef std::array<double, 3> P3;
  for (i64 i = 0; i + 1 < nleaf; i++) {
    Cell& ci = cells[i];
    int sdim = 0;  // first maximum of the half extents
    for (int k = 1; k < 3; k++)
      if (ci.R[sdim] < ci.R[k]) sdim = k;
    i64 b0 = ci.body[0], b1 = ci.body[1];
    P3* first = reinterpret_cast<P3*>(bodies + 3 * b0);
    P3* last = reinterpret_cast<P3*>(bodies + 3 * b1);
    // Same comparator and the same std::sort as the reference, so equal
    // keys (which random inputs do not produce) would also land the same.
    std::sort(first, last, [=](P3& a, P3& b) { return a[sdim] < b[sdim]; });
    i64 c0 = 2 * i + 1;
    ci.child[0] = c0;
    ci.child[1] = c0 + 2;
    i64 mid = b0 + (b1 - b0) / 2;
    cells[c0].body[0] = b0;
    cells[c0].body[1] = mid;
    cells[c0 + 1].body[0] = mid;
    cells[c0 + 1].body[1] = b1;
    bounds(bodies + 3 * b0, mid - b0, cells[c0].R, cells[c0].C);
    bounds(bodies + 3 * mid, b1 - mid, cells[c0 + 1].R, cells[c0 + 1].C);
  }
}

// Geometric, leaf-capped binary tree (build extension for strongly
// non-uniform bodies).  Same cells, sort and bounds as build_binary_tree,
// but a cell is cut where its bounding box is halved along the longest
// extent (the first body at or past the box centre) rather than at the
// median, and the cut is clamped so that each child can still give every one
// of its h = 2^(levels - l - 1) leaves between leaf_min and leaf_max bodies:
// left count in [max(leaf_min h, n - leaf_max h), min(leaf_max h, n -
// leaf_min h)].  By induction from the root (leaf_min 2^levels <= N <=
// leaf_max 2^levels) every leaf ends with leaf_min..leaf_max bodies, while
// boxes follow the geometry wherever the density allows.
void build_binary_tree_capped(Cell* cells, double* bodies, i64 nbodies, i64 levels, i64 leaf_min, i64 leaf_max) {
  cells[0].body[0] = 0;
  cells[0].body[1] = nbodies;
  bounds(bodies, nbodies, cells[0].R, cells[0].C);
  const i64 nleaf = (i64)1 << levels;
  typedef std::array<double, 3> P3;
  i64 level = 0;
  for (i64 i = 0; i + 1 < nleaf; i++) {
    if (i + 1 >= ((i64)2 << level)) level++;  // cells of level l are [2^l - 1, 2^(l+1) - 1)
    Cell& ci = cells[i];
    int sdim = 0;
    for (int k = 1; k < 3; k++)
      if (ci.R[sdim] < ci.R[k]) sdim = k;
    const i64 b0 = ci.body[0], b1 = ci.body[1], n = b1 - b0;
    P3* first = reinterpret_cast<P3*>(bodies + 3 * b0);
    P3* last = reinterpret_cast<P3*>(bodies + 3 * b1);
    std::sort(first, last, [=](P3& a, P3& b) { return a[sdim] < b[sdim]; });
    const double cut = ci.C[sdim];
    i64 left = std::lower_bound(first, last, cut, [=](const P3& a, double v) { return a[sdim] < v; }) - first;
    const i64 h = (i64)1 << (levels - level - 1);
    const i64 lo = std::max(leaf_min * h, n - leaf_max * h), hi = std::min(leaf_max * h, n - leaf_min * h);
    left = lo <= hi ? std::min(std::max(left, lo), hi) : n / 2;
    const i64 c0 = 2 * i + 1, mid = b0 + left;
    ci.child[0] = c0;
    ci.child[1] = c0 + 2;
    cells[c0].body[0] = b0;
    cells[c0].body[1] = mid;
    cells[c0 + 1].body[0] = mid;
    cells[c0 + 1].body[1] = b1;
    bounds(bodies + 3 * b0, mid - b0, cells[c0].R, cells[c0].C);
    bounds(bodies + 3 * mid, b1 - mid, cells[c0 + 1].R, cells[c0 + 1].C);
  }
}

PairCSR build_pair_csr(char kind, const std::vector<Cell>& cells, double theta) {
  // Dual-tree descent from (0, 0), taken one tree level at a time; the
  // emitted pairs are sorted afterwards exactly as CSR::CSR sorts them.
  std::vector<std::pair<i64, i64>> out, cur{{0, 0}}, next;
  bool want_far = kind == 'F' || kind == 'f';
  while (!cur.empty()) {
    next.clear();
    for (auto& p : cur) {
      const Cell& a = cells[p.first];
      const Cell& b = cells[p.second];
      double dC = 0., dR1 = 0., dR2 = 0.;
      for (int k = 0; k < 3; k++) {
        double d = a.C[k] - b.C[k];
        dC = dC + d * d;
      }
      for (int k = 0; k < 3; k++) dR1 = dR1 + a.R[k] * a.R[k];
      for (int k = 0; k < 3; k++) dR2 = dR2 + b.R[k] * b.R[k];
      bool admis = dC > theta * (dR1 + dR2);
      if (admis == want_far) out.push_back(p);
      if (!admis && a.child[0] >= 0 && b.child[0] >= 0)
        for (i64 k = a.child[0]; k < a.child[1]; k++)
          for (i64 l = b.child[0]; l < b.child[1]; l++) next.emplace_back(k, l);
    }
    cur.swap(next);
  }
  std::sort(out.begin(), out.end());
  PairCSR csr;
  i64 nc = (i64)cells.size();
  csr.row.assign(nc + 1, 0);
  csr.col.resize(out.size());
  for (size_t k = 0; k < out.size(); k++) {
    csr.row[out[k].first + 1]++;
    csr.col[k] = out[k].second;
  }
  for (i64 i = 0; i < nc; i++) csr.row[i + 1] += csr.row[i];
  return csr;
}

void sample_far_list(const std::vector<std::pair<i64, i64>>& ranges, i64 samples, std::vector<int>& out) {
  i64 total = 0;
  for (auto& r : ranges) total += r.second - r.first;
  out.clear();
  if (total == 0) return;
  i64 keep = (samples <= 0 || samples >= total) ? total : samples;
  out.resize(keep);
  // Walk the concatenated list once; targets are increasing.
  size_t ri = 0;
  i64 base = 0;
  for (i64 j = 0; j < keep; j++) {
    i64 t = (keep == total) ? j : (j * total) / samples;
    while (t >= base + (ranges[ri].second - ranges[ri].first)) {
      base += ranges[ri].second - ranges[ri].first;
      ri++;
    }
    out[j] = (int)(ranges[ri].first + (t - base));
  }
}

}  // namespace h2b

namespace h2b {

void sample_far_list_geometric(const std::vector<std::pair<i64, i64>>& ranges, const std::vector<i64>& gstart,
                               i64 samples, std::vector<int>& out) {
  const int G = (int)gstart.size();
  std::vector<i64> gsize(G, 0), alloc(G, 0);
  i64 total = 0;
  for (int g = 0; g < G; g++) {
    i64 r1 = g + 1 < G ? gstart[g + 1] : (i64)ranges.size();
    for (i64 r = gstart[g]; r < r1; r++) gsize[g] += ranges[r].second - ranges[r].first;
    total += gsize[g];
  }
  out.clear();
  if (total == 0) return;
  if (samples <= 0 || samples >= total) {
    sample_far_list(ranges, 0, out);
    return;
  }
  // Nearest group (the box's own level, last in the list) first: half of
  // what is left, then half again for each level further out; the farthest
  // group takes the rest.  Shares a small group cannot use move outward
  // first and then inward.
  i64 rem = samples;
  for (int g = G - 1; g >= 0; g--) {
    i64 share = g == 0 ? rem : (rem + 1) / 2;
    alloc[g] = std::min(gsize[g], share);
    rem -= alloc[g];
  }
  for (int g = G - 1; g >= 0 && rem > 0; g--) {
    i64 extra = std::min(gsize[g] - alloc[g], rem);
    alloc[g] += extra;
    rem -= extra;
  }
  for (int g = 0; g < G; g++) {
    if (alloc[g] == 0) continue;
    i64 r1 = g + 1 < G ? gstart[g + 1] : (i64)ranges.size();
    std::vector<std::pair<i64, i64>> sub(ranges.begin() + gstart[g], ranges.begin() + r1);
    std::vector<int> part;
    sample_far_list(sub, alloc[g] == gsize[g] ? 0 : alloc[g], part);
    out.insert(out.end(), part.begin(), part.end());
  }
}

}  // namespace h2b
