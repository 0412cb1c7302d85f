// Host supernode partition for matrices the reference's symbolic phase has not analysed
// (the batched path factors hundreds of generated matrices at once).  The reference builds
// its partition inside analyze_p2 (cholesky/sw_LSparsity.h:590-605, relaxed supernodes
// with nrelax = {4, 16, 48}, zrelax = {0.8, 0.1, 0.05}, examples/sw_choleskyTest01.cpp:112-113);
// this is an independent implementation of the same kind of partition.
//
// Input: the lower CSC pattern of an already ordered matrix (P A P^T).  Steps:
//   1. elimination tree (Liu's algorithm with path compression);
//   2. exact column counts of L by row-subtree traversal: for every row i, walk from each
//      k < i with A(i, k) != 0 up the tree until a node already marked for i; every visited
//      node's column contains row i;
//   3. supernodes: column j joins the supernode [start, j) when parent(j-1) == j (so the
//      supernode is a chain of the tree), the width stays within max_width, and the
//      explicit zeros of the merged supernode pass the relaxation test.  For a chain the
//      merged supernode has (j - start) + colcount(j) rows (every column's structure
//      below the chain lies inside the structure of the chain's last column), so its zeros
//      are exact: width x rows - width (width - 1) / 2 - sum of the columns' counts.
//      Relaxation (zero fraction z of the merged supernode's entries): always merge when z
//      is 0 or width <= nrelax[0]; else merge when (width <= nrelax[1] and z < zrelax[0]) or
//      (width <= nrelax[2] and z < zrelax[1]) or z < zrelax[2].
// The result is a partition in the reference's blockSet format; build_layout turns it into
// the BCSC layout, update lists and level schedule.
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "swc_internal.h"

namespace swc {

bool supernode_partition(int n, const int *c, const int *r, const int nrelax[3],
                         const double zrelax[3], int max_width, std::vector<int> &super,
                         std::string &err) {
  if (n <= 0 || !c || !r || max_width <= 0) {
    err = "invalid arguments";
    return false;
  }
  // row lists of the strictly lower triangle: for row i, the columns k < i with A(i,k) != 0
  std::vector<int> rp(n + 1, 0);
  for (int k = 0; k < n; ++k) {
    if (c[k + 1] < c[k]) {
      err = "column pointers must be non-decreasing";
      return false;
    }
    for (int p = c[k]; p < c[k + 1]; ++p) {
      const int i = r[p];
      if (i < 0 || i >= n) {
        err = "row index out of range";
        return false;
      }
      if (i > k) rp[i + 1]++;
    }
  }
  for (int i = 0; i < n; ++i) rp[i + 1] += rp[i];
  std::vector<int> rk(rp[n]);
  {
    std::vector<int> fill(rp.begin(), rp.end() - 1);
    for (int k = 0; k < n; ++k)
      for (int p = c[k]; p < c[k + 1]; ++p)
        if (r[p] > k) rk[fill[r[p]]++] = k;
  }
  // 1. elimination tree
  std::vector<int> parent(n, -1), anc(n, -1);
  for (int i = 0; i < n; ++i)
    for (int q = rp[i]; q < rp[i + 1]; ++q) {
      int k = rk[q];
      while (k != -1 && k < i) {
        const int next = anc[k];
        anc[k] = i;
        if (next == -1) parent[k] = i;
        k = next;
      }
    }
  // 2. column counts (diagonal included)
  std::vector<int64_t> colcount(n, 1);
  std::vector<int> mark(n, -1);
  for (int i = 0; i < n; ++i) {
    mark[i] = i;
    for (int q = rp[i]; q < rp[i + 1]; ++q) {
      int k = rk[q];
      while (k != -1 && mark[k] != i) {
        colcount[k]++;
        mark[k] = i;
        k = parent[k];
      }
    }
  }
  // 3. chains of the tree, relaxed
  super.clear();
  super.push_back(0);
  int start = 0;
  int64_t sumcc = colcount[0];
  for (int j = 1; j < n; ++j) {
    bool merge = parent[j - 1] == j && (j - start + 1) <= max_width;
    if (merge) {
      const int64_t width = j - start + 1;
      const int64_t rows = (j - start) + colcount[j];
      const int64_t entries = width * rows - width * (width - 1) / 2;
      const int64_t zeros = entries - (sumcc + colcount[j]);
      const double z = (double)zeros / (double)entries;
      merge = zeros == 0 || width <= nrelax[0] || (width <= nrelax[1] && z < zrelax[0]) ||
              (width <= nrelax[2] && z < zrelax[1]) || z < zrelax[2];
    }
    if (merge) {
      sumcc += colcount[j];
    } else {
      super.push_back(j);
      start = j;
      sumcc = colcount[j];
    }
  }
  super.push_back(n);
  return true;
}

}  // namespace swc
