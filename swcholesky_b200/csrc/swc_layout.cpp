// Host-side supernodal layout builder.
//
// Given the lower CSC pattern of P A P^T and a supernode partition (blockSet), it builds
// the reference's column-compressed supernodal layout -- Li_ptr, lC, Ls -- the update
// lists (prune sets), the supernodal elimination tree and a level schedule in the
// reference's H-level array format.  These are the arrays the reference's symbolic phase
// hands to the numeric executor (cholesky/sw_LSparsity.h:598-665, consumed by
// cholesky/sw_parallel_PB_Cholesky_05.c:193-207).
//
// Layout rules (reference BCSC, common/def.h:123-210, cholesky/sw_LSparsity.h:611-638):
//   * the row list of supernode s is sorted and starts with its own columns;
//   * it is the union of the sub-diagonal pattern of A's columns in s and of the
//     off-diagonal rows of every child supernode (the supernodal symbolic factorization);
//   * Li_ptr[j] = start of the row list of col2sup[j] for every column j,
//     Li_ptr[n] = total length;
//   * lC[j] = value offset of column j; a supernode is an nsrow x nscol column-major
//     block, so lC[j+1] - lC[j] = nsrow of its supernode.
// Update list of s = every descendant d whose row list meets the columns of s, in
// increasing supernode order (a topological order, since supernodes are numbered in a
// postorder of the supernodal etree).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "swc_internal.h"

namespace swc {

bool build_layout(int n, const int *c, const int *r, const int *blockSet, int supNo,
                  Layout &out, std::string &err) {
  if (n <= 0 || supNo <= 0 || !c || !r || !blockSet) {
    err = "invalid arguments";
    return false;
  }
  if (blockSet[0] != 0 || blockSet[supNo] != n) {
    err = "blockSet must start at 0 and end at n";
    return false;
  }
  std::vector<int> col2sup(n);
  for (int s = 0; s < supNo; ++s) {
    if (blockSet[s + 1] <= blockSet[s]) {
      err = "blockSet must be strictly increasing";
      return false;
    }
    for (int j = blockSet[s]; j < blockSet[s + 1]; ++j) col2sup[j] = s;
  }
  std::vector<int> mark(n, -1);
  std::vector<std::vector<int>> children(supNo);
  std::vector<int> rows;
  out.n = n;
  out.nsuper = supNo;
  out.rowptr.assign(supNo + 1, 0);
  out.Ls.clear();
  out.sparent.assign(supNo, -1);
  for (int s = 0; s < supNo; ++s) {
    int f = blockSet[s], l = blockSet[s + 1];
    rows.clear();
    for (int j = f; j < l; ++j) {
      mark[j] = s;
      rows.push_back(j);
    }
    for (int j = f; j < l; ++j)
      for (int p = c[j]; p < c[j + 1]; ++p) {
        int i = r[p];
        if (i < 0 || i >= n) {
          err = "row index out of range";
          return false;
        }
        if (i >= f && mark[i] != s) {
          mark[i] = s;
          rows.push_back(i);
        }
      }
    for (int ch : children[s]) {
      int64_t b = out.rowptr[ch], e = out.rowptr[ch + 1];
      for (int64_t q = b; q < e; ++q) {
        int i = out.Ls[q];
        if (i >= f && mark[i] != s) {
          mark[i] = s;
          rows.push_back(i);
        }
      }
    }
    std::sort(rows.begin() + (l - f), rows.end());
    out.Ls.insert(out.Ls.end(), rows.begin(), rows.end());
    out.rowptr[s + 1] = (int64_t)out.Ls.size();
    if ((int)rows.size() > l - f) {
      int par = col2sup[rows[l - f]];
      out.sparent[s] = par;
      children[par].push_back(s);
    }
  }
  // Li_ptr / lC per column
  out.Li_ptr.assign(n + 1, 0);
  out.lC.assign(n + 1, 0);
  int64_t xo = 0;
  for (int s = 0; s < supNo; ++s) {
    int f = blockSet[s], l = blockSet[s + 1];
    int64_t m = out.rowptr[s + 1] - out.rowptr[s];
    for (int j = f; j < l; ++j) {
      out.Li_ptr[j] = out.rowptr[s];
      out.lC[j] = xo;
      xo += m;
    }
  }
  out.Li_ptr[n] = out.rowptr[supNo];
  out.lC[n] = xo;
  out.xsize = xo;
  // update lists: for each descendant d, the distinct supernodes its off-diagonal rows hit
  std::vector<std::pair<int, int>> pairs;  // (target, source)
  for (int d = 0; d < supNo; ++d) {
    int w = blockSet[d + 1] - blockSet[d];
    int last = -1;
    for (int64_t q = out.rowptr[d] + w; q < out.rowptr[d + 1]; ++q) {
      int t = col2sup[out.Ls[q]];
      if (t != last) {
        pairs.emplace_back(t, d);
        last = t;
      }
    }
  }
  std::sort(pairs.begin(), pairs.end());
  out.prunePtr.assign(supNo + 1, 0);
  out.pruneSet.resize(pairs.size());
  for (size_t k = 0; k < pairs.size(); ++k) {
    out.prunePtr[pairs[k].first + 1]++;
    out.pruneSet[k] = pairs[k].second;
  }
  for (int s = 0; s < supNo; ++s) out.prunePtr[s + 1] += out.prunePtr[s];
  // level schedule: level = height above the leaves; one partition per supernode
  std::vector<int> level(supNo, 0);
  int nlev = 0;
  for (int s = 0; s < supNo; ++s) {
    nlev = std::max(nlev, level[s] + 1);
    int p = out.sparent[s];
    if (p >= 0) level[p] = std::max(level[p], level[s] + 1);
  }
  out.levelPtr.assign(nlev + 1, 0);
  for (int s = 0; s < supNo; ++s) out.levelPtr[level[s] + 1]++;
  for (int l = 0; l < nlev; ++l) out.levelPtr[l + 1] += out.levelPtr[l];
  out.partition.resize(supNo);
  std::vector<int> fill(out.levelPtr.begin(), out.levelPtr.end() - 1);
  for (int s = 0; s < supNo; ++s) out.partition[fill[level[s]]++] = s;
  out.parPtr.resize(supNo + 1);
  for (int k = 0; k <= supNo; ++k) out.parPtr[k] = k;
  return true;
}

}  // namespace swc
