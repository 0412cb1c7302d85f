// Fill-reducing ordering for general sparse symmetric matrices (host).
//
// The reference takes its ordering as an input (GIVEN, cholesky/sw_LSparsity.h:461-468:
// without a permutation file analyze_p2 asserts) and ships no working ordering of its own
// (its AMD, cholesky/AMD.h, is incomplete).  This is the project's own nested dissection
// for any graph:
//
//   * the adjacency graph of the pattern (both triangles, no self loops) is split
//     recursively; a disconnected subgraph is split into its components first;
//   * a connected subgraph is bisected by a vertex separator taken from a breadth-first
//     level structure (George and Liu, "Computer Solution of Large Sparse Positive
//     Definite Systems", 1981, chapter 8): from a pseudo-peripheral start vertex (repeated
//     breadth-first searches from a minimum-degree vertex of the last level until the
//     eccentricity stops growing) the levels L_0 .. L_h are formed, and for a split level m
//     the separator is the vertices of L_m (or L_m+1) that have a neighbour in L_m+1 (or
//     L_m); everything before it is one part and everything after it the other, so no
//     edge joins the parts.  Among the split levels the smallest separator whose smaller
//     part holds at least 30% of the rest is kept (the best-balanced one when none does),
//     over a few start vertices;
//   * the parts are ordered first, the separator last;
//   * subgraphs of at most `leaf` (<= 64) vertices are ordered by exact minimum degree
//     (elimination simulated on 64-bit adjacency masks, ties to the lowest index).
//
// perm[k] = original index of the vertex at new position k, the convention of the
// reference's permutation files.
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "swc_internal.h"

namespace swc {

namespace {

struct Graph {
  int n = 0;
  std::vector<int64_t> ptr;
  std::vector<int> adj;
};

bool build_graph(int n, const int *c, const int *r, Graph &g, std::string &err) {
  g.n = n;
  std::vector<int64_t> deg((size_t)n + 1, 0);
  for (int j = 0; j < n; ++j) {
    if (c[j + 1] < c[j]) { err = "column pointers not monotone"; return false; }
    for (int p = c[j]; p < c[j + 1]; ++p) {
      const int i = r[p];
      if (i < 0 || i >= n) { err = "row index out of range"; return false; }
      if (i == j) continue;
      deg[i + 1]++;
      deg[j + 1]++;
    }
  }
  for (int j = 0; j < n; ++j) deg[j + 1] += deg[j];
  std::vector<int> tmp(deg[n]);
  std::vector<int64_t> fill(deg.begin(), deg.end() - 1);
  for (int j = 0; j < n; ++j)
    for (int p = c[j]; p < c[j + 1]; ++p) {
      const int i = r[p];
      if (i == j) continue;
      tmp[fill[i]++] = j;
      tmp[fill[j]++] = i;
    }
  // sort and deduplicate each list (a full pattern lists every edge twice)
  g.ptr.assign((size_t)n + 1, 0);
  g.adj.clear();
  g.adj.reserve(tmp.size());
  for (int v = 0; v < n; ++v) {
    auto b = tmp.begin() + deg[v], e = tmp.begin() + deg[v + 1];
    std::sort(b, e);
    e = std::unique(b, e);
    g.adj.insert(g.adj.end(), b, e);
    g.ptr[v + 1] = (int64_t)g.adj.size();
  }
  return true;
}

struct Task {
  std::vector<int> verts;
  int64_t lo;   // first output position of this subgraph
};

class Dissector {
 public:
  Dissector(const Graph &g, const NdOptions &opt, std::vector<int64_t> &perm)
      : g_(g), opt_(opt), perm_(perm), tag_(g.n, -1), level_(g.n, -1) {}

  void run() {
    std::vector<Task> stack;
    Task all;
    all.verts.resize(g_.n);
    for (int v = 0; v < g_.n; ++v) all.verts[v] = v;
    all.lo = 0;
    stack.push_back(std::move(all));
    while (!stack.empty()) {
      Task t = std::move(stack.back());
      stack.pop_back();
      const int id = next_tag_++;
      for (int v : t.verts) tag_[v] = id;
      if ((int)t.verts.size() <= std::min(opt_.leaf, 64)) {
        min_degree(t, id);
        continue;
      }
      std::vector<std::vector<int>> comps;
      components(t.verts, id, comps);
      if (comps.size() > 1) {
        int64_t lo = t.lo;
        for (auto &cv : comps) {
          Task s;
          s.lo = lo;
          lo += (int64_t)cv.size();
          s.verts = std::move(cv);
          stack.push_back(std::move(s));
        }
        continue;
      }
      std::vector<int> A, B, S;
      bisect(t.verts, id, A, B, S);
      // parts first, separator last
      int64_t pos = t.lo + (int64_t)A.size() + (int64_t)B.size();
      for (int v : S) perm_[pos++] = v;
      Task ta, tb;
      ta.lo = t.lo;
      ta.verts = std::move(A);
      tb.lo = t.lo + (int64_t)ta.verts.size();
      tb.verts = std::move(B);
      if (!tb.verts.empty()) stack.push_back(std::move(tb));
      if (!ta.verts.empty()) stack.push_back(std::move(ta));
    }
  }

 private:
  const Graph &g_;
  const NdOptions &opt_;
  std::vector<int64_t> &perm_;
  std::vector<int> tag_, level_;
  int next_tag_ = 0;

  void components(const std::vector<int> &verts, int id, std::vector<std::vector<int>> &out) {
    std::vector<int> queue;
    for (int v : verts) level_[v] = -1;
    for (int s : verts) {
      if (level_[s] >= 0) continue;
      queue.clear();
      queue.push_back(s);
      level_[s] = 0;
      for (size_t h = 0; h < queue.size(); ++h) {
        const int v = queue[h];
        for (int64_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) {
          const int u = g_.adj[p];
          if (tag_[u] == id && level_[u] < 0) {
            level_[u] = 0;
            queue.push_back(u);
          }
        }
      }
      out.push_back(queue);
    }
  }

  int degree_in(int v, int id) const {
    int d = 0;
    for (int64_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) d += tag_[g_.adj[p]] == id;
    return d;
  }

  // Breadth-first levels of the subgraph from s; returns the number of levels and fills
  // order (vertices by level) and level_ of every vertex of the subgraph.
  int bfs(int s, int id, const std::vector<int> &verts, std::vector<int> &order,
          std::vector<int> &level_start) {
    for (int v : verts) level_[v] = -1;
    order.clear();
    level_start.clear();
    order.push_back(s);
    level_[s] = 0;
    level_start.push_back(0);
    int cur = 0;
    for (size_t h = 0; h < order.size(); ++h) {
      const int v = order[h];
      if (level_[v] != cur) {
        cur = level_[v];
        level_start.push_back((int)h);
      }
      for (int64_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) {
        const int u = g_.adj[p];
        if (tag_[u] == id && level_[u] < 0) {
          level_[u] = level_[v] + 1;
          order.push_back(u);
        }
      }
    }
    level_start.push_back((int)order.size());
    return cur + 1;
  }

  // Pseudo-peripheral vertex reached from s (George-Liu): last level's minimum-degree
  // vertex until the eccentricity stops growing.
  int pseudo_peripheral(int s, int id, const std::vector<int> &verts) {
    std::vector<int> order, ls;
    int h = bfs(s, id, verts, order, ls);
    for (int it = 0; it < 8; ++it) {
      int best = -1, bd = 1 << 30;
      for (int k = ls[h - 1]; k < ls[h]; ++k) {
        const int d = degree_in(order[k], id);
        if (d < bd) { bd = d; best = order[k]; }
      }
      const int h2 = bfs(best, id, verts, order, ls);
      s = best;
      if (h2 <= h) break;
      h = h2;
    }
    return s;
  }

  struct Split {
    int start = -1, m = -1, upper = 0;   // separator from level m (upper = 0) or m + 1 (1)
    int64_t sep = 0, a = 0, b = 0;
  };

  static bool better(const Split &x, const Split &y, int64_t total) {
    if (y.start < 0) return true;
    auto balanced = [&](const Split &s) {
      return std::min(s.a, s.b) >= (int64_t)(0.3 * (double)(total - s.sep));
    };
    const bool bx = balanced(x), by = balanced(y);
    if (bx != by) return bx;
    if (bx) return x.sep < y.sep || (x.sep == y.sep && std::llabs(x.a - x.b) < std::llabs(y.a - y.b));
    return std::min(x.a, x.b) > std::min(y.a, y.b);
  }

  void bisect(const std::vector<int> &verts, int id, std::vector<int> &A, std::vector<int> &B,
              std::vector<int> &S) {
    const int64_t total = (int64_t)verts.size();
    int mind = 1 << 30, s0 = verts[0];
    for (int v : verts) {
      const int d = degree_in(v, id);
      if (d < mind) { mind = d; s0 = v; }
    }
    std::vector<int> starts;
    int s = pseudo_peripheral(s0, id, verts);
    starts.push_back(s);
    std::vector<int> order, ls;
    for (int t = 1; t < opt_.trials; ++t) {
      // the far end of the previous start's level structure, then the vertex in its middle
      const int h = bfs(starts.back(), id, verts, order, ls);
      const int cand = t == 1 ? order.back() : order[ls[h / 2]];
      if (std::find(starts.begin(), starts.end(), cand) == starts.end())
        starts.push_back(pseudo_peripheral(cand, id, verts));
    }
    Split best;
    for (int st : starts) {
      const int h = bfs(st, id, verts, order, ls);
      if (h < 3) continue;
      // per level: vertices with a neighbour in the next / previous level
      std::vector<int64_t> up(h, 0), down(h, 0);
      for (int v : verts) {
        const int l = level_[v];
        bool nu = false, nd = false;
        for (int64_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) {
          const int u = g_.adj[p];
          if (tag_[u] != id) continue;
          nu |= level_[u] == l + 1;
          nd |= level_[u] == l - 1;
        }
        up[l] += nu;
        down[l] += nd;
      }
      for (int m = 1; m + 1 < h; ++m) {
        const int64_t before = ls[m], at = ls[m + 1] - ls[m];
        // separator in level m: its vertices with a neighbour in level m + 1
        Split x;
        x.start = st; x.m = m; x.upper = 0;
        x.sep = up[m];
        x.a = before + (at - up[m]);
        x.b = total - before - at;
        if (better(x, best, total)) best = x;
        // separator in level m + 1: its vertices with a neighbour in level m
        Split y;
        y.start = st; y.m = m; y.upper = 1;
        y.sep = down[m + 1];
        y.a = before + at;
        y.b = total - y.a - y.sep;
        if (better(y, best, total)) best = y;
      }
    }
    A.clear(); B.clear(); S.clear();
    if (best.start < 0) {
      // diameter below 3 from every start (a nearly complete subgraph): no useful
      // separator; order it as one block, lowest degree first
      S = verts;
      std::stable_sort(S.begin(), S.end(),
                       [&](int x, int y) { return degree_in(x, id) < degree_in(y, id); });
      return;
    }
    bfs(best.start, id, verts, order, ls);
    const int m = best.m;
    for (int v : verts) {
      const int l = level_[v];
      bool nu = false, nd = false;
      for (int64_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) {
        const int u = g_.adj[p];
        if (tag_[u] != id) continue;
        nu |= level_[u] == l + 1;
        nd |= level_[u] == l - 1;
      }
      if (best.upper == 0) {
        if (l < m || (l == m && !nu)) A.push_back(v);
        else if (l == m) S.push_back(v);
        else B.push_back(v);
      } else {
        if (l <= m) A.push_back(v);
        else if (l == m + 1 && nd) S.push_back(v);
        else B.push_back(v);
      }
    }
  }

  // Exact minimum degree on a subgraph of at most 64 vertices (adjacency bit masks).
  void min_degree(const Task &t, int id) {
    const int k = (int)t.verts.size();
    std::vector<int> local(k);
    std::vector<uint64_t> adj(k, 0);
    for (int i = 0; i < k; ++i) level_[t.verts[i]] = i;   // local index
    for (int i = 0; i < k; ++i) {
      const int v = t.verts[i];
      for (int64_t p = g_.ptr[v]; p < g_.ptr[v + 1]; ++p) {
        const int u = g_.adj[p];
        if (tag_[u] == id) adj[i] |= 1ULL << level_[u];
      }
    }
    uint64_t alive = k == 64 ? ~0ULL : ((1ULL << k) - 1ULL);
    for (int pos = 0; pos < k; ++pos) {
      int best = -1, bd = 1 << 30;
      for (int i = 0; i < k; ++i)
        if ((alive >> i) & 1ULL) {
          const int d = __builtin_popcountll(adj[i] & alive);
          if (d < bd) { bd = d; best = i; }
        }
      const uint64_t nb = adj[best] & alive & ~(1ULL << best);
      for (uint64_t m = nb; m; m &= m - 1) {
        const int u = __builtin_ctzll(m);
        adj[u] |= nb & ~(1ULL << u);   // the neighbours of the eliminated vertex form a clique
      }
      alive &= ~(1ULL << best);
      perm_[t.lo + pos] = t.verts[best];
    }
  }
};

}  // namespace

bool nested_dissection_order(int n, const int *c, const int *r, const NdOptions &opt,
                             std::vector<int64_t> &perm, std::string &err) {
  if (n <= 0 || !c || !r) { err = "empty matrix"; return false; }
  if (opt.leaf < 1 || opt.trials < 1) { err = "leaf and trials must be positive"; return false; }
  Graph g;
  if (!build_graph(n, c, r, g, err)) return false;
  perm.assign((size_t)n, -1);
  Dissector dis(g, opt, perm);
  dis.run();
  std::vector<char> seen((size_t)n, 0);
  for (int64_t v : perm) {
    if (v < 0 || v >= n || seen[v]) { err = "internal: ordering is not a permutation"; return false; }
    seen[v] = 1;
  }
  return true;
}

}  // namespace swc
