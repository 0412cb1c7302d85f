// Engine: validates and uploads the symbolic structure, derives the level schedule and
// the task lists of every kernel, and runs the factorization on one CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>

#include "swc_engine.h"

namespace swc {

namespace {

template <typename T>
bool upload(T *&dst, const T *src, size_t count, cudaStream_t st, std::string &err) {
  if (dst) { cudaFree(dst); dst = nullptr; }
  size_t bytes = sizeof(T) * std::max<size_t>(count, 1);
  cudaError_t e = cudaMalloc(&dst, bytes);
  if (e == cudaSuccess && count) e = cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    err = std::string("device upload: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

bool small_class(int w, int64_t m, const Tuning &T) {
  return w <= std::min(T.small_max_w, SMALL_MAX_W) && m <= std::min(T.small_max_m, SMALL_MAX_M) &&
         (int64_t)w * m <= std::min(T.small_max_elems, SMALL_MAX_ELEMS);
}

// shared memory of the small-class kernel for an m x w panel: panel, rows, relative
// indices (+ padding to 8 bytes), pivot column, staging slab
int64_t small_smem(int w, int64_t m) {
  return 8 * m * w + 8 * m + 8 + 8 * (int64_t)w + 8 * (int64_t)SMALL_SLAB;
}

// One update tile of the tiled class with the descendants that touch it.
struct TileWork {
  int4 task;                 // (s, r0, c0, first pair -- filled when flattened)
  std::vector<int4> pairs;   // (d, a0, b0, na | nb << 16)
  std::vector<TcPair> tc;    // the same pairs with the tile rows / columns they feed
  double flops = 0, bytes = 0;
};

// Mask of the first n bits (n <= 64).
inline unsigned long long low_bits(int n) { return n >= 64 ? ~0ULL : ((1ULL << n) - 1ULL); }

// Splits every update d -> s of the prune set into the 64x64 tiles of s it touches.  The
// rows of d at or below s's first column map monotonically into s's row list, so each
// tile receives one contiguous run of d's rows for its row range and one for its column
// range.  Appends one TileWork per touched tile (row-major tile order).
bool build_update_pairs(int s, int f, int w, int m, const std::vector<int> &super,
                        const std::vector<int64_t> &rowptr, const int *Ls, const int *prunePtr,
                        const int *pruneSet, std::vector<TileWork> &out, std::string &err) {
  const int ntr = (m + TB - 1) / TB, ntc = (w + TB - 1) / TB;
  std::vector<int> tile_of((size_t)ntr * ntc, -1);
  std::vector<TileWork> tiles;
  const int *rows_s = Ls + rowptr[s];
  std::vector<int> pos;
  struct Run { int tile, start, count; };
  std::vector<Run> runs;
  for (int q = prunePtr[s]; q < prunePtr[s + 1]; ++q) {
    const int d = pruneSet[q];
    const int *rd = Ls + rowptr[d];
    const int md = (int)(rowptr[d + 1] - rowptr[d]);
    const int wd = super[d + 1] - super[d];
    const int lb = (int)(std::lower_bound(rd, rd + md, f) - rd);
    pos.clear();
    int k = 0;
    for (int i = lb; i < md; ++i) {
      while (k < m && rows_s[k] < rd[i]) ++k;
      if (k == m || rows_s[k] != rd[i]) {
        err = "row structure of a descendant is not contained in its ancestor's";
        return false;
      }
      pos.push_back(k);
    }
    runs.clear();
    for (int i = 0; i < (int)pos.size(); ++i) {
      const int tl = pos[i] / TB;
      if (runs.empty() || runs.back().tile != tl) runs.push_back({tl, lb + i, 1});
      else runs.back().count++;
    }
    for (const Run &cr : runs) {
      if ((int64_t)cr.tile * TB >= w) break;   // column runs: positions < w only
      int nb = 0;
      unsigned long long cmask = 0;
      for (int i = cr.start - lb; i < cr.start - lb + cr.count; ++i)
        if (pos[i] < w) {
          ++nb;
          cmask |= 1ULL << (pos[i] - cr.tile * TB);
        }
      if (nb == 0) continue;
      for (const Run &rr : runs) {
        if (rr.tile < cr.tile) continue;
        unsigned long long rmask = 0;
        for (int i = rr.start - lb; i < rr.start - lb + rr.count; ++i)
          rmask |= 1ULL << (pos[i] - rr.tile * TB);
        const int key = rr.tile * ntc + cr.tile;
        if (tile_of[key] < 0) {
          tile_of[key] = (int)tiles.size();
          TileWork tw;
          tw.task = make_int4(s, rr.tile * TB, cr.tile * TB, 0);
          tiles.push_back(std::move(tw));
        }
        TileWork &tw = tiles[tile_of[key]];
        tw.pairs.push_back(make_int4(d, rr.start, cr.start, rr.count | (nb << 16)));
        tw.tc.push_back(TcPair{d, rr.start, cr.start, wd << 16, rmask, cmask});
        tw.flops += 2.0 * rr.count * nb * wd;
        tw.bytes += 8.0 * (rr.count + nb) * wd;
      }
    }
  }
  for (TileWork &tw : tiles) {
    tw.bytes += 16.0 * TB * TB;
    out.push_back(std::move(tw));
  }
  return true;
}

}  // namespace

Engine::Engine(int device) : device_(device) {
  cudaSetDevice(device_);
  const char *ng = getenv("SWC_NO_GRAPH");
  use_graph_ = !(ng && ng[0] == '1');
  cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking);
  stream_ = own_stream_;
  cudaStreamCreateWithFlags(&aux_stream_, cudaStreamNonBlocking);
  cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming);
  cudaStreamCreateWithFlags(&small_stream_, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&grp_stream_, cudaStreamNonBlocking);
  for (int k = 0; k < 2; ++k) cudaEventCreateWithFlags(&ev_grp_[k], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ev_sfork_, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ev_sjoin_, cudaEventDisableTiming);
  cudaMallocHost(&h_status_, kStatusWords * sizeof(int));
}

Engine::~Engine() {
  release();
  if (d_stage_) cudaFree(d_stage_);
  if (h_status_) cudaFreeHost(h_status_);
  if (h_norms_) cudaFreeHost(h_norms_);
  if (own_stream_) cudaStreamDestroy(own_stream_);
  if (aux_stream_) cudaStreamDestroy(aux_stream_);
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  if (ev_join_) cudaEventDestroy(ev_join_);
  if (small_stream_) cudaStreamDestroy(small_stream_);
  if (grp_stream_) cudaStreamDestroy(grp_stream_);
  for (int k = 0; k < 2; ++k)
    if (ev_grp_[k]) cudaEventDestroy(ev_grp_[k]);
  if (ev_sfork_) cudaEventDestroy(ev_sfork_);
  if (ev_sjoin_) cudaEventDestroy(ev_sjoin_);
}

void Engine::release() {
  void *ptrs[] = {d_super_, d_Ls_, d_Ap_, d_Ai_, d_rowptr_, d_xptr_, d_upd_ptr_, d_upd_, d_upd_lbub_,
                  d_Ax_, dL_, d_status_, d_small_, d_big_, d_asm_, d_panel_, d_upd_tasks_,
                  d_syrk_, d_pairs_, d_upd_end_, d_dinv_, d_dinv_off_, d_diag_,
                  d_slist_, d_cptr_, d_cidx_, d_flags_, d_fchain_, d_bchain_, d_scontrib_, d_sgather_, d_csr_rp_, d_csr_ci_,
                  d_csr_map_,
                  d_csr_val_, d_contrib_, d_work_, d_norms_, d_persist_, d_qctr_, d_npart_,
                  d_tiny_, d_dense_tasks_, d_dense_toff_, d_dense_ver_, d_swarp_,
                  d_Lk_, d_xk_, d_xk16_, d_tmaps_, d_tc_pairs_, d_syrk_pairs_, d_syrk_end_,
                  d_sc_tiles_, d_sc_base_, d_sc_coff_, d_sc_rel_, d_sc_relidx_, d_sc_maps_,
                  d_sc_maps16_,
                  d_sc_small_, d_sc_dense_};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  release_adjoint();
  d_super_ = d_Ls_ = d_Ap_ = d_Ai_ = nullptr;
  d_rowptr_ = d_xptr_ = nullptr;
  d_upd_ptr_ = d_upd_ = nullptr;
  d_upd_lbub_ = nullptr;
  d_Ax_ = dL_ = nullptr;
  d_status_ = d_small_ = d_big_ = nullptr;
  d_asm_ = d_panel_ = nullptr;
  d_upd_tasks_ = d_syrk_ = d_pairs_ = nullptr;
  d_upd_end_ = nullptr;
  d_dinv_ = nullptr;
  d_dinv_off_ = nullptr;
  d_diag_ = nullptr;
  d_dense_tasks_ = nullptr;
  d_dense_toff_ = d_dense_ver_ = nullptr;
  dense_ver_len_ = 0;
  d_slist_ = d_cptr_ = d_cidx_ = d_flags_ = nullptr;
  d_swarp_ = nullptr;
  d_fchain_ = d_bchain_ = nullptr;
  d_scontrib_ = d_sgather_ = nullptr;
  d_csr_rp_ = d_csr_ci_ = d_csr_map_ = nullptr;
  d_csr_val_ = d_contrib_ = d_work_ = d_norms_ = nullptr;
  d_persist_ = d_qctr_ = d_tiny_ = nullptr;
  d_Lk_ = nullptr;
  d_xk_ = d_xk16_ = nullptr;
  d_tmaps_ = nullptr;
  d_tc_pairs_ = d_syrk_pairs_ = nullptr;
  d_syrk_end_ = nullptr;
  d_sc_tiles_ = nullptr;
  d_sc_small_ = nullptr;
  d_sc_dense_ = nullptr;
  d_sc_base_ = d_sc_coff_ = nullptr;
  d_sc_rel_ = d_sc_relidx_ = nullptr;
  d_sc_maps_ = d_sc_maps16_ = nullptr;
  kmirror_len_ = 0;
  tiny_ctas_ = 0;
  d_npart_ = nullptr;
  persist_ctas_ = 0;
  release_solve_graphs();
  if (d_sx_) cudaFree(d_sx_);
  d_sx_ = nullptr;
  work_nrhs_ = 0;
  for (int k = 0; k < 3; ++k) {
    if (graph_exec_[k]) cudaGraphExecDestroy(graph_exec_[k]);
    if (graph_[k]) cudaGraphDestroy(graph_[k]);
    graph_exec_[k] = nullptr;
    graph_[k] = nullptr;
  }
}

// Dataflow tasks of the dense factorization of one tiled-class panel (w columns, m rows),
// see k_dense_persist.  The updates of tile (I, C) by column blocks 0 .. C-1 (0 .. C-2 for
// a diagonal tile, whose last one its diagonal task applies) are grouped: the last block
// alone (off-diagonal tiles), then groups of `group` blocks back to block 0, so the
// updates the next TRSM waits for stay short and the older ones run as longer products.
// Each task gets its bottom level: its cost plus the longest chain of costs of the tasks
// that wait for it (diagonal block 4; full TRSM tile 1; update 0.6 + 0.4 per block;
// scaled by the tile's fill).  Tasks are generated in a topological order; sorting by
// decreasing bottom level keeps one (every task's bottom level exceeds its successors' by
// at least its own cost) and starts the longest chains first.
struct DenseTask {
  double bl;
  int4 t;
};

static inline int dense_code(int kind, int step, int first) {
  return kind | (step << 2) | (first << 17);
}

static void dense_panel_tasks(int s, int w, int m, int group, std::vector<DenseTask> &out) {
  const int nb = (w + TB - 1) / TB, mb = (m + TB - 1) / TB;
  const double per_elem = 1.0 / (TB * TB), min_frac = 0.25;
  struct Node {
    int4 t;
    double cost, succ = 0.0;
    int pred[3] = {-1, -1, -1};
  };
  std::vector<Node> nodes;
  std::vector<int> last((size_t)nb * mb, -1);      // [C * mb + I]: last task that set ver(I, C)
  std::vector<int> trsm((size_t)nb * mb, -1);      // [J * mb + I]: aligned TRSM task of (I, J)
  auto add = [&](int4 t, double cost, int p0, int p1, int p2) {
    Node nd;
    nd.t = t;
    nd.cost = cost;
    nd.pred[0] = p0;
    nd.pred[1] = p1;
    nd.pred[2] = p2;
    nodes.push_back(nd);
    return (int)nodes.size() - 1;
  };
  for (int J = 0; J < nb; ++J) {
    const int c0 = J * TB, bw = std::min(TB, w - c0);
    // diagonal block J: waits for the diagonal tile's updates (through J-2) and TRSM (J, J-1)
    const int d = add(make_int4(s, c0, c0, dense_code(0, J, 0)), 4.0, last[(size_t)J * mb + J],
                      J > 0 ? trsm[(size_t)(J - 1) * mb + J] : -1, -1);
    last[(size_t)J * mb + J] = d;
    // TRSM of the rows below it: waits for the diagonal block and the covered tiles' updates
    for (int r0 = c0 + bw; r0 < m; r0 += TB) {
      const int nr = std::min(TB, m - r0);
      const int I0 = r0 / TB, I1 = (r0 + nr - 1) / TB;
      const int p1 = I0 != J ? last[(size_t)J * mb + I0] : -1;
      const int p2 = I1 != J && I1 != I0 ? last[(size_t)J * mb + I1] : -1;
      const int t = add(make_int4(s, r0, 0, dense_code(1, J, 0)),
                        std::max(min_frac, nr * bw * per_elem), d, p1, p2);
      if (bw == TB) {
        trsm[(size_t)J * mb + I0] = t;
        last[(size_t)J * mb + I0] = t;
      }
    }
    // update groups ending at block J: tile (I, C), C > J
    for (int C = J + 1; C < nb; ++C)
      for (int I = C; I < mb; ++I) {
        int first;
        if (I > C && J == C - 1) first = J;                          // the last block alone
        else if (J <= C - 2 && (C - 2 - J) % group == 0) first = std::max(0, J - group + 1);
        else continue;
        const int nrow = std::min(TB, m - I * TB), ncol = std::min(TB, w - C * TB);
        const double cost = std::max(min_frac, nrow * ncol * per_elem) * (0.6 + 0.4 * (J - first + 1));
        const int u = add(make_int4(s, I * TB, C * TB, dense_code(2, J, first)), cost,
                          last[(size_t)C * mb + I], trsm[(size_t)J * mb + I],
                          trsm[(size_t)J * mb + C]);
        last[(size_t)C * mb + I] = u;
      }
  }
  // bottom levels, successors before predecessors
  for (int k = (int)nodes.size() - 1; k >= 0; --k) {
    const double bl = nodes[k].cost + nodes[k].succ;
    nodes[k].succ = bl;   // now the bottom level
    for (int q = 0; q < 3; ++q)
      if (nodes[k].pred[q] >= 0) nodes[nodes[k].pred[q]].succ = std::max(nodes[nodes[k].pred[q]].succ, bl);
  }
  for (const Node &nd : nodes) out.push_back({nd.succ, nd.t});
}

// Replays the waits of k_dense_persist on the host, in list order, with the tile versions
// every earlier task leaves: true when no task waits for a later one, i.e. the persistent
// walk cannot stall whatever the number of resident CTAs.
static bool dense_order_ok(const int4 *tasks, int count, const std::vector<int> &super,
                           const std::vector<int64_t> &rowptr, const std::vector<int> &toff,
                           std::vector<int> &ver) {
  for (int k = 0; k < count; ++k) {
    const int4 t = tasks[k];
    const int s = t.x, kind = t.w & 3, step = (t.w >> 2) & 0x7fff, first = t.w >> 17;
    const int w = super[s + 1] - super[s];
    const int m = (int)(rowptr[s + 1] - rowptr[s]);
    const int mb = (m + TB - 1) / TB;
    int *V = ver.data() + toff[s];
    if (kind == 0) {
      if (step > 0 && (V[step * mb + step] < step - 1 || V[(step - 1) * mb + step] < step))
        return false;
      V[step * mb + step] = step + 1;
    } else if (kind == 1) {
      const int nr = std::min(TB, m - t.y);
      if (V[step * mb + step] < step + 1) return false;
      for (int I = t.y / TB; I <= (t.y + nr - 1) / TB; ++I)
        if (I != step && V[step * mb + I] < step) return false;
      if (t.y % TB == 0 && w - step * TB >= TB) V[step * mb + t.y / TB] = step + 1;
    } else {
      const int I = t.y / TB, C = t.z / TB;
      if (V[C * mb + I] < first || V[step * mb + I] < step + 1 || V[step * mb + C] < step + 1)
        return false;
      V[C * mb + I] = step + 1;
    }
  }
  return true;
}

bool build_plan(int n, const int *c, const int *r, const int64_t *lC, const int *Ls,
                const int64_t *Li_ptr, const int *blockSet, int supNo, const int *prunePtr,
                const int *pruneSet, HostSym &H, Plan &P, std::string &err, const Tuning &T) {
  // ---- host-side validation of the symbolic arrays (no device work on bad input) ----
  if (n <= 0 || supNo <= 0 || !c || !r || !lC || !Ls || !Li_ptr || !blockSet || !prunePtr ||
      !pruneSet) {
    err = "null or empty symbolic input";
    return false;
  }
  if (blockSet[0] != 0 || blockSet[supNo] != n) {
    err = "blockSet must start at 0 and end at n";
    return false;
  }
  std::vector<int> super(blockSet, blockSet + supNo + 1);
  std::vector<int64_t> rowptr(supNo + 1), xptr(supNo);
  for (int s = 0; s < supNo; ++s) {
    int f = super[s], l = super[s + 1];
    if (l <= f) { err = "blockSet must be strictly increasing"; return false; }
    int64_t m = Li_ptr[l] - Li_ptr[f];
    if (m < l - f) { err = "supernode has fewer rows than columns"; return false; }
    for (int j = f; j < l; ++j) {
      if (Li_ptr[j] != Li_ptr[f] || lC[j + 1] - lC[j] != m) {
        err = "Li_ptr / lC are not a supernodal layout";
        return false;
      }
    }
    rowptr[s] = Li_ptr[f];
    xptr[s] = lC[f];
    for (int64_t q = Li_ptr[f]; q < Li_ptr[l]; ++q) {
      int64_t k = q - Li_ptr[f];
      if (Ls[q] < 0 || Ls[q] >= n || (k < l - f && Ls[q] != f + k) ||
          (k > 0 && Ls[q] <= Ls[q - 1])) {
        err = "row list of a supernode is not sorted / does not start with its columns";
        return false;
      }
    }
  }
  rowptr[supNo] = Li_ptr[n];
  int64_t nls = Li_ptr[n];
  int64_t xsize = lC[n];
  int64_t nnz = c[n];
  for (int j = 0; j < n; ++j)
    if (c[j + 1] < c[j]) { err = "column pointers of A not monotone"; return false; }
  for (int s = 0; s <= supNo; ++s)
    if (s < supNo && prunePtr[s + 1] < prunePtr[s]) { err = "prunePtr not monotone"; return false; }
  int nprune = prunePtr[supNo];
  for (int q = 0; q < nprune; ++q)
    if (pruneSet[q] < 0 || pruneSet[q] >= supNo) { err = "pruneSet entry out of range"; return false; }
  for (int s = 0; s < supNo; ++s)
    for (int q = prunePtr[s]; q < prunePtr[s + 1]; ++q)
      if (pruneSet[q] >= s) { err = "prune set holds a non-descendant"; return false; }

  // ---- supernodal etree and levels ----
  std::vector<int> col2sup(n);
  for (int s = 0; s < supNo; ++s)
    for (int j = super[s]; j < super[s + 1]; ++j) col2sup[j] = s;
  std::vector<int> level(supNo, 0);
  int nlev = 0;
  for (int s = 0; s < supNo; ++s) {
    int w = super[s + 1] - super[s];
    int64_t m = rowptr[s + 1] - rowptr[s];
    nlev = std::max(nlev, level[s] + 1);
    if (m > w) {
      int p = col2sup[Ls[rowptr[s] + w]];
      if (p <= s) { err = "supernodes are not numbered children before parents"; return false; }
      level[p] = std::max(level[p], level[s] + 1);
    }
  }
  // every update source must sit on an earlier level than its target
  for (int s = 0; s < supNo; ++s)
    for (int q = prunePtr[s]; q < prunePtr[s + 1]; ++q)
      if (level[pruneSet[q]] >= level[s]) { err = "prune set is not consistent with the etree"; return false; }

  // ---- persistent bottom sets: tiny supernodes whose whole subtree is tiny (one warp
  // each), then small supernodes whose whole subtree is tiny or small (one CTA each) ----
  std::vector<char> in_tiny(supNo, 0), in_persist(supNo, 0);
  {
    std::vector<char> kids_tiny(supNo, 1), kids_ok(supNo, 1);
    for (int s = 0; s < supNo; ++s) {
      const int w = super[s + 1] - super[s];
      const int64_t m = rowptr[s + 1] - rowptr[s];
      in_tiny[s] = T.tiny && kids_tiny[s] && m <= TINY_M && (int64_t)w * m <= TINY_ELEMS;
      if (!in_tiny[s])
        in_persist[s] = T.persist && kids_ok[s] && small_class(w, m, T) &&
                        small_smem(w, m) <= T.persist_max_smem;
      if (m > w) {
        const int p = col2sup[Ls[rowptr[s] + w]];
        if (!in_tiny[s]) kids_tiny[p] = 0;
        if (!in_tiny[s] && !in_persist[s]) kids_ok[p] = 0;
      }
    }
  }

  // ---- plan ----
  P = Plan();
  P.waves.resize(nlev);
  P.dense_toff.assign(supNo, -1);
  std::vector<std::vector<int>> by_level(nlev);
  for (int s = 0; s < supNo; ++s) by_level[level[s]].push_back(s);
  int launches = 2;
  std::vector<TileWork> wave_tiles;
  for (int lv = 0; lv < nlev; ++lv) {
    Wave &W = P.waves[lv];
    W.small_off = (int)P.small_list.size();
    W.asm_off = (int)P.asm_tasks.size();
    W.upd_off = (int)P.upd_tasks.size();
    std::vector<int> big;
    for (int s : by_level[lv]) {
      int w = super[s + 1] - super[s];
      int64_t m = rowptr[s + 1] - rowptr[s];
      if (in_tiny[s]) {
        P.tiny_list.push_back(s);
      } else if (in_persist[s]) {
        P.persist_list.push_back(s);
        P.persist_smem = std::max<int>(P.persist_smem, (int)small_smem(w, m));
      } else if (small_class(w, m, T)) {
        P.small_list.push_back(s);
        W.small_smem = std::max<int>(W.small_smem, (int)small_smem(w, m));
      } else {
        big.push_back(s);
      }
    }
    W.small_cnt = (int)P.small_list.size() - W.small_off;
    W.big_off = (int)P.big_list.size();
    W.big_cnt = (int)big.size();
    P.big_list.insert(P.big_list.end(), big.begin(), big.end());
    int maxnb = 0;
    for (int s : big) {
      int f = super[s], w = super[s + 1] - f;
      int m = (int)(rowptr[s + 1] - rowptr[s]);
      for (int j = f; j < f + w; ++j) P.asm_tasks.push_back(make_int2(s, j));
      if (prunePtr[s + 1] > prunePtr[s] &&
          !build_update_pairs(s, f, w, m, super, rowptr, Ls, prunePtr, pruneSet, wave_tiles,
                              err))
        return false;
      maxnb = std::max(maxnb, (w + TB - 1) / TB);
    }
    W.asm_cnt = (int)P.asm_tasks.size() - W.asm_off;
    // heaviest tiles first (shorter tail); ties keep supernode / tile order
    std::stable_sort(wave_tiles.begin(), wave_tiles.end(),
                     [](const TileWork &a, const TileWork &b) { return a.flops > b.flops; });
    for (TileWork &tw : wave_tiles) {
      tw.task.w = (int)P.upd_pairs.size();
      P.upd_pairs.insert(P.upd_pairs.end(), tw.pairs.begin(), tw.pairs.end());
      P.tc_pairs.insert(P.tc_pairs.end(), tw.tc.begin(), tw.tc.end());
      P.upd_tasks.push_back(tw.task);
      P.upd_end.push_back((int)P.upd_pairs.size());
      P.work.flops[K_UPDATE] += tw.flops;
      P.work.bytes[K_UPDATE] += tw.bytes;
    }
    wave_tiles.clear();
    W.upd_cnt = (int)P.upd_tasks.size() - W.upd_off;
    for (int j = 0; j < maxnb; ++j) {
      W.panel_off.push_back((int)P.panel_tasks.size());
      W.syrk_off.push_back((int)P.syrk_tasks.size());
      W.diag_off.push_back((int)P.diag_list.size());
      W.scd_off.push_back((int)P.sc_dense.size());
      std::vector<ScTile> grouped;   // after the step's next-column tiles
      for (int s : big) {
        int w = super[s + 1] - super[s];
        int m = (int)(rowptr[s + 1] - rowptr[s]);
        int c0 = j * TB;
        if (c0 >= w) continue;
        int bw = std::min(TB, w - c0);
        for (int r0 = c0 + bw; r0 < m; r0 += TB) P.panel_tasks.push_back(make_int2(s, r0));
        // trailing updates of step j: column j+1 (the next TRSM reads it) by block j alone;
        // a column C >= j+2 by the group of blocks that closes at step j (blocks j-G+1..j,
        // at the steps j = C-2, C-2-G, ...), so it receives blocks 0..C-2 in groups and
        // block C-1 at step C-1, and every tile is read and written once per group
        const int G = std::max(1, T.dense_group);
        for (int cc = c0 + TB; cc < w; cc += TB) {
          const int C = cc / TB;
          int first;
          if (C == j + 1) first = j;
          else if ((C - 2 - j) % G == 0) first = std::max(0, j - G + 1);
          else continue;
          if (T.scatter) {   // the same update as 128-row x one-column-block dense tiles
            const int kc = c0 + bw - first * TB;
            for (int r0 = cc == c0 + TB ? cc + TB : cc; r0 < m; r0 += 128)
              (C == j + 1 ? P.sc_dense : grouped)
                  .push_back(ScTile{s, r0, cc, (kc + 31) / 32, m, first * TB,
                                    std::min(TB, w - cc), 1, 0, 0});
          }
          for (int r0 = cc; r0 < m; r0 += TB)
            if (!(cc == c0 + TB && r0 == cc)) {   // next diagonal tile: the TRSM task's update
              // .w: the task's own index: its product (column blocks first..j) in syrk_pairs
              P.syrk_pairs.push_back(TcPair{s, r0, cc, (first * TB) | ((c0 + bw - first * TB) << 16),
                                            low_bits(std::min(TB, m - r0)),
                                            low_bits(std::min(TB, w - cc))});
              P.syrk_tasks.push_back(make_int4(s, r0, cc, (int)P.syrk_tasks.size()));
              P.syrk_end.push_back((int)P.syrk_tasks.size());
            }
        }
        if (c0 + TB < w) P.diag_list.push_back(s);
      }
      W.panel_cnt.push_back((int)P.panel_tasks.size() - W.panel_off.back());
      W.syrk_cnt.push_back((int)P.syrk_tasks.size() - W.syrk_off.back());
      W.diag_cnt.push_back((int)P.diag_list.size() - W.diag_off.back());
      W.scd_nc.push_back((int)P.sc_dense.size() - W.scd_off.back());
      P.sc_dense.insert(P.sc_dense.end(), grouped.begin(), grouped.end());
      W.scd_cnt.push_back((int)P.sc_dense.size() - W.scd_off.back());
    }
    launches += (W.small_cnt > 0) + (W.asm_cnt > 0) + (W.upd_cnt > 0);
    int widest = 0;
    for (int s : big) widest = std::max(widest, super[s + 1] - super[s]);
    if (T.dense_dataflow && !big.empty() && (widest + TB - 1) / TB < (1 << 14)) {
      std::vector<DenseTask> dt;
      for (int s : big) {
        const int w = super[s + 1] - super[s];
        const int m = (int)(rowptr[s + 1] - rowptr[s]);
        P.dense_toff[s] = (int)P.dense_tiles;
        P.dense_tiles += (int64_t)((w + TB - 1) / TB) * ((m + TB - 1) / TB);
        if (P.dense_tiles > INT32_MAX) { err = "too many dense tiles"; return false; }
        dense_panel_tasks(s, w, m, std::max(1, T.dense_group), dt);
      }
      std::stable_sort(dt.begin(), dt.end(),
                       [](const DenseTask &a, const DenseTask &b) { return a.bl > b.bl; });
      W.dense_off = (int)P.dense_tasks.size();
      W.dense_cnt = (int)dt.size();
      for (const DenseTask &d : dt) P.dense_tasks.push_back(d.t);
      std::vector<int> ver(P.dense_tiles, 0);
      if (!dense_order_ok(P.dense_tasks.data() + W.dense_off, W.dense_cnt, super, rowptr,
                          P.dense_toff, ver)) {
        err = "internal: dense task order is not topological";
        return false;
      }
      launches += 1;
    } else {
      launches += (W.big_cnt > 0);
      for (int j = 0; j < maxnb; ++j)
        launches += (W.panel_cnt[j] > 0) + (W.syrk_cnt[j] > 0) + (W.diag_cnt[j] > 0);
    }
  }
  if (!P.persist_list.empty()) launches += 1;
  if (!P.tiny_list.empty()) launches += 1;
  P.launches = launches;

  // ---- right-looking updates of the split-TF32 mode: the contribution of every descendant
  // d to tiled-class targets, C = B B^T over the rows of d from the first one whose column
  // belongs to a tiled supernode, as 128x128 tiles of one dense product, launched in the
  // level after d's own (every target sits on a later level) ----
  if (T.scatter && !P.big_list.empty()) {
    std::vector<char> tiled(supNo, 0);
    for (int s : P.big_list) tiled[s] = 1;
    std::vector<std::vector<ScTile>> by_wave(nlev);
    std::vector<std::vector<int2>> small_by_wave(nlev);
    P.sc_coff.assign(supNo, 0);
    P.sc_used.assign(supNo, 0);
    for (int d = 0; d < supNo; ++d) {
      const int wd = super[d + 1] - super[d];
      const int md = (int)(rowptr[d + 1] - rowptr[d]);
      const int *rd = Ls + rowptr[d];
      int c0 = wd;
      while (c0 < md && !tiled[col2sup[rd[c0]]]) ++c0;
      if (c0 == md) continue;
      P.sc_coff[d] = (int64_t)P.sc_base.size() - c0;
      for (int j = c0; j < md;) {
        const int s = col2sup[rd[j]];
        int je = j;
        while (je < md && col2sup[rd[je]] == s) ++je;
        if (!tiled[s]) {
          P.sc_base.insert(P.sc_base.end(), (size_t)(je - j), (int64_t)-1);
          P.sc_rel.insert(P.sc_rel.end(), (size_t)(je - j), 0);
        } else {
          // positions of rows j.. of d in the row list of s (contained in it: s is an
          // ancestor of d)
          const int *rs = Ls + rowptr[s];
          const int ms = (int)(rowptr[s + 1] - rowptr[s]);
          const int64_t rbase = (int64_t)P.sc_relidx.size() - j;
          if ((int64_t)P.sc_relidx.size() + (md - j) > INT32_MAX) {
            err = "relative indices of the right-looking updates exceed 2^31 entries";
            return false;
          }
          int k = (int)(std::lower_bound(rs, rs + ms, rd[j]) - rs);
          for (int i = j; i < md; ++i) {
            while (k < ms && rs[k] < rd[i]) ++k;
            if (k == ms || rs[k] != rd[i]) {
              err = "row structure of a descendant is not contained in its ancestor's";
              return false;
            }
            P.sc_relidx.push_back(k);
          }
          for (int q = j; q < je; ++q) {
            P.sc_base.push_back(xptr[s] + (int64_t)(rd[q] - super[s]) * ms);
            P.sc_rel.push_back((int)rbase);
          }
        }
        j = je;
      }
      const int nk = (wd + 31) / 32, r = md - c0;
      if (r <= 128 && (int64_t)wd * ((r + 31) & ~31) <= SC_SMALL_ELEMS) {
        small_by_wave[level[d] + 1].push_back(make_int2(d, c0));   // FP64 on the CUDA cores
        continue;
      }
      const int kcut = T.scatter_kmax > 0 ? std::max(1, T.scatter_kmax / 32) : nk;
      for (int i0 = c0; i0 < md; i0 += 128)
        for (int j0 = c0; j0 <= i0; j0 += 128) {
          for (int kb = 0; kb < nk; kb += kcut)
            by_wave[level[d] + 1].push_back(
                ScTile{d, i0, j0, std::min(kcut, nk - kb), md, kb * 32, 128, 0, P.sc_coff[d], 0});
          P.sc_flops += 2.0 * 128 * 128 * wd;
        }
      P.sc_used[d] |= 1;
    }
    // dense tiles of its own factorization: A operands through the 128-row maps, B through
    // the 64-row maps
    for (int s : P.big_list) P.sc_used[s] |= 3;
    // every tile's supernode has the maps its loads use
    for (const ScTile &t : P.sc_tiles)
      if (!(P.sc_used[t.d] & 1)) { err = "internal: scatter tile without its tensor maps"; return false; }
    for (const ScTile &t : P.sc_dense)
      if ((P.sc_used[t.d] & 3) != 3) { err = "internal: dense tile without its tensor maps"; return false; }
    // per level: larger K first (a shorter tail); one descendant's tiles stay together
    int sc_launches = 0;
    for (int lv = 0; lv < nlev; ++lv) {
      std::vector<ScTile> &v = by_wave[lv];
      std::stable_sort(v.begin(), v.end(),
                       [](const ScTile &a, const ScTile &b) { return a.nk > b.nk; });
      P.waves[lv].sc_off = (int)P.sc_tiles.size();
      P.waves[lv].sc_cnt = (int)v.size();
      P.sc_tiles.insert(P.sc_tiles.end(), v.begin(), v.end());
      P.waves[lv].scs_off = (int)P.sc_small.size();
      P.waves[lv].scs_cnt = (int)small_by_wave[lv].size();
      P.sc_small.insert(P.sc_small.end(), small_by_wave[lv].begin(), small_by_wave[lv].end());
      sc_launches += !v.empty() + !small_by_wave[lv].empty();
    }
    // one assemble launch up front instead of one per level; scatter instead of tile-owner
    int asm_l = 0, upd_l = 0;
    for (const Wave &W : P.waves) {
      asm_l += W.asm_cnt > 0;
      upd_l += W.upd_cnt > 0;
    }
    P.launches_scatter = launches - asm_l - upd_l + (asm_l > 0) + sc_launches;
  } else {
    P.launches_scatter = launches;
  }

  // ---- algorithmic work per kernel class (one factorization) ----
  {
    KernelStats &K = P.work;
    std::vector<int> all_small(P.small_list);
    all_small.insert(all_small.end(), P.persist_list.begin(), P.persist_list.end());
    all_small.insert(all_small.end(), P.tiny_list.begin(), P.tiny_list.end());
    for (int s : all_small) {
      int f = super[s], w = super[s + 1] - f;
      int64_t m = rowptr[s + 1] - rowptr[s];
      double fl = 0, by = 0;
      for (int q = prunePtr[s]; q < prunePtr[s + 1]; ++q) {
        int d = pruneSet[q];
        const int *b = Ls + rowptr[d], *e = Ls + rowptr[d + 1];
        int64_t lb = std::lower_bound(b, e, f) - b, ub = std::lower_bound(b, e, f + w) - b;
        int64_t nr = (e - b) - lb, n1 = ub - lb;
        int wd = super[d + 1] - super[d];
        fl += 2.0 * (n1 * nr - n1 * (n1 - 1) / 2) * wd;
        by += 8.0 * nr * wd;
      }
      fl += (double)w * w * w / 3.0 + (double)(m - w) * w * w;
      by += 16.0 * m * w + 12.0 * (c[f + w] - c[f]);
      K.flops[K_SMALL] += fl;
      K.bytes[K_SMALL] += by;
    }
    for (const int4 &t : P.syrk_tasks) {
      int s = t.x, w = super[s + 1] - super[s];
      int64_t m = rowptr[s + 1] - rowptr[s];
      int nrow = (int)std::min<int64_t>(TB, m - t.y), ncol = std::min(TB, w - t.z);
      const int kc = P.syrk_pairs[t.w].kk >> 16;
      K.flops[K_SYRK] += 2.0 * nrow * ncol * kc;
      K.bytes[K_SYRK] += 8.0 * (2.0 * nrow * ncol + (nrow + ncol) * kc);
    }
    // dense factorization of the tiled class: POTRF + TRSM per column block
    for (int lv = 0; lv < nlev; ++lv)
      for (int s : by_level[lv]) {
        int w = super[s + 1] - super[s];
        int64_t m = rowptr[s + 1] - rowptr[s];
        if (small_class(w, m, T)) continue;
        for (int c0 = 0; c0 < w; c0 += TB) {
          int bw = std::min(TB, w - c0);
          K.flops[K_PANEL] += (double)bw * bw * bw / 3.0 + (double)(m - c0 - bw) * bw * bw;
          K.bytes[K_PANEL] += 16.0 * (m - c0) * bw;
        }
        // each entry of A in the supernode's columns: row index and value read, one value of
        // the panel written (the rest of the panel is zeroed by the memset)
        K.bytes[K_ASSEMBLE] += 20.0 * (c[super[s + 1]] - c[super[s]]);
      }
    if (!P.dense_tasks.empty()) {   // one launch does the trailing updates too: one class
      K.flops[K_PANEL] += K.flops[K_SYRK];
      K.bytes[K_PANEL] += K.bytes[K_SYRK];
      K.flops[K_SYRK] = K.bytes[K_SYRK] = 0.0;
    }
  }
  H.dinv_off.assign(supNo, -1);
  H.ndinv = 0;
  for (int s : P.big_list) {
    H.dinv_off[s] = (int)H.ndinv;
    H.ndinv += (super[s + 1] - super[s] + TB - 1) / TB;
  }
  H.super = std::move(super);
  H.rowptr = std::move(rowptr);
  H.xptr = std::move(xptr);
  H.nls = nls;
  H.xsize = xsize;
  H.nnz = nnz;
  H.nprune = nprune;
  H.upd_lbub.resize(nprune);
  for (int t = 0; t < supNo; ++t)
    for (int q = prunePtr[t]; q < prunePtr[t + 1]; ++q) {
      const int d = pruneSet[q], wd = H.super[d + 1] - H.super[d];
      const int *b = Ls + H.rowptr[d] + wd, *e = Ls + H.rowptr[d + 1];
      const int lb = (int)(std::lower_bound(b, e, H.super[t]) - b) + wd;
      const int ub = (int)(std::lower_bound(b, e, H.super[t + 1]) - b) + wd;
      H.upd_lbub[q] = make_int2(lb, ub);
    }
  return true;
}

bool check_scatter_plan(int n, const int *Ls, const HostSym &H, const Plan &P, const Tuning &T,
                        std::string &err) {
  if (P.sc_coff.empty()) return true;
  const std::vector<int> &super = H.super;
  const int ns = (int)super.size() - 1;
  std::vector<int> col2sup(n), level(ns, 0), wave_of(ns, -1);
  for (int s = 0; s < ns; ++s)
    for (int j = super[s]; j < super[s + 1]; ++j) col2sup[j] = s;
  for (int s = 0; s < ns; ++s) {
    const int w = super[s + 1] - super[s];
    if (H.rowptr[s + 1] - H.rowptr[s] > w)
      level[col2sup[Ls[H.rowptr[s] + w]]] = std::max(level[col2sup[Ls[H.rowptr[s] + w]]], level[s] + 1);
  }
  std::vector<char> tiled(ns, 0);
  for (size_t lv = 0; lv < P.waves.size(); ++lv)
    for (int k = P.waves[lv].big_off; k < P.waves[lv].big_off + P.waves[lv].big_cnt; ++k) {
      tiled[P.big_list[k]] = 1;
      wave_of[P.big_list[k]] = (int)lv;
    }
  auto fail = [&](const std::string &what, long long a, long long b) {
    err = "scatter plan check: " + what + " (" + std::to_string(a) + ", " + std::to_string(b) + ")";
    return false;
  };
  // 1. per descendant: the column table and the relative indices address, for every entry
  //    (i, j), i >= j, from its first row with a tiled-class target, the entry of L a direct
  //    lookup finds (rs[pos] == rd[i] in the target's sorted row list identifies it)
  std::vector<int> first(ns, -1);
  for (int d = 0; d < ns; ++d) {
    const int wd = super[d + 1] - super[d];
    const int md = (int)(H.rowptr[d + 1] - H.rowptr[d]);
    const int *rd = Ls + H.rowptr[d];
    int c0 = wd;
    while (c0 < md && !tiled[col2sup[rd[c0]]]) ++c0;
    if (c0 == md) continue;
    first[d] = c0;
    for (int j = c0; j < md; ++j) {
      const int s = col2sup[rd[j]];
      const int64_t base = P.sc_base[P.sc_coff[d] + j];
      if (!tiled[s]) {
        if (base != -1) return fail("small-class target with an address, descendant/column", d, j);
        continue;
      }
      const int ms = (int)(H.rowptr[s + 1] - H.rowptr[s]);
      if (base != H.xptr[s] + (int64_t)(rd[j] - super[s]) * ms)
        return fail("column address, descendant/column", d, j);
      const int *rs = Ls + H.rowptr[s];
      const int64_t rel = P.sc_rel[P.sc_coff[d] + j];
      for (int i = j; i < md; ++i) {
        const int pos = P.sc_relidx[rel + i];
        if (pos < 0 || pos >= ms || rs[pos] != rd[i]) return fail("relative index, descendant/row", d, i);
      }
    }
  }
  // 2. every descendant with a tiled-class target is handled once, in the level after its
  //    own: by one CUDA-core task, or by tiles whose K ranges cover its width exactly once
  //    for every 128 x 128 block of its lower triangle from that first row
  std::vector<int> nsmall(ns, 0);
  std::vector<std::vector<const ScTile *>> tiles_of(ns);
  for (size_t lv = 0; lv < P.waves.size(); ++lv) {
    const Wave &W = P.waves[lv];
    for (int q = W.scs_off; q < W.scs_off + W.scs_cnt; ++q) {
      const int d = P.sc_small[q].x;
      if (level[d] + 1 != (int)lv || P.sc_small[q].y != first[d])
        return fail("CUDA-core task level or first row, descendant/level", d, (long long)lv);
      ++nsmall[d];
    }
    for (int t = W.sc_off; t < W.sc_off + W.sc_cnt; ++t) {
      const ScTile &tl = P.sc_tiles[t];
      if (tl.d < 0 || tl.d >= ns || level[tl.d] + 1 != (int)lv)
        return fail("tile level, tile/level", t, (long long)lv);
      tiles_of[tl.d].push_back(&tl);
    }
  }
  for (int d = 0; d < ns; ++d) {
    const int c0 = first[d];
    const int wd = super[d + 1] - super[d];
    const int md = (int)(H.rowptr[d + 1] - H.rowptr[d]);
    const int nk = (wd + 31) / 32;
    if (c0 < 0) {
      if (nsmall[d] || !tiles_of[d].empty()) return fail("work for a descendant without tiled targets", d, 0);
      continue;
    }
    if (nsmall[d] + (tiles_of[d].empty() ? 0 : 1) != 1) return fail("descendant handled twice or never", d, nsmall[d]);
    if (nsmall[d]) continue;
    const int nb = (md - c0 + 127) / 128;
    std::vector<std::vector<std::pair<int, int>>> kr((size_t)nb * nb);
    for (const ScTile *tl : tiles_of[d]) {
      if (tl->md != md || tl->ncol != 128 || tl->dense || tl->co != P.sc_coff[d] ||
          (tl->i0 - c0) % 128 || (tl->j0 - c0) % 128 || tl->j0 < c0 || tl->j0 > tl->i0 ||
          tl->i0 >= md || tl->k0 % 32 || tl->nk <= 0)
        return fail("tile fields, descendant/row", d, tl->i0);
      kr[(size_t)((tl->i0 - c0) / 128) * nb + (tl->j0 - c0) / 128].push_back({tl->k0 / 32, tl->nk});
    }
    for (int bi = 0; bi < nb; ++bi)
      for (int bj = 0; bj <= bi; ++bj) {
        std::vector<std::pair<int, int>> &v = kr[(size_t)bi * nb + bj];
        std::sort(v.begin(), v.end());
        int at = 0;
        for (const auto &p : v) {
          if (p.first != at) return fail("K ranges of a tile leave a gap or overlap, descendant/block", d, bi);
          at += p.second;
        }
        if (at != nk) return fail("K ranges of a tile do not cover the width, descendant/block", d, bi);
      }
  }
  // 3. trailing updates of the dense steps: for every tiled supernode, column block C and K
  //    block b < C, the rows that receive b tile [C*64 + 64, m) when b = C - 1 (the diagonal
  //    tile gets that block from the diagonal-block kernel) and [C*64, m) otherwise, every
  //    row exactly once, from the tiles of step b's group
  const int G = std::max(1, T.dense_group);
  std::map<std::tuple<int, int, int>, std::vector<std::pair<int, int>>> rows;   // (s, C, b)
  for (size_t lv = 0; lv < P.waves.size(); ++lv) {
    const Wave &W = P.waves[lv];
    for (size_t j = 0; j < W.scd_off.size(); ++j)
      for (int t = W.scd_off[j]; t < W.scd_off[j] + W.scd_cnt[j]; ++t) {
        const ScTile &tl = P.sc_dense[t];
        const int s = tl.d;
        if (s < 0 || s >= ns || !tiled[s] || wave_of[s] != (int)lv) return fail("dense tile's supernode, tile", t, s);
        const int w = super[s + 1] - super[s];
        const int m = (int)(H.rowptr[s + 1] - H.rowptr[s]);
        const int C = tl.j0 / TB;
        const int b0 = tl.k0 / TB, b1 = (std::min(w, tl.k0 + 32 * tl.nk) + TB - 1) / TB;
        if (!tl.dense || tl.md != m || tl.j0 % TB || tl.k0 % TB || tl.ncol != std::min(TB, w - tl.j0) ||
            b1 - 1 != (int)j || C <= (int)j || tl.i0 < tl.j0 || tl.i0 >= m ||
            tl.k0 + 32 * tl.nk < std::min(w, b1 * TB) || b1 - b0 > G)
          return fail("dense tile fields, tile/step", t, (long long)j);
        // the step's next-column tiles (the next TRSM's column, launched on the chain's
        // stream) come first, then the grouped ones (launched beside the next steps)
        if ((t - W.scd_off[j] < W.scd_nc[j]) != (C == (int)j + 1))
          return fail("next-column and grouped dense tiles out of order, tile/step", t, (long long)j);
        for (int b = b0; b < b1; ++b) rows[std::make_tuple(s, C, b)].push_back({tl.i0, std::min(m, tl.i0 + 128)});
      }
  }
  for (int s = 0; s < ns; ++s) {
    if (!tiled[s]) continue;
    const int w = super[s + 1] - super[s];
    const int m = (int)(H.rowptr[s + 1] - H.rowptr[s]);
    for (int C = 1; C * TB < w; ++C)
      for (int b = 0; b < C; ++b) {
        const int lo = b == C - 1 ? C * TB + TB : C * TB;
        auto it = rows.find(std::make_tuple(s, C, b));
        if (lo >= m) {
          if (it != rows.end()) return fail("dense rows below the supernode, supernode/block", s, C);
          continue;
        }
        if (it == rows.end()) return fail("column block misses a K block, supernode/block", s, C);
        std::vector<std::pair<int, int>> &v = it->second;
        std::sort(v.begin(), v.end());
        int at = lo;
        for (const auto &p : v) {
          if (p.first != at) return fail("dense rows leave a gap or overlap, supernode/block", s, C);
          at = p.second;
        }
        if (at != m) return fail("dense rows do not reach the last row, supernode/block", s, C);
        rows.erase(it);
      }
  }
  if (!rows.empty()) return fail("dense tiles outside the lower column blocks", (long long)rows.size(), 0);
  return true;
}

// Per-level task lists of the supernodal solves (no device work).
void build_solve_plan(int n, const int *Ls, const HostSym &H, SolvePlan &SP) {
  const int supNo = (int)H.super.size() - 1;
  const std::vector<int> &super = H.super;
  const std::vector<int64_t> &rowptr = H.rowptr;
  const int64_t nls = H.nls;
  SP = SolvePlan();
  std::vector<int> lev(supNo, 0);
  int nl = 0;
  std::vector<int> col2sup(n);
  for (int s = 0; s < supNo; ++s)
    for (int j = super[s]; j < super[s + 1]; ++j) col2sup[j] = s;
  for (int s = 0; s < supNo; ++s) {
    const int w = super[s + 1] - super[s];
    const int64_t m = rowptr[s + 1] - rowptr[s];
    nl = std::max(nl, lev[s] + 1);
    if (m > w) {
      const int p = col2sup[Ls[rowptr[s] + w]];
      lev[p] = std::max(lev[p], lev[s] + 1);
    }
    SP.max_w = std::max(SP.max_w, w);
  }
  std::vector<std::vector<int>> bylev(nl);
  for (int s = 0; s < supNo; ++s) bylev[lev[s]].push_back(s);
  auto warp_size_ok = [&](int s) {
    const int w = super[s + 1] - super[s];
    const int64_t m = rowptr[s + 1] - rowptr[s];
    return H.dinv_off[s] < 0 && w <= SOLVE_WARP_W && m - w <= SOLVE_WARP_ROWS;
  };
  std::vector<int> warp_level(nl, 0);
  for (int l = 0; l < nl; ++l) {
    int cnt = 0;
    for (int s : bylev[l]) cnt += warp_size_ok(s);
    warp_level[l] = cnt >= SOLVE_WARP_LEVEL_MIN;
  }
  for (int l = 0; l < nl; ++l) {
    SP.level_off.push_back((int)SP.list.size());
    SP.warp_off.push_back((int)SP.warp_list.size());
    SP.chain_off.push_back((int)SP.fchain.size());
    SP.contrib_off.push_back((int)SP.contrib_tasks.size());
    SP.gather_off.push_back((int)SP.gather_tasks.size());
    std::vector<int2> narrow, wide;
    // 128-row tasks of 8 warps for the wide supernodes only when the level has enough of
    // them to fill the GPU; otherwise 32-row tasks of 32 warps (more, shorter CTAs)
    int64_t n128 = 0;
    for (int s : bylev[l]) {
      const int w = super[s + 1] - super[s];
      const int64_t m = rowptr[s + 1] - rowptr[s];
      if (w > SOLVE_NARROW_W && (H.dinv_off[s] >= 0 || !(warp_level[l] && warp_size_ok(s))))
        n128 += (m - w + SOLVE_CONTRIB_WIDE_ROWS - 1) / SOLVE_CONTRIB_WIDE_ROWS;
    }
    const bool wide_level = n128 >= SOLVE_CONTRIB_WIDE_MIN;
    for (int s : bylev[l]) {
      const int w = super[s + 1] - super[s];
      const int m = (int)(rowptr[s + 1] - rowptr[s]);
      if (H.dinv_off[s] >= 0) {   // tiled class: chained solves through the block inverses
        const int nb = (w + TB - 1) / TB;
        for (int k = 0; k < nb; ++k) SP.fchain.push_back(make_int2(s, k));
        for (int k = nb - 1; k >= 0; --k) SP.bchain.push_back(make_int2(s, k));
      } else if (warp_level[l] && warp_size_ok(s)) {
        SP.warp_list.push_back(s);   // its contributions and gathers are done by the warp
        continue;
      } else {
        SP.list.push_back(s);
      }
      if (w > SOLVE_CONTRIB_BIG_W || (w > SOLVE_NARROW_W && !wide_level))
        for (int r0 = w; r0 < m; r0 += SOLVE_CONTRIB_ROWS) SP.contrib_tasks.push_back(make_int2(s, r0));
      else if (w > SOLVE_NARROW_W)
        for (int r0 = w; r0 < m; r0 += SOLVE_CONTRIB_WIDE_ROWS) wide.push_back(make_int2(s, r0));
      else
        for (int r0 = w; r0 < m; r0 += SOLVE_CONTRIB_ROWS) narrow.push_back(make_int2(s, r0));
      if (m > w)
        for (int j0 = 0; j0 < w; j0 += SOLVE_GATHER_COLS) SP.gather_tasks.push_back(make_int2(s, j0));
    }
    SP.contrib_big.push_back((int)SP.contrib_tasks.size() - SP.contrib_off.back());
    SP.contrib_wide.push_back((int)wide.size());
    SP.contrib_tasks.insert(SP.contrib_tasks.end(), wide.begin(), wide.end());
    SP.contrib_tasks.insert(SP.contrib_tasks.end(), narrow.begin(), narrow.end());
  }
  SP.level_off.push_back((int)SP.list.size());
  SP.warp_off.push_back((int)SP.warp_list.size());
  SP.chain_off.push_back((int)SP.fchain.size());
  SP.contrib_off.push_back((int)SP.contrib_tasks.size());
  SP.gather_off.push_back((int)SP.gather_tasks.size());
  SP.contrib_len = nls - n;
  // column contribution lists: off-diagonal row a of supernode d (a >= w_d) feeds column
  // Ls[a] through contribution (rowptr[d] - super[d]) + (a - w_d)
  SP.cptr.assign(n + 1, 0);
  for (int d = 0; d < supNo; ++d) {
    const int w = super[d + 1] - super[d];
    for (int64_t q = rowptr[d] + w; q < rowptr[d + 1]; ++q) SP.cptr[Ls[q] + 1]++;
  }
  for (int j = 0; j < n; ++j) SP.cptr[j + 1] += SP.cptr[j];
  SP.cidx.resize(SP.cptr[n]);
  std::vector<int> fillc(SP.cptr.begin(), SP.cptr.end() - 1);
  for (int d = 0; d < supNo; ++d) {
    const int w = super[d + 1] - super[d];
    for (int64_t q = rowptr[d] + w; q < rowptr[d + 1]; ++q)
      SP.cidx[fillc[Ls[q]]++] = (int)((rowptr[d] - super[d]) + (q - rowptr[d] - w));
  }
}

// The streaming tasks of a solve plan whose supernodes sit in `level` (by_warp: solved by
// one warp, which does its own contributions and gathers): forward contribution tasks cover
// each off-diagonal row once, backward gather tasks each 16-column group once, and the
// per-column contribution lists name each contribution once, under the row it belongs to.
static bool check_solve_tasks(int n, const int *Ls, const HostSym &H, const SolvePlan &SP,
                              const std::vector<int> &level, const std::vector<char> &by_warp,
                              std::string &err) {
  const int supNo = (int)H.super.size() - 1;
  const std::vector<int> &super = H.super;
  const std::vector<int64_t> &rowptr = H.rowptr;
  const int nl = (int)SP.level_off.size() - 1;
  const int64_t clen = SP.contrib_len;
  auto bad = [&](const std::string &m) {
    err = "solve plan: " + m;
    return false;
  };
  std::vector<char> row_done(std::max<int64_t>(clen, 1), 0);
  std::vector<char> col_done(n, 0);
  for (int l = 0; l < nl; ++l) {
    const int t0 = SP.contrib_off[l], t1 = SP.contrib_off[l + 1];
    const int nbig = SP.contrib_big[l], nwide = SP.contrib_wide[l];
    if (nbig < 0 || nwide < 0 || nbig + nwide > t1 - t0) return bad("contribution classes");
    for (int k = t0; k < t1; ++k) {
      const int s = SP.contrib_tasks[k].x, r0 = SP.contrib_tasks[k].y;
      if (s < 0 || s >= supNo || level[s] != l || by_warp[s])
        return bad("contribution task of a supernode not solved by a CTA in its level");
      const int w = super[s + 1] - super[s];
      const int m = (int)(rowptr[s + 1] - rowptr[s]);
      const int span = (k - t0 >= nbig && k - t0 < nbig + nwide) ? SOLVE_CONTRIB_WIDE_ROWS
                                                                 : SOLVE_CONTRIB_ROWS;
      if (r0 < w || r0 >= m || (r0 - w) % span != 0) return bad("contribution rows misaligned");
      for (int a = r0; a < std::min(m, r0 + span); ++a) {
        const int64_t idx = (rowptr[s] - super[s]) + (a - w);
        if (row_done[idx]) return bad("an off-diagonal row in two contribution tasks");
        row_done[idx] = 1;
      }
    }
    for (int k = SP.gather_off[l]; k < SP.gather_off[l + 1]; ++k) {
      const int s = SP.gather_tasks[k].x, j0 = SP.gather_tasks[k].y;
      if (s < 0 || s >= supNo || level[s] != l || by_warp[s])
        return bad("gather task of a supernode not solved by a CTA in its level");
      const int w = super[s + 1] - super[s];
      if (rowptr[s + 1] - rowptr[s] == w || j0 < 0 || j0 >= w || j0 % SOLVE_GATHER_COLS != 0)
        return bad("gather columns misaligned");
      if (col_done[super[s] + j0]) return bad("a column group in two gather tasks");
      col_done[super[s] + j0] = 1;
    }
  }
  // coverage, and the contribution lists: row of each contribution
  std::vector<int> row_of(std::max<int64_t>(clen, 1), -1);
  for (int s = 0; s < supNo; ++s) {
    const int w = super[s + 1] - super[s];
    const int m = (int)(rowptr[s + 1] - rowptr[s]);
    for (int a = w; a < m; ++a) {
      const int64_t idx = (rowptr[s] - super[s]) + (a - w);
      row_of[idx] = Ls[rowptr[s] + a];
      if (!by_warp[s] && !row_done[idx]) return bad("an off-diagonal row in no contribution task");
    }
    if (by_warp[s] || m == w) continue;
    for (int j0 = 0; j0 < w; j0 += SOLVE_GATHER_COLS)
      if (!col_done[super[s] + j0]) return bad("a column group in no gather task");
  }
  if ((int64_t)SP.cptr.size() != n + 1 || SP.cptr[0] != 0 || SP.cptr[n] != clen ||
      (int64_t)SP.cidx.size() != clen)
    return bad("contribution lists of the wrong size");
  std::fill(row_done.begin(), row_done.end(), 0);
  for (int j = 0; j < n; ++j) {
    if (SP.cptr[j + 1] < SP.cptr[j]) return bad("contribution list pointers decrease");
    for (int q = SP.cptr[j]; q < SP.cptr[j + 1]; ++q) {
      const int idx = SP.cidx[q];
      if (idx < 0 || idx >= clen || row_done[idx] || row_of[idx] != j)
        return bad("column " + std::to_string(j) + "'s contribution list");
      row_done[idx] = 1;
    }
  }
  return true;
}

bool check_solve_plan(int n, const int *Ls, const HostSym &H, const SolvePlan &SP,
                      std::string &err) {
  const int supNo = (int)H.super.size() - 1;
  const std::vector<int> &super = H.super;
  const std::vector<int64_t> &rowptr = H.rowptr;
  const int nl = (int)SP.level_off.size() - 1;
  auto bad = [&](const std::string &m) {
    err = "solve plan: " + m;
    return false;
  };
  if (nl < 0 || (int)SP.warp_off.size() != nl + 1 || (int)SP.chain_off.size() != nl + 1 ||
      (int)SP.contrib_off.size() != nl + 1 || (int)SP.gather_off.size() != nl + 1 ||
      (int)SP.contrib_big.size() != nl || (int)SP.contrib_wide.size() != nl ||
      SP.fchain.size() != SP.bchain.size())
    return bad("per-level offsets of unequal length");
  if (SP.contrib_len != H.nls - n) return bad("contribution length");
  // every supernode in exactly one level, by exactly one kind of task
  std::vector<int> level(supNo, -1);
  std::vector<char> by_warp(supNo, 0);
  auto place = [&](int s, int l) {
    if (s < 0 || s >= supNo) return false;
    if (level[s] >= 0 && level[s] != l) return false;
    level[s] = l;
    return true;
  };
  for (int l = 0; l < nl; ++l) {
    for (int k = SP.level_off[l]; k < SP.level_off[l + 1]; ++k) {
      const int s = SP.list[k];
      if (!place(s, l) || H.dinv_off[s] >= 0) return bad("small supernode misplaced");
    }
    for (int k = SP.warp_off[l]; k < SP.warp_off[l + 1]; ++k) {
      const int s = SP.warp_list[k];
      if (!place(s, l) || H.dinv_off[s] >= 0) return bad("warp supernode misplaced");
      const int w = super[s + 1] - super[s];
      if (w > SOLVE_WARP_W || rowptr[s + 1] - rowptr[s] - w > SOLVE_WARP_ROWS)
        return bad("supernode too large for one warp");
      by_warp[s] = 1;
    }
    // chained blocks: one per 64 columns, forward increasing, backward decreasing
    const int c0 = SP.chain_off[l], c1 = SP.chain_off[l + 1];
    for (int k = c0; k < c1;) {
      const int s = SP.fchain[k].x;
      if (!place(s, l) || H.dinv_off[s] < 0) return bad("chained supernode misplaced");
      const int nb = (super[s + 1] - super[s] + TB - 1) / TB;
      if (k + nb > c1) return bad("chain cut short");
      for (int b = 0; b < nb; ++b)
        if (SP.fchain[k + b].x != s || SP.fchain[k + b].y != b ||
            SP.bchain[k + b].x != s || SP.bchain[k + b].y != nb - 1 - b)
          return bad("chain blocks out of order");
      k += nb;
    }
  }
  std::vector<int> col2sup(n);
  for (int s = 0; s < supNo; ++s)
    for (int j = super[s]; j < super[s + 1]; ++j) col2sup[j] = s;
  std::vector<int> seen(supNo, 0);
  for (int l = 0; l < nl; ++l) {
    for (int k = SP.level_off[l]; k < SP.level_off[l + 1]; ++k) seen[SP.list[k]]++;
    for (int k = SP.warp_off[l]; k < SP.warp_off[l + 1]; ++k) seen[SP.warp_list[k]]++;
    for (int k = SP.chain_off[l]; k < SP.chain_off[l + 1]; ++k)
      if (SP.fchain[k].y == 0) seen[SP.fchain[k].x]++;
  }
  for (int s = 0; s < supNo; ++s) {
    if (seen[s] != 1) return bad("supernode " + std::to_string(s) + " solved " +
                                 std::to_string(seen[s]) + " times");
    const int w = super[s + 1] - super[s];
    if (rowptr[s + 1] - rowptr[s] > w) {
      const int p = col2sup[Ls[rowptr[s] + w]];   // the parent: first off-diagonal row's
      if (level[p] <= level[s]) return bad("a parent not in a later level");
    }
  }
  return check_solve_tasks(n, Ls, H, SP, level, by_warp, err);
}

bool Engine::analyze(int n, const int *c, const int *r, const int64_t *lC, const int *Ls,
                     const int64_t *Li_ptr, const int *blockSet, int supNo,
                     const int *prunePtr, const int *pruneSet, std::string &err) {
  cudaSetDevice(device_);
  if (!kernels_configure(err) || !update_tc_configure(err) || !scatter_tc_configure(err))
    return false;
  HostSym H;
  Plan P;
  if (!build_plan(n, c, r, lC, Ls, Li_ptr, blockSet, supNo, prunePtr, pruneSet, H, P, err,
                  tuning_))
    return false;
  const std::vector<int> &super = H.super;
  const std::vector<int64_t> &rowptr = H.rowptr, &xptr = H.xptr;
  const int64_t nls = H.nls, xsize = H.xsize, nnz = H.nnz;
  const int nprune = H.nprune;

  // ---- solve plan: levels of the supernodal etree, per-level task lists ----
  SolvePlan SP;
  build_solve_plan(n, Ls, H, SP);
  if (!solve_configure(SP.max_w, err)) return false;
  // ---- full CSR of the symmetric matrix for residuals: entry -> index into A2 values ----
  std::vector<int> csr_rp(n + 1, 0), csr_ci, csr_map;
  {
    for (int j = 0; j < n; ++j)
      for (int p = c[j]; p < c[j + 1]; ++p) {
        csr_rp[r[p] + 1]++;
        if (r[p] != j) csr_rp[j + 1]++;
      }
    for (int i = 0; i < n; ++i) csr_rp[i + 1] += csr_rp[i];
    csr_ci.resize(csr_rp[n]);
    csr_map.resize(csr_rp[n]);
    std::vector<int> fill(csr_rp.begin(), csr_rp.end() - 1);
    for (int j = 0; j < n; ++j)
      for (int p = c[j]; p < c[j + 1]; ++p) {
        const int i = r[p];
        csr_ci[fill[i]] = j;
        csr_map[fill[i]++] = p;
        if (i != j) {
          csr_ci[fill[j]] = i;
          csr_map[fill[j]++] = p;
        }
      }
  }

  // ---- upload ----
  release();
  cudaStream_t st = stream_;
  std::vector<int64_t> rp(rowptr);
  bool ok = upload(d_super_, super.data(), super.size(), st, err) &&
            upload(d_rowptr_, rp.data(), rp.size(), st, err) &&
            upload(d_Ls_, Ls, (size_t)nls, st, err) &&
            upload(d_xptr_, xptr.data(), xptr.size(), st, err) &&
            upload(d_Ap_, c, (size_t)n + 1, st, err) &&
            upload(d_Ai_, r, (size_t)nnz, st, err) &&
            upload(d_upd_ptr_, prunePtr, (size_t)supNo + 1, st, err) &&
            upload(d_upd_, pruneSet, (size_t)nprune, st, err) &&
            upload(d_upd_lbub_, H.upd_lbub.data(), H.upd_lbub.size(), st, err) &&
            upload(d_small_, P.small_list.data(), P.small_list.size(), st, err) &&
            upload(d_persist_, P.persist_list.data(), P.persist_list.size(), st, err) &&
            upload(d_tiny_, P.tiny_list.data(), P.tiny_list.size(), st, err) &&
            upload(d_big_, P.big_list.data(), P.big_list.size(), st, err) &&
            upload(d_diag_, P.diag_list.data(), P.diag_list.size(), st, err) &&
            upload(d_asm_, P.asm_tasks.data(), P.asm_tasks.size(), st, err) &&
            upload(d_upd_tasks_, P.upd_tasks.data(), P.upd_tasks.size(), st, err) &&
            upload(d_upd_end_, P.upd_end.data(), P.upd_end.size(), st, err) &&
            upload(d_pairs_, P.upd_pairs.data(), P.upd_pairs.size(), st, err) &&
            upload(d_panel_, P.panel_tasks.data(), P.panel_tasks.size(), st, err) &&
            upload(d_syrk_, P.syrk_tasks.data(), P.syrk_tasks.size(), st, err) &&
            upload(d_syrk_pairs_, P.syrk_pairs.data(), P.syrk_pairs.size(), st, err) &&
            upload(d_syrk_end_, P.syrk_end.data(), P.syrk_end.size(), st, err) &&
            upload(d_tc_pairs_, P.tc_pairs.data(), P.tc_pairs.size(), st, err) &&
            upload(d_sc_tiles_, P.sc_tiles.data(), P.sc_tiles.size(), st, err) &&
            upload(d_sc_small_, P.sc_small.data(), P.sc_small.size(), st, err) &&
            upload(d_sc_dense_, P.sc_dense.data(), P.sc_dense.size(), st, err) &&
            upload(d_sc_base_, P.sc_base.data(), P.sc_base.size(), st, err) &&
            upload(d_sc_coff_, P.sc_coff.data(), P.sc_coff.size(), st, err) &&
            upload(d_sc_rel_, P.sc_rel.data(), P.sc_rel.size(), st, err) &&
            upload(d_sc_relidx_, P.sc_relidx.data(), P.sc_relidx.size(), st, err) &&
            upload(d_dense_tasks_, P.dense_tasks.data(), P.dense_tasks.size(), st, err) &&
            upload(d_dense_toff_, P.dense_toff.data(), P.dense_toff.size(), st, err) &&
            upload(d_dinv_off_, H.dinv_off.data(), H.dinv_off.size(), st, err) &&
            upload(d_slist_, SP.list.data(), SP.list.size(), st, err) &&
            upload(d_swarp_, SP.warp_list.data(), SP.warp_list.size(), st, err) &&
            upload(d_cptr_, SP.cptr.data(), SP.cptr.size(), st, err) &&
            upload(d_cidx_, SP.cidx.data(), SP.cidx.size(), st, err) &&
            upload(d_fchain_, SP.fchain.data(), SP.fchain.size(), st, err) &&
            upload(d_bchain_, SP.bchain.data(), SP.bchain.size(), st, err) &&
            upload(d_scontrib_, SP.contrib_tasks.data(), SP.contrib_tasks.size(), st, err) &&
            upload(d_sgather_, SP.gather_tasks.data(), SP.gather_tasks.size(), st, err) &&
            upload(d_csr_rp_, csr_rp.data(), csr_rp.size(), st, err) &&
            upload(d_csr_ci_, csr_ci.data(), csr_ci.size(), st, err) &&
            upload(d_csr_map_, csr_map.data(), csr_map.size(), st, err);
  if (!ok) return false;
  cudaError_t e = cudaMalloc(&d_Ax_, sizeof(double) * std::max<int64_t>(nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&dL_, sizeof(double) * std::max<int64_t>(xsize, 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_status_, kStatusWords * sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(d_status_, 0, kStatusWords * sizeof(int), st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_status_ + 4, &wait_budget_, sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMalloc(&d_flags_, sizeof(int) * std::max<int64_t>(H.ndinv, 1));
  if (e == cudaSuccess) e = cudaMemsetAsync(d_flags_, 0, sizeof(int) * std::max<int64_t>(H.ndinv, 1), st);
  if (e == cudaSuccess)
    e = cudaMalloc(&d_dinv_, sizeof(double) * TB * TB * std::max<int64_t>(H.ndinv, 1));
  if (e == cudaSuccess)
    e = cudaMalloc(&d_csr_val_, sizeof(double) * std::max<size_t>(csr_ci.size(), 1));
  // queue head of the CTA walk, done flags, queue head of the warp walk
  if (e == cudaSuccess) e = cudaMalloc(&d_qctr_, sizeof(int) * ((size_t)supNo + 2));
  if (e == cudaSuccess && !P.tiny_list.empty()) tiny_ctas_ = tiny_ctas((int)P.tiny_list.size());
  if (e == cudaSuccess && !P.persist_list.empty())
    persist_ctas_ = persist_ctas(P.persist_smem, (int)P.persist_list.size());
  // dense dataflow: one queue head per wave, then the tile version counters
  dense_ver_len_ = (int64_t)P.waves.size() + P.dense_tiles;
  if (e == cudaSuccess && !P.dense_tasks.empty())
    e = cudaMalloc(&d_dense_ver_, sizeof(int) * dense_ver_len_);
  for (Wave &W : P.waves)
    if (W.dense_cnt > 0) W.dense_ctas = dense_ctas(W.dense_cnt);

  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("device allocation: ") + cudaGetErrorString(e);
    return false;
  }
  n_ = n;
  nsuper_ = supNo;
  xsize_ = xsize;
  nnz_ = nnz;
  plan_ = std::move(P);
  splan_ = std::move(SP);
  nflags_ = H.ndinv;
  csr_nnz_ = (int64_t)csr_ci.size();
  sym_.n = n;
  sym_.nsuper = supNo;
  sym_.super = d_super_;
  sym_.rowptr = d_rowptr_;
  sym_.Ls = d_Ls_;
  sym_.xptr = d_xptr_;
  sym_.Ap = d_Ap_;
  sym_.Ai = d_Ai_;
  sym_.Ax = d_Ax_;
  sym_.upd_ptr = d_upd_ptr_;
  sym_.upd = d_upd_;
  sym_.L = dL_;
  sym_.status = d_status_;
  sym_.dinv = d_dinv_;
  sym_.Lf = nullptr;
  sym_.xk = nullptr;
  sym_.dinv_off = d_dinv_off_;
  kmirror_len_ = kmirror_layout(H.super, H.rowptr, h_xk_);
  hsym_ = H;
  h_Ls_.assign(Ls, Ls + nls);

  return true;
}

void Engine::launch_all(std::vector<std::pair<int, cudaEvent_t>> *prof, int prec) {
  // split products on tcgen05: split-TF32 (cp.async or TMA staging) or BF16x3
  const int variant = prec == 2 ? UT_VARIANT_BF16
                                : (tuning_.tc_tma ? UT_VARIANT_TF32_TMA : UT_VARIANT_TF32);
  cudaStream_t st = stream_;
  // mixed modes: right-looking descendant updates through the scatter kernel (tensor maps
  // of the mode's mirror format), unless a tile-owner plan (split-TF32 plans 6, 7) is set
  const bool scatter = prec != 0 && !plan_.sc_coff.empty();
  const bool bf16 = prec == 2;
  void *sc_maps = bf16 ? d_sc_maps16_ : d_sc_maps_;
  // the trailing updates of the dense steps: split dense tiles of the scatter kernel (two
  // SMs left to the concurrent diagonal-block kernel), else FP64
  const bool syrk_tc = scatter && !tuning_.syrk_fp64;
  auto syrk = [&](const Wave &W, int j) {
    if (syrk_tc)
      launch_scatter_tc(sym_, sc_maps, d_sc_dense_ + W.scd_off[j], W.scd_cnt[j], scatter_cols(),
                        2, bf16, st);
    else
      launch_syrk_step(sym_, d_syrk_ + W.syrk_off[j], d_syrk_pairs_, W.syrk_cnt[j], st);
  };
  // With profiling on, every launch is preceded by an event and followed by one.
  auto mark = [&](int kind, int count) {
    if (!prof || count <= 0) return;
    cudaEvent_t ev;
    cudaEventCreate(&ev);
    cudaEventRecord(ev, st);
    prof->emplace_back(kind, ev);
  };
  // right-looking updates: contributions reach a target from the level after each
  // descendant's, so every tiled panel is assembled up front
  const ScatterCols sc_cols = scatter_cols();
  mark(K_MEMSET, 1);
  cudaMemsetAsync(dL_, 0, sizeof(double) * xsize_, st);
  launch_init_status(d_status_, st);
  mark(-1, 1);
  if (scatter && !plan_.asm_tasks.empty()) {
    mark(K_ASSEMBLE, 1);
    launch_assemble(sym_, d_asm_, (int)plan_.asm_tasks.size(), st);
    mark(-1, 1);
  }
  if (!plan_.tiny_list.empty() || !plan_.persist_list.empty())
    cudaMemsetAsync(d_qctr_, 0, sizeof(int) * (nsuper_ + 2), st);
  if (d_dense_ver_) cudaMemsetAsync(d_dense_ver_, 0, sizeof(int) * dense_ver_len_, st);
  if (!plan_.tiny_list.empty()) {
    mark(K_SMALL, 1);
    launch_factor_tiny_persist(sym_, d_upd_lbub_, d_tiny_, (int)plan_.tiny_list.size(), tiny_ctas_,
                               d_qctr_,
                               d_qctr_ + 1 + nsuper_, st);
    mark(-1, 1);
  }
  if (!plan_.persist_list.empty()) {
    mark(K_SMALL, 1);
    launch_factor_small_persist(sym_, d_upd_lbub_, d_persist_, (int)plan_.persist_list.size(),
                                plan_.persist_smem, persist_ctas_, d_qctr_, st);
    mark(-1, 1);
  }
  for (const Wave &W : plan_.waves) {
    // the wave's small supernodes read only earlier waves' panels and write only their own,
    // so they run beside the wave's tiled work (updates and dense steps) on a second
    // stream, joined before the next wave (whose updates and supernodes read them)
    const bool side = !prof && W.small_cnt > 0 && W.big_cnt > 0;
    if (side) {
      cudaEventRecord(ev_sfork_, st);
      cudaStreamWaitEvent(small_stream_, ev_sfork_, 0);
      launch_factor_small(sym_, d_upd_lbub_, d_small_ + W.small_off, W.small_cnt, W.small_smem,
                          small_stream_);
      cudaEventRecord(ev_sjoin_, small_stream_);
    } else {
      mark(K_SMALL, W.small_cnt);
      launch_factor_small(sym_, d_upd_lbub_, d_small_ + W.small_off, W.small_cnt, W.small_smem, st);
      mark(-1, W.small_cnt);
    }
    if (scatter) {
      mark(K_UPDATE, W.scs_cnt);
      launch_scatter_small(sym_, d_sc_small_ + W.scs_off, W.scs_cnt, sc_cols, st);
      mark(-1, W.scs_cnt);
      mark(K_UPDATE, W.sc_cnt);
      launch_scatter_tc(sym_, sc_maps, d_sc_tiles_ + W.sc_off, W.sc_cnt, sc_cols, 0, bf16, st);
      mark(-1, W.sc_cnt);
    } else {
    mark(K_ASSEMBLE, W.asm_cnt);
    launch_assemble(sym_, d_asm_ + W.asm_off, W.asm_cnt, st);
    mark(-1, W.asm_cnt);
    mark(K_UPDATE, W.upd_cnt);
    if (prec != 0)
      launch_update_tc(sym_, d_tmaps_, d_upd_tasks_ + W.upd_off, d_upd_end_ + W.upd_off,
                       d_tc_pairs_, W.upd_cnt, variant, false, st);
    else
      launch_update_tiles(sym_, d_upd_tasks_ + W.upd_off, d_upd_end_ + W.upd_off, d_pairs_,
                          W.upd_cnt, st);
    mark(-1, W.upd_cnt);
    }
    if (W.dense_cnt > 0) {
      // the whole dense factorization of the wave in one dataflow launch
      mark(K_PANEL, 1);
      const int wave = (int)(&W - plan_.waves.data());
      launch_dense_persist(sym_, d_dense_tasks_ + W.dense_off, W.dense_cnt, W.dense_ctas,
                           d_dense_toff_, d_dense_ver_ + plan_.waves.size(), d_dense_ver_ + wave,
                           st);
      mark(-1, 1);
      if (side) cudaStreamWaitEvent(st, ev_sjoin_, 0);
      continue;
    }
    mark(K_PANEL, W.big_cnt);
    launch_diag_step(sym_, d_big_ + W.big_off, W.big_cnt, 0, st);
    mark(-1, W.big_cnt);
    for (size_t j = 0; j < W.panel_off.size(); ++j) {
      mark(K_PANEL, W.panel_cnt[j]);
      launch_trsm_step(sym_, d_panel_ + W.panel_off[j], W.panel_cnt[j], (int)j, st);
      mark(-1, W.panel_cnt[j]);
      if (syrk_tc && !prof) {
        // look-ahead: the step's trailing update split in two.  Column block j+1 (the next
        // TRSM reads it) on this stream; the grouped updates of the later columns on a third
        // stream, where they may run on beside the next TRSM: only the diagonal block two
        // steps on (the next iteration's diagonal-block launch) waits for them
        cudaEventRecord(ev_fork_, st);
        if (W.diag_cnt[j] > 0) {
          cudaStreamWaitEvent(aux_stream_, ev_fork_, 0);
          if (j > 0) cudaStreamWaitEvent(aux_stream_, ev_grp_[(j - 1) & 1], 0);
          launch_diag_step(sym_, d_diag_ + W.diag_off[j], W.diag_cnt[j], (int)j + 1, aux_stream_);
          cudaEventRecord(ev_join_, aux_stream_);
        }
        const int nc = W.scd_nc[j];
        cudaStreamWaitEvent(grp_stream_, ev_fork_, 0);
        launch_scatter_tc(sym_, sc_maps, d_sc_dense_ + W.scd_off[j] + nc, W.scd_cnt[j] - nc,
                          scatter_cols(), tuning_.grouped_reserve, bf16, grp_stream_);
        cudaEventRecord(ev_grp_[j & 1], grp_stream_);
        launch_scatter_tc(sym_, sc_maps, d_sc_dense_ + W.scd_off[j], nc, scatter_cols(), 2, bf16, st);
        if (W.diag_cnt[j] > 0) cudaStreamWaitEvent(st, ev_join_, 0);
        if (j + 1 == W.panel_off.size()) cudaStreamWaitEvent(st, ev_grp_[j & 1], 0);
      } else if (prof) {
        // profiled runs keep one stream so every launch is bracketed by its own events
        mark(K_PANEL, W.diag_cnt[j]);
        launch_diag_step(sym_, d_diag_ + W.diag_off[j], W.diag_cnt[j], (int)j + 1, st);
        mark(-1, W.diag_cnt[j]);
        mark(K_SYRK, W.syrk_cnt[j]);
        syrk(W, (int)j);
        mark(-1, W.syrk_cnt[j]);
      } else if (W.diag_cnt[j] > 0) {
        // fork: next diagonal block on the auxiliary stream, trailing update here; join
        cudaEventRecord(ev_fork_, st);
        cudaStreamWaitEvent(aux_stream_, ev_fork_, 0);
        launch_diag_step(sym_, d_diag_ + W.diag_off[j], W.diag_cnt[j], (int)j + 1, aux_stream_);
        cudaEventRecord(ev_join_, aux_stream_);
        syrk(W, (int)j);
        cudaStreamWaitEvent(st, ev_join_, 0);
      } else {
        syrk(W, (int)j);
      }
    }
    if (side) cudaStreamWaitEvent(st, ev_sjoin_, 0);
  }
}

bool Engine::set_mode(int prec, std::string &err) {
  if (prec != 0 && !d_Lk_) {   // the K-major split mirror, its format arrays, tensor maps
    const size_t mb = tensor_map_bytes() * (size_t)nsuper_;
    const size_t nx = h_xk_.size();   // nsuper + 1: offsets, then the format entry
    std::vector<unsigned char> maps(mb);
    std::vector<int64_t> xk16(h_xk_);
    xk16[nx - 1] = 1;
    cudaError_t e = cudaMalloc(&d_Lk_, sizeof(float) * std::max<int64_t>(kmirror_len_, 8));
    if (e == cudaSuccess) e = cudaMalloc(&d_xk_, sizeof(int64_t) * nx);
    if (e == cudaSuccess) e = cudaMalloc(&d_xk16_, sizeof(int64_t) * nx);
    if (e == cudaSuccess) e = cudaMalloc(&d_tmaps_, std::max<size_t>(mb, 128));
    if (e != cudaSuccess) {
      err = std::string("mirror allocation: ") + cudaGetErrorString(e);
      return false;
    }
    if (!build_tensor_maps(hsym_.super, hsym_.rowptr, h_xk_, d_Lk_, maps.data(), err)) return false;
    for (int f = 0; f < 2 && !plan_.sc_coff.empty(); ++f) {
      // plane maps of the right-looking update tiles, split-TF32 (f = 0) and BF16x3 layouts
      std::vector<unsigned char> sm(tensor_map_bytes() * scatter_maps_count(nsuper_, f == 1), 0);
      if (!build_scatter_maps(hsym_.super, hsym_.rowptr, h_xk_, plan_.sc_used, d_Lk_, f == 1,
                              sm.data(), err))
        return false;
      void *&dst = f ? d_sc_maps16_ : d_sc_maps_;
      e = cudaMalloc(&dst, sm.size());
      if (e == cudaSuccess) e = cudaMemcpy(dst, sm.data(), sm.size(), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        err = std::string("scatter tensor maps: ") + cudaGetErrorString(e);
        return false;
      }
    }
    e = cudaMemcpy(d_xk_, h_xk_.data(), sizeof(int64_t) * nx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_xk16_, xk16.data(), sizeof(int64_t) * nx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_tmaps_, maps.data(), mb, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      err = std::string("mirror set-up: ") + cudaGetErrorString(e);
      return false;
    }
  }
  sym_.Lf = prec != 0 ? reinterpret_cast<float2 *>(d_Lk_) : nullptr;
  sym_.xk = prec == 2 ? d_xk16_ : prec == 1 ? d_xk_ : nullptr;
  return true;
}

int Engine::factor(const double *values, bool values_on_device, int *info, std::string &err,
                   int prec) {
  if (prec < 0 || prec > 2) { err = "unknown precision mode"; return -1; }
  if (!dL_) { err = "factor before analyze"; return -1; }
  cudaSetDevice(device_);
  if (!set_mode(prec, err)) return -1;
  cudaStream_t st = stream_;
  // values always reach the kernels through d_Ax_, so a captured graph stays valid
  cudaError_t e = cudaMemcpyAsync(d_Ax_, values, sizeof(double) * nnz_,
                                  values_on_device ? cudaMemcpyDeviceToDevice
                                                   : cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) { err = std::string("values upload: ") + cudaGetErrorString(e); return -1; }
  h2d_bytes_ = values_on_device ? 0 : (int64_t)sizeof(double) * nnz_;
  if (use_graph_) {
    // The whole launch sequence is fixed by the structure (and the mode): capture it once
    // per mode, replay it.
    cudaGraph_t &g = graph_[prec];
    cudaGraphExec_t &ge = graph_exec_[prec];
    if (!ge) {
      e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        launch_all(nullptr, prec);
        e = cudaStreamEndCapture(st, &g);
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
      if (e != cudaSuccess) { err = std::string("graph capture: ") + cudaGetErrorString(e); return -1; }
    }
    e = cudaGraphLaunch(ge, st);
    if (e != cudaSuccess) { err = std::string("graph launch: ") + cudaGetErrorString(e); return -1; }
  } else {
    launch_all(nullptr, prec);
  }
  return finish(info, err);
}

int Engine::factor_profiled(const double *values, bool values_on_device, int *info,
                            KernelStats &out, std::string &err, int prec) {
  if (prec < 0 || prec > 2) { err = "unknown precision mode"; return -1; }
  if (!dL_) { err = "factor before analyze"; return -1; }
  cudaSetDevice(device_);
  if (!set_mode(prec, err)) return -1;
  cudaStream_t st = stream_;
  cudaError_t e = cudaMemcpyAsync(d_Ax_, values, sizeof(double) * nnz_,
                                  values_on_device ? cudaMemcpyDeviceToDevice
                                                   : cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) { err = std::string("values upload: ") + cudaGetErrorString(e); return -1; }
  std::vector<std::pair<int, cudaEvent_t>> prof;
  launch_all(&prof, prec);
  int rc = finish(info, err);
  out = plan_.work;
  for (int k = 0; k < K_NKINDS; ++k) { out.launches[k] = 0; out.ms[k] = 0; }
  for (size_t i = 0; i + 1 < prof.size(); i += 2) {
    float ms = 0;
    cudaEventElapsedTime(&ms, prof[i].second, prof[i + 1].second);
    int k = prof[i].first;
    out.launches[k] += 1;
    out.ms[k] += ms;
  }
  for (auto &pe : prof) cudaEventDestroy(pe.second);
  return rc;
}

int Engine::finish(int *info, std::string &err) {
  cudaStream_t st = stream_;
  // full-CSR values of this matrix for residuals, and ||A||_inf
  launch_gather_vals((int)csr_nnz_, d_csr_map_, d_Ax_, d_csr_val_, st);
  cudaError_t e = cudaMemcpyAsync(h_status_, d_status_, 4 * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) { err = std::string("factor: ") + cudaGetErrorString(e); return -1; }
  if (h_status_[1]) { err = "symbolic structure inconsistent with the matrix pattern"; return -2; }
  if (h_status_[3]) {
    err = "timeout: a persistent walk of the factorization waited longer than its budget "
          "(descendant supernode or dense tile)";
    return -3;
  }
  if (h_status_[0] != INT_MAX) {
    if (info) *info = h_status_[0];
    err = "matrix is not positive definite";
    return 1;
  }
  if (info) *info = 0;
  return 0;
}

bool Engine::download(double *lValues, bool to_device, std::string &err) {
  if (!dL_) { err = "download before factor"; return false; }
  cudaSetDevice(device_);
  cudaError_t e = cudaMemcpyAsync(lValues, dL_, sizeof(double) * xsize_,
                                  to_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  stream_);
  d2h_bytes_ = to_device ? 0 : (int64_t)sizeof(double) * xsize_;
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) { err = std::string("download: ") + cudaGetErrorString(e); return false; }
  return true;
}

bool Engine::set_wait_budget(long long polls, std::string &err) {
  wait_budget_ = polls < 0 ? kDefaultWaitBudget : (int)std::min<long long>(polls, INT_MAX);
  if (!d_status_) return true;   // written at the next analyze
  cudaSetDevice(device_);
  cudaError_t e = cudaMemcpyAsync(d_status_ + 4, &wait_budget_, sizeof(int),
                                  cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) { err = std::string("wait budget: ") + cudaGetErrorString(e); return false; }
  return true;
}

double *Engine::staging(size_t doubles, std::string &err) {
  cudaSetDevice(device_);
  if (doubles > stage_len_) {
    if (d_stage_) cudaFree(d_stage_);
    d_stage_ = nullptr;
    stage_len_ = 0;
    cudaError_t e = cudaMalloc(&d_stage_, sizeof(double) * doubles);
    if (e != cudaSuccess) {
      d_stage_ = nullptr;
      err = std::string("staging buffer: ") + cudaGetErrorString(e);
      return nullptr;
    }
    stage_len_ = doubles;
  }
  return d_stage_;
}

bool Engine::ensure_work(int nrhs, std::string &err) {
  if (nrhs <= work_nrhs_) return true;
  release_solve_graphs();   // they hold the old buffers
  if (d_sx_) cudaFree(d_sx_);
  d_sx_ = nullptr;
  if (d_contrib_) cudaFree(d_contrib_);
  if (d_work_) cudaFree(d_work_);
  if (d_norms_) cudaFree(d_norms_);
  if (h_norms_) cudaFreeHost(h_norms_);
  if (d_npart_) cudaFree(d_npart_);
  d_contrib_ = d_work_ = d_norms_ = h_norms_ = d_npart_ = nullptr;
  cudaError_t e = cudaMalloc(&d_contrib_, sizeof(double) * std::max<int64_t>(splan_.contrib_len, 1) * nrhs);
  // work: r, d, p, q vectors (4 * n * nrhs) + row sums
  if (e == cudaSuccess) e = cudaMalloc(&d_work_, sizeof(double) * ((size_t)4 * n_ * nrhs + n_));
  if (e == cudaSuccess) e = cudaMalloc(&d_norms_, sizeof(double) * 8 * (nrhs + 1));
  if (e == cudaSuccess) e = cudaMallocHost(&h_norms_, sizeof(double) * 8 * (nrhs + 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_npart_, sizeof(double) * norm_scratch_doubles(nrhs));
  if (e == cudaSuccess) e = cudaMalloc(&d_sx_, sizeof(double) * (size_t)n_ * nrhs);
  if (e != cudaSuccess) {
    err = std::string("solve workspace: ") + cudaGetErrorString(e);
    work_nrhs_ = 0;
    return false;
  }
  work_nrhs_ = nrhs;
  return true;
}

void Engine::release_solve_graphs() {
  for (auto &g : solve_graphs_) cudaGraphExecDestroy(g.second);
  solve_graphs_.clear();
}

// The solve of nrhs right-hand sides held in d_sx_ as one CUDA graph (its launch sequence
// and buffers are fixed by the structure and nrhs); captured on first use, nullptr when the
// capture fails (the caller then launches directly).
cudaGraphExec_t Engine::solve_graph(int nrhs) {
  for (auto &g : solve_graphs_)
    if (g.first == nrhs) return g.second;
  cudaStream_t st = stream_;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return nullptr;
  run_solve_with(d_sx_, nrhs, d_contrib_);
  cudaError_t e = cudaStreamEndCapture(st, &graph);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  solve_graphs_.emplace_back(nrhs, exec);
  return exec;
}

// x := (L L^T)^{-1} x for device x (n x nrhs): the solve graph on a copy of x in d_sx_,
// or direct launches without graphs.
void Engine::run_solve(double *x, int nrhs) {
  cudaGraphExec_t g = use_graph_ ? solve_graph(nrhs) : nullptr;
  if (!g) {
    run_solve_with(x, nrhs, d_contrib_);
    return;
  }
  const size_t bytes = sizeof(double) * (size_t)n_ * nrhs;
  cudaMemcpyAsync(d_sx_, x, bytes, cudaMemcpyDeviceToDevice, stream_);
  cudaGraphLaunch(g, stream_);
  cudaMemcpyAsync(x, d_sx_, bytes, cudaMemcpyDeviceToDevice, stream_);
}

// Forward then backward supernodal solve, level by level, with the contribution scratch
// `contrib` (one double per off-diagonal row of L per right-hand side).  The chained blocks'
// counters are cleared first and every block takes part in every pass, in the order
// forward r = 0 .. nrhs - 1, then backward r = 0 .. nrhs - 1, so the pass numbers (epochs
// r + 1 forward, nrhs + r + 1 backward) are the same in every solve and a graph of this
// sequence can be replayed.
void Engine::run_solve_with(double *x, int nrhs, double *contrib) {
  cudaStream_t st = stream_;
  const SolvePlan &SP = splan_;
  const int nl = (int)SP.level_off.size() - 1;
  const int smem = (int)sizeof(double) * std::max(SP.max_w, 1);
  const int64_t cs = std::max<int64_t>(SP.contrib_len, 1);
  const int base = 0;
  cudaMemsetAsync(d_flags_, 0, sizeof(int) * std::max<int64_t>(nflags_, 1), st);
  cudaMemsetAsync(d_status_ + 2, 0, sizeof(int), st);
  for (int l = 0; l < nl; ++l) {
    launch_fwd_warp(sym_, d_swarp_ + SP.warp_off[l], SP.warp_off[l + 1] - SP.warp_off[l], x,
                    contrib, d_cptr_, d_cidx_, n_, nrhs, cs, st);
    launch_fwd_diag(sym_, d_slist_ + SP.level_off[l], SP.level_off[l + 1] - SP.level_off[l], smem,
                    x, contrib, d_cptr_, d_cidx_, n_, nrhs, cs, st);
    for (int r = 0; r < nrhs; ++r)
      launch_fwd_chain(sym_, d_fchain_ + SP.chain_off[l], SP.chain_off[l + 1] - SP.chain_off[l],
                       x + (size_t)r * n_, contrib + (size_t)r * cs, d_cptr_, d_cidx_, d_flags_,
                       base + r + 1, n_, cs, st);
    launch_fwd_contrib(sym_, d_scontrib_ + SP.contrib_off[l], SP.contrib_off[l + 1] - SP.contrib_off[l],
                       SP.contrib_big[l], SP.contrib_wide[l], x, contrib, n_, nrhs, cs, st);
  }
  for (int l = nl - 1; l >= 0; --l) {
    launch_bwd_gather(sym_, d_sgather_ + SP.gather_off[l], SP.gather_off[l + 1] - SP.gather_off[l],
                      x, n_, nrhs, st);
    launch_bwd_diag(sym_, d_slist_ + SP.level_off[l], SP.level_off[l + 1] - SP.level_off[l], smem,
                    x, n_, nrhs, st);
    launch_bwd_warp(sym_, d_swarp_ + SP.warp_off[l], SP.warp_off[l + 1] - SP.warp_off[l], x, n_,
                    nrhs, st);
    for (int r = 0; r < nrhs; ++r)
      launch_bwd_chain(sym_, d_bchain_ + SP.chain_off[l], SP.chain_off[l + 1] - SP.chain_off[l],
                       x + (size_t)r * n_, d_flags_, base + nrhs + r + 1, st);
  }
}

// After a synchronised solve: did a chained block wait time out?
bool Engine::solve_status_ok(std::string &err) {
  cudaError_t e = cudaMemcpy(h_status_ + 2, d_status_ + 2, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) { err = std::string("solve status: ") + cudaGetErrorString(e); return false; }
  if (h_status_[2]) {
    err = "timeout: a chained block of the triangular solve waited longer than its budget for "
          "its predecessor";
    return false;
  }
  return true;
}

bool Engine::solve(const double *b, double *x, int nrhs, std::string &err) {
  if (!dL_) { err = "solve before factor"; return false; }
  cudaSetDevice(device_);
  if (!ensure_work(nrhs, err)) return false;
  cudaError_t e = cudaSuccess;
  if (x != b) e = cudaMemcpyAsync(x, b, sizeof(double) * n_ * nrhs, cudaMemcpyDeviceToDevice, stream_);
  if (e != cudaSuccess) { err = std::string("solve: ") + cudaGetErrorString(e); return false; }
  run_solve(x, nrhs);
  e = cudaStreamSynchronize(stream_);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) { err = std::string("solve: ") + cudaGetErrorString(e); return false; }
  return solve_status_ok(err);
}

bool Engine::refine(const double *b, double *x, int nrhs, double tol, int maxit, RefineInfo &info,
                    std::string &err) {
  if (!dL_) { err = "refine before factor"; return false; }
  cudaSetDevice(device_);
  if (!ensure_work(nrhs, err)) return false;
  cudaStream_t st = stream_;
  const size_t len = (size_t)n_ * nrhs;
  double *r = d_work_, *dv = r + len, *pv = dv + len, *qv = pv + len, *rows = qv + len;
  auto sync_norms = [&](int count) -> bool {
    cudaError_t e = cudaMemcpyAsync(h_norms_, d_norms_, sizeof(double) * 2 * count,
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { err = std::string("refine: ") + cudaGetErrorString(e); return false; }
    return true;
  };
  // ||A||_inf
  launch_rowabs(n_, d_csr_rp_, d_csr_val_, rows, st);
  launch_norms(n_, 1, rows, nullptr, d_norms_, d_npart_, st);
  if (!sync_norms(1)) return false;
  anorm_ = h_norms_[0];
  // residual r = b - A x and backward errors; returns the max over right-hand sides
  std::vector<double> berr(nrhs, 0.0);
  auto residual = [&](const double *xx) -> bool {
    launch_spmv(n_, d_csr_rp_, d_csr_ci_, d_csr_val_, xx, r, nrhs, st);
    launch_residual(len, b, r, st);
    launch_norms(n_, nrhs, r, nullptr, d_norms_, d_npart_, st);
    launch_norms(n_, nrhs, xx, nullptr, d_norms_ + 2 * nrhs, d_npart_, st);
    if (!sync_norms(2 * nrhs)) return false;
    for (int k = 0; k < nrhs; ++k) {
      const double rn = h_norms_[2 * k], xn = h_norms_[2 * (nrhs + k)];
      berr[k] = (xn > 0 && anorm_ > 0) ? rn / (anorm_ * xn) : rn;
    }
    return true;
  };
  auto worst = [&]() { return *std::max_element(berr.begin(), berr.end()); };
  // x0 = solve(b)
  cudaMemcpyAsync(x, b, sizeof(double) * len, cudaMemcpyDeviceToDevice, st);
  run_solve(x, nrhs);
  if (!residual(x)) return false;
  info.method = 0;
  info.iterations = 0;
  double prev = worst(), cur = prev;
  int stall = 0;
  while (cur > tol && info.iterations < maxit) {
    cudaMemcpyAsync(dv, r, sizeof(double) * len, cudaMemcpyDeviceToDevice, st);
    run_solve(dv, nrhs);
    launch_axpy(len, 1.0, dv, x, st);
    info.method = 1;
    info.iterations++;
    if (!residual(x)) return false;
    cur = worst();
    stall = (cur > 0.5 * prev) ? stall + 1 : 0;
    prev = cur;
    if (stall >= 2) break;
  }
  if (cur > tol && stall >= 2) {
    // factor-preconditioned conjugate gradients, one right-hand side at a time
    info.method = 2;
    for (int k = 0; k < nrhs; ++k) {
      double *xk = x + (size_t)k * n_, *rk = r + (size_t)k * n_;
      double *zk = dv + (size_t)k * n_, *pk = pv + (size_t)k * n_, *qk = qv + (size_t)k * n_;
      const double *bk = b + (size_t)k * n_;
      auto norms1 = [&](const double *a, const double *bb) -> bool {
        launch_norms(n_, 1, a, bb, d_norms_, d_npart_, st);
        return sync_norms(1);
      };
      launch_spmv(n_, d_csr_rp_, d_csr_ci_, d_csr_val_, xk, rk, 1, st);
      launch_residual((size_t)n_, bk, rk, st);
      cudaMemcpyAsync(zk, rk, sizeof(double) * n_, cudaMemcpyDeviceToDevice, st);
      run_solve(zk, 1);
      cudaMemcpyAsync(pk, zk, sizeof(double) * n_, cudaMemcpyDeviceToDevice, st);
      if (!norms1(rk, zk)) return false;
      double rz = h_norms_[1];
      for (int it = 0; it < maxit * 10; ++it) {
        launch_spmv(n_, d_csr_rp_, d_csr_ci_, d_csr_val_, pk, qk, 1, st);
        if (!norms1(pk, qk)) return false;
        const double pq = h_norms_[1];
        if (!(pq > 0)) break;
        const double alpha = rz / pq;
        launch_axpy((size_t)n_, alpha, pk, xk, st);
        launch_axpy((size_t)n_, -alpha, qk, rk, st);
        info.iterations++;
        if (!norms1(rk, nullptr)) return false;
        const double rn = h_norms_[0];
        if (!norms1(xk, nullptr)) return false;
        const double bk_err = rn / (anorm_ * h_norms_[0]);
        if (bk_err <= tol) break;
        cudaMemcpyAsync(zk, rk, sizeof(double) * n_, cudaMemcpyDeviceToDevice, st);
        run_solve(zk, 1);
        if (!norms1(rk, zk)) return false;
        const double rz2 = h_norms_[1];
        const double beta = rz2 / rz;
        rz = rz2;
        launch_xpby((size_t)n_, zk, beta, pk, st);   // p = z + beta p
      }
    }
    if (!residual(x)) return false;
  }
  info.berr = berr;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { err = std::string("refine: ") + cudaGetErrorString(e); return false; }
  return solve_status_ok(err);
}

bool Engine::solve_in_scratch(const double *b, double *x, int nrhs, double *scratch,
                              int64_t capacity, std::string &err) {
  if (!dL_) { err = "solve before factor"; return false; }
  const SolvePlan &SP = splan_;
  const int64_t cs = std::max<int64_t>(SP.contrib_len, 1);
  if (nrhs <= 0 || cs * nrhs > capacity) {
    err = "solve needs " + std::to_string(cs * (nrhs > 0 ? nrhs : 1)) +
          " doubles of scratch (off-diagonal rows of L times right-hand sides); the fixed "
          "scratch holds " + std::to_string(capacity);
    return false;
  }
  cudaSetDevice(device_);
  cudaStream_t st = stream_;
  cudaError_t e = cudaSuccess;
  if (x != b) e = cudaMemcpyAsync(x, b, sizeof(double) * n_ * nrhs, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) { err = std::string("solve: ") + cudaGetErrorString(e); return false; }
  run_solve_with(x, nrhs, scratch);
  e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) { err = std::string("solve: ") + cudaGetErrorString(e); return false; }
  return solve_status_ok(err);
}

}  // namespace swc
