// Internal declarations shared by the host code and the CUDA kernels of libswchol_b200.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace swc {

// Supernodal layout in the reference's BCSC conventions plus derived schedule arrays.
struct Layout {
  int n = 0, nsuper = 0;
  int64_t xsize = 0;
  std::vector<int64_t> rowptr;   // per supernode: start of its row list in Ls (nsuper+1)
  std::vector<int> Ls;           // row lists
  std::vector<int64_t> Li_ptr;   // per column (n+1)
  std::vector<int64_t> lC;       // per column (n+1)
  std::vector<int> sparent;      // supernodal etree, -1 = root
  std::vector<int> prunePtr, pruneSet;
  std::vector<int> levelPtr, parPtr, partition;
};

bool build_layout(int n, const int *c, const int *r, const int *blockSet, int supNo,
                  Layout &out, std::string &err);

// Supernode partition of an ordered lower CSC pattern (elimination tree, column counts,
// relaxed chains); super receives nsuper + 1 entries.
bool supernode_partition(int n, const int *c, const int *r, const int nrelax[3],
                         const double zrelax[3], int max_width, std::vector<int> &super,
                         std::string &err);

// A symmetric matrix read from a Matrix Market file: its lower triangle in CSC form, rows
// sorted, diagonal present (explicit zero when the file has none) in every column.
struct MtxLower {
  int n = 0;
  std::vector<int> colptr, rowind;
  std::vector<double> values;
};
bool read_matrix_market(const char *path, MtxLower &out, std::string &err);
bool write_matrix_market(const char *path, int n, const int *c, const int *r, const double *v,
                         std::string &err);
// Raw permutation files: n native size_t values (new position k holds original index perm[k]).
bool read_perm_file(const char *path, int n, std::vector<int64_t> &perm, std::string &err);
bool write_perm_file(const char *path, int n, const int64_t *perm, std::string &err);

// Fill-reducing ordering of a general sparse symmetric matrix given by its lower (or full)
// CSC pattern: nested dissection by level-structure vertex separators, minimum degree on
// the leaves.  perm[k] = original index at new position k.
struct NdOptions {
  int leaf = 64;           // subgraphs at most this large are ordered by minimum degree
  int trials = 3;          // pseudo-peripheral starting vertices tried per bisection
};
bool nested_dissection_order(int n, const int *c, const int *r, const NdOptions &opt,
                             std::vector<int64_t> &perm, std::string &err);

// Tile edge used by every tiled kernel.
constexpr int TB = 64;

// Task shapes of the solve's streaming kernels: rows of an off-diagonal block per forward
// contribution task, columns per backward gather task.
constexpr int SOLVE_CONTRIB_ROWS = 32;
constexpr int SOLVE_CONTRIB_WIDE_ROWS = 128;   // rows of a wide supernode's contribution task
constexpr int SOLVE_CONTRIB_BIG_W = 512;       // wider: 32-row tasks of 32 warps each
constexpr int SOLVE_CONTRIB_WIDE_MIN = 300;    // 128-row tasks only on levels with this many
constexpr int SOLVE_GATHER_COLS = 16;
constexpr int SOLVE_NARROW_W = 64;   // contribution tasks of supernodes this narrow: a warp each
// Supernodes of the small class at most this wide, with at most SOLVE_WARP_ROWS rows below
// the diagonal block, are solved by one warp each (both directions, fused) on levels that
// hold at least SOLVE_WARP_LEVEL_MIN of them (enough warps to fill the GPU; a CTA per
// supernode is faster on levels of fewer, larger ones).
constexpr int SOLVE_WARP_W = 32;
constexpr int SOLVE_WARP_ROWS = 256;
constexpr int SOLVE_WARP_LEVEL_MIN = 4096;

// Size classes of the executor (the B200 counterpart of the reference's triple queue,
// cholesky/tripleQueue.c:17-170): a supernode whose whole panel fits in shared memory is
// factored by one CTA, updates included; every other supernode goes through the tiled
// path (tile-owner updates, then a blocked right-looking dense factorization).
constexpr int SMALL_MAX_W = 64;
constexpr int SMALL_MAX_ELEMS = 12288;  // panel doubles held in shared memory (96 KB)
constexpr int SMALL_MAX_M = 2048;
// Shared-memory slab (doubles) through which a small supernode stages a descendant's rows,
// a column chunk at a time, before forming its update.
constexpr int SMALL_SLAB = 2048;   // >= SMALL_MAX_M: one full column always fits

// Tiny supernodes: one warp each (panel and row lists in a per-warp shared-memory slice).
constexpr int TINY_ELEMS = 1024;
constexpr int TINY_M = 256;
constexpr int TINY_SLAB = 512;     // >= TINY_M
static_assert(SMALL_SLAB >= SMALL_MAX_M && TINY_SLAB >= TINY_M, "a slab holds one full column");

// Execution-plan parameters (defaults above; the batched path's autotuner varies them).
struct Tuning {
  // size-class limits, at most the constants above.  Supernodes above 1,024 rows or 4,096
  // panel entries go through the tiled path: their updates then come from the descendants'
  // tiles over the whole GPU, where a CTA per supernode would walk a long descendant list
  // alone (grid3d_60: the split-TF32 factor 9.7 -> 9.3 ms)
  int small_max_w = SMALL_MAX_W;
  int small_max_m = 1024;
  int small_max_elems = 4096;
  int tiny = 1;                          // bottom tiny supernodes: one warp each, one launch
  int persist = 1;                       // bottom small supernodes in one persistent launch
  int persist_max_smem = 24 * 1024;      // shared-memory cap of a persistent supernode (bytes)
  int dense_dataflow = 0;                // dense steps of a wave: one dataflow launch (else
                                         // three launches per 64-column step)
  int dense_group = 4;                   // column blocks per grouped trailing update
  int grouped_reserve = 48;              // mixed modes: SMs the grouped trailing updates
                                         // leave to the next TRSM and diagonal block
  int syrk_fp64 = 0;                     // mixed modes: trailing SYRK steps in FP64 (DMMA)
                                         // instead of split dense tiles of the scatter
                                         // kernel
  int tc_tma = 0;                        // split-TF32 tile-owner tcgen05 updates: stage
                                         // operands with TMA gather4 loads, not cp.async
  int scatter = 1;                       // mixed modes: right-looking updates (dense
                                         // 128x128 tiles, FP64 atomic scatter) instead of
                                         // the tile-owner gather
  int scatter_kmax = 0;                  // right-looking tiles: columns of K per tile (a
                                         // multiple of 32; 0 = the descendant's width).
                                         // Shorter FP32 accumulations, summed in FP64 by
                                         // the scatter's atomic adds
};

}  // namespace swc
