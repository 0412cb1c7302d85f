// The numeric-factorization engine: device-resident symbolic data, the execution plan
// derived from it, and the launch sequence of the FP64 supernodal factorization.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "swc_internal.h"

namespace swc {

// Device view of one analysed matrix, passed by value to every kernel.
struct DevSym {
  int n, nsuper;
  const int *super;       // nsuper+1: first column of each supernode
  const int64_t *rowptr;  // nsuper+1: start of each supernode's row list in Ls
  const int *Ls;          // row lists
  const int64_t *xptr;    // nsuper: offset of each supernode's values in L
  const int *Ap;          // lower CSC of P A P^T
  const int *Ai;
  const double *Ax;
  const int *upd_ptr;     // update lists (prune sets)
  const int *upd;
  double *L;              // supernodal values (the reference's lValues)
  int *status;            // [0] = smallest failing column + 1 (INT_MAX if none),
                          // [1] = structure error flag, [2] = solve wait timeout,
                          // [3] = factorization wait timeout (persistent walk),
                          // [4] = poll budget of every bounded wait (set by the host)
  float2 *Lf;             // split mirror of L in K-major form (mixed-precision modes only,
                          // else null): supernode s at (float *)Lf + xk[s]
  const int64_t *xk;      // per supernode: offset (floats) of its mirror; xk[nsuper]: the
                          // format, 0 hi / lo TF32 planes, 1 hi / mid / lo bfloat16 planes
                          // (rows of kmirror_pitch_tf32 / _bf16 elements)
  double *dinv;           // scratch: inverses of the 64x64 diagonal blocks of the tiled class
  const int *dinv_off;    // per supernode: first block of its inverses in dinv (-1: none)
};

// Status words per handle (see DevSym::status) and the default poll budget of a wait.
constexpr int kStatusWords = 8;
constexpr int kDefaultWaitBudget = 1 << 24;

// Poll budget of a bounded device-side wait, as the host set it in status[4].
__device__ __forceinline__ long long wait_budget(const int *status) {
  return (long long)*(volatile const int *)&status[4];
}

// Row pitch (elements) of a supernode of width w in the K-major split mirror: rows start on
// 128-byte boundaries, so every 32-column K chunk of a row is one aligned 128-byte (TF32) or
// 64-byte (bfloat16) run.
__host__ __device__ __forceinline__ int kmirror_pitch_tf32(int w) { return (w + 31) & ~31; }
__host__ __device__ __forceinline__ int kmirror_pitch_bf16(int w) { return (w + 63) & ~63; }

// One (64x64 tile, descendant) product of the tcgen05 update kernel: rows a0.. of
// supernode d feed the tile rows set in rmask (in order), rows b0.. the tile columns set in
// cmask; the product runs over columns k0 .. k0 + kcnt - 1 of d (kk = k0 | kcnt << 16).
struct __align__(16) TcPair {
  int d, a0, b0, kk;
  unsigned long long rmask, cmask;
};

// Right-looking split-TF32 updates (swc_scatter_tc.cu).  Tiles (d, i0, j0, K chunks): the
// 128x128 block of d's contribution whose rows start at row i0 and columns at row j0 of d's
// row list.  Column table: entry coff[d] + j (row j of d, used as a column of C) holds the
// first entry in L of the target column (-1: the target is not of the tiled class) and the
// offset r such that relidx[r + i] is the position of d's row i in that target's row list.
struct ScatterCols {
  const int64_t *base;
  const int *rel;
  const int64_t *coff;
  const int *relidx;
};
// One tile of a contribution: supernode d, first row i0 and first column j0 (rows of d's row
// list), nk K chunks of 32 columns from column k0 of d, d's rows md, ncol columns (128, or at
// most 64 for a dense tile) and d's column-table offset co.  dense: a trailing update of the
// dense factorization of d itself (target = d's own columns j0.., row i at position i; no
// table), else a descendant's contribution to its tiled-class ancestors (128x128).
struct __align__(16) ScTile {
  int d, i0, j0, nk, md, k0, ncol, dense;
  int64_t co, pad;
};
// One level of the schedule (supernodes whose descendants all belong to earlier levels).
struct Wave {
  int small_off = 0, small_cnt = 0;
  int small_smem = 0;
  int asm_off = 0, asm_cnt = 0;    // (supernode, column) tasks of the tiled class
  int upd_off = 0, upd_cnt = 0;    // (supernode, row tile, column tile) update tasks
  int big_off = 0, big_cnt = 0;    // tiled-class supernodes (block 0 POTRF)
  std::vector<int> panel_off, panel_cnt;  // per column block step: TRSM tiles
  std::vector<int> syrk_off, syrk_cnt;
  std::vector<int> diag_off, diag_cnt;    // per step j: supernodes whose block j+1 exists
  std::vector<int> scd_off, scd_cnt;      // per step j: the trailing updates as dense tiles,
  std::vector<int> scd_nc;                //   the first scd_nc of them for column block j+1
                                          // (split-TF32 mode)
  int dense_off = 0, dense_cnt = 0;       // dataflow tasks of the dense factorization
  int dense_ctas = 0;
  int sc_off = 0, sc_cnt = 0;   // right-looking update tiles of the descendants of the level
                                // before (split-TF32 mode)
  int scs_off = 0, scs_cnt = 0; // the same level's small contributions
};

// Kernel classes, for per-kernel timing (profiled factorization) and flop accounting.
enum KernelKind { K_MEMSET = 0, K_SMALL, K_ASSEMBLE, K_UPDATE, K_PANEL, K_SYRK, K_NKINDS };

struct KernelStats {
  int launches[K_NKINDS] = {0};
  double ms[K_NKINDS] = {0};
  double flops[K_NKINDS] = {0};   // algorithmic flops of one factorization
  double bytes[K_NKINDS] = {0};   // algorithmic DRAM bytes of one factorization
};

struct Plan {
  std::vector<Wave> waves;
  std::vector<int> small_list;
  std::vector<int> big_list;
  std::vector<int2> asm_tasks;
  std::vector<int4> upd_tasks;     // (s, r0, c0, first pair)
  std::vector<int> upd_end;        // one past the last pair of each task
  std::vector<int4> upd_pairs;     // (d, a0, b0, na | nb << 16)
  std::vector<TcPair> tc_pairs;    // the same pairs for the tcgen05 kernel (tile masks)
  std::vector<TcPair> syrk_pairs;  // per SYRK task: its product (s, r0, c0, step block)
  std::vector<int> syrk_end;       // per SYRK task: one past its pair (its index + 1)
  std::vector<int2> panel_tasks;
  std::vector<int4> syrk_tasks;
  std::vector<int> diag_list;
  std::vector<int> tiny_list;      // tiny supernodes of the warp walk, in level order
  std::vector<int> persist_list;   // small supernodes of the persistent walk, in level order
  std::vector<int4> dense_tasks;   // (s, r0, c0, step << 2 | kind), per wave in topological order
  std::vector<int> dense_toff;     // per supernode: first tile version counter (-1: none)
  int64_t dense_tiles = 0;         // tile version counters in total
  // right-looking updates (split-TF32 mode): tiles, the column table and relative indices
  // (ScatterCols), supernodes that own tiles
  std::vector<ScTile> sc_tiles;
  std::vector<int2> sc_small;        // (d, c0) tasks of the small contributions
  std::vector<ScTile> sc_dense;      // trailing updates of the dense steps as tiles
  std::vector<int64_t> sc_base, sc_coff;
  std::vector<int> sc_rel, sc_relidx;
  std::vector<char> sc_used;
  double sc_flops = 0;               // executed flops of the tiles (128x128 blocks)
  int persist_smem = 0;
  int launches = 0;  // kernel launches per factorization
  int launches_scatter = 0;  // the same in the mixed modes with right-looking updates
  KernelStats work;  // algorithmic flops/bytes per kernel class
};


// Triangular solves and refinement (swc_solve.cu)
bool solve_configure(int max_w, std::string &err);
void launch_fwd_diag(const DevSym &S, const int *list, int count, int smem, double *y,
                     const double *contrib, const int *cptr, const int *cidx, int n, int nrhs,
                     int64_t cstride, cudaStream_t st);
void launch_fwd_contrib(const DevSym &S, const int2 *tasks, int count, int nbig, int nwide,
                        const double *y, double *contrib, int n, int nrhs, int64_t cstride,
                        cudaStream_t st);
void launch_bwd_gather(const DevSym &S, const int2 *tasks, int count, double *x, int n, int nrhs,
                       cudaStream_t st);
void launch_bwd_diag(const DevSym &S, const int *list, int count, int smem, double *x, int n,
                     int nrhs, cudaStream_t st);
// small supernodes, one warp each: forward (contributions in, diagonal solve, contributions
// of the rows below out) and backward (gather from ancestors, transposed diagonal solve)
void launch_fwd_warp(const DevSym &S, const int *list, int count, double *y, double *contrib,
                     const int *cptr, const int *cidx, int n, int nrhs, int64_t cstride,
                     cudaStream_t st);
void launch_bwd_warp(const DevSym &S, const int *list, int count, double *x, int n, int nrhs,
                     cudaStream_t st);
void launch_fwd_chain(const DevSym &S, const int2 *tasks, int count, double *y,
                      const double *contrib, const int *cptr, const int *cidx, int *flags,
                      int epoch, int n, int64_t cstride, cudaStream_t st);
void launch_bwd_chain(const DevSym &S, const int2 *tasks, int count, double *x, int *flags,
                      int epoch, cudaStream_t st);
void launch_spmv(int n, const int *rp, const int *ci, const double *val, const double *x,
                 double *y, int nrhs, cudaStream_t st);
void launch_gather_vals(int nnz, const int *map, const double *ax, double *val, cudaStream_t st);
void launch_residual(size_t len, const double *b, double *r, cudaStream_t st);
void launch_axpy(size_t len, double a, const double *x, double *y, cudaStream_t st);
void launch_xpby(size_t len, const double *z, double beta, double *p, cudaStream_t st);
void launch_norms(int n, int nrhs, const double *x, const double *y, double *out, double *part,
                  cudaStream_t st);
int norm_scratch_doubles(int nrhs);
void launch_rowabs(int n, const int *rp, const double *val, double *out, cudaStream_t st);

// Per-level task lists of the solves.
struct SolvePlan {
  std::vector<int> level_off;       // small-class supernodes of level l:
  std::vector<int> list;            //   list[level_off[l] .. level_off[l+1])
  std::vector<int> warp_off;        // small supernodes solved by one warp each (level l):
  std::vector<int> warp_list;       //   warp_list[warp_off[l] .. warp_off[l+1])
  std::vector<int> chain_off;       // (s, block) tasks of the tiled class in level l:
  std::vector<int2> fchain, bchain; //   forward (increasing block) / backward (decreasing)
  std::vector<int> contrib_off;     // (s, r0) tasks of level l: contrib_big[l] tasks of very
  std::vector<int> contrib_big;     //   wide supernodes, contrib_wide[l] of wide ones (a CTA
  std::vector<int> contrib_wide;    //   each), then narrow ones (a warp)
  std::vector<int2> contrib_tasks;
  std::vector<int> gather_off;      // (s, j0) tasks of level l
  std::vector<int2> gather_tasks;
  int max_w = 0;
  int64_t contrib_len = 0;          // off-diagonal rows in total (one contribution each)
  std::vector<int> cptr, cidx;      // per column: contributions it receives (CSR)
};

// Result of a refined solve, per right-hand side.
struct RefineInfo {
  std::vector<double> berr;         // final backward error ||b - A x|| / (||A|| ||x||), inf-norms
  int iterations = 0;               // refinement steps (or CG iterations after the fallback)
  int method = 0;                   // 0: direct solve sufficed, 1: refinement, 2: CG fallback
};

// Host copy of the per-supernode arrays the kernels index by.
struct HostSym {
  std::vector<int> super;
  std::vector<int64_t> rowptr, xptr;
  int64_t nls = 0, xsize = 0, nnz = 0;
  int nprune = 0;
  std::vector<int> dinv_off;   // per supernode: first diagonal-block inverse (-1: none)
  std::vector<int2> upd_lbub;  // per update-list entry: the descendant's row range in the target
  int64_t ndinv = 0;           // diagonal-block inverses in total
};

// Validates the symbolic arrays and derives the execution plan (no device work).
bool build_plan(int n, const int *c, const int *r, const int64_t *lC, const int *Ls,
                const int64_t *Li_ptr, const int *blockSet, int supNo, const int *prunePtr,
                const int *pruneSet, HostSym &H, Plan &P, std::string &err,
                const Tuning &T = Tuning());

// Host check of a plan's right-looking update tables (a no-op without them): every scattered
// entry's address against a direct lookup in the target's row list, every descendant's
// lower triangle covered once per column of K, every tile in the level after its
// descendant's, every column block of the dense steps' trailing updates receiving each
// earlier block once, each step's next-column tiles ahead of its grouped ones.  False with
// a message on the first violation.
bool check_scatter_plan(int n, const int *Ls, const HostSym &H, const Plan &P, const Tuning &T,
                        std::string &err);

// Per-level task lists of the supernodal solves (no device work).
void build_solve_plan(int n, const int *Ls, const HostSym &H, SolvePlan &SP);

// Host check of a solve plan: every supernode solved once (by its CTA or its warp, or, in
// the tiled class, by one chained block per 64 columns, forward in increasing and backward
// in decreasing block order), in a level after the levels of its children; every
// off-diagonal row of a supernode not solved by a warp in exactly one forward contribution
// task of its level, and each of its 16-column groups in exactly one backward gather task;
// every column's contribution list naming exactly the contributions of the rows equal to
// it.  False with a message on the first violation.
bool check_solve_plan(int n, const int *Ls, const HostSym &H, const SolvePlan &SP,
                      std::string &err);

struct AdjointPlan;   // reverse-sweep schedule of the adjoint (swc_adjoint.cu)

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  bool analyze(int n, const int *c, const int *r, const int64_t *lC, const int *Ls,
               const int64_t *Li_ptr, const int *blockSet, int supNo, const int *prunePtr,
               const int *pruneSet, std::string &err);
  // values: the A2 values (host or device).  Returns 0 on success, 1 if not SPD
  // (*info = failing column + 1), <0 on errors.
  // prec: 0 FP64; 1 / 2: Schur updates of the tiled class as split-TF32 / BF16x3
  // tensor-core products (the C ABI's mode numbers).
  int factor(const double *values, bool values_on_device, int *info, std::string &err,
             int prec = 0);
  // The same factorization with a CUDA event pair around every launch; fills per-class
  // launch counts and device milliseconds (no other difference).
  int factor_profiled(const double *values, bool values_on_device, int *info,
                      KernelStats &out, std::string &err, int prec = 0);
  // x = (L L^T)^{-1} b for nrhs right-hand sides (device pointers, leading dimension n).
  bool solve(const double *b, double *x, int nrhs, std::string &err);
  // The same solve with the contribution scratch supplied by the caller (capacity in
  // doubles); allocates nothing.  Fails if the scratch is too small.
  bool solve_in_scratch(const double *b, double *x, int nrhs, double *scratch,
                        int64_t capacity, std::string &err);
  // FP64 iterative refinement with the factor (falls back to factor-preconditioned CG when
  // refinement stalls); device pointers.
  bool refine(const double *b, double *x, int nrhs, double tol, int maxit, RefineInfo &info,
              std::string &err);
  // Device staging buffer of at least `doubles` entries (host-vector calls of the C ABI);
  // allocated on first use and grown when needed, freed with the engine.  nullptr on error.
  double *staging(size_t doubles, std::string &err);
  int64_t h2d_bytes() const { return h2d_bytes_; }
  int64_t d2h_bytes() const { return d2h_bytes_; }
  bool download(double *lValues, bool to_device, std::string &err);
  cudaStream_t stream() const { return stream_; }
  void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
  // Plan parameters used by the next analyze.
  void set_tuning(const Tuning &t) { tuning_ = t; }
  const Tuning &tuning() const { return tuning_; }
  // Poll budget of the device-side waits (status[4]); < 0 restores the default.
  bool set_wait_budget(long long polls, std::string &err);
  int64_t xsize() const { return xsize_; }
  int n() const { return n_; }
  int64_t nnz() const { return nnz_; }
  int nsuper() const { return nsuper_; }
  const Plan &plan() const { return plan_; }
  double *device_L() const { return dL_; }
  // kernel launches of one factorization in the given mode
  int launches_per_factor(int prec = 0) const {
    return prec != 0 ? plan_.launches_scatter : plan_.launches;
  }

  // Adjoint (swc_adjoint.cu), on the current factor; device pointers, grad has one entry
  // per stored nonzero of A.
  bool logdet(double *out, std::string &err);
  bool selected_inverse(std::string &err);   // Z = A^{-1} on the pattern of L
  const double *selected_inverse_ptr() const { return d_adj_Z_; }
  bool logdet_grad(double *grad, std::string &err);
  bool solve_grad(const double *x, const double *lam, double *grad, std::string &err);

  // Backward error ||b - A x||_inf / (||A||_inf ||x||_inf) of every diagonal block of A
  // (rows d_seg[k] .. d_seg[k+1]; a batch's matrices); device b, x; berr on the host.
  bool segment_berr(const int64_t *d_seg, int nseg, const double *b, const double *x,
                    double *berr, std::string &err);

 private:
  bool prepare_adjoint(std::string &err);
  void release_adjoint();
  std::shared_ptr<AdjointPlan> adj_;
  HostSym hsym_;
  std::vector<int> h_Ls_;
  int4 *d_adj_units_ = nullptr;
  int64_t *d_adj_tinv_off_ = nullptr, *d_adj_seg_tbl_ = nullptr;
  int2 *d_adj_tasks_ = nullptr;
  int *d_adj_wave_units_ = nullptr, *d_adj_ut_begin_ = nullptr, *d_adj_ut_end_ = nullptr;
  int *d_adj_rowseg_ = nullptr, *d_adj_seg_t_ = nullptr, *d_adj_seg_S_ = nullptr;
  int *d_adj_tbl_ = nullptr;
  double *d_adj_Z_ = nullptr, *d_adj_U_ = nullptr, *d_adj_tinv_ = nullptr, *d_adj_P_ = nullptr;
  double *d_adj_partial_ = nullptr;

  void release();
  void launch_all(std::vector<std::pair<int, cudaEvent_t>> *prof = nullptr, int prec = 0);
  bool set_mode(int prec, std::string &err);
  int finish(int *info, std::string &err);
  int64_t h2d_bytes_ = 0, d2h_bytes_ = 0;
  int wait_budget_ = kDefaultWaitBudget;
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaStream_t own_stream_ = nullptr;
  int n_ = 0, nsuper_ = 0;
  int64_t xsize_ = 0, nnz_ = 0;
  // device buffers
  int *d_super_ = nullptr, *d_Ls_ = nullptr, *d_Ap_ = nullptr, *d_Ai_ = nullptr;
  int64_t *d_rowptr_ = nullptr, *d_xptr_ = nullptr;
  int *d_upd_ptr_ = nullptr, *d_upd_ = nullptr;
  int2 *d_upd_lbub_ = nullptr;
  double *d_Ax_ = nullptr, *dL_ = nullptr, *d_dinv_ = nullptr;
  int *d_dinv_off_ = nullptr;
  int *d_status_ = nullptr, *h_status_ = nullptr;
  int *d_small_ = nullptr, *d_big_ = nullptr, *d_diag_ = nullptr;
  int4 *d_dense_tasks_ = nullptr;
  int *d_dense_toff_ = nullptr, *d_dense_ver_ = nullptr;   // ver: wave queue heads, tile counters
  int64_t dense_ver_len_ = 0;
  cudaStream_t aux_stream_ = nullptr;          // second branch of each dense step
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
  cudaStream_t small_stream_ = nullptr;        // a wave's small supernodes, beside its tiled work
  cudaEvent_t ev_sfork_ = nullptr, ev_sjoin_ = nullptr;
  cudaStream_t grp_stream_ = nullptr;          // grouped trailing updates of the dense steps
  cudaEvent_t ev_grp_[2] = {nullptr, nullptr};
  int2 *d_asm_ = nullptr, *d_panel_ = nullptr;
  int4 *d_upd_tasks_ = nullptr, *d_syrk_ = nullptr, *d_pairs_ = nullptr;
  int *d_upd_end_ = nullptr;
  cudaGraph_t graph_[3] = {nullptr, nullptr, nullptr};          // one per precision mode
  cudaGraphExec_t graph_exec_[3] = {nullptr, nullptr, nullptr};
  float *d_Lk_ = nullptr;                      // K-major split mirror (either mixed mode)
  int64_t *d_xk_ = nullptr, *d_xk16_ = nullptr;   // its offsets + format (TF32 / BF16x3)
  void *d_tmaps_ = nullptr;                    // one tensor map per supernode (over d_Lk_)
  std::vector<int64_t> h_xk_;
  int64_t kmirror_len_ = 0;
  TcPair *d_tc_pairs_ = nullptr, *d_syrk_pairs_ = nullptr;
  int *d_syrk_end_ = nullptr;
  ScTile *d_sc_tiles_ = nullptr;               // right-looking update tiles and their tables
  int2 *d_sc_small_ = nullptr;
  ScTile *d_sc_dense_ = nullptr;
  int64_t *d_sc_base_ = nullptr, *d_sc_coff_ = nullptr;
  int *d_sc_rel_ = nullptr, *d_sc_relidx_ = nullptr;
  void *d_sc_maps_ = nullptr;                  // tensor maps of the mirror's planes (over
  void *d_sc_maps16_ = nullptr;                //   d_Lk_): split-TF32 and BF16x3 layouts
  ScatterCols scatter_cols() const { return {d_sc_base_, d_sc_rel_, d_sc_coff_, d_sc_relidx_}; }
  bool use_graph_ = true;
  Tuning tuning_;
  int *d_persist_ = nullptr, *d_qctr_ = nullptr, *d_tiny_ = nullptr;
  int persist_ctas_ = 0, tiny_ctas_ = 0;
  Plan plan_;
  DevSym sym_{};
  // solve data
  SolvePlan splan_;
  int *d_slist_ = nullptr, *d_cptr_ = nullptr, *d_cidx_ = nullptr, *d_flags_ = nullptr;
  int *d_swarp_ = nullptr;
  int2 *d_fchain_ = nullptr, *d_bchain_ = nullptr;
  int64_t nflags_ = 0;
  double *d_sx_ = nullptr;                                         // solve graphs' vectors
  std::vector<std::pair<int, cudaGraphExec_t>> solve_graphs_;      // per nrhs
  cudaGraphExec_t solve_graph(int nrhs);
  void release_solve_graphs();
  int2 *d_scontrib_ = nullptr, *d_sgather_ = nullptr;
  int *d_csr_rp_ = nullptr, *d_csr_ci_ = nullptr, *d_csr_map_ = nullptr;
  double *d_csr_val_ = nullptr;
  int64_t csr_nnz_ = 0;
  double *d_contrib_ = nullptr, *d_work_ = nullptr, *d_norms_ = nullptr, *h_norms_ = nullptr;
  double *d_npart_ = nullptr;   // slices of the norm reductions
  double *d_stage_ = nullptr;
  size_t stage_len_ = 0;
  int work_nrhs_ = 0;
  double anorm_ = 0.0;
  bool ensure_work(int nrhs, std::string &err);
  void run_solve(double *x, int nrhs);
  void run_solve_with(double *x, int nrhs, double *contrib);
  bool solve_status_ok(std::string &err);
};

// kernel launch wrappers (swc_kernels.cu)
// lbub: per update-list entry (s, d), the first row of d's row list at or below s's first
// column and the first below its last column (computed on the host)
void launch_factor_small(const DevSym &S, const int2 *lbub, const int *list, int count, int smem,
                         cudaStream_t st);
// persistent small-class walk: CTAs to launch (occupancy x SMs, at most count) and the launch
int persist_ctas(int smem, int count);
int tiny_ctas(int count);
void launch_factor_tiny_persist(const DevSym &S, const int2 *lbub, const int *order, int count,
                                int ctas, int *qctr, int *qhead, cudaStream_t st);
void launch_factor_small_persist(const DevSym &S, const int2 *lbub, const int *order, int count,
                                 int smem, int ctas, int *qctr, cudaStream_t st);
void launch_assemble(const DevSym &S, const int2 *tasks, int count, cudaStream_t st);
void launch_update_tiles(const DevSym &S, const int4 *tasks, const int *task_end,
                         const int4 *pairs, int count, cudaStream_t st);
void launch_diag_step(const DevSym &S, const int *list, int count, int step, cudaStream_t st);
void launch_trsm_step(const DevSym &S, const int2 *tasks, int count, int step, cudaStream_t st);
// tasks (s, r0, c0, product index): prod[index].kk names the column blocks applied
void launch_syrk_step(const DevSym &S, const int4 *tasks, const TcPair *prod, int count,
                      cudaStream_t st);
// dense factorization of a wave's tiled-class panels as one persistent dataflow launch:
// tasks in topological order, per-supernode first tile counter (toff), tile version
// counters and the queue head (both zeroed before the launch)
int dense_ctas(int count);
void launch_dense_persist(const DevSym &S, const int4 *tasks, int count, int ctas, const int *toff,
                          int *ver, int *qhead, cudaStream_t st);
void launch_init_status(int *status, cudaStream_t st);
bool kernels_configure(std::string &err);
// split-precision tile updates on tcgen05 (swc_update_tc.cu): K-major mirror layout
// (offsets per supernode and the format entry, total floats), one tensor map per supernode
// for the TMA staging (host array of nsuper entries of tensor_map_bytes() each), the launch
// over tile tasks
bool update_tc_configure(std::string &err);
int64_t kmirror_layout(const std::vector<int> &super, const std::vector<int64_t> &rowptr,
                       std::vector<int64_t> &xk);
bool build_tensor_maps(const std::vector<int> &super, const std::vector<int64_t> &rowptr,
                       const std::vector<int64_t> &xk, float *Lk, void *maps_host,
                       std::string &err);
size_t tensor_map_bytes();
// variants: split-TF32 staged with cp.async (four producer warps) or with TMA gather4 loads;
// BF16x3 staged with cp.async
constexpr int UT_VARIANT_TF32 = 0, UT_VARIANT_TF32_TMA = 1, UT_VARIANT_BF16 = 2;
int update_tc_ctas(int count);   // CTAs of a launch over `count` tiles (at most one per SM)
// shared_sm: the launch runs next to another kernel (the diagonal-block kernel of the dense
// steps) and keeps shared memory for it
void launch_update_tc(const DevSym &S, const void *maps, const int4 *tasks, const int *task_end,
                      const TcPair *pairs, int count, int variant, bool shared_sm,
                      cudaStream_t st);

// Right-looking split-TF32 updates (swc_scatter_tc.cu): ScatterCols, ScTile above.
bool scatter_tc_configure(std::string &err);
// tensor maps over the K-major split mirror (scatter_maps_count entries): plane p (TF32: hi,
// lo; BF16x3: hi, mid, lo) of supernode d at [(box * planes + p) * nsuper + d], box 0 with
// 128-row boxes (used[d] & 1), box 1 with 64-row boxes (used[d] & 2)
size_t scatter_maps_count(int nsuper, bool bf16);
bool build_scatter_maps(const std::vector<int> &super, const std::vector<int64_t> &rowptr,
                        const std::vector<int64_t> &xk, const std::vector<char> &used, float *Lk,
                        bool bf16, void *maps_host, std::string &err);
// reserve: SMs left free for a kernel running at the same time (the diagonal-block kernel
// of the dense steps); bf16: the mirror holds BF16x3 planes (else split-TF32)
void launch_scatter_tc(const DevSym &S, const void *maps, const ScTile *tiles, int count,
                       const ScatterCols &C, int reserve, bool bf16, cudaStream_t st);
// Small contributions (a descendant whose rows from c0 number at most 128 and whose width
// times those rows, rounded up to 32, is at most SC_SMALL_ELEMS): one CTA per (d, c0) task,
// FP64 products from L on the CUDA cores, the same atomic scatter.
constexpr int SC_SMALL_ELEMS = 4096;
void launch_scatter_small(const DevSym &S, const int2 *tasks, int count, const ScatterCols &C,
                          cudaStream_t st);

}  // namespace swc
