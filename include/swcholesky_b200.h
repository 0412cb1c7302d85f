/* libswchol_b200 -- supernodal sparse Cholesky numeric factorization on NVIDIA B200.
 *
 * C ABI.  Plain pointers and sizes; no CUDA or PyTorch types in any signature (streams and
 * device pointers travel as void*).  Every function that can fail returns an int status
 * (SWC_OK = 0) and leaves a message for swc_last_error(), except the drop-in
 * sw_cholesky_left_par_05, which keeps the reference's "1 = success" convention.
 *
 * Layout conventions are the reference's BCSC (swCholesky common/def.h:123-210):
 *   blockSet[s] .. blockSet[s+1]-1 are the columns of supernode s (supNo supernodes);
 *   Ls[Li_ptr[j] ..] is the sorted row list of the supernode holding column j;
 *   lValues[lC[j] ..] holds column j; a supernode is an nsrow x nscol column-major block.
 */
#ifndef SWCHOLESKY_B200_H
#define SWCHOLESKY_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SWC_OK 0
#define SWC_NOT_SPD 1          /* a pivot was <= 0 or NaN; *info = failing column + 1 */
#define SWC_INVALID_INPUT 2    /* symbolic arrays rejected by host-side validation */
#define SWC_CUDA_ERROR 3
#define SWC_STRUCTURE_ERROR 4  /* pattern of A does not fit the supernodal structure */
#define SWC_NOT_READY 5        /* call order violated (e.g. factor before analyze) */
#define SWC_TIMEOUT 6          /* a bounded device-side wait ran out (see swc_set_wait_budget);
                                  the kernels returned and the handle stays usable */

/* factorization modes */
#define SWC_MODE_FP64 0        /* every operation in FP64 */
#define SWC_MODE_MIXED_TF32X3 1 /* the Schur updates of the wide supernodes (descendant updates
                                   and the trailing updates of their dense factorization) as
                                   split-TF32 products on the tcgen05 tensor cores (each value
                                   as hi + lo TF32 pieces, the products hi hi' + lo hi' +
                                   hi lo', FP32 accumulation over a descendant's width or
                                   over the column blocks of one trailing update), added to L
                                   in FP64; POTRF, TRSM and small supernodes in FP64.  Pair
                                   with swc_refine. */
#define SWC_MODE_MIXED_BF16X3 2 /* the same Schur updates as BF16x3 split products on
                                   tcgen05: each value as three bfloat16 pieces, the six piece
                                   products down to the third order (about FP32 accuracy),
                                   FP32 accumulation, added to L in FP64 */

typedef struct swc_handle *swc_handle_t;

/* ---- drop-in for the reference numeric executor ------------------------------------
 * Replaces sw_cholesky_left_par_05 (PRUNE build), cholesky/sw_parallel_PB_Cholesky_05.h:52-66,
 * called from examples/sw_choleskyTest01.cpp:223-232.  Same arguments, same meaning: A2 =
 * lower CSC of P A P^T (c, r, values), the BCSC layout (lC, Ls, Li_ptr, blockSet, supNo),
 * the prune sets and the H-level schedule from analyze_p2; lValues (L->xsize doubles, zeroed
 * by the caller) receives L in place.  timing, levelSet, nPar, chunk, threads, super_max,
 * col_max and nodCost are accepted and ignored, as in the reference (levelSet is never
 * allocated by its inspector: cholesky/InspectionLevel_06.h:28).  The factorization runs on
 * the current CUDA device through a process-wide handle; inputs are uploaded, L is
 * downloaded before returning.  Returns 1 on success and 0 on failure (non-SPD matrix or
 * invalid input); swc_last_info() gives the failing column + 1 of a non-SPD matrix. */
int sw_cholesky_left_par_05(int n, int *c, int *r, double *values, size_t *lC, int *Ls,
                            size_t *Li_ptr, double *lValues, int *blockSet, int supNo,
                            double *timing, int *prunePtr, int *pruneSet, int nLevels,
                            int *levelPtr, int *levelSet, int nPar, int *parPtr,
                            int *partition, int chunk, int threads, int super_max,
                            int col_max, double *nodCost);

/* Info of the last sw_cholesky_left_par_05 call: 0, or failing column + 1. */
int swc_last_info(void);

/* Message of the last failing call on this thread ("" if none). */
const char *swc_last_error(void);

/* ---- handle API: device-resident factorization -----------------------------------
 * No reference counterpart: the reference re-reads host arrays on every call.  A handle
 * keeps the symbolic structure and L on one GPU so that refactorization, solves and
 * refinement need no host traffic. */
int swc_create(swc_handle_t *handle, int device);
int swc_destroy(swc_handle_t handle);
/* Stream used by every later call on the handle (a cudaStream_t; NULL restores the
 * handle's own stream). */
int swc_set_stream(swc_handle_t handle, void *stream);
void *swc_get_stream(swc_handle_t handle);
/* Execution plan used by the next swc_analyze / swc_batch_analyze on the handle: one of
 * the candidates swc_batch_autotune tries.  0: default (supernodes of at most 1,024 rows
 * and 4,096 panel entries in the small class, persistent walk up to 24 KB of shared memory
 * per supernode); 1: persistent small-supernode walk up to 100 KB; 2: no persistent walk
 * (one launch per level); 3: larger small-class limits (2,048 rows, 12,288 entries, walk up
 * to 48 KB: fewer tiled supernodes); 4: the dense
 * factorization of each level's tiled supernodes as one persistent dataflow launch
 * instead of three launches per 64-column step; 5: in the mixed modes, the trailing SYRK
 * steps of the dense factorization in FP64 (DMMA) instead of split tcgen05 tiles; 6 and 7:
 * in the mixed modes, the descendant updates by the tile-owner gather kernel (split-TF32
 * operands staged by TMA gather4 loads, 6, or by cp.async, 7; BF16x3 by cp.async) instead
 * of the right-looking dense products with an FP64 atomic scatter, and the trailing SYRK
 * steps in FP64; 8 and 9: in the mixed modes, the right-looking products cut into tiles
 * of at most 256 (8) or 128 (9) columns of K, each accumulated in FP32 on the tensor
 * cores and summed in FP64 by the scatter (a more accurate factor for more atomic adds).
 * SWC_INVALID_INPUT for other values. */
int swc_set_plan(swc_handle_t handle, int plan);

/* Poll budget of the handle's device-side waits: the persistent walks of the
 * factorization (a supernode waiting for its descendants, a dense tile for its
 * predecessors) and the chained blocks of the triangular solves (a block waiting for the
 * one before it).  A wait that is still unserved after `polls` polls gives up, the other
 * waits of the launch give up with it, the kernels return, and the call fails with
 * SWC_TIMEOUT.  Default 2^24 polls (seconds); polls < 0 restores it, 0 fails every wait
 * that is not already served.  Takes effect for the next call.  No reference counterpart
 * (the reference's level barriers are pthread joins). */
int swc_set_wait_budget(swc_handle_t handle, long long polls);

/* Uploads and validates the structure.  Arguments as in sw_cholesky_left_par_05
 * (values excluded).  levelPtr/parPtr/partition may be NULL: the executor derives its own
 * level schedule from the supernodal etree. */
int swc_analyze(swc_handle_t handle, int n, const int *c, const int *r, const size_t *lC,
                const int *Ls, const size_t *Li_ptr, const int *blockSet, int supNo,
                const int *prunePtr, const int *pruneSet, int nLevels, const int *levelPtr,
                const int *parPtr, const int *partition);

/* Numeric factorization with the A2 values (nnz(A2) doubles, in the order of r).
 * values_on_device != 0: values is a device pointer on the handle's GPU.  *info = 0, or
 * the failing column + 1 (status SWC_NOT_SPD). */
int swc_factor(swc_handle_t handle, const double *values, int values_on_device, int mode,
               int *info);

/* Copies L (xsize doubles, reference layout) to host (to_device == 0) or device memory. */
int swc_get_L(swc_handle_t handle, double *lValues, int to_device);

/* x = (L L^T)^{-1} b with the handle's factor, in the factor's (permuted) ordering, for
 * nrhs right-hand sides stored column by column (leading dimension n).  on_device != 0: b
 * and x are device pointers on the handle's GPU.  Supernodal forward and backward solves,
 * level by level; the forward solve is the reference's blockedLsolve
 * (triangularSolve/Triangular_BCSC.h:14-48) in gather form; the backward solve has no
 * reference counterpart. */
int swc_solve(swc_handle_t handle, const double *b, double *x, int nrhs, int on_device);

/* Solve with FP64 iterative refinement against A (the values of the last factor):
 * x_{k+1} = x_k + (L L^T)^{-1} (b - A x_k) until the backward error
 * ||b - A x||_inf / (||A||_inf ||x||_inf) <= tol for every right-hand side, at most maxit
 * steps; when refinement stalls (two steps without halving the error) it falls back to
 * conjugate gradients preconditioned with the factor.  berr (nrhs doubles), iterations and
 * method (0 direct, 1 refinement, 2 CG) may be NULL.  No reference counterpart. */
int swc_refine(swc_handle_t handle, const double *b, double *x, int nrhs, int on_device,
               double tol, int maxit, double *berr, int *iterations, int *method);

/* Allocation-free variant of swc_solve, for callers that cannot allocate device memory
 * when they solve (their device memory is owned by a pool that forbids further CUDA
 * allocations, their host only allows allocation at start-up, or the implicit
 * synchronisation of cudaMalloc is not acceptable in their loop).  No counterpart in the
 * reference.  Same result as swc_solve with on_device = 1 (b and x are device pointers on
 * the handle's GPU; the handle was analysed and factored before); its scratch is a fixed
 * array of SWC_SOLVE_NOALLOC_MAX doubles (8 MiB) in the library's device image, held by
 * every GPU that loads the library until the process exits.  It needs (number of
 * off-diagonal rows of L) x nrhs doubles, i.e. (Li_ptr[n] - n) * nrhs <= SWC_SOLVE_NOALLOC_MAX,
 * and returns SWC_INVALID_INPUT with a message otherwise.  The first call on a device looks
 * up the scratch's device address; make that first call before any stream capture.  All
 * calls on a GPU share the scratch: overlapping calls race and must be serialised by the
 * caller.  Nothing in the scratch needs clearing between calls. */
#define SWC_SOLVE_NOALLOC_MAX 1048576
int swc_solve_noalloc(swc_handle_t handle, const double *b, double *x, int nrhs);

/* ---- adjoint (no reference counterpart: the reference computes no derivatives) -----
 * All three work on the handle's current factor (any mode) and on the stored nonzeros of
 * A2 = P A P^T (lower triangle, the `values` of swc_factor; a stored off-diagonal value
 * stands for both A_ij and A_ji).  Vectors are in the factor's ordering.
 *
 * swc_logdet: log det A = 2 sum_j log L_jj.
 * swc_logdet_grad: grad[p] = d log det A / d values[p] = (A^{-1})_ij (2 - delta_ij), from
 *   the selected inverse of A on the pattern of L (reverse sweep over the elimination
 *   tree).  grad has c[n] doubles.
 * swc_solve_grad: for a scalar f(x) with x = A^{-1} b and lam = A^{-1} df/dx (one more
 *   solve), grad[p] = df / d values[p] = -(lam_i x_j + lam_j x_i), or -lam_i x_i on the
 *   diagonal.  x and lam have n doubles, grad c[n]; df/db is lam itself. */
int swc_logdet(swc_handle_t handle, double *logdet);
int swc_logdet_grad(swc_handle_t handle, double *grad, int on_device);
int swc_solve_grad(swc_handle_t handle, const double *x, const double *lam, double *grad,
                   int on_device);

/* Device pointer to the handle's L (xsize doubles), valid until the next analyze. */
const double *swc_device_L(swc_handle_t handle);

/* sizes[0..5] = n, nsuper, xsize, kernel launches per factorization, host-to-device and
 * device-to-host bytes of the last factor / get_L call. */
int swc_sizes(swc_handle_t handle, long long *sizes);

/* Kernel classes reported by swc_profile (arrays of SWC_NKINDS entries, in this order). */
#define SWC_NKINDS 6   /* memset, small, assemble, update, panel, syrk */

/* One factorization, as swc_factor, with a CUDA event pair around every kernel launch:
 * per kernel class the number of launches, the summed device milliseconds, and the
 * algorithmic flops and DRAM bytes of one factorization.  Any output may be NULL. */
int swc_profile(swc_handle_t handle, const double *values, int values_on_device, int mode,
                int *info, int *launches, double *ms, double *flops, double *bytes);

/* Host-only: validates the structure (as swc_analyze does) and describes the execution
 * plan (candidate `plan`, as swc_set_plan) without touching a GPU; for plan 4 the dataflow
 * task order is checked (every wait served by an earlier task) as at analysis, and the
 * tables of the mixed modes' right-looking updates are checked against a direct lookup
 * (every scattered entry's address in L, each descendant's contribution covered once per
 * column of K, the dense steps' trailing updates covering each column block once), and
 * so are the solves' task lists (every supernode solved once, after its children; every
 * off-diagonal row in one forward contribution task, every 16-column group in one backward
 * gather task, each contribution listed once under its column);
 * SWC_INVALID_INPUT with the first violation in swc_last_error().
 * stats[0..19] = levels, kernel launches per factorization,
 * small-class supernodes, tiled-class supernodes, update tiles, update (tile, descendant)
 * pairs, TRSM tiles, SYRK tiles, then per kernel class (memset, small, assemble, update,
 * panel, syrk) the algorithmic flops [8..13] and DRAM bytes [14..19] of one
 * factorization.  No reference counterpart. */
int swc_plan_stats(int n, const int *c, const int *r, const size_t *lC, const int *Ls,
                   const size_t *Li_ptr, const int *blockSet, int supNo, const int *prunePtr,
                   const int *pruneSet, int plan, double *stats);

/* ---- host layout builder ---------------------------------------------------------
 * Builds the BCSC layout the reference's analyze_p2 produces for a given supernode
 * partition (cholesky/sw_LSparsity.h:598-665): Li_ptr, lC and Ls, the prune sets
 * (descendants in increasing order), the supernodal etree, and a level schedule in the
 * H-level array format (one partition per supernode, levels by etree height).
 * swc_layout_sizes gives sizes[0..3] = len(Ls), len(pruneSet), xsize, nLevels. */
int swc_layout_sizes(int n, const int *c, const int *r, const int *blockSet, int supNo,
                     long long *sizes);
int swc_layout(int n, const int *c, const int *r, const int *blockSet, int supNo,
               size_t *lC, int *Ls, size_t *Li_ptr, int *sparent, int *prunePtr,
               int *pruneSet, int *levelPtr, int *parPtr, int *partition);

/* ---- batched factorization (no reference counterpart) ------------------------------
 * nmat independent SPD matrices, each already ordered (P_k A_k P_k^T, lower CSC): n[k]
 * columns, column pointers c (n[k] + 1 entries per matrix, each starting at 0, the
 * matrices' arrays concatenated) and row indices r (local to the matrix, concatenated).
 * The handle then holds them as ONE block-diagonal matrix of N = sum n[k] columns with
 * the library's own supernode partition: swc_factor takes the matrices' values
 * concatenated in the same order, swc_solve / swc_refine the right-hand sides
 * concatenated, and the whole batch is factored by one CUDA graph replay.
 * swc_batch_autotune times the factorization of the batch for each supernode grouping and
 * plan candidate and keeps the fastest (choice[0] = partition, choice[1] = plan,
 * *best_ms = its time); cache_path (may be NULL) is a text file of earlier results keyed
 * by structure and mode.  swc_batch_berr gives every matrix's backward error
 * ||b - A x||_inf / (||A||_inf ||x||_inf) for concatenated b and x (nmat doubles). */
int swc_batch_analyze(swc_handle_t handle, int nmat, const int *n, const int *c, const int *r);
int swc_batch_autotune(swc_handle_t handle, const double *values, int values_on_device,
                       int mode, const char *cache_path, int *choice, double *best_ms);
int swc_batch_berr(swc_handle_t handle, const double *b, const double *x, int on_device,
                   double *berr);

/* Host-only supernode partition of an ordered matrix, for matrices the reference's
 * analyze_p2 has not seen (the batched path): elimination tree, exact column counts, and
 * relaxed chains with the reference's relaxation parameters (nrelax = {4, 16, 48},
 * zrelax = {0.8, 0.1, 0.05} when NULL) and supernodes at most max_width wide.  blockSet
 * needs room for n + 1 entries; *supNo receives the number of supernodes.  Pair with
 * swc_layout.  No reference counterpart as a function (it is part of analyze_p2). */
int swc_supernodes(int n, const int *c, const int *r, const int *nrelax, const double *zrelax,
                   int max_width, int *blockSet, int *supNo);

/* ---- input files and fill-reducing ordering (host only) ---------------------------
 * swc_read_mtx replaces the reference's readMatrix (common/Util.h:77-179): a Matrix Market
 * coordinate file of a square real or integer matrix, symmetric or general (a general one
 * must be numerically symmetric), entries in any order, duplicates summed, upper entries of
 * a symmetric file mirrored, comments and blank lines anywhere before the entries, empty
 * columns allowed.  Result: the lower triangle in CSC form (n + 1 column pointers, row
 * indices sorted, the diagonal present in every column -- an explicit 0 where the file has
 * none) in arrays allocated with malloc; release each with swc_free.  Malformed files fail
 * with SWC_INVALID_INPUT and a message (the reference's reader returns false or silently
 * misreads).  swc_write_mtx writes a lower CSC matrix as a symmetric coordinate file that
 * both readers accept (1-based, column by column).
 * swc_read_perm / swc_write_perm replace the raw permutation read of the reference's driver
 * (examples/sw_choleskyTest01.cpp:70-82): n native size_t values, perm[k] = original index
 * at new position k; the reader checks the file's length and that it is a permutation.
 * swc_order_nd: the project's own fill-reducing ordering for any sparse symmetric pattern
 * (lower or full CSC): nested dissection by breadth-first level-structure separators,
 * exact minimum degree on subgraphs of at most `leaf` vertices (<= 64; 0 for the default
 * 64).  The reference needs the ordering as an input file (cholesky/sw_LSparsity.h:461-468). */
int swc_read_mtx(const char *path, int *n, int **colptr, int **rowind, double **values);
void swc_free(void *p);
int swc_write_mtx(const char *path, int n, const int *colptr, const int *rowind,
                  const double *values);
int swc_read_perm(const char *path, int n, size_t *perm);
int swc_write_perm(const char *path, int n, const size_t *perm);
int swc_order_nd(int n, const int *colptr, const int *rowind, int leaf, size_t *perm);

#ifdef __cplusplus
}
#endif

#endif /* SWCHOLESKY_B200_H */
