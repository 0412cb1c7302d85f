/* Test oracle only: a thin C wrapper around the reference's own host symbolic phase
 * (analyze_p2, cholesky/sw_LSparsity.h:248-702) and its FP64 numeric executor
 * (sw_cholesky_left_par_05_check, cholesky/sw_parallel_PB_Cholesky_05_check.c:43-692),
 * compiled from the reference sources where they lie by oracle/Makefile.
 *
 * It reproduces exactly what the reference driver does between reading the matrix and
 * the factor call (examples/sw_choleskyTest01.cpp:99-232):
 *   - nrelax = {4,16,48}, zrelax = {0.8,0.1,0.05}            (:112-113)
 *   - analyze_p2(1, A, NULL, NULL, nrelax, zrelax, n, ...)    (:138-144)
 *   - A1 = ptranspose(A, 2, L->Perm), A2 = ptranspose(A1, 2)  (:198-199)
 *   - the factor call with super_max = maxSupWid+1, col_max = maxCol+1 (:223-232)
 * and exposes every array so tests can compare against them and the bench can time the
 * reference on the same inputs.  swc_ref_read_matrix runs the reference's Matrix Market
 * reader (readMatrix, common/Util.h:77-179) for the reader's parity tests.  Nothing in the
 * product links this file. */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sys/time.h>
#include <unistd.h>
#include <fcntl.h>

// Same include order as the reference driver (examples/sw_choleskyTest01.cpp:11-18); the
// headers are not self-contained and rely on it.
#include "Ordering.h"
#include "Inspection_Prune.h"
#include "Inspection_Block.h"
#include "Util.h"
#include "PB_Cholesky.h"
#include "sw_LSparsity.h"
#include "sw_parallel_PB_Cholesky_05.h"

extern "C" void swc_ref_set_blas_threads(int t);

namespace {

struct RefSym {
  int n = 0;
  CSC *A = nullptr;   // caller's lower CSC (copied)
  CSC *A2 = nullptr;  // lower CSC of P A P^T with sorted rows
  BCSC *L = nullptr;
  int *prunePtr = nullptr, *pruneSet = nullptr;
  int nLevels = 0, nPar = 0;
  int *levelPtr = nullptr, *levelSet = nullptr, *parPtr = nullptr, *partition = nullptr;
  int maxSupWid = 0, maxCol = 0;
  double symbolic_seconds = 0.0;
};

double now_s() {
  struct timeval t;
  gettimeofday(&t, nullptr);
  return t.tv_sec + 1e-6 * t.tv_usec;
}

// The reference prints progress on stdout; route it to /dev/null while it runs so the
// caller's own stdout (e.g. a one-line JSON report) stays clean.
struct QuietStdout {
  int saved = -1;
  QuietStdout() {
    fflush(stdout);
    std::cout.flush();
    saved = dup(1);
    int fd = open("/dev/null", O_WRONLY);
    if (fd >= 0) { dup2(fd, 1); close(fd); }
  }
  ~QuietStdout() {
    fflush(stdout);
    std::cout.flush();
    if (saved >= 0) { dup2(saved, 1); close(saved); }
  }
};

}  // namespace

extern "C" {

/* Runs the reference symbolic phase on the lower triangle of A (CSC, sorted rows,
 * every column non-empty, as readMatrix requires: common/Util.h:97-176) with the
 * user permutation perm (size_t[n], as the driver reads it: sw_choleskyTest01.cpp:70-80).
 * Returns an opaque handle, or NULL on failure. */
void *swc_ref_analyze(int n, const int *Ap, const int *Ai, const double *Ax,
                      const long long *perm, int costParam, int levelParam,
                      int finalSeqNode) {
  QuietStdout quiet;
  RefSym *h = new RefSym;
  h->n = n;
  int nnz = Ap[n];
  CSC *A = new CSC;
  std::memset(A, 0, sizeof(CSC));
  A->nzmax = nnz;
  A->ncol = A->nrow = n;
  A->stype = -1;
  A->xtype = CHOLMOD_REAL;
  A->packed = TRUE;
  A->sorted = TRUE;
  A->p = new int[n + 1];
  A->i = new int[nnz];
  A->x = new double[nnz];
  A->nz = nullptr;
  std::memcpy(A->p, Ap, sizeof(int) * (n + 1));
  std::memcpy(A->i, Ai, sizeof(int) * nnz);
  std::memcpy(A->x, Ax, sizeof(double) * nnz);
  h->A = A;

  size_t *inPerm = new size_t[n];
  for (int k = 0; k < n; ++k) inPerm[k] = (size_t)perm[k];
  int nrelax[3] = {4, 16, 48};
  double zrelax[3] = {0.8, 0.1, 0.05};
  int status = 0;
  double orderingTime = 0;
  double t0 = now_s();
  h->L = analyze_p2(1, A, NULL, NULL, nrelax, zrelax, n, h->prunePtr, h->pruneSet,
                    h->nLevels, h->levelPtr, h->levelSet, h->nPar, h->parPtr,
                    h->partition, costParam, levelParam, finalSeqNode, status,
                    h->maxSupWid, h->maxCol, orderingTime, inPerm);
  h->symbolic_seconds = now_s() - t0;
  delete[] inPerm;
  if (!h->L) { delete h; return nullptr; }
  CSC *A1 = ptranspose(A, 2, h->L->Perm, NULL, 0, status);
  h->A2 = ptranspose(A1, 2, NULL, NULL, 0, status);
  allocateAC(A1, 0, 0, 0, FALSE);
  return h;
}

/* sizes[0..11] = n, nsuper, xsize, len(Ls), nnz(A2), nLevels, nParts, len(partition),
 *               len(pruneSet), maxSupWid, maxCol, symbolic time in microseconds */
void swc_ref_sizes(void *hv, long long *sizes) {
  RefSym *h = (RefSym *)hv;
  BCSC *L = h->L;
  int n = h->n, ns = (int)L->nsuper;
  int nparts = h->levelPtr[h->nLevels];
  sizes[0] = n;
  sizes[1] = ns;
  sizes[2] = (long long)L->xsize;
  sizes[3] = (long long)L->i_ptr[n];
  sizes[4] = h->A2->p[n];
  sizes[5] = h->nLevels;
  sizes[6] = nparts;
  sizes[7] = h->parPtr[nparts];
  sizes[8] = h->prunePtr[ns];
  sizes[9] = h->maxSupWid;
  sizes[10] = h->maxCol;
  sizes[11] = (long long)(h->symbolic_seconds * 1e6);
}

/* Copies out every array the numeric phase consumes (plus Perm, ColCount and the
 * supernodal etree).  Any pointer may be NULL to skip that array. */
void swc_ref_arrays(void *hv, int *perm, int *colcount, int *super, int *sparent,
                    int *Ls, long long *lC, long long *Li_ptr, int *A2p, int *A2i,
                    double *A2x, int *prunePtr, int *pruneSet, int *levelPtr,
                    int *parPtr, int *partition) {
  RefSym *h = (RefSym *)hv;
  BCSC *L = h->L;
  int n = h->n, ns = (int)L->nsuper;
  int nparts = h->levelPtr[h->nLevels];
  if (perm) std::memcpy(perm, L->Perm, sizeof(int) * n);
  if (colcount) std::memcpy(colcount, L->ColCount, sizeof(int) * n);
  if (super) std::memcpy(super, L->super, sizeof(int) * (ns + 1));
  if (sparent) std::memcpy(sparent, L->sParent, sizeof(int) * ns);
  if (Ls) std::memcpy(Ls, L->s, sizeof(int) * L->i_ptr[n]);
  if (lC) for (int j = 0; j <= n; ++j) lC[j] = (long long)L->p[j];
  if (Li_ptr) for (int j = 0; j <= n; ++j) Li_ptr[j] = (long long)L->i_ptr[j];
  if (A2p) std::memcpy(A2p, h->A2->p, sizeof(int) * (n + 1));
  if (A2i) std::memcpy(A2i, h->A2->i, sizeof(int) * h->A2->p[n]);
  if (A2x) std::memcpy(A2x, h->A2->x, sizeof(double) * h->A2->p[n]);
  if (prunePtr) std::memcpy(prunePtr, h->prunePtr, sizeof(int) * (ns + 1));
  if (pruneSet) std::memcpy(pruneSet, h->pruneSet, sizeof(int) * h->prunePtr[ns]);
  if (levelPtr) std::memcpy(levelPtr, h->levelPtr, sizeof(int) * (h->nLevels + 1));
  if (parPtr) std::memcpy(parPtr, h->parPtr, sizeof(int) * (nparts + 1));
  if (partition) std::memcpy(partition, h->partition, sizeof(int) * h->parPtr[nparts]);
}

/* Runs the reference FP64 numeric executor on the analysed structure.  values: the
 * A2 values to factor (NULL = the ones analysed).  lValues (xsize doubles) is zeroed
 * here, as the driver does before each call (sw_choleskyTest01.cpp:208-210).
 * threads > 0 sets the OpenBLAS thread count.  Returns the wall time in seconds of the
 * factor call alone, timed with gettimeofday as the driver does (:221-238); *ret gets the
 * executor's return value. */
double swc_ref_factor(void *hv, const double *values, double *lValues, int threads,
                      int *ret) {
  RefSym *h = (RefSym *)hv;
  BCSC *L = h->L;
  int n = h->n;
  if (threads > 0) swc_ref_set_blas_threads(threads);
  if (values) std::memcpy(h->A2->x, values, sizeof(double) * h->A2->p[n]);
  std::memset(lValues, 0, sizeof(double) * L->xsize);
  double timing[8] = {0};
  double t;
  int r;
  {
    QuietStdout quiet;
    double t0 = now_s();
    r = sw_cholesky_left_par_05_check(
        n, h->A2->p, h->A2->i, h->A2->x, L->p, L->s, L->i_ptr, lValues, L->super,
        (int)L->nsuper, timing, h->prunePtr, h->pruneSet, h->nLevels, h->levelPtr,
        h->levelSet, h->nPar, h->parPtr, h->partition, 0, 1, h->maxSupWid + 1,
        h->maxCol + 1, NULL);
    t = now_s() - t0;
  }
  if (ret) *ret = r;
  return t;
}

void swc_ref_free(void *hv) {
  RefSym *h = (RefSym *)hv;
  if (!h) return;
  // The reference's own driver leaks most of these too; free what we own.
  allocateAC(h->A2, 0, 0, 0, FALSE);
  delete[] h->A->p;
  delete[] h->A->i;
  delete[] h->A->x;
  delete h->A;
  delete h;
}

// The reference's readMatrix on a file: 1 and the lower CSC arrays (new[]-allocated, free
// with swc_ref_free_matrix) on success, 0 when it reports failure.
int swc_ref_read_matrix(const char *path, long long *n, long long *nnz, int **col, int **row,
                        double **val) {
  size_t nn = 0, nz = 0;
  int *c = nullptr, *r = nullptr;
  double *v = nullptr;
  if (!readMatrix(std::string(path), nn, nz, c, r, v)) return 0;
  *n = (long long)nn;
  *nnz = (long long)nz;
  *col = c;
  *row = r;
  *val = v;
  return 1;
}

void swc_ref_free_matrix(int *col, int *row, double *val) {
  delete[] col;
  delete[] row;
  delete[] val;
}

}  // extern "C"
