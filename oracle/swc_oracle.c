/* TEST ORACLE ONLY.  A plain-C restatement of the reference's FP64 left-looking
 * supernodal numeric factorization and of the layout-compatible supernodal solves.
 * It is the checker for the CUDA library, never part of it: only tests, the smoke check
 * and the CPU-baseline leg of the benchmark load it.
 *
 * Layout (reference BCSC, common/def.h:123-210 and cholesky/sw_LSparsity.h:611-638):
 *   supernode s spans columns blockSet[s] .. blockSet[s+1]-1; its sorted row list is
 *   Ls[Li_ptr[blockSet[s]] .. Li_ptr[blockSet[s+1]]); its values are a column-major
 *   nsrow x nscol block at lValues + lC[blockSet[s]] with leading dimension nsrow.
 *
 * The dense kernels are written out as loops (no BLAS) so the oracle depends on nothing
 * but libm; the loop order of the update is the reference's: one descendant at a time in
 * prune-set order, each contribution formed in full and then subtracted. */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

/* contrib = S S^T (lower, ndrow1 x ndrow1) and contrib[ndrow1:, :] = B S^T, the dsyrk_/dgemm_
 * pair of cholesky/sw_parallel_PB_Cholesky_05_check.c:230-257: S = src (ndrow1 rows),
 * B = srcL (ndrow3 rows), both with leading dimension lda and k columns; contrib has
 * leading dimension ldc = nSupRs = ndrow1 + ndrow3. */
static void contrib_syrk_gemm(int ndrow1, int ndrow3, int k, const double *src,
                              const double *srcL, int lda, double *contrib, int ldc) {
  for (int j = 0; j < ndrow1; ++j) {
    for (int i = j; i < ndrow1 + ndrow3; ++i) {
      const double *a = (i < ndrow1) ? (src + i) : (srcL + (i - ndrow1));
      const double *b = src + j;
      double acc = 0.0;
      for (int p = 0; p < k; ++p) acc += a[(size_t)p * lda] * b[(size_t)p * lda];
      contrib[(size_t)j * ldc + i] = acc;
    }
  }
}

/* In-place lower Cholesky of the n x n diagonal block (leading dimension lda): the
 * dpotrf_ call of _check.c:319-324.  Returns 0, or j+1 for the first column whose pivot
 * is not positive (or NaN), as the reference's dpotrf2_single does
 * (BLAS-sw/dpotrf2_single.c:14-17). */
static int potrf_lower(int n, double *a, int lda) {
  for (int j = 0; j < n; ++j) {
    double d = a[(size_t)j * lda + j];
    for (int p = 0; p < j; ++p) d -= a[(size_t)p * lda + j] * a[(size_t)p * lda + j];
    if (!(d > 0.0)) return j + 1;
    d = sqrt(d);
    a[(size_t)j * lda + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double v = a[(size_t)j * lda + i];
      for (int p = 0; p < j; ++p) v -= a[(size_t)p * lda + i] * a[(size_t)p * lda + j];
      a[(size_t)j * lda + i] = v / d;
    }
  }
  return 0;
}

/* B := B L^{-T} for B (m x n, leading dimension ldb), L lower n x n (lda): the dtrsm_
 * ('R','L','T','N') call of _check.c:349-355. */
static void trsm_rltn(int m, int n, const double *l, int lda, double *b, int ldb) {
  for (int j = 0; j < n; ++j) {
    double d = l[(size_t)j * lda + j];
    for (int i = 0; i < m; ++i) {
      double v = b[(size_t)j * ldb + i];
      for (int p = 0; p < j; ++p) v -= b[(size_t)p * ldb + i] * l[(size_t)p * lda + j];
      b[(size_t)j * ldb + i] = v / d;
    }
  }
}

/* Factor one supernode s (0-based), cholesky/sw_parallel_PB_Cholesky_05_check.c:141-365:
 * row map, copy of A into the panel, updates from every descendant in the prune set,
 * POTRF on the diagonal block, TRSM below it.  Returns 0 or the failing global column+1. */
static int factor_supernode(int s, const int *c, const int *r, const double *values,
                            const size_t *lC, const int *Ls, const size_t *Li_ptr,
                            double *lValues, const int *blockSet, const int *prunePtr,
                            const int *pruneSet, int *map, double *contribs) {
  int curCol = blockSet[s], nxtCol = blockSet[s + 1];
  int supWdt = nxtCol - curCol;
  int nSupR = (int)(Li_ptr[nxtCol] - Li_ptr[curCol]);
  /* row map (_check.c:147-149) */
  for (size_t i = Li_ptr[curCol], cnt = 0; i < Li_ptr[nxtCol]; ++i) map[Ls[i]] = (int)cnt++;
  /* copy A into L (_check.c:152-161) */
  for (int i = curCol; i < nxtCol; ++i)
    for (int j = c[i]; j < c[i + 1]; ++j) lValues[lC[i] + map[r[j]]] = values[j];
  double *cur = &lValues[lC[curCol]];
  /* updates from the prune set, in order (_check.c:174-300) */
  for (int q = prunePtr[s]; q < prunePtr[s + 1]; ++q) {
    int lSN = pruneSet[q];
    int cSN = blockSet[lSN], cNSN = blockSet[lSN + 1];
    size_t b0 = Li_ptr[cSN], b1 = Li_ptr[cNSN];
    int nSNRCur = (int)(b1 - b0);
    int supWdts = cNSN - cSN;
    /* overlap search (_check.c:190-209): lb = first row >= curCol, ub = last row < nxtCol */
    int lb = 0, ub = 0, sw = 1;
    for (size_t j = b0; j < b1; ++j) {
      if (Ls[j] >= curCol && sw) { lb = (int)(j - b0); sw = 0; }
      if (Ls[j] < nxtCol && !sw) ub = (int)(j - b0);
      if (Ls[j] >= nxtCol) break;
    }
    int nSupRs = nSNRCur - lb;
    int ndrow1 = ub - lb + 1;
    int ndrow3 = nSupRs - ndrow1;
    const double *src = &lValues[lC[cSN] + lb];
    const double *srcL = &lValues[lC[cSN] + ub + 1];
    contrib_syrk_gemm(ndrow1, ndrow3, supWdts, src, srcL, nSNRCur, contribs, nSupRs);
    /* scatter-subtract of the lower trapezoid (_check.c:282-295) */
    for (int i2 = 0; i2 < ndrow1; ++i2) {
      int col = map[Ls[b0 + i2 + lb]];
      for (int j2 = i2; j2 < nSupRs; ++j2) {
        int cRow = Ls[b0 + j2 + lb];
        cur[(size_t)col * nSupR + map[cRow]] -= contribs[(size_t)i2 * nSupRs + j2];
      }
    }
  }
  int info = potrf_lower(supWdt, cur, nSupR);
  if (info) return curCol + info;
  trsm_rltn(nSupR - supWdt, supWdt, cur, nSupR, cur + supWdt, nSupR);
  return 0;
}

/* The whole factor in the reference's schedule order: coarse levels in order, the
 * partitions of each level, the supernodes of each partition in order
 * (_check.c:127-141 and :447-456; partition[k] is a 0-based supernode id).  lValues must
 * be zeroed by the caller, as in the reference driver (examples/sw_choleskyTest01.cpp:
 * 208-210).  Returns 1 on success; on a non-positive pivot stops and returns 0 with
 * *info = failing global column + 1 (the reference prints and breaks, _check.c:320-323). */
int swc_oracle_factor(int n, const int *c, const int *r, const double *values,
                      const size_t *lC, const int *Ls, const size_t *Li_ptr,
                      double *lValues, const int *blockSet, int supNo, const int *prunePtr,
                      const int *pruneSet, int nLevels, const int *levelPtr,
                      const int *parPtr, const int *partition, int *info) {
  int super_max = 0, col_max = 0;
  for (int s = 0; s < supNo; ++s) {
    int w = blockSet[s + 1] - blockSet[s];
    int m = (int)(Li_ptr[blockSet[s + 1]] - Li_ptr[blockSet[s]]);
    if (w > super_max) super_max = w;
    if (m > col_max) col_max = m;
  }
  int *map = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  double *contribs = (double *)malloc(sizeof(double) * (size_t)(super_max + 1) * (col_max + 1));
  if (info) *info = 0;
  int ok = 1;
  for (int l = 0; l < nLevels && ok; ++l)
    for (int p = levelPtr[l]; p < levelPtr[l + 1] && ok; ++p)
      for (int k = parPtr[p]; k < parPtr[p + 1]; ++k) {
        int e = factor_supernode(partition[k], c, r, values, lC, Ls, Li_ptr, lValues,
                                 blockSet, prunePtr, pruneSet, map, contribs);
        if (e) { if (info) *info = e; ok = 0; break; }
      }
  free(map);
  free(contribs);
  return ok;
}

/* Supernodal forward solve L y = b in place (x holds b on entry), following the
 * reference's blockedLsolve (triangularSolve/Triangular_BCSC.h:14-48): a dense lower
 * solve on the diagonal block, then x[rows below] -= L_below * x[cols]. */
static void lsolve(const size_t *lC, const int *Ls, const size_t *Li_ptr,
                   const double *lValues, const int *blockSet, int supNo, double *x) {
  for (int s = 0; s < supNo; ++s) {
    int c0 = blockSet[s], c1 = blockSet[s + 1], w = c1 - c0;
    int m = (int)(Li_ptr[c1] - Li_ptr[c0]);
    const double *Lp = lValues + lC[c0];
    const int *rows = Ls + Li_ptr[c0];
    for (int j = 0; j < w; ++j) {
      x[c0 + j] /= Lp[(size_t)j * m + j];
      double xj = x[c0 + j];
      for (int i = j + 1; i < w; ++i) x[c0 + i] -= Lp[(size_t)j * m + i] * xj;
    }
    for (int i = w; i < m; ++i) {
      double acc = 0.0;
      for (int j = 0; j < w; ++j) acc += Lp[(size_t)j * m + i] * x[c0 + j];
      x[rows[i]] -= acc;
    }
  }
}

/* Supernodal backward solve L^T x = y in place: supernodes in reverse order,
 * x[cols] -= L_below^T x[rows below], then a dense upper solve with the diagonal block. */
static void ltsolve(const size_t *lC, const int *Ls, const size_t *Li_ptr,
                    const double *lValues, const int *blockSet, int supNo, double *x) {
  for (int s = supNo - 1; s >= 0; --s) {
    int c0 = blockSet[s], c1 = blockSet[s + 1], w = c1 - c0;
    int m = (int)(Li_ptr[c1] - Li_ptr[c0]);
    const double *Lp = lValues + lC[c0];
    const int *rows = Ls + Li_ptr[c0];
    for (int j = w - 1; j >= 0; --j) {
      double v = x[c0 + j];
      for (int i = w; i < m; ++i) v -= Lp[(size_t)j * m + i] * x[rows[i]];
      for (int i = j + 1; i < w; ++i) v -= Lp[(size_t)j * m + i] * x[c0 + i];
      x[c0 + j] = v / Lp[(size_t)j * m + j];
    }
  }
}

/* Solves (L L^T) x = b for nrhs right-hand sides stored column by column (leading
 * dimension n), all in the permuted ordering. */
void swc_oracle_solve(int n, const size_t *lC, const int *Ls, const size_t *Li_ptr,
                      const double *lValues, const int *blockSet, int supNo, double *x,
                      int nrhs) {
  for (int k = 0; k < nrhs; ++k) {
    lsolve(lC, Ls, Li_ptr, lValues, blockSet, supNo, x + (size_t)k * n);
    ltsolve(lC, Ls, Li_ptr, lValues, blockSet, supNo, x + (size_t)k * n);
  }
}

/* y = A x for the symmetric matrix whose lower triangle is the CSC (c, r, values). */
void swc_oracle_symv(int n, const int *c, const int *r, const double *values,
                     const double *x, double *y) {
  memset(y, 0, sizeof(double) * (size_t)n);
  for (int j = 0; j < n; ++j)
    for (int p = c[j]; p < c[j + 1]; ++p) {
      int i = r[p];
      y[i] += values[p] * x[j];
      if (i != j) y[j] += values[p] * x[i];
    }
}
