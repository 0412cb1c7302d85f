/* Test oracle only.  The reference numeric executor, built with -DXMATH, calls the
 * Fortran BLAS/LAPACK symbols dsyrk_/dgemm_/dpotrf_/dtrsm_
 * (cholesky/sw_parallel_PB_Cholesky_05_check.c:230,254,319,349).  On Sunway these come
 * from the closed xMath library (makefile:29).  Here they are routed to the OpenBLAS
 * that scipy ships (exported with a scipy_ prefix), which the linker resolves at build
 * time.  The shim adds nothing: it forwards every argument unchanged. */
#include <stddef.h>

void scipy_dsyrk_(const char *, const char *, const int *, const int *, const double *,
                  const double *, const int *, const double *, double *, const int *,
                  size_t, size_t);
void scipy_dgemm_(const char *, const char *, const int *, const int *, const int *,
                  const double *, const double *, const int *, const double *, const int *,
                  const double *, double *, const int *, size_t, size_t);
void scipy_dpotrf_(const char *, const int *, double *, const int *, int *, size_t);
void scipy_dtrsm_(const char *, const char *, const char *, const char *, const int *,
                  const int *, const double *, const double *, const int *, double *,
                  const int *, size_t, size_t, size_t, size_t);
void scipy_openblas_set_num_threads(int);

void dsyrk_(const char *uplo, const char *trans, const int *n, const int *k,
            const double *alpha, const double *a, const int *lda, const double *beta,
            double *c, const int *ldc) {
  scipy_dsyrk_(uplo, trans, n, k, alpha, a, lda, beta, c, ldc, 1, 1);
}

void dgemm_(const char *ta, const char *tb, const int *m, const int *n, const int *k,
            const double *alpha, const double *a, const int *lda, const double *b,
            const int *ldb, const double *beta, double *c, const int *ldc) {
  scipy_dgemm_(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, 1, 1);
}

void dpotrf_(const char *uplo, const int *n, double *a, const int *lda, int *info) {
  scipy_dpotrf_(uplo, n, a, lda, info, 1);
}

void dtrsm_(const char *side, const char *uplo, const char *ta, const char *diag,
            const int *m, const int *n, const double *alpha, const double *a,
            const int *lda, double *b, const int *ldb) {
  scipy_dtrsm_(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb, 1, 1, 1, 1);
}

void swc_ref_set_blas_threads(int t) { scipy_openblas_set_num_threads(t); }
