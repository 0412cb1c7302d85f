/* Prototypes for the BLAS/LAPACK symbols the reference executor calls without
 * declaring them; force-included when compiling that file for the oracle. */
#ifndef SWC_ORACLE_BLAS_SHIM_H
#define SWC_ORACLE_BLAS_SHIM_H
void dsyrk_(const char *, const char *, const int *, const int *, const double *,
            const double *, const int *, const double *, double *, const int *);
void dgemm_(const char *, const char *, const int *, const int *, const int *,
            const double *, const double *, const int *, const double *, const int *,
            const double *, double *, const int *);
void dpotrf_(const char *, const int *, double *, const int *, int *);
void dtrsm_(const char *, const char *, const char *, const char *, const int *,
            const int *, const double *, const double *, const int *, double *,
            const int *);
#endif
