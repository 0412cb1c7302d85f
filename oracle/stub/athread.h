/* Host stand-in for the Sunway athread runtime header, used only to compile the
 * reference numeric executor on x86 for the test oracle.  The reference calls
 * athread_init() once per factorization (cholesky/sw_parallel_PB_Cholesky_05_check.c:57);
 * on the host there is no CPE cluster to bring up, so it does nothing. */
#ifndef SWC_ORACLE_ATHREAD_STUB_H
#define SWC_ORACLE_ATHREAD_STUB_H
static inline int athread_init(void) { return 0; }
#endif
