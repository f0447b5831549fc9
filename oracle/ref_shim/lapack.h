/* Stand-in for MATLAB's lapack.h, written for this checker: the LAPACK
 * routines fmex/solve3d.c calls, bound to numpy's ILP64 OpenBLAS.  Test
 * infrastructure only. */
#ifndef TTG_REF_SHIM_LAPACK_H
#define TTG_REF_SHIM_LAPACK_H

#define dgeqrf_ scipy_dgeqrf_64_
#define dorgqr_ scipy_dorgqr_64_
#define dgesv_ scipy_dgesv_64_

void dgeqrf_(long* m, long* n, double* a, long* lda, double* tau, double* work, long* lwork,
             long* info);
void dorgqr_(long* m, long* n, long* k, double* a, long* lda, double* tau, double* work,
             long* lwork, long* info);
void dgesv_(long* n, long* nrhs, double* a, long* lda, long* ipiv, double* b, long* ldb,
            long* info);

#endif
