/* Stand-in for MATLAB's blas.h, written for this checker: the BLAS routines
 * fmex/solve3d.c calls, bound to the ILP64 OpenBLAS that numpy ships
 * (symbols scipy_<name>_64_, 64-bit integers -- the reference passes
 * `long` everywhere).  Test infrastructure only. */
#ifndef TTG_REF_SHIM_BLAS_H
#define TTG_REF_SHIM_BLAS_H

#define dcopy_ scipy_dcopy_64_
#define daxpy_ scipy_daxpy_64_
#define dscal_ scipy_dscal_64_
#define ddot_ scipy_ddot_64_
#define dnrm2_ scipy_dnrm2_64_
#define dgemv_ scipy_dgemv_64_
#define dgemm_ scipy_dgemm_64_
#define dtrsv_ scipy_dtrsv_64_

void dcopy_(long* n, double* x, long* incx, double* y, long* incy);
void daxpy_(long* n, double* a, double* x, long* incx, double* y, long* incy);
void dscal_(long* n, double* a, double* x, long* incx);
double ddot_(long* n, double* x, long* incx, double* y, long* incy);
double dnrm2_(long* n, double* x, long* incx);
void dgemv_(char* trans, long* m, long* n, double* alpha, double* a, long* lda, double* x,
            long* incx, double* beta, double* y, long* incy);
void dgemm_(char* ta, char* tb, long* m, long* n, long* k, double* alpha, double* a, long* lda,
            double* b, long* ldb, double* beta, double* c, long* ldc);
void dtrsv_(char* uplo, char* trans, char* diag, long* n, double* a, long* lda, double* x,
            long* incx);

#endif
