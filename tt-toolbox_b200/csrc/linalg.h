// FP64 dense factorizations on the device (QR, SVD, LU solve).
#pragma once
#include "kernels.h"

namespace ttg {

// Failures of the library factorizations (LAPACK info != 0) are accumulated
// into the context's device error slot 4 without a host round trip; call
// check_factorizations() after a sequence to turn them into an error.
void check_factorizations(Context* c);

// Thin QR of the m x n column-major A (lda = m): Q (m x k, ld m) and
// R (k x n, ld k), k = min(m, n).  A is not modified.  Householder QR with
// LAPACK's sign convention (geqrf/orgqr), as MATLAB's qr(A,0).
// lapack_signs = false lets tall inputs (m >= 4n, 8 <= n <= 96) take a
// shifted Cholesky QR (linalg.cu): the same factorization up to the signs of
// Q's columns and R's rows, which the TT sweeps treat as a gauge; inputs too
// close to rank deficiency for it fall back to the Householder QR.
int64_t qr_f64(Context* c, int64_t m, int64_t n, const double* A, double* Q, double* R,
               bool lapack_signs = false);

// Economy SVD A = U diag(S) VT of the m x n column-major A:
// U (m x k, ld m), S (k) on the device, VT (k x n, ld k), k = min(m, n).
// A is not modified.  Returns k.  Tall inputs (m >= 2n) are reduced by a QR
// first; wide inputs are transposed.
int64_t svd_f64(Context* c, int64_t m, int64_t n, const double* A, double* U, double* S,
                double* VT);

// The same economy SVD by cuSOLVER's bidiagonal QR (gesvd): the fallback
// of the rounding sweep when a Jacobi SVD reaches its sweep limit, as
// round.m:64-74 falls back to svds when MATLAB's svd does not converge.
int64_t svd_f64_fallback(Context* c, int64_t m, int64_t n, const double* A, double* U,
                         double* S, double* VT);

// Solve the square N x N system B X = RHS (nrhs columns) by LU with partial
// pivoting; RHS is overwritten by X.  B is not modified.
void lu_solve_f64(Context* c, int64_t N, const double* B, double* rhs, int64_t nrhs = 1);

// R = triu(A(0:k, 0:n)) (k x n, ld k) from a geqrf output (ld lda).
void extract_triu_f64(Context* c, int64_t k, int64_t n, const double* A, int64_t lda, double* R);

}  // namespace ttg
