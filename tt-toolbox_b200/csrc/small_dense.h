// Single-CTA FP64 factorizations of small matrices (small_dense.cu).
#pragma once
#include "kernels.h"

namespace ttg {

// True when an m x n Householder QR fits in one CTA's shared memory.
bool small_qr_fits(int64_t m, int64_t n);
// Thin Householder QR in one CTA: Q (m x k, ld m), R (k x n, ld k).
void small_qr_f64(Context* c, int64_t m, int64_t n, const double* A, int64_t lda, double* Q,
                  double* R);
// Thin Householder QR of a skinny m x n matrix (n <= 8, any m >= n) in one
// CTA working from global memory: Q (m x n, ld m), R (n x n, ld n); the
// signs of k_house_qr / LAPACK.
bool skinny_qr_fits(int64_t m, int64_t n);
void skinny_qr_f64(Context* c, int64_t m, int64_t n, const double* A, int64_t lda, double* Q,
                   double* R);
// Cholesky factor of a shifted Gram matrix and its inverse, one CTA:
// R' R = G + shift_factor * trace(G) * I, Rinv = R^{-1} (n x n, ld n, upper).
// A non-positive pivot sets *flag (nullptr: the context's factorization
// error slot).
// X <- B^{-1} X (n x n B, n x nrhs X, column-major) by one-CTA LU with
// partial pivoting; an exactly zero pivot sets error slot 4.
bool lu_small_fits(int64_t n, int64_t nrhs);
void lu_small_f64(Context* c, int64_t n, const double* B, double* X, int64_t nrhs);
bool chol_inv_fits(int64_t n);
void chol_inv_f64(Context* c, int64_t n, const double* G, int64_t ldg, double shift_factor,
                  double* R, double* Rinv, int* flag = nullptr);
// One-sided Jacobi SVD of a square n x n matrix: U (n x n), S (n, descending),
// VT (n x n), all with leading dimension n.  via_transpose rotates the
// columns of A^T instead of A (same factors of A on output): for the R factor
// of a QR this is the Drmac-Veselic preconditioned Jacobi, which needs far
// fewer sweeps when the singular values decay (about 9 instead of 20-28 at a
// decay of 1e-8 to 1e-14 over 50-64 columns).
void jacobi_svd_f64(Context* c, int64_t n, const double* A, int64_t lda, double* U, double* S,
                    double* VT, bool via_transpose = false);
// One-sided Jacobi SVD of a tall m x n matrix (m >= n, n <= 8, m n <= 16384)
// rotated directly in one CTA: U (m x n, ld m, orthonormal columns), S (n,
// descending), VT (n x n, ld n).
bool svd_tall_small_fits(int64_t m, int64_t n);
void svd_tall_small_f64(Context* c, int64_t m, int64_t n, const double* A, int64_t lda, double* U,
                        double* S, double* VT);

}  // namespace ttg
