// Single-CTA FP64 factorizations of small matrices (small_dense.cu).
#pragma once
#include "kernels.h"

namespace ttg {

// True when an m x n Householder QR fits in one CTA's shared memory.
bool small_qr_fits(int64_t m, int64_t n);
// Thin Householder QR in one CTA: Q (m x k, ld m), R (k x n, ld k).
void small_qr_f64(Context* c, int64_t m, int64_t n, const double* A, int64_t lda, double* Q,
                  double* R);
// Batch of one-CTA QRs: matrix b is m x n at A + b sA (lda); Q_b (m x k,
// ld m) at Q + b sQ; R_b (k x n, leading dimension ldr) at R + b sR.
void small_qr_batched_f64(Context* c, int64_t batch, int64_t m, int64_t n, const double* A,
                          int64_t lda, int64_t sA, double* Q, int64_t sQ, double* R, int64_t ldr,
                          int64_t sR);
// Most rows an n-column one-CTA QR can hold.
int64_t small_qr_max_rows(int64_t n);
// One-sided Jacobi SVD of a square n x n matrix: U (n x n), S (n, descending),
// VT (n x n), all with leading dimension n.
void jacobi_svd_f64(Context* c, int64_t n, const double* A, int64_t lda, double* U, double* S,
                    double* VT);

}  // namespace ttg
