// Centre block-Jacobi local preconditioner ('cjacobi', MEX prec = 1).
#pragma once
#include "kernels.h"

namespace ttg {

// Largest mode size the one-CTA block LU handles (n x n FP64 in shared memory).
constexpr int64_t JAC_MAX_N = 128;

// J [rx1, n, n, rx2]: for every rank pair (i, k) the n x n block
//   inv( sum_{al,be} Phi1[i,i,al] A[al,:,:,be] Phi2[k,be,k] )
// stored at J[i + rx1 (j + n (m + n k))] (row j, column m).
// Phi1 [rx1, rx1, ra1], A [ra1, n, n, ra2], Phi2 [rx2, ra2, rx2].
// A singular block raises the context's factorization error slot.
void jac_gen_c_f64(Context* c, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1, int64_t ra2,
                   const double* Phi1, const double* A, const double* Phi2, double* J);

// y[i, j, k] = sum_m J[i, j, m, k] x[i, m, k]   (x, y natural layout, y != x).
void jac_apply_c_f64(Context* c, int64_t rx1, int64_t n, int64_t rx2, const double* J,
                     const double* x, double* y);

// All three block-Jacobi local preconditioners of solve/solve3d_2ml.m:21-70
// (prec = MEX code: 1 'cjacobi', 2 'ljacobi', 3 'rjacobi'):
//   1: n x n blocks per rank pair (i, k)          (layout as jac_gen_c_f64)
//   2: (rx1 n) x (rx1 n) blocks per k, J[(i,j), (a,m), k]  =
//      inv(sum_{al,be} Phi1[:,:,al] (x) A[al,:,:,be] Phi2[k,be,k])
//   3: (n rx2) x (n rx2) blocks per i, J[(j,k), (m,q), i]  =
//      inv(sum_{al,be} Phi1[i,i,al] A[al,:,:,be] (x) Phi2[:,be,:])
// jac_size() doubles for J; the 2 / 3 blocks must fit JAC_MAX_ELEMS.
constexpr int64_t JAC_MAX_ELEMS = int64_t(1) << 28;  // 2 GiB of FP64
int64_t jac_size(int prec, int64_t rx1, int64_t n, int64_t rx2);
void jac_gen_f64(Context* c, int prec, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1,
                 int64_t ra2, const double* Phi1, const double* A, const double* Phi2, double* J);
// y = P x (natural layouts, y != x); scratch: 2 rx1 n rx2 doubles (prec 3).
void jac_apply_f64(Context* c, int prec, int64_t rx1, int64_t n, int64_t rx2, const double* J,
                   const double* x, double* y, double* scratch);
// Invert nblocks contiguous B x B blocks in place (one-CTA Gauss-Jordan up
// to JAC_MAX_N, LU and B X = I beyond).
void inv_blocks_f64(Context* c, int64_t B, int64_t nblocks, double* J);

}  // namespace ttg
