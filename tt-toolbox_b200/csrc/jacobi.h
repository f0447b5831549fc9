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

}  // namespace ttg
