// Mixed-precision local solve: low-precision Krylov solver inside an FP64
// iterative-refinement loop on the local residual.
#pragma once
#include "amen.h"

namespace ttg {

// dres = rhs - B sol_prev (FP64), nres = ||dres||, nrhs = ||rhs|| are given.
// bsol_out (nullable, N doubles): receives B sol (FP64) when the refinement
// loop computed it for the returned sol (result.have_bsol).  prec 1: the
// centre block-Jacobi right preconditioner ('cjacobi') in the low-precision
// Krylov solves and in the FP64 fallback.
LocalSolveResult local_solve_mixed(Context* c, const MvDims& d, const double* Phi1,
                                   const double* A, const double* Phi2, const double* rhs,
                                   const double* dres, double nres, double nrhs, double tol,
                                   const double* sol_prev, int64_t nrestart, int64_t niters,
                                   double* sol, double* bsol_out = nullptr, int prec = 0);

}  // namespace ttg
