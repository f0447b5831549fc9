// Local Krylov solvers.
#pragma once
#include <functional>

#include "local_ops.h"

namespace ttg {

// y = B x for the local operator (any precision); x, y device vectors of sz.
using ApplyFn = std::function<void(const double* x, double* y)>;

struct GmresResult {
  int64_t iters = 0;    // Krylov steps
  int64_t matvecs = 0;  // operator applications
  double relres = 0.0;  // final estimate |tau|/||r0||
};

// Right-preconditioned GMRES with Householder Arnoldi and Givens rotations,
// the algorithm of fmex/solve3d.c:339-518 (dgmresr_hh), no preconditioner.
// Starts from sol = 0; stops when |tau_{j+1}|/||rhs|| < tol or after niters
// restarts of nrestart steps.  sol (device, sz) receives the solution.
GmresResult gmres_hh_f64(Context* c, const ApplyFn& apply, const double* rhs, int64_t sz,
                         int64_t nrestart, double tol, int64_t niters, double* sol);

}  // namespace ttg
