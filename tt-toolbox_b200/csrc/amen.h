#pragma once
#include "gmres.h"

namespace ttg {

// Local solve with the semantics of the MEX gateway solve3d_2, residual branch
// (fmex/solve3d_2.c:254-279): dres = rhs - B sol_prev, GMRES on dres with
// tolerance tol / max(||dres||/||rhs||, tol), sol = sol_prev + dsol.
// precision TTG_FP64 runs dgmresr_hh on FP64 matvecs; TTG_MIXED runs the
// low-precision Krylov solver inside an FP64 refinement loop.
struct LocalSolveResult {
  int64_t iters = 0;
  int64_t matvecs = 0;
  int64_t matvecs_fp64 = 0;
  // The solver's last FP64 refinement matvec was B sol for the returned sol
  // and was stored in the caller's bsol_out buffer.
  bool have_bsol = false;
};
LocalSolveResult local_solve(Context* c, const MvDims& d, const double* Phi1, const double* A,
                             const double* Phi2, const double* rhs, double tol,
                             const double* sol_prev, int64_t nrestart, int64_t niters,
                             double* sol, int precision, int prec = 0);

// Solve on context c (its stream, allocator and solver handle); the inputs
// may belong to another context of the same device.  The result handle
// belongs to out_ctx (nullptr: c) and its core is drawn from out_ctx's
// allocator.
ttg_tt_s* amen_solve(Context* c, ttg_tt_s* A, ttg_tt_s* y, double tol, const ttg_amen_opts& o,
                     ttg_tt_s* x0, ttg_tt_s* z0, ttg_amen_stats* stats,
                     Context* out_ctx = nullptr);

// ALS(t+z) solve of solve/alstpz_solve.m (kicktype 'svd'): nswp sweeps of
// rounding, residual enrichment of rank kickrank and one ALS sweep.  Uses
// the fields nswp, max_full_size, local_restart, local_iters, kickrank,
// resid_damp, local_prec, precision, verb and seed of o.  Stats: sweeps,
// per-sweep max_res / max_dx, local solves, Krylov steps, max rank,
// launches, host-clock time.
ttg_tt_s* alstpz_solve(Context* c, ttg_tt_s* A, ttg_tt_s* y, double tol, const ttg_amen_opts& o,
                       ttg_tt_s* x0, ttg_amen_stats* stats);

// Right-orthogonal random TT of rank r (tt_rand(n,d,r,-1), core/tt_rand.m:40-62)
// with entries from the device hash generator.
ttg_tt_s* tt_rand_device(Context* c, const std::vector<int64_t>& n, int64_t r, uint64_t seed);

}  // namespace ttg
