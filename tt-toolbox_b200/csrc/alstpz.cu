// ALS(t+z) solver on the device: restates solve/alstpz_solve.m on its
// default path (kicktype 'svd', the MEX local solver, no symmetrisation).
//
// Every sweep (there is no convergence test: all nswp sweeps run, :138):
//   x = round(x, tol)                                     (:140)
//   z = round(y - A x, tol, kickrank)                     (:189-195)
//   x = x + 0 z   (z's directions join x's bases, weight zero; :199-201)
//   one ALS sweep (als_solve, :217-428): right-to-left QR orthogonalisation
//   with interfaces, then left-to-right local solves, each solution split by
//   QR into the next core.
// The rounding, the exact residual and the rank concatenation are the
// library's device TT algebra (round.cu, tt_algebra.cu); the local solve is
// the MEX solver's (amen.cu: local_solve, solve3d_2.c:254-279); interfaces
// are the reference's compute_next_Phi without normalisation (the reference
// calls it with one output, :297-298, :396-397).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <vector>

#include "amen.h"
#include "linalg.h"
#include "local_ops.h"
#include "round.h"

namespace ttg {

namespace {

// Status of a C-ABI call made from inside the library, as an error.
void ok(int code) {
  if (code != TTG_OK) fail(code, "%s", ttg_last_error());
}

struct Owned {  // a TT handle freed at scope exit
  ttg_tt_s* t = nullptr;
  explicit Owned(ttg_tt_s* h = nullptr) : t(h) {}
  Owned(const Owned&) = delete;
  Owned& operator=(const Owned&) = delete;
  ~Owned() {
    if (t) ttg_tt_free(t);
  }
  ttg_tt_s* release() {
    ttg_tt_s* h = t;
    t = nullptr;
    return h;
  }
};

// One ALS sweep (als_solve, solve/alstpz_solve.m:217-428) on the cores crx
// (ranks rx), in place.  res_prev / dx of every core go to the device slots
// sl[3 i + 0..2] (res_prev, ||sol - sol_prev||, ||sol||).
void als_sweep(Context* c, ttg_tt_s* A, ttg_tt_s* y, double tol, const ttg_amen_opts& o,
               std::vector<DBuf<double>>& crx, std::vector<int64_t>& rx, double* sl,
               int64_t* gmres_iters, int64_t* local_solves) {
  const int64_t d = y->d;
  const std::vector<int64_t>& n = y->n;
  const std::vector<int64_t>& ry = y->r;
  const std::vector<int64_t>& ra = A->r;
  auto cry = [&](int64_t k) { return y->core + y->ps[k]; };
  auto crA = [&](int64_t k) { return A->core + A->ps[k]; };
  std::vector<DBuf<double>> phia(d + 1), phiy(d + 1);
  for (int64_t k : {int64_t(0), d}) {                                   // :270-271
    phia[k].reset(c, 1);
    fill_f64(c, 1, 1.0, phia[k].p());
    phiy[k].reset(c, 1);
    fill_f64(c, 1, 1.0, phiy[k].p());
  }
  // Orthogonalisation (:286-299)
  for (int64_t i = d - 1; i >= 1; --i) {
    const int64_t ncols = n[i] * rx[i + 1];
    DBuf<double> crT(c, ncols * rx[i]);
    transpose_f64(c, rx[i], ncols, crx[i].p(), rx[i], crT.p(), ncols);
    const int64_t kq = std::min(ncols, rx[i]);
    DBuf<double> Q(c, ncols * kq), rv(c, kq * rx[i]);
    qr_f64(c, ncols, rx[i], crT.p(), Q.p(), rv.p());                   // :288
    const int64_t m2 = rx[i - 1] * n[i - 1];
    DBuf<double> cr2(c, m2 * kq);
    gemm_f64(c, false, true, m2, kq, rx[i], 1.0, crx[i - 1].p(), m2, 0, rv.p(), kq, 0, 0.0,
             cr2.p(), m2, 0, 1);                                        // :289-291
    rx[i] = kq;                                                         // :292
    crx[i].reset(c, kq * ncols);
    transpose_f64(c, ncols, kq, Q.p(), ncols, crx[i].p(), kq);          // :293
    crx[i - 1] = std::move(cr2);                                        // :294
    phia[i].reset(c, rx[i] * ra[i] * rx[i]);                            // :297
    next_phi_f64(c, 1, rx[i], n[i], rx[i + 1], rx[i], rx[i + 1], ra[i], ra[i + 1],
                 phia[i + 1].p(), crx[i].p(), crA(i), crx[i].p(), phia[i].p());
    phiy[i].reset(c, ry[i] * rx[i]);                                    // :298
    next_phi_f64(c, 1, rx[i], n[i], rx[i + 1], ry[i], ry[i + 1], 1, 1, phiy[i + 1].p(),
                 crx[i].p(), nullptr, cry(i), phiy[i].p());
  }
  const double real_tol = (tol / std::sqrt(double(d))) / o.resid_damp;   // :318
  DBuf<double> s2(c, 2);
  for (int64_t i = 0; i < d; ++i) {                                     // :305
    const double* Phi1 = phia[i].p();
    const double* Phi2 = phia[i + 1].p();
    MvDims md{rx[i], rx[i], ra[i], n[i], n[i], rx[i + 1], ra[i + 1], rx[i + 1]};
    const int64_t N = md.in_size();
    // rhs = phiy_i * y_i * phiy_{i+1}  (:311-316)
    DBuf<double> t(c, rx[i] * n[i] * ry[i + 1]), rhs(c, N);
    gemm_f64(c, false, false, rx[i], n[i] * ry[i + 1], ry[i], 1.0, phiy[i].p(), rx[i], 0, cry(i),
             ry[i], 0, 0.0, t.p(), rx[i], 0, 1);
    gemm_f64(c, false, false, rx[i] * n[i], rx[i + 1], ry[i + 1], 1.0, t.p(), rx[i] * n[i], 0,
             phiy[i + 1].p(), ry[i + 1], 0, 0.0, rhs.p(), rx[i] * n[i], 0, 1);
    dot_f64(c, N, rhs.p(), nullptr, s2.p() + 1, true);                  // :317 norm_rhs
    const double* sol_prev = crx[i].p();                                // :319
    DBuf<double> sol(c, N), res(c, N);
    const bool full = N < o.max_full_size;                              // :321
    DBuf<double> B;
    if (full) {                                                         // :322-336
      B.reset(c, N * N);
      assemble_local_f64(c, rx[i], n[i], rx[i + 1], ra[i], ra[i + 1], Phi1, crA(i), Phi2, B.p());
      gemm_f64(c, false, false, N, 1, N, 1.0, B.p(), N, 0, sol_prev, N, 0, 0.0, res.p(), N, 0, 1);
    } else {                                                            // :341
      local_matvec_f64(c, md, Phi1, crA(i), Phi2, sol_prev, res.p());
    }
    axpby_f64(c, N, -1.0, rhs.p(), 1.0, res.p());                       // B sol_prev - rhs
    dot_f64(c, N, res.p(), nullptr, s2.p(), true);
    double h[2];
    read_scalars(c, s2.p(), h, 2);
    const double res_prev = h[0] / h[1];                                // :333, :341
    fill_f64(c, 1, res_prev, sl + 3 * i);
    if (res_prev > real_tol) {
      if (full) {
        copy_f64(c, N, rhs.p(), sol.p());
        lu_solve_f64(c, N, B.p(), sol.p(), 1);                          // :335
      } else {                                                          // :344-349
        LocalSolveResult lr = local_solve(c, md, Phi1, crA(i), Phi2, rhs.p(), real_tol, sol_prev,
                                          o.local_restart, o.local_iters, sol.p(), o.precision,
                                          o.local_prec);
        *gmres_iters += lr.iters;
        *local_solves += 1;
      }
    } else {
      copy_f64(c, N, sol_prev, sol.p());
    }
    diffnrm_f64(c, N, sol.p(), sol_prev, sl + 3 * i + 1, true);          // :371
    dot_f64(c, N, sol.p(), nullptr, sl + 3 * i + 2, true);
    if (i < d - 1) {                                                    // :380-402
      const int64_t m = rx[i] * n[i];
      const int64_t k = std::min(m, rx[i + 1]);
      DBuf<double> u(c, m * k), v(c, k * rx[i + 1]);
      qr_f64(c, m, rx[i + 1], sol.p(), u.p(), v.p());                   // :380
      const int64_t nc = n[i + 1] * rx[i + 2];
      DBuf<double> v2(c, k * nc);
      gemm_f64(c, false, false, k, nc, rx[i + 1], 1.0, v.p(), k, 0, crx[i + 1].p(), rx[i + 1], 0,
               0.0, v2.p(), k, 0, 1);                                   // :390
      rx[i + 1] = k;                                                    // :400
      crx[i] = std::move(u);                                            // :401
      crx[i + 1] = std::move(v2);                                       // :402
      phia[i + 1].reset(c, rx[i + 1] * ra[i + 1] * rx[i + 1]);          // :396
      next_phi_f64(c, 0, rx[i], n[i], rx[i + 1], rx[i], rx[i + 1], ra[i], ra[i + 1], phia[i].p(),
                   crx[i].p(), crA(i), crx[i].p(), phia[i + 1].p());
      phiy[i + 1].reset(c, rx[i + 1] * ry[i + 1]);                      // :397
      next_phi_f64(c, 0, rx[i], n[i], rx[i + 1], ry[i], ry[i + 1], 1, 1, phiy[i].p(), crx[i].p(),
                   nullptr, cry(i), phiy[i + 1].p());
    } else {
      crx[i] = std::move(sol);                                          // :405
    }
  }
}

// A new tensor handle holding the cores crx (ranks rx).
ttg_tt_s* assemble_tt(Context* c, const std::vector<int64_t>& n, const std::vector<int64_t>& rx,
                      const std::vector<DBuf<double>>& crx) {
  std::unique_ptr<ttg_tt_s> t(new ttg_tt_s());
  t->ctx = c;
  t->d = int64_t(n.size());
  t->is_matrix = false;
  t->n = n;
  t->r = rx;
  t->ps.assign(t->d + 1, 0);
  for (int64_t k = 0; k < t->d; ++k) t->ps[k + 1] = t->ps[k] + rx[k] * n[k] * rx[k + 1];
  t->numel = t->ps[t->d];
  t->core = static_cast<double*>(c->alloc->get(sizeof(double) * std::max<int64_t>(t->numel, 1)));
  Owned guard(t.release());  // freed with its core if a copy launch fails
  for (int64_t k = 0; k < guard.t->d; ++k)
    copy_f64(c, guard.t->ps[k + 1] - guard.t->ps[k], crx[k].p(), guard.t->core + guard.t->ps[k]);
  return guard.release();
}

}  // namespace

ttg_tt_s* alstpz_solve(Context* c, ttg_tt_s* A, ttg_tt_s* y, double tol, const ttg_amen_opts& o,
                       ttg_tt_s* x0, ttg_amen_stats* stats) {
  TTG_REQUIRE(A->is_matrix, "A must be a TT matrix");
  TTG_REQUIRE(!y->is_matrix, "y must be a TT tensor");
  TTG_REQUIRE(y->ctx == A->ctx && y->ctx == c, "A and y belong to different contexts");
  TTG_REQUIRE(A->d == y->d, "A.d != y.d");
  const int64_t d = y->d;
  TTG_REQUIRE(d >= 2, "alstpz_solve needs d >= 2");
  for (int64_t k = 0; k < d; ++k) {
    TTG_REQUIRE(A->n[k] == A->m[k], "alstpz_solve needs a square operator (core %lld)",
                (long long)k);
    TTG_REQUIRE(A->n[k] == y->n[k], "mode size mismatch at core %lld", (long long)k);
  }
  TTG_REQUIRE(A->r[0] == 1 && A->r[d] == 1 && y->r[0] == 1 && y->r[d] == 1,
              "border ranks must be 1");
  TTG_REQUIRE(o.nswp >= 1 && o.nswp <= TTG_MAX_SWEEPS_RECORDED && o.local_restart >= 1 &&
                  o.local_iters >= 1 && o.kickrank >= 0 && o.resid_damp > 0,
              "invalid options");
  TTG_REQUIRE(o.local_prec >= 0 && o.local_prec <= 3, "local_prec %d is unknown", o.local_prec);
  TTG_REQUIRE(3 * d <= 4096, "alstpz_solve: d = %lld cores is more than the per-sweep "
              "residual read holds (1365)", (long long)d);
  TTG_REQUIRE(o.precision == TTG_FP64 || o.precision == TTG_MIXED, "unknown precision %d",
              o.precision);
  TTG_REQUIRE(o.local_prec <= 1 || o.precision == TTG_FP64,
              "'ljacobi' and 'rjacobi' run with precision TTG_FP64 only");
  require_finite(A, "A");
  require_finite(y, "y");
  if (x0) {
    TTG_REQUIRE(!x0->is_matrix && x0->d == d && x0->ctx == c, "x0 shape mismatch");
    for (int64_t k = 0; k < d; ++k) TTG_REQUIRE(x0->n[k] == y->n[k], "x0 mode size mismatch");
    TTG_REQUIRE(x0->r[0] == 1 && x0->r[d] == 1, "x0 border ranks must be 1");
    require_finite(x0, "x0");
  }
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t la0 = c->launches;
  // x = tt_rand(n, d, 2) when no initial guess is given (:116-118)
  Owned x;
  if (x0) {
    std::vector<DBuf<double>> cr(d);
    for (int64_t k = 0; k < d; ++k) {
      const int64_t sz = x0->ps[k + 1] - x0->ps[k];
      cr[k].reset(c, sz);
      copy_f64(c, sz, x0->core + x0->ps[k], cr[k].p());
    }
    x.t = assemble_tt(c, y->n, x0->r, cr);
  } else {
    x.t = tt_rand_device(c, y->n, 2, o.seed);
  }
  DBuf<double> sl(c, 3 * d);
  int64_t gmres_iters = 0, local_solves = 0, sweeps = 0;
  std::vector<double> max_res, max_dx;
  for (int64_t swp = 0; swp < o.nswp; ++swp) {                          // :138
    Owned xr(round_tt(x.t, tol, {}, TTG_FP64, nullptr));                // :140
    ttg_tt_free(x.release());
    if (o.kickrank > 0) {                                               // :189-201
      ttg_tt_s* ax = nullptr;
      ok(ttg_tt_matvec(A, xr.t, &ax));
      Owned Ax(ax);
      ttg_tt_s* zz = nullptr;
      ok(ttg_tt_axpby(1.0, y, -1.0, Ax.t, &zz));                        // y - A*x
      Owned ZZ(zz);
      Owned z(round_tt(ZZ.t, tol, {o.kickrank}, TTG_FP64, nullptr));
      ttg_tt_s* xe = nullptr;
      ok(ttg_tt_axpby(1.0, xr.t, 0.0, z.t, &xe));                       // x + 0*z
      ttg_tt_free(xr.release());
      xr.t = xe;
    }
    std::vector<int64_t> rx = xr.t->r;
    std::vector<DBuf<double>> crx(d);
    for (int64_t k = 0; k < d; ++k) {
      const int64_t sz = xr.t->ps[k + 1] - xr.t->ps[k];
      crx[k].reset(c, sz);
      copy_f64(c, sz, xr.t->core + xr.t->ps[k], crx[k].p());
    }
    als_sweep(c, A, y, tol, o, crx, rx, sl.p(), &gmres_iters, &local_solves);
    x.t = assemble_tt(c, y->n, rx, crx);
    std::vector<double> h(3 * d);
    read_scalars(c, sl.p(), h.data(), int(3 * d));
    double mr = 0.0, md = 0.0;
    for (int64_t i = 0; i < d; ++i) {
      mr = std::max(mr, h[3 * i]);                                      // :373
      md = std::max(md, h[3 * i + 2] > 0 ? h[3 * i + 1] / h[3 * i + 2] : 0.0);  // :371-372
    }
    max_res.push_back(mr);
    max_dx.push_back(md);
    ++sweeps;
    if (o.verb)
      fprintf(stderr, "=alstpz_solve= sweep %lld, max_dx: %3.3e, max_res: %3.3e, mrank: %lld\n",
              (long long)sweeps, md, mr,
              (long long)*std::max_element(x.t->r.begin(), x.t->r.end()));
  }
  if (stats) {
    *stats = ttg_amen_stats{};
    stats->sweeps = sweeps;
    for (int64_t s = 0; s < sweeps && s < TTG_MAX_SWEEPS_RECORDED; ++s) {
      stats->max_res[s] = max_res[s];
      stats->max_dx[s] = max_dx[s];
    }
    stats->local_solves = local_solves;
    stats->gmres_iters = gmres_iters;
    stats->max_rank = *std::max_element(x.t->r.begin(), x.t->r.end());
    stats->launches = c->launches - la0;
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return x.release();
}

}  // namespace ttg
