// AMEn solver on the device: restates solve/amen_solve2.m:67-831 on its
// default option path (kicktype 'als', trunc_norm 'residual', no local
// preconditioner, MEX local solver).
//
// All cores, interfaces (Phi) and local vectors live on the device, and so
// does the scalar bookkeeping of the reference (nrmsa/nrmsy/nrmsx/nrmsc,
// the local residuals and the per-sweep maxima): small device kernels update
// it in stream order.  The host reads device values only where the
// algorithm branches on them: the local-solve tolerance (one read per core),
// the rank of the residual-based truncation (one read per chunk of 16
// candidates), the Krylov stopping test, and the per-sweep stopping test.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "amen.h"
#include "jacobi.h"
#include "linalg.h"
#include "mixed.h"
#include "round.h"

namespace ttg {

LocalSolveResult local_solve_from_residual(Context* c, const MvDims& d, const double* Phi1,
                                           const double* A, const double* Phi2,
                                           const double* rhs, const double* dres, double nres,
                                           double nrhs, double tol, const double* sol_prev,
                                           int64_t nrestart, int64_t niters, double* sol,
                                           int precision, int prec = 0,
                                           double* bsol_out = nullptr) {
  TTG_REQUIRE(prec >= 0 && prec <= 3,
              "local preconditioner %d is unknown (0 none, 1 'cjacobi', 2 'ljacobi', "
              "3 'rjacobi')", prec);
  if (precision == TTG_MIXED) {
    TTG_REQUIRE(prec == 0 || prec == 1,
                "the mixed-precision local solve has the 'cjacobi' preconditioner only");
    return local_solve_mixed(c, d, Phi1, A, Phi2, rhs, dres, nres, nrhs, tol, sol_prev, nrestart,
                             niters, sol, bsol_out, prec);
  }
  LocalSolveResult out;
  const int64_t sz = d.in_size();
  if (nrestart > sz) nrestart = sz;                                   // solve3d_2.c:184
  DBuf<double> t1(c, d.t1_size()), t2(c, d.t2_size()), J, pw, js;
  if (prec != 0) {                                                    // solve3d_2.c:212-231
    J.reset(c, jac_size(prec, d.rx1, d.n, d.rx2));
    pw.reset(c, sz);
    if (prec == 3) js.reset(c, 2 * sz);
    jac_gen_f64(c, prec, d.rx1, d.n, d.rx2, d.ra1, d.ra2, Phi1, A, Phi2, J.p());
  }
  auto mv = [&](const double* x, double* y) {
    if (prec != 0) {  // right preconditioning: B P x
      jac_apply_f64(c, prec, d.rx1, d.n, d.rx2, J.p(), x, pw.p(), js.p());
      local_matvec_f64(c, d, Phi1, A, Phi2, pw.p(), y, t1.p(), t2.p());
    } else {
      local_matvec_f64(c, d, Phi1, A, Phi2, x, y, t1.p(), t2.p());
    }
  };
  double tol_prev = nres / nrhs;                                      // :263
  if (tol_prev < tol) tol_prev = tol;                                 // :264
  GmresResult g = gmres_hh_f64(c, mv, dres, sz, nrestart, tol / tol_prev, niters, sol);  // :267
  if (prec != 0) {                                                    // :272-274
    jac_apply_f64(c, prec, d.rx1, d.n, d.rx2, J.p(), sol, pw.p(), js.p());
    copy_f64(c, sz, pw.p(), sol);
  }
  axpby_f64(c, sz, 1.0, sol_prev, 1.0, sol);                          // :277-278
  out.iters = g.iters;
  out.matvecs_fp64 += g.matvecs;
  return out;
}

LocalSolveResult local_solve(Context* c, const MvDims& d, const double* Phi1, const double* A,
                             const double* Phi2, const double* rhs, double tol,
                             const double* sol_prev, int64_t nrestart, int64_t niters,
                             double* sol, int precision, int prec) {
  const int64_t sz = d.in_size();
  DBuf<double> dres(c, sz), s2(c, 2);
  local_matvec_f64(c, d, Phi1, A, Phi2, sol_prev, dres.p());          // solve3d_2.c:257
  axpby_f64(c, sz, 1.0, rhs, -1.0, dres.p());                         // :259-262
  dot_f64(c, sz, dres.p(), nullptr, s2.p(), true);
  dot_f64(c, sz, rhs, nullptr, s2.p() + 1, true);
  double h[2];
  read_scalars(c, s2.p(), h, 2);
  LocalSolveResult r = local_solve_from_residual(c, d, Phi1, A, Phi2, rhs, dres.p(), h[0], h[1],
                                                 tol, sol_prev, nrestart, niters, sol, precision,
                                                 prec);
  r.matvecs_fp64 += 1;
  return r;
}

namespace {

struct Core {
  DBuf<double> buf;
  double* p() const { return buf.p(); }
};

// Optional phase breakdown (TTG_PROFILE=1): synchronises at phase
// boundaries and accumulates host-clock time per phase.
struct PhaseProf {
  bool on = false;
  Context* c = nullptr;
  std::chrono::steady_clock::time_point t0;
  std::map<std::string, double> ms;
  std::string name;
  void start(Context* cc) {
    const char* e = getenv("TTG_PROFILE");
    on = e && e[0] == '1';
    c = cc;
    fb0 = c->mixed_fallbacks;
  }
  void mark(const char* n) {
    if (!on) return;
    sync(c);
    auto t = std::chrono::steady_clock::now();
    if (!name.empty()) ms[name] += std::chrono::duration<double, std::milli>(t - t0).count();
    name = n;
    t0 = t;
  }
  int64_t fb0 = 0;
  void report() {
    if (!on) return;
    mark("");
    fprintf(stderr, "[ttg profile] mixed local solves finished in FP64: %lld\n",
            (long long)(c->mixed_fallbacks - fb0));
    double tot = 0;
    for (auto& kv : ms) tot += kv.second;
    for (auto& kv : ms)
      fprintf(stderr, "[ttg profile] %-14s %9.2f ms  (%4.1f%%)\n", kv.first.c_str(), kv.second,
              100.0 * kv.second / (tot > 0 ? tot : 1));
  }
};

// Device scalar slots of one solve.
struct Scalars {
  DBuf<double> buf;
  int64_t d = 0;
  enum Fixed : int64_t {
    NRMSC = 0, NRHS, RES_PREV, RES_NEW, THR, MAXRES, MAXDX, T0, T1, T2, T3, NFIXED
  };
  static constexpr int64_t NCAND = 64;  // candidate residual slots
  double* p(int64_t k) const { return buf.p() + k; }
  double* a(int64_t i) const { return buf.p() + NFIXED + NCAND + i; }            // nrmsa
  double* y(int64_t i) const { return buf.p() + NFIXED + NCAND + (d - 1) + i; }  // nrmsy
  double* x(int64_t i) const { return buf.p() + NFIXED + NCAND + 2 * (d - 1) + i; }  // nrmsx
  double* cand(int64_t k) const { return buf.p() + NFIXED + k; }
  void init(Context* c, int64_t dd) {
    d = dd;
    const int64_t total = NFIXED + NCAND + 3 * (d - 1);
    buf.reset(c, total);
    fill_f64(c, total, 1.0, buf.p());                                 // :277-282
  }
};

// ||B x - rhs|| into *out (device), FP64 local matvec.
void local_residual_dev(Context* c, const MvDims& d, const double* Phi1, const double* A,
                        const double* Phi2, const double* x, const double* rhs, double* tmp,
                        double* t1, double* t2, double* out) {
  local_matvec_f64(c, d, Phi1, A, Phi2, x, tmp, t1, t2);
  diffnrm_f64(c, d.out_size(), tmp, rhs, out, true);
}

void dense_residual_dev(Context* c, int64_t N, const double* B, const double* x,
                        const double* rhs, double* tmp, double* out) {
  gemm_f64(c, false, false, N, 1, N, 1.0, B, N, 0, x, N, 0, 0.0, tmp, N, 0, 1);
  diffnrm_f64(c, N, tmp, rhs, out, true);
}

// Free a TT handle whose core the context's recorded work may still use.
void release_tt(Context* c, ttg_tt_s* t) {
  if (c->rec) {
    rec_free(c->rec, t->core, sizeof(double) * size_t(t->numel));
    delete t;
  } else {
    ttg_tt_free(t);
  }
}

// Normalise in place by the Frobenius norm, the norm (1 if zero) into *slot
// (compute_next_Phi with nargout > 1, amen_solve2.m:907-914).
void normalize_dev(Context* c, int64_t n, double* x, double* slot) {
  dot_f64(c, n, x, nullptr, slot, true);
  normalize_by_dev(c, n, x, slot);
}

}  // namespace

ttg_tt_s* tt_rand_device(Context* c, const std::vector<int64_t>& n, int64_t r, uint64_t seed) {
  const int64_t d = int64_t(n.size());
  std::vector<int64_t> rr(d + 1, r);
  rr[0] = 1;
  rr[d] = 1;
  std::vector<DBuf<double>> cores(d);
  uint64_t off = 0;
  for (int64_t i = d - 1; i >= 0; --i) {           // tt_rand.m:52-57 (RL)
    const int64_t m = n[i] * rr[i + 1], k0 = rr[i];
    DBuf<double> G(c, m * k0);
    randn_f64(c, m * k0, seed, off, G.p());
    off += uint64_t(m * k0);
    const int64_t k = std::min(m, k0);
    DBuf<double> Q(c, m * k), R(c, k * k0);
    qr_f64(c, m, k0, G.p(), Q.p(), R.p());
    rr[i] = k;
    cores[i].reset(c, k * m);
    transpose_f64(c, m, k, Q.p(), m, cores[i].p(), k);
  }
  auto* t = new ttg_tt_s();
  t->ctx = c;
  t->d = d;
  t->is_matrix = false;
  t->n = n;
  t->r = rr;
  t->ps.assign(d + 1, 0);
  for (int64_t k = 0; k < d; ++k) t->ps[k + 1] = t->ps[k] + rr[k] * n[k] * rr[k + 1];
  t->numel = t->ps[d];
  t->core = static_cast<double*>(c->alloc->get(sizeof(double) * t->numel));
  for (int64_t k = 0; k < d; ++k) copy_f64(c, t->ps[k + 1] - t->ps[k], cores[k].p(), t->core + t->ps[k]);
  sync(c);
  return t;
}

ttg_tt_s* amen_solve(Context* c, ttg_tt_s* Ah, ttg_tt_s* yh, double tol, const ttg_amen_opts& o,
                     ttg_tt_s* x0h, ttg_tt_s* z0h, ttg_amen_stats* stats, Context* out_ctx) {
  if (!out_ctx) out_ctx = c;
  TTG_REQUIRE(Ah->is_matrix, "A must be a TT matrix");
  TTG_REQUIRE(!yh->is_matrix, "y must be a TT tensor");
  TTG_REQUIRE(yh->ctx == Ah->ctx, "A and y belong to different contexts");
  TTG_REQUIRE(Ah->d == yh->d, "A.d != y.d");
  const int64_t d = yh->d;
  TTG_REQUIRE(d >= 2, "amen_solve needs d >= 2");
  for (int64_t k = 0; k < d; ++k) {
    TTG_REQUIRE(Ah->n[k] == Ah->m[k],
                "AMEn does not know how to solve rectangular systems (core %lld)", (long long)k);  // :216-218
    TTG_REQUIRE(Ah->n[k] == yh->n[k], "mode size mismatch at core %lld", (long long)k);
  }
  TTG_REQUIRE(Ah->r[0] == 1 && Ah->r[d] == 1 && yh->r[0] == 1 && yh->r[d] == 1,
              "border ranks must be 1");
  TTG_REQUIRE(o.trunc_norm == 1, "only trunc_norm 'residual' is implemented");
  TTG_REQUIRE(o.local_prec >= 0 && o.local_prec <= 3,
              "local_prec %d is unknown (0 = none, 1 'cjacobi', 2 'ljacobi', 3 'rjacobi')",
              o.local_prec);
  TTG_REQUIRE(o.local_prec <= 1 || o.precision == TTG_FP64,
              "'ljacobi' and 'rjacobi' run with precision TTG_FP64 only");
  TTG_REQUIRE(o.precision == TTG_FP64 || o.precision == TTG_MIXED, "unknown precision %d",
              o.precision);
  TTG_REQUIRE(o.nswp >= 1 && o.local_restart >= 1 && o.local_iters >= 1 && o.rmax >= 1 &&
                  o.kickrank >= 0,
              "invalid options");
  require_finite(c, {{Ah, "A"}, {yh, "y"}, {x0h, "x0"}, {z0h, "z0"}});
  const std::vector<int64_t> n = yh->n;
  const int64_t nswp = o.nswp, rmax = o.rmax, max_full_size = o.max_full_size;
  const int64_t kickrank = o.kickrank;
  const double resid_damp = o.resid_damp;
  const double tol_exit = o.tol_exit > 0 ? o.tol_exit : tol;            // :156-158
  const bool use_z = kickrank > 0;                                      // :246
  const double real_tol = (tol / std::sqrt(double(d))) / resid_damp;   // :466

  // Device time of the solve from an event pair; a solve of a grouped batch
  // (recorded stream work) takes the host clock instead.
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const auto host_t0 = std::chrono::steady_clock::now();
  if (!c->rec) {
    TTG_CUDA(cudaEventCreate(&e0));
    TTG_CUDA(cudaEventCreate(&e1));
    TTG_CUDA(cudaEventRecord(e0, c->stream));
  }
  const int64_t mv0 = c->matvecs, fl0 = c->matvec_flops, la0 = c->launches;
  const double flk0[2] = {c->mv_flops[0], c->mv_flops[1]};
  const double byl0 = c->mv_bytes_lp;
  const int64_t mvk0[2] = {c->mv_count[0], c->mv_count[1]};
  c->ev_collect();
  const double msk0[2] = {c->mv_ms[0], c->mv_ms[1]};
  c->time_matvec = o.timing != 0 && !c->rec;
  struct TimingOff {
    Context* c;
    ~TimingOff() { c->time_matvec = false; }
  } timing_off{c};
  memset_async(c, c->d_err, 0, 8 * sizeof(int));

  PhaseProf prof;
  prof.start(c);
  prof.mark("init");
  // Initial guesses (:222-224, :250-252).
  // Given guesses are checked before the random ones are drawn, so a
  // rejected call holds no device tensor.
  if (x0h) {
    TTG_REQUIRE(x0h->d == d && !x0h->is_matrix, "x0 shape mismatch");
    for (int64_t k = 0; k < d; ++k) TTG_REQUIRE(x0h->n[k] == n[k], "x0 mode size mismatch");
    TTG_REQUIRE(x0h->r[0] == 1 && x0h->r[d] == 1, "x0 border ranks must be 1");
  }
  if (use_z && z0h) {
    TTG_REQUIRE(z0h->d == d && !z0h->is_matrix, "z0 shape mismatch");
    for (int64_t k = 0; k < d; ++k) TTG_REQUIRE(z0h->n[k] == n[k], "z0 mode size mismatch");
    TTG_REQUIRE(z0h->r[0] == 1 && z0h->r[d] == 1, "z0 border ranks must be 1");
  }
  ttg_tt_s* x0own = nullptr;
  ttg_tt_s* z0own = nullptr;
  if (!x0h) x0h = x0own = tt_rand_device(c, n, 2, o.seed);
  if (use_z && !z0h) z0h = z0own = tt_rand_device(c, n, kickrank, o.seed ^ 0x5bd1e995ull);

  std::vector<int64_t> rx = x0h->r, ry = yh->r, ra = Ah->r, rz;
  std::vector<Core> crx(d), crz(d);
  for (int64_t k = 0; k < d; ++k) {
    const int64_t sz = x0h->ps[k + 1] - x0h->ps[k];
    crx[k].buf.reset(c, sz);
    copy_f64(c, sz, x0h->core + x0h->ps[k], crx[k].p());
  }
  if (use_z) {
    rz = z0h->r;
    for (int64_t k = 0; k < d; ++k) {
      const int64_t sz = z0h->ps[k + 1] - z0h->ps[k];
      crz[k].buf.reset(c, sz);
      copy_f64(c, sz, z0h->core + z0h->ps[k], crz[k].p());
    }
  }
  if (x0own) release_tt(c, x0own);
  if (z0own) release_tt(c, z0own);
  auto cry = [&](int64_t k) { return yh->core + yh->ps[k]; };
  auto crA = [&](int64_t k) { return Ah->core + Ah->ps[k]; };

  std::vector<Core> phia(d + 1), phiy(d + 1), phiza(d + 1), phizy(d + 1);
  for (int64_t k : {int64_t(0), d}) {                                   // :243-249
    for (auto* v : {&phia, &phiy, &phiza, &phizy}) {
      (*v)[k].buf.reset(c, 1);
      fill_f64(c, 1, 1.0, (*v)[k].p());
    }
  }
  Scalars S;
  S.init(c, d);                                  // nrmsa = nrmsy = nrmsx = nrmsc = 1 (:277-282)
  double* NC = S.p(Scalars::NRMSC);
  bool last_sweep = false;
  int64_t local_solves = 0, gmres_iters = 0, mv_fp64 = 0;
  int64_t swp_done = 0;
  int64_t trace_len = 0;

  for (int64_t swp = 1; swp <= nswp; ++swp) {                           // :296
    // ------------- right-to-left orthogonalisation (:299-438)
    int64_t rznew = 0;
    for (int64_t i = d - 1; i >= 1; --i) {
      prof.mark("rl_z");
      if (use_z && !last_sweep) {                                       // :301-324
        DBuf<double> zt;  // (n*rz_{i+1}) x k, to be orthogonalised
        int64_t kz = 0;
        const int64_t ncols = n[i] * rz[i + 1];
        if (swp > 1) {
          MvDims zd{rz[i], rx[i], ra[i], n[i], n[i], rx[i + 1], ra[i + 1], rz[i + 1]};
          DBuf<double> crzAt(c, zd.out_size());
          local_matvec_f64(c, zd, phiza[i].p(), crA(i), phiza[i + 1].p(), crx[i].p(), crzAt.p());
          mv_fp64++;
          DBuf<double> t(c, rz[i] * n[i] * ry[i + 1]), crzy(c, rz[i] * n[i] * rz[i + 1]);
          gemm_f64(c, false, false, rz[i], n[i] * ry[i + 1], ry[i], 1.0, phizy[i].p(), rz[i], 0,
                   cry(i), ry[i], 0, 0.0, t.p(), rz[i], 0, 1);
          gemm_f64(c, false, false, rz[i] * n[i], rz[i + 1], ry[i + 1], 1.0, t.p(), rz[i] * n[i], 0,
                   phizy[i + 1].p(), ry[i + 1], 0, 0.0, crzy.p(), rz[i] * n[i], 0, 1);
          axpby_dev(c, zd.out_size(), -1.0, crzAt.p(), NC, crzy.p());  // :309 crzy*nrmsc - crzAt
          const int64_t K = std::min(rz[i], ncols);
          DBuf<double> U(c, rz[i] * K), Sv(c, K), VT(c, K * ncols);
          svd_f64(c, rz[i], ncols, crzy.p(), U.p(), Sv.p(), VT.p());     // :311
          kz = std::min(kickrank, K);                                     // :312
          // The rows of V' are orthonormal, so the QR of :320 returns them
          // up to column signs (a gauge of z): they are the new core.
          rznew = kz;
          crz[i].buf.reset(c, kz * ncols);
          copy2d_f64(c, kz, ncols, VT.p(), K, crz[i].p(), kz);            // :322-323
        } else {
          kz = rz[i];
          zt.reset(c, ncols * kz);
          transpose_f64(c, rz[i], ncols, crz[i].p(), rz[i], zt.p(), ncols);  // :317
          const int64_t kq = std::min(ncols, kz);
          DBuf<double> Q(c, ncols * kq), R(c, kq * kz);
          qr_f64(c, ncols, kz, zt.p(), Q.p(), R.p());                    // :320
          rznew = kq;
          crz[i].buf.reset(c, kq * ncols);
          transpose_f64(c, ncols, kq, Q.p(), ncols, crz[i].p(), kq);     // :322-323
        }
      }
      if (swp > 1)                                                      // :325-328
        scalar_op(c, SC_NRMSC_DIV, NC, S.y(i - 1), S.a(i - 1), S.x(i - 1));
      prof.mark("rl_qr");
      // QR of x_i^T (:331-342)
      const int64_t ncols = n[i] * rx[i + 1];
      DBuf<double> crT(c, ncols * rx[i]);
      transpose_f64(c, rx[i], ncols, crx[i].p(), rx[i], crT.p(), ncols);
      const int64_t kq = std::min(ncols, rx[i]);
      DBuf<double> Q(c, ncols * kq), rv(c, kq * rx[i]);
      qr_f64(c, ncols, rx[i], crT.p(), Q.p(), rv.p());
      // cr2 = x_{i-1} * rv^T (:347-349)
      const int64_t m2 = rx[i - 1] * n[i - 1];
      DBuf<double> cr2(c, m2 * kq);
      gemm_f64(c, false, true, m2, kq, rx[i], 1.0, crx[i - 1].p(), m2, 0, rv.p(), kq, 0, 0.0,
               cr2.p(), m2, 0, 1);
      normalize_dev(c, m2 * kq, cr2.p(), S.p(Scalars::T0));            // :351-356
      scalar_op(c, SC_MUL, S.x(i - 1), S.p(Scalars::T0));              // :357
      rx[i] = kq;                                                         // :359
      crx[i].buf.reset(c, kq * ncols);
      transpose_f64(c, ncols, kq, Q.p(), ncols, crx[i].p(), kq);          // :360-362
      crx[i - 1].buf = std::move(cr2);
      prof.mark("rl_phi");
      // Interfaces (:364-365)
      phia[i].buf.reset(c, rx[i] * ra[i] * rx[i]);
      next_phi_f64(c, 1, rx[i], n[i], rx[i + 1], rx[i], rx[i + 1], ra[i], ra[i + 1],
                   phia[i + 1].p(), crx[i].p(), crA(i), crx[i].p(), phia[i].p());
      normalize_dev(c, rx[i] * ra[i] * rx[i], phia[i].p(), S.a(i - 1));
      phiy[i].buf.reset(c, ry[i] * rx[i]);
      next_phi_f64(c, 1, rx[i], n[i], rx[i + 1], ry[i], ry[i + 1], 1, 1, phiy[i + 1].p(),
                   crx[i].p(), nullptr, cry(i), phiy[i].p());
      normalize_dev(c, ry[i] * rx[i], phiy[i].p(), S.y(i - 1));
      scalar_op(c, SC_NRMSC_MUL, NC, S.y(i - 1), S.a(i - 1), S.x(i - 1));  // :372
      if (use_z && !last_sweep) {                                         // :432-436
        rz[i] = rznew;
        phiza[i].buf.reset(c, rx[i] * ra[i] * rz[i]);
        next_phi_f64(c, 1, rz[i], n[i], rz[i + 1], rx[i], rx[i + 1], ra[i], ra[i + 1],
                     phiza[i + 1].p(), crz[i].p(), crA(i), crx[i].p(), phiza[i].p());
        scale_dev_f64(c, rx[i] * ra[i] * rz[i], phiza[i].p(), phiza[i].p(), nullptr, S.a(i - 1));
        phizy[i].buf.reset(c, ry[i] * rz[i]);
        next_phi_f64(c, 1, rz[i], n[i], rz[i + 1], ry[i], ry[i + 1], 1, 1, phizy[i + 1].p(),
                     crz[i].p(), nullptr, cry(i), phizy[i].p());
        scale_dev_f64(c, ry[i] * rz[i], phizy[i].p(), phizy[i].p(), nullptr, S.y(i - 1));
      }
    }

    // ------------- left-to-right solve sweep (:444-791)
    fill_f64(c, 2, 0.0, S.p(Scalars::MAXRES));  // max_res = max_dx = 0 (:440-441)
    for (int64_t i = 0; i < d; ++i) {
      prof.mark("lr_rhs");
      const double* Phi1 = phia[i].p();
      const double* Phi2 = phia[i + 1].p();
      const double* A1 = crA(i);
      MvDims md{rx[i], rx[i], ra[i], n[i], n[i], rx[i + 1], ra[i + 1], rx[i + 1]};
      const int64_t N = md.in_size();
      const double* sol_prev = crx[i].p();
      // y1 = y_i * nrmsc (:453); rhs = phiy_i * y1 * phiy_{i+1} (:456-461)
      const int64_t ysz = ry[i] * n[i] * ry[i + 1];
      DBuf<double> y1(c, ysz);
      scale_dev_f64(c, ysz, cry(i), y1.p(), NC, nullptr);
      DBuf<double> t(c, rx[i] * n[i] * ry[i + 1]), rhs(c, N);
      gemm_f64(c, false, false, rx[i], n[i] * ry[i + 1], ry[i], 1.0, phiy[i].p(), rx[i], 0,
               y1.p(), ry[i], 0, 0.0, t.p(), rx[i], 0, 1);
      gemm_f64(c, false, false, rx[i] * n[i], rx[i + 1], ry[i + 1], 1.0, t.p(), rx[i] * n[i], 0,
               phiy[i + 1].p(), ry[i + 1], 0, 0.0, rhs.p(), rx[i] * n[i], 0, 1);
      dot_f64(c, N, rhs.p(), nullptr, S.p(Scalars::NRHS), true);         // :462
      prof.mark("lr_solve");
      const bool full = N < max_full_size;                                // :468
      DBuf<double> sol(c, N), tmp(c, N), B, t1(c, md.t1_size()), t2(c, md.t2_size());
      bool have_bsol = false;  // tmp = B sol (FP64) after the local solve
      int64_t step_iters = -1;  // Krylov steps of this local solve (trace)
      if (full) {
        B.reset(c, N * N);
        assemble_local_f64(c, rx[i], n[i], rx[i + 1], ra[i], ra[i + 1], Phi1, A1, Phi2, B.p());
        dense_residual_dev(c, N, B.p(), sol_prev, rhs.p(), tmp.p(), S.p(Scalars::T0));  // :482
        copy_f64(c, N, rhs.p(), sol.p());
        lu_solve_f64(c, N, B.p(), sol.p(), 1);                            // :486
        dense_residual_dev(c, N, B.p(), sol.p(), rhs.p(), tmp.p(), S.p(Scalars::T1));   // :487
        scalar_op(c, SC_DIV, S.p(Scalars::RES_PREV), S.p(Scalars::T0), S.p(Scalars::NRHS));
        scalar_op(c, SC_DIV, S.p(Scalars::RES_NEW), S.p(Scalars::T1), S.p(Scalars::NRHS));
      } else {
        // dres = rhs - B sol_prev serves both res_prev (:495) and the MEX
        // local solver's initial residual (solve3d_2.c:257-263).
        DBuf<double> dres(c, N);
        local_matvec_f64(c, md, Phi1, A1, Phi2, sol_prev, dres.p(), t1.p(), t2.p());
        mv_fp64++;
        axpby_f64(c, N, 1.0, rhs.p(), -1.0, dres.p());
        dot_f64(c, N, dres.p(), nullptr, S.p(Scalars::T0), true);
        scalar_op(c, SC_DIV, S.p(Scalars::RES_PREV), S.p(Scalars::T0), S.p(Scalars::NRHS));
        // one read of the slots NRHS .. T0
        double h[Scalars::T0 - Scalars::NRHS + 1];
        read_scalars(c, S.p(Scalars::NRHS), h, int(Scalars::T0 - Scalars::NRHS + 1));
        const double norm_rhs = h[0], nres = h[Scalars::T0 - Scalars::NRHS];
        if (norm_rhs > 0) {                                               // :497
          LocalSolveResult lr = local_solve_from_residual(
              c, md, Phi1, A1, Phi2, rhs.p(), dres.p(), nres, norm_rhs, real_tol, sol_prev,
              o.local_restart, o.local_iters, sol.p(), o.precision, o.local_prec,
              tmp.p());                                                   // :501
          local_solves++;
          gmres_iters += lr.iters;
          step_iters = lr.iters;
          mv_fp64 += lr.matvecs_fp64;
          if (lr.have_bsol) {  // the refinement's last FP64 matvec was B sol: reuse it
            diffnrm_f64(c, N, tmp.p(), rhs.p(), S.p(Scalars::T1), true);  // :504
          } else {
            local_residual_dev(c, md, Phi1, A1, Phi2, sol.p(), rhs.p(), tmp.p(), t1.p(), t2.p(),
                               S.p(Scalars::T1));                         // :504
            mv_fp64++;
          }
          have_bsol = true;
          scalar_op(c, SC_DIV, S.p(Scalars::RES_NEW), S.p(Scalars::T1), S.p(Scalars::NRHS));
        } else {
          fill_f64(c, N, 0.0, sol.p());
          fill_f64(c, 1, 0.0, S.p(Scalars::RES_NEW));
        }
      }
      // dx = ||sol - sol_prev|| / ||sol|| ; max_dx, max_res (:519-521)
      diffnrm_f64(c, N, sol.p(), sol_prev, S.p(Scalars::T2), true);
      dot_f64(c, N, sol.p(), nullptr, S.p(Scalars::T3), true);
      scalar_op(c, SC_DIV_NZ, S.p(Scalars::T2), S.p(Scalars::T2), S.p(Scalars::T3));
      scalar_op(c, SC_MAXUPD, S.p(Scalars::MAXDX), S.p(Scalars::T2));
      scalar_op(c, SC_MAXUPD, S.p(Scalars::MAXRES), S.p(Scalars::RES_PREV));

      prof.mark("lr_trunc");
      // Truncation (:530-601)
      const int64_t M = rx[i] * n[i], r2 = rx[i + 1];
      DBuf<double> u, v;  // u: M x r ; v: r2 x r
      int64_t r = 0;
      if (kickrank >= 0 && i < d - 1) {
        const int64_t K = std::min(M, r2);
        DBuf<double> U(c, M * K), Sv(c, K), VT(c, K * r2);
        svd_f64(c, M, r2, sol.p(), U.p(), Sv.p(), VT.p());               // :533
        // thr = max(real_tol*resid_damp, res_new) (:547)
        scalar_op(c, SC_MAX_CONST, S.p(Scalars::THR), S.p(Scalars::RES_NEW), nullptr, nullptr,
                  real_tol * resid_damp);
        // Candidate ranks rr = K-1, K-2, ..., 1 (:539-550): the rank is the
        // first candidate whose residual exceeds thr, as in the loop.  The
        // residuals come from rank-one images of the SVD terms when B sol is
        // at hand; otherwise (zero rhs, dense branch) one local residual per
        // candidate, evaluated in growing batches with one read per batch.
        int64_t found = -1, next = K - 1, batch = 1;
        if (have_bsol && next >= 1) {
          // rhs - B(U_rr S_rr V_rr^T) = (rhs - B sol) + sum_{k >= rr} s_k B(u_k v_k^T):
          // candidates in chunks of up to 16, each chunk one rank-one image
          // contraction and one fused running-norm pass, one read-back.
          const int64_t C = CUMNORM_MAXC;
          DBuf<double> R(c, N), W(c, N * std::min(C, next)),
              scr(c, rank1_scratch_size(md, std::min(C, next))),
              part(c, cumulative_norms_part_size(c));
          copy_f64(c, N, rhs.p(), R.p());
          axpby_f64(c, N, -1.0, tmp.p(), 1.0, R.p());
          while (next >= 1 && found < 0) {
            const int64_t nb = std::min(C, next);
            const int64_t k0 = next - nb + 1;  // chunk covers rr = next .. k0
            rank1_images_f64(c, md, Phi1, A1, Phi2, U.p(), M, VT.p(), K, Sv.p(), k0, nb, W.p(),
                             scr.p());
            cumulative_norms_f64(c, N, nb, R.p(), W.p(), part.p(), S.cand(0));
            first_exceeding(c, nb, S.cand(0), S.p(Scalars::NRHS), S.p(Scalars::THR),
                            S.p(Scalars::T3));
            double hb;
            read_scalars(c, S.p(Scalars::T3), &hb, 1);
            if (hb >= 0.0) found = next - int64_t(hb);
            next -= nb;
          }
        }
        DBuf<double> us(c, M * K), cursol(c, M * r2);
        while (next >= 1 && found < 0) {
          const int64_t nb = std::min<int64_t>(std::min(batch, next), Scalars::NCAND);
          for (int64_t b = 0; b < nb; ++b) {
            const int64_t rr = next - b;
            copy2d_f64(c, M, rr, U.p(), M, us.p(), M, Sv.p());
            gemm_f64(c, false, false, M, r2, rr, 1.0, us.p(), M, 0, VT.p(), K, 0, 0.0,
                     cursol.p(), M, 0, 1);
            if (full) {
              dense_residual_dev(c, N, B.p(), cursol.p(), rhs.p(), tmp.p(), S.cand(b));
            } else {
              local_residual_dev(c, md, Phi1, A1, Phi2, cursol.p(), rhs.p(), tmp.p(), t1.p(),
                                 t2.p(), S.cand(b));
              mv_fp64++;
            }
          }
          first_exceeding(c, nb, S.cand(0), S.p(Scalars::NRHS), S.p(Scalars::THR),
                          S.p(Scalars::T3));
          double hb;
          read_scalars(c, S.p(Scalars::T3), &hb, 1);
          if (hb >= 0.0) found = next - int64_t(hb);
          next -= nb;
          batch *= 2;
        }
        // MATLAB leaves the loop variable at 1 when no candidate breaks the
        // loop; an empty loop (K == 1) gives K.
        r = (found >= 1 ? found : (K - 1 >= 1 ? 1 : K - 1)) + 1;          // :551
        r = std::min(r, K);                                               // :593
        r = std::min(r, rmax);                                            // :594
        u.reset(c, M * r);
        copy_f64(c, M * r, U.p(), u.p());                                 // :603
        v.reset(c, r2 * r);                                               // :604 v = V(:,1:r)*diag(s)
        DBuf<double> vtmp(c, r2 * r);
        transpose_f64(c, r, r2, VT.p(), K, vtmp.p(), r2);
        copy2d_f64(c, r2, r, vtmp.p(), r2, v.p(), r2, Sv.p());
      } else {                                                             // :596-601
        const int64_t K = std::min(M, r2);
        DBuf<double> Q(c, M * K), R(c, K * r2);
        qr_f64(c, M, r2, sol.p(), Q.p(), R.p());
        r = K;
        u = std::move(Q);
        v.reset(c, r2 * K);
        transpose_f64(c, K, r2, R.p(), K, v.p(), r2);
      }

      if (o.trace) {  // decision record of this step (one extra read)
        if (trace_len < o.trace_cap) {
          double rr[2];
          read_scalars(c, S.p(Scalars::RES_PREV), rr, 2);
          ttg_amen_step& t = o.trace[trace_len];
          t.sweep = swp;
          t.core = i;
          t.rank = i < d - 1 ? r : -1;
          t.iters = step_iters;
          t.res_prev = rr[0];
          t.res_new = rr[1];
        }
        trace_len++;
      }

      prof.mark("lr_z");
      DBuf<double> uv;
      if ((use_z && !last_sweep) || (i < d - 1 && kickrank > 0 && !last_sweep)) {
        uv.reset(c, M * r2);
        gemm_f64(c, false, true, M, r2, r, 1.0, u.p(), M, 0, v.p(), r2, 0, 0.0, uv.p(), M, 0, 1);
      }
      if (use_z && !last_sweep) {                                          // :605-623
        MvDims zd{rz[i], rx[i], ra[i], n[i], n[i], rx[i + 1], ra[i + 1], rz[i + 1]};
        DBuf<double> crzAt(c, zd.out_size());
        local_matvec_f64(c, zd, phiza[i].p(), A1, phiza[i + 1].p(), uv.p(), crzAt.p());
        mv_fp64++;
        DBuf<double> tz(c, rz[i] * n[i] * ry[i + 1]), crzy(c, rz[i] * n[i] * rz[i + 1]);
        gemm_f64(c, false, false, rz[i], n[i] * ry[i + 1], ry[i], 1.0, phizy[i].p(), rz[i], 0,
                 y1.p(), ry[i], 0, 0.0, tz.p(), rz[i], 0, 1);
        gemm_f64(c, false, false, rz[i] * n[i], rz[i + 1], ry[i + 1], 1.0, tz.p(), rz[i] * n[i], 0,
                 phizy[i + 1].p(), ry[i + 1], 0, 0.0, crzy.p(), rz[i] * n[i], 0, 1);
        axpby_f64(c, zd.out_size(), -1.0, crzAt.p(), 1.0, crzy.p());       // :612
        const int64_t mz = rz[i] * n[i];
        const int64_t K = std::min(mz, rz[i + 1]);
        DBuf<double> U(c, mz * K), Sv(c, K), VT(c, K * rz[i + 1]);
        svd_f64(c, mz, rz[i + 1], crzy.p(), U.p(), Sv.p(), VT.p());       // :613
        const int64_t kz = std::min(kickrank, K);                          // :614
        // U has orthonormal columns: the QR of :619 returns its first kz
        // columns up to signs (a gauge of z).
        rznew = kz;
        crz[i].buf.reset(c, mz * kz);
        copy_f64(c, mz * kz, U.p(), crz[i].p());                           // :621-622
      }

      if (i < d - 1) {                                                     // :625
        prof.mark("lr_kick");
        if (kickrank > 0 && !last_sweep) {                                 // :626
          MvDims ld{rx[i], rx[i], ra[i], n[i], n[i], rx[i + 1], ra[i + 1], rz[i + 1]};
          DBuf<double> leftresid(c, ld.out_size());
          local_matvec_f64(c, ld, Phi1, A1, phiza[i + 1].p(), uv.p(), leftresid.p());  // :702
          mv_fp64++;
          // lefty = phiy{i} * y1 (:704) is t, already formed for the rhs (:456)
          DBuf<double> uk(c, M * rz[i + 1]);
          gemm_f64(c, false, false, M, rz[i + 1], ry[i + 1], 1.0, t.p(), M, 0, phizy[i + 1].p(),
                   ry[i + 1], 0, 0.0, uk.p(), M, 0, 1);                     // :706
          axpby_f64(c, M * rz[i + 1], -1.0, leftresid.p(), 1.0, uk.p());   // :707
          // [u, rv] = qr([u, uk]) ; v = [v, 0] * rv.'  (:713-716)
          const int64_t radd = rz[i + 1], wcols = r + radd;
          const int64_t kq = std::min(M, wcols);
          if (M >= wcols) {
            // u has orthonormal columns (left singular vectors), so a QR of
            // [u, uk] is [u, Q2] with Q2 an orthonormal basis of uk's part
            // orthogonal to u, and rv = [I, u'uk; 0, R2]: then v*rv(:,1:r)' =
            // [v, 0].  This is the reference's factorization up to the column
            // signs LAPACK would choose (a gauge of the TT representation).
            // Two projection passes, then a QR of the M x radd block.  When a
            // column of uk lies (numerically) in span(u), the QR of the
            // projected block is not reliably orthogonal to u: a third
            // projection and QR run, gated on the device by the columns' loss
            // of norm (no host round trip).
            DBuf<double> w(c, M * radd), C(c, r * radd), Q2(c, M * radd), R2(c, radd * radd),
                G(c, 2 * radd * radd);
            DBuf<int> keep(c, 1);
            copy_f64(c, M * radd, uk.p(), w.p());
            gemm_f64(c, true, false, radd, radd, M, 1.0, w.p(), M, 0, w.p(), M, 0, 0.0, G.p(),
                     radd, 0, 1);
            auto project = [&]() {
              gemm_f64(c, true, false, r, radd, M, 1.0, u.p(), M, 0, w.p(), M, 0, 0.0, C.p(), r,
                       0, 1);
              gemm_f64(c, false, false, M, radd, r, -1.0, u.p(), M, 0, C.p(), r, 0, 1.0, w.p(), M,
                       0, 1);
            };
            project();
            project();
            gemm_f64(c, true, false, radd, radd, M, 1.0, w.p(), M, 0, w.p(), M, 0, 0.0,
                     G.p() + radd * radd, radd, 0, 1);
            collapse_flag(c, radd, G.p(), radd, G.p() + radd * radd, radd, 1e-8, keep.p());
            qr_f64(c, M, radd, w.p(), Q2.p(), R2.p());
            {
              SkipGuard guard(c, keep.p());  // runs only when a column collapsed
              copy_f64(c, M * radd, Q2.p(), w.p());
              project();
              qr_f64(c, M, radd, w.p(), Q2.p(), R2.p());
            }
            DBuf<double> Q(c, M * kq), vn(c, r2 * kq);
            copy_f64(c, M * r, u.p(), Q.p());
            copy_f64(c, M * radd, Q2.p(), Q.p() + M * r);
            fill_f64(c, r2 * kq, 0.0, vn.p());
            copy_f64(c, r2 * r, v.p(), vn.p());
            u = std::move(Q);
            v = std::move(vn);
          } else {
            DBuf<double> uu(c, M * wcols);
            copy_f64(c, M * r, u.p(), uu.p());
            copy_f64(c, M * radd, uk.p(), uu.p() + M * r);
            DBuf<double> Q(c, M * kq), rv(c, kq * wcols);
            qr_f64(c, M, wcols, uu.p(), Q.p(), rv.p());
            // v_new (r2 x kq) = v (r2 x r) * rv(:, 1:r)^T  (the zero block drops out)
            DBuf<double> vn(c, r2 * kq);
            gemm_f64(c, false, true, r2, kq, r, 1.0, v.p(), r2, 0, rv.p(), kq, 0, 0.0, vn.p(), r2,
                     0, 1);
            u = std::move(Q);
            v = std::move(vn);
          }
          r = kq;
        }
        // v = v.' * x_{i+1}  (:732-734)
        const int64_t nc = n[i + 1] * rx[i + 2];
        DBuf<double> vx(c, r * nc);
        gemm_f64(c, true, false, r, nc, r2, 1.0, v.p(), r2, 0, crx[i + 1].p(), r2, 0, 0.0, vx.p(),
                 r, 0, 1);
        scalar_op(c, SC_NRMSC_DIV, NC, S.y(i), S.a(i), S.x(i));           // :737
        normalize_dev(c, r * nc, vx.p(), S.p(Scalars::T0));               // :739-744
        scalar_op(c, SC_MUL, S.x(i), S.p(Scalars::T0));                   // :745
        prof.mark("lr_phi");
        // Interfaces (:751-752)
        phia[i + 1].buf.reset(c, r * r * ra[i + 1]);
        next_phi_f64(c, 0, rx[i], n[i], r, rx[i], r, ra[i], ra[i + 1], phia[i].p(), u.p(), A1,
                     u.p(), phia[i + 1].p());
        normalize_dev(c, r * r * ra[i + 1], phia[i + 1].p(), S.a(i));
        phiy[i + 1].buf.reset(c, r * ry[i + 1]);
        next_phi_f64(c, 0, rx[i], n[i], r, ry[i], ry[i + 1], 1, 1, phiy[i].p(), u.p(), nullptr,
                     cry(i), phiy[i + 1].p());
        normalize_dev(c, r * ry[i + 1], phiy[i + 1].p(), S.y(i));
        scalar_op(c, SC_NRMSC_MUL, NC, S.y(i), S.a(i), S.x(i));           // :754
        rx[i + 1] = r;                                                     // :765-767
        crx[i].buf = std::move(u);
        crx[i + 1].buf = std::move(vx);
        if (use_z && !last_sweep) {                                        // :770-774
          rz[i + 1] = rznew;
          phiza[i + 1].buf.reset(c, rz[i + 1] * rx[i + 1] * ra[i + 1]);
          next_phi_f64(c, 0, rz[i], n[i], rz[i + 1], rx[i], rx[i + 1], ra[i], ra[i + 1],
                       phiza[i].p(), crz[i].p(), A1, crx[i].p(), phiza[i + 1].p());
          scale_dev_f64(c, rz[i + 1] * rx[i + 1] * ra[i + 1], phiza[i + 1].p(), phiza[i + 1].p(),
                        nullptr, S.a(i));
          phizy[i + 1].buf.reset(c, rz[i + 1] * ry[i + 1]);
          next_phi_f64(c, 0, rz[i], n[i], rz[i + 1], ry[i], ry[i + 1], 1, 1, phizy[i].p(),
                       crz[i].p(), nullptr, cry(i), phizy[i + 1].p());
          scale_dev_f64(c, rz[i + 1] * ry[i + 1], phizy[i + 1].p(), phizy[i + 1].p(), nullptr,
                        S.y(i));
        }
      } else {
        crx[i].buf = std::move(sol);                                       // :778-779
      }
    }
    swp_done = swp;
    double mm[2];
    read_scalars(c, S.p(Scalars::MAXRES), mm, 2);
    const double max_res = mm[0], max_dx = mm[1];
    int64_t maxr = 0;
    for (auto v : rx) maxr = std::max(maxr, v);
    if (stats && swp <= TTG_MAX_SWEEPS_RECORDED) {
      stats->max_res[swp - 1] = max_res;
      stats->max_dx[swp - 1] = max_dx;
    }
    if (o.verb > 0)
      fprintf(stderr, "=amen_solve= sweep %lld, max_dx: %3.3e, max_res: %3.3e, max_rank: %lld\n",
              (long long)swp, max_dx, max_res, (long long)maxr);            // :793-795
    if (last_sweep) break;                                                 // :797-799
    if (max_res < tol_exit) last_sweep = true;                             // :806-808
  }

  prof.report();
  // Distribute the norms (:816-820) and assemble the output.
  std::vector<double> hx(d - 1);
  read_scalars(c, S.x(0), hx.data(), int(d - 1));
  double lsum = 0.0;
  for (double v : hx) lsum += std::log(v);
  const double nx = std::exp(lsum / double(d));
  auto* out = new ttg_tt_s();
  out->ctx = out_ctx;
  out->d = d;
  out->is_matrix = false;
  out->n = n;
  out->r = rx;
  out->ps.assign(d + 1, 0);
  for (int64_t k = 0; k < d; ++k) out->ps[k + 1] = out->ps[k] + rx[k] * n[k] * rx[k + 1];
  out->numel = out->ps[d];
  out->core = static_cast<double*>(out_ctx->alloc->get(sizeof(double) * out->numel));
  for (int64_t k = 0; k < d; ++k)
    axpby_f64(c, out->ps[k + 1] - out->ps[k], nx, crx[k].p(), 0.0, out->core + out->ps[k]);
  float ms = 0.f;
  if (!c->rec) {
    TTG_CUDA(cudaEventRecord(e1, c->stream));
    TTG_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  int herr[8];
  read_device(c, herr, c->d_err, sizeof(herr));
  if (c->rec)
    ms = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                         host_t0)
                   .count());
  if (herr[0] || herr[1] || herr[2]) {
    release_tt(c, out);
    fail(TTG_ERR_TIMEOUT, "a bounded device-side wait timed out (codes %d %d %d)", herr[0],
         herr[1], herr[2]);
  }
  if (herr[4]) {
    release_tt(c, out);
    fail(TTG_ERR_SOLVER, "a device factorization reported a non-zero LAPACK info");
  }
  if (herr[3]) {  // MATLAB's svd errors when it does not converge (amen_solve2.m:533)
    release_tt(c, out);
    fail(TTG_ERR_NOCONV, "a Jacobi SVD reached its sweep limit (%d sweeps)",
         c->jacobi_max_sweeps);
  }
  if (stats) {
    stats->sweeps = swp_done;
    stats->matvecs = c->matvecs - mv0;
    stats->matvecs_fp64 = mv_fp64;
    stats->local_solves = local_solves;
    stats->gmres_iters = gmres_iters;
    int64_t mr = 0;
    for (auto v : rx) mr = std::max(mr, v);
    stats->max_rank = mr;
    stats->ms_total = ms;
    stats->matvec_gflop = double(c->matvec_flops - fl0) * 1e-9;
    stats->launches = c->launches - la0;
    c->ev_collect();
    stats->matvecs_lp = c->mv_count[1] - mvk0[1];
    stats->gflop_lp = (c->mv_flops[1] - flk0[1]) * 1e-9;
    stats->gbyte_lp = (c->mv_bytes_lp - byl0) * 1e-9;
    stats->ms_lp = c->mv_ms[1] - msk0[1];
    stats->gflop_fp64 = (c->mv_flops[0] - flk0[0]) * 1e-9;
    stats->ms_fp64 = c->mv_ms[0] - msk0[0];
    stats->ms_matvec = o.precision == TTG_MIXED ? stats->ms_lp : stats->ms_fp64;
    stats->trace_len = trace_len;
  }
  return out;
}

}  // namespace ttg
