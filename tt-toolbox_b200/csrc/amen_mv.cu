// AMEn approximate matrix-by-vector product y ~ A x on the device.
//
// Restates core/amen_mv.m:1-419 on its default option path (tt_matrix
// operator, renorm 'direct', fkick false, kickrank2 0, init_qr true).  Every
// core of y is in turn replaced by the projection of A x onto the other
// cores' interfaces -- the local matvec bfun3 of the AMEn solver with bra y
// and ket x (amen_mv.m:224) -- then truncated by an SVD to tol ||s|| /
// sqrt(d) (:244-248, :318-322).  A rank-kickrank auxiliary TT z tracks the
// projected error and enriches y in the backward half-sweeps (:327-355).
// All cores and interfaces stay on the device; the host reads the singular
// values for the rank decisions and one norm per sweep.
#include <algorithm>
#include <cmath>
#include <vector>

#include "amen.h"
#include "linalg.h"
#include "local_ops.h"
#include "round.h"

using namespace ttg;

namespace {

struct Buf {
  DBuf<double> b;
  double* p() const { return b.p(); }
};

// Phi /= ||Phi|| (norm into *slot; 1 when zero): compute_next_Phi with
// nargout > 1 (amen_mv.m:596-602).
void normalize_phi(Context* c, int64_t n, double* x, double* slot) {
  dot_f64(c, n, x, nullptr, slot, true);
  normalize_by_dev(c, n, x, slot);
}

// Thin QR with Q into dst (m x k), k returned.
int64_t qr_q(Context* c, int64_t m, int64_t n, const double* a, DBuf<double>& dst) {
  const int64_t k = std::min(m, n);
  DBuf<double> R(c, k * n);
  dst.reset(c, m * k);
  qr_f64(c, m, n, a, dst.p(), R.p());
  return k;
}

}  // namespace

extern "C" {

int ttg_amen_mv_opts_default(ttg_amen_mv_opts* o) {
  if (!o) return TTG_ERR_INVALID;
  *o = ttg_amen_mv_opts{};
  o->nswp = 20;      // amen_mv.m:55
  o->kickrank = 4;   // :56
  o->init_qr = 1;    // :61
  o->seed = 0x5eed;
  return TTG_OK;
}

int ttg_amen_mv(ttg_tt A, ttg_tt x, double tol, const ttg_amen_mv_opts* opts, ttg_tt y0,
                ttg_tt z0, ttg_tt* y_out, ttg_tt* z_out, int64_t* sweeps_out) {
  TTG_API_BEGIN
  TTG_REQUIRE(A && x && y_out, "NULL argument");
  *y_out = nullptr;
  if (z_out) *z_out = nullptr;
  TTG_REQUIRE(A->is_matrix && !x->is_matrix, "A must be a TT matrix and x a TT tensor");
  TTG_REQUIRE(A->ctx == x->ctx, "operands belong to different contexts");
  TTG_REQUIRE(std::isfinite(tol) && tol > 0, "tol must be > 0");
  ttg_amen_mv_opts o;
  if (opts)
    o = *opts;
  else
    ttg_amen_mv_opts_default(&o);
  TTG_REQUIRE(o.nswp >= 1 && o.kickrank >= 0, "invalid options");
  const int64_t d = x->d;
  TTG_REQUIRE(A->d == d && d >= 2, "A and x need the same number (>= 2) of cores");
  for (int64_t k = 0; k < d; ++k)
    TTG_REQUIRE(A->m[k] == x->n[k] && A->n[k] == A->m[k],
                "core %lld: square A cores matching x are required", (long long)k);
  TTG_REQUIRE(A->r[0] == 1 && A->r[d] == 1 && x->r[0] == 1 && x->r[d] == 1,
              "border ranks must be 1");
  Context* c = A->ctx;
  TTG_CUDA(cudaSetDevice(c->device));
  require_finite(A, "A");
  require_finite(x, "x");
  require_finite(y0, "y0");
  require_finite(z0, "z0");
  TTG_CUDA(cudaMemsetAsync(c->d_err, 0, 8 * sizeof(int), c->stream));
  const std::vector<int64_t>& n = A->n;
  const std::vector<int64_t>& ra = A->r;
  const std::vector<int64_t>& rx = x->r;
  const bool use_z = o.kickrank > 0;
  auto Ak = [&](int64_t k) { return A->core + A->ps[k]; };
  auto xk = [&](int64_t k) { return x->core + x->ps[k]; };

  // Initial guesses (:130-137): given, or right-orthogonal random TTs.
  ttg_tt_s* y0own = nullptr;
  ttg_tt_s* z0own = nullptr;
  if (!y0) y0 = y0own = tt_rand_device(c, n, 2, uint64_t(o.seed));
  if (use_z && !z0) z0 = z0own = tt_rand_device(c, n, o.kickrank, uint64_t(o.seed) ^ 0x9e37ull);
  struct Own {
    ttg_tt_s *a, *b;
    ~Own() {
      if (a) ttg_tt_free(a);
      if (b) ttg_tt_free(b);
    }
  } own{y0own, z0own};
  TTG_REQUIRE(y0->ctx == c && !y0->is_matrix && y0->d == d, "y0 shape mismatch");
  if (use_z) TTG_REQUIRE(z0->ctx == c && !z0->is_matrix && z0->d == d, "z0 shape mismatch");
  for (int64_t k = 0; k < d; ++k) {
    TTG_REQUIRE(y0->n[k] == n[k], "y0 mode size mismatch");
    if (use_z) TTG_REQUIRE(z0->n[k] == n[k], "z0 mode size mismatch");
  }
  std::vector<int64_t> ry = y0->r, rz;
  std::vector<Buf> y(d), z(d);
  for (int64_t k = 0; k < d; ++k) {
    const int64_t sz = ry[k] * n[k] * ry[k + 1];
    y[k].b.reset(c, sz);
    copy_f64(c, sz, y0->core + y0->ps[k], y[k].p());
  }
  if (use_z) {
    rz = z0->r;
    for (int64_t k = 0; k < d; ++k) {
      const int64_t sz = rz[k] * n[k] * rz[k + 1];
      z[k].b.reset(c, sz);
      copy_f64(c, sz, z0->core + z0->ps[k], z[k].p());
    }
  }
  // Interfaces: phiyax 'lr' [ry, rx, ra], 'rl' [rx, ra, ry]; phizax likewise
  // with z as bra; phizy 'lr' [rz, ry], 'rl' [ry, rz] (:142-155).
  std::vector<Buf> phiyax(d + 1), phizax(d + 1), phizy(d + 1);
  for (int64_t k : {int64_t(0), d}) {
    phiyax[k].b.reset(c, 1);
    fill_f64(c, 1, 1.0, phiyax[k].p());
    if (use_z) {
      phizax[k].b.reset(c, 1);
      phizy[k].b.reset(c, 1);
      fill_f64(c, 1, 1.0, phizax[k].p());
      fill_f64(c, 1, 1.0, phizy[k].p());
    }
  }
  DBuf<double> nrms(c, d), sc(c, 4);  // sc[0] = dx, sc[1] = max_dx, sc[2] scratch
  fill_f64(c, d, 1.0, nrms.p());                                           // :157

  auto lr_y = [&](int64_t i) {  // phiyax{i+1} = compute_next_Phi(.., y{i}, A{i}, x{i}, 'lr')
    phiyax[i + 1].b.reset(c, ry[i + 1] * rx[i + 1] * ra[i + 1]);
    next_phi_f64(c, 0, ry[i], n[i], ry[i + 1], rx[i], rx[i + 1], ra[i], ra[i + 1],
                 phiyax[i].p(), y[i].p(), Ak(i), xk(i), phiyax[i + 1].p());
    normalize_phi(c, ry[i + 1] * rx[i + 1] * ra[i + 1], phiyax[i + 1].p(), nrms.p() + i);
  };
  auto lr_z = [&](int64_t i) {  // :212-213 / :306-307
    phizax[i + 1].b.reset(c, rz[i + 1] * rx[i + 1] * ra[i + 1]);
    next_phi_f64(c, 0, rz[i], n[i], rz[i + 1], rx[i], rx[i + 1], ra[i], ra[i + 1],
                 phizax[i].p(), z[i].p(), Ak(i), xk(i), phizax[i + 1].p());
    scale_dev_f64(c, rz[i + 1] * rx[i + 1] * ra[i + 1], phizax[i + 1].p(), phizax[i + 1].p(),
                  nullptr, nrms.p() + i);
    phizy[i + 1].b.reset(c, rz[i + 1] * ry[i + 1]);
    next_phi_f64(c, 0, rz[i], n[i], rz[i + 1], ry[i], ry[i + 1], 1, 1, phizy[i].p(), z[i].p(),
                 nullptr, y[i].p(), phizy[i + 1].p());
  };
  auto rl_y = [&](int64_t i) {  // :364
    phiyax[i].b.reset(c, rx[i] * ra[i] * ry[i]);
    next_phi_f64(c, 1, ry[i], n[i], ry[i + 1], rx[i], rx[i + 1], ra[i], ra[i + 1],
                 phiyax[i + 1].p(), y[i].p(), Ak(i), xk(i), phiyax[i].p());
    normalize_phi(c, rx[i] * ra[i] * ry[i], phiyax[i].p(), nrms.p() + i);
  };
  auto rl_z = [&](int64_t i) {  // :376-377
    phizax[i].b.reset(c, rx[i] * ra[i] * rz[i]);
    next_phi_f64(c, 1, rz[i], n[i], rz[i + 1], rx[i], rx[i + 1], ra[i], ra[i + 1],
                 phizax[i + 1].p(), z[i].p(), Ak(i), xk(i), phizax[i].p());
    scale_dev_f64(c, rx[i] * ra[i] * rz[i], phizax[i].p(), phizax[i].p(), nullptr,
                  nrms.p() + i);
    phizy[i].b.reset(c, ry[i] * rz[i]);
    next_phi_f64(c, 1, rz[i], n[i], rz[i + 1], ry[i], ry[i + 1], 1, 1, phizy[i + 1].p(),
                 z[i].p(), nullptr, y[i].p(), phizy[i].p());
  };
  // QR of the left-unfolded core i, R/||R||_F pushed into core i+1 (:162-175).
  auto orth_left = [&](std::vector<Buf>& t, std::vector<int64_t>& r, int64_t i) {
    const int64_t m = r[i] * n[i], cols = r[i + 1], k = std::min(m, cols);
    DBuf<double> Q(c, m * k), R(c, k * cols), nr(c, 1);
    qr_f64(c, m, cols, t[i].p(), Q.p(), R.p());
    normalize_phi(c, k * cols, R.p(), nr.p());
    const int64_t nc = n[i + 1] * r[i + 2];
    DBuf<double> nx(c, k * nc);
    gemm_f64(c, false, false, k, nc, cols, 1.0, R.p(), k, 0, t[i + 1].p(), cols, 0, 0.0, nx.p(),
             k, 0, 1);
    r[i + 1] = k;
    t[i].b = std::move(Q);
    t[i + 1].b = std::move(nx);
  };

  for (int64_t i = 0; i < d - 1; ++i) {                                   // :160-214
    if (o.init_qr) orth_left(y, ry, i);
    lr_y(i);
    if (use_z) {
      orth_left(z, rz, i);
      lr_z(i);
    }
  }

  int64_t i = d - 1, dir = -1, swp = 1, sweeps = 0;                        // :216-219
  fill_f64(c, 1, 0.0, sc.p() + 1);
  DBuf<double> cry;
  const double chop = tol / std::sqrt(double(d));
  while (swp <= o.nswp) {                                                  // :221
    // projection of A x onto the interfaces (:223-230)
    MvDims md{ry[i], rx[i], ra[i], n[i], n[i], rx[i + 1], ra[i + 1], ry[i + 1]};
    const int64_t N = md.out_size();
    cry.reset(c, N);
    local_matvec_f64(c, md, phiyax[i].p(), Ak(i), phiyax[i + 1].p(), xk(i), cry.p());
    dot_f64(c, N, cry.p(), nullptr, nrms.p() + i, true);
    normalize_by_dev(c, N, cry.p(), nrms.p() + i);
    diffnrm_f64(c, N, cry.p(), y[i].p(), sc.p(), true);                    // :232
    scalar_op(c, SC_MAXUPD, sc.p() + 1, sc.p());                           // :233
    if (dir > 0 && i < d - 1) {                                            // :237
      const int64_t M = ry[i] * n[i], C = ry[i + 1], K = std::min(M, C);
      DBuf<double> U(c, M * K), S(c, K), VT(c, K * C);
      svd_f64(c, M, C, cry.p(), U.p(), S.p(), VT.p());                     // :244
      std::vector<double> hs(K);
      read_scalars(c, S.p(), hs.data(), int(K));
      double ns = 0.0;
      for (double v : hs) ns += v * v;
      const int64_t r = my_chop2(hs.data(), K, chop * std::sqrt(ns));       // :246
      DBuf<double> u(c, M * r), v(c, C * r), vt(c, C * r);
      copy_f64(c, M * r, U.p(), u.p());
      transpose_f64(c, r, C, VT.p(), K, vt.p(), C);                        // V(:,1:r)
      copy2d_f64(c, C, r, vt.p(), C, v.p(), C, S.p());                     // * diag(s)
      DBuf<double> crz;
      if (use_z) {                                                         // :251-262
        DBuf<double> uv(c, M * C);
        gemm_f64(c, false, true, M, C, r, 1.0, u.p(), M, 0, v.p(), C, 0, 0.0, uv.p(), M, 0, 1);
        MvDims zd{rz[i], rx[i], ra[i], n[i], n[i], rx[i + 1], ra[i + 1], rz[i + 1]};
        crz.reset(c, zd.out_size());
        local_matvec_f64(c, zd, phizax[i].p(), Ak(i), phizax[i + 1].p(), xk(i), crz.p());
        DBuf<double> ys(c, M * rz[i + 1]), yz(c, rz[i] * n[i] * rz[i + 1]);
        gemm_f64(c, false, false, M, rz[i + 1], C, 1.0, uv.p(), M, 0, phizy[i + 1].p(), C, 0,
                 0.0, ys.p(), M, 0, 1);                                    // ys = cry*phizy{i+1}
        gemm_f64(c, false, false, rz[i], n[i] * rz[i + 1], ry[i], 1.0, phizy[i].p(), rz[i], 0,
                 ys.p(), ry[i], 0, 0.0, yz.p(), rz[i], 0, 1);              // phizy{i}*yz
        scale_dev_f64(c, zd.out_size(), crz.p(), crz.p(), nullptr, nrms.p() + i);
        axpby_f64(c, zd.out_size(), -1.0, yz.p(), 1.0, crz.p());           // crz/nrms - yz
      }
      y[i].b = std::move(u);                                               // :287
      const int64_t nc = n[i + 1] * ry[i + 2];
      DBuf<double> nx(c, r * nc);
      gemm_f64(c, true, false, r, nc, C, 1.0, v.p(), C, 0, y[i + 1].p(), C, 0, 0.0, nx.p(), r, 0,
               1);                                                         // v.'*cr2
      y[i + 1].b = std::move(nx);
      ry[i + 1] = r;
      lr_y(i);                                                             // :296
      if (use_z) {                                                         // :299-308
        const int64_t mz = rz[i] * n[i];
        rz[i + 1] = qr_q(c, mz, rz[i + 1], crz.p(), z[i].b);
        lr_z(i);
      }
    } else if (dir < 0 && i > 0) {                                         // :311
      const int64_t M = ry[i], C = n[i] * ry[i + 1], K = std::min(M, C);
      DBuf<double> U(c, M * K), S(c, K), VT(c, K * C);
      svd_f64(c, M, C, cry.p(), U.p(), S.p(), VT.p());                     // :318
      std::vector<double> hs(K);
      read_scalars(c, S.p(), hs.data(), int(K));
      double ns = 0.0;
      for (double v : hs) ns += v * v;
      int64_t r = my_chop2(hs.data(), K, chop * std::sqrt(ns));
      DBuf<double> u(c, M * r), v(c, C * r);
      transpose_f64(c, r, C, VT.p(), K, v.p(), C);                         // :321 V(:,1:r)
      copy2d_f64(c, M, r, U.p(), M, u.p(), M, S.p());                      // :322 U*diag(s)
      DBuf<double> crz;
      if (use_z) {                                                         // :325-355
        DBuf<double> uv(c, M * C);
        gemm_f64(c, false, true, M, C, r, 1.0, u.p(), M, 0, v.p(), C, 0, 0.0, uv.p(), M, 0, 1);
        MvDims zd{rz[i], rx[i], ra[i], n[i], n[i], rx[i + 1], ra[i + 1], rz[i + 1]};
        crz.reset(c, zd.out_size());
        local_matvec_f64(c, zd, phizax[i].p(), Ak(i), phizax[i + 1].p(), xk(i), crz.p());
        DBuf<double> ys(c, rz[i] * C), yz(c, rz[i] * n[i] * rz[i + 1]);
        gemm_f64(c, false, false, rz[i], C, M, 1.0, phizy[i].p(), rz[i], 0, uv.p(), M, 0, 0.0,
                 ys.p(), rz[i], 0, 1);                                     // ys = phizy{i}*cry
        gemm_f64(c, false, false, rz[i] * n[i], rz[i + 1], ry[i + 1], 1.0, ys.p(),
                 rz[i] * n[i], 0, phizy[i + 1].p(), ry[i + 1], 0, 0.0, yz.p(), rz[i] * n[i], 0,
                 1);                                                       // yz*phizy{i+1}
        scale_dev_f64(c, zd.out_size(), crz.p(), crz.p(), nullptr, nrms.p() + i);
        axpby_f64(c, zd.out_size(), -1.0, yz.p(), 1.0, crz.p());           // :336
        // crs = bfun3(phizax{i}, A{i}, phiyax{i+1}, x{i}) / nrms - ys (:344-346)
        MvDims sd{rz[i], rx[i], ra[i], n[i], n[i], rx[i + 1], ra[i + 1], ry[i + 1]};
        DBuf<double> crs(c, sd.out_size());
        local_matvec_f64(c, sd, phizax[i].p(), Ak(i), phiyax[i + 1].p(), xk(i), crs.p());
        scale_dev_f64(c, sd.out_size(), crs.p(), crs.p(), nullptr, nrms.p() + i);
        axpby_f64(c, sd.out_size(), -1.0, ys.p(), 1.0, crs.p());
        // v = qr([v, crs.']); u = [u, 0] * R.'  (:347-354)
        const int64_t w = r + rz[i];
        DBuf<double> vv(c, C * w);
        copy_f64(c, C * r, v.p(), vv.p());
        transpose_f64(c, rz[i], C, crs.p(), rz[i], vv.p() + C * r, C);
        const int64_t k2 = std::min(C, w);
        DBuf<double> Q(c, C * k2), R(c, k2 * w);
        qr_f64(c, C, w, vv.p(), Q.p(), R.p());
        DBuf<double> un(c, M * k2);
        gemm_f64(c, false, true, M, k2, r, 1.0, u.p(), M, 0, R.p(), k2, 0, 0.0, un.p(), M, 0, 1);
        u = std::move(un);
        v = std::move(Q);
        r = k2;
      }
      const int64_t mp = ry[i - 1] * n[i - 1];                             // :357-360
      DBuf<double> prev(c, mp * r), yi(c, r * C);
      gemm_f64(c, false, false, mp, r, M, 1.0, y[i - 1].p(), mp, 0, u.p(), M, 0, 0.0, prev.p(),
               mp, 0, 1);
      transpose_f64(c, C, r, v.p(), C, yi.p(), r);
      y[i - 1].b = std::move(prev);
      y[i].b = std::move(yi);
      ry[i] = r;
      rl_y(i);                                                             // :364
      if (use_z) {                                                         // :366-378
        const int64_t cz = n[i] * rz[i + 1];
        DBuf<double> czt(c, cz * rz[i]), Q;
        transpose_f64(c, rz[i], cz, crz.p(), rz[i], czt.p(), cz);
        const int64_t k = qr_q(c, cz, rz[i], czt.p(), Q);
        z[i].b.reset(c, k * cz);
        transpose_f64(c, cz, k, Q.p(), cz, z[i].p(), k);
        rz[i] = k;
        rl_z(i);
      }
    }
    if ((dir > 0 && i == d - 1) || (dir < 0 && i == 0)) {                  // :387
      if (dir > 0) {
        sweeps = swp;
        double mdx = 0.0;
        read_scalars(c, sc.p() + 1, &mdx, 1);
        if (o.verb > 0)
          fprintf(stderr, "amen-mv: swp=%lld, max_dx=%3.3e, max_r=%lld\n", (long long)swp, mdx,
                  (long long)*std::max_element(ry.begin(), ry.end()));
        if (mdx < tol || swp == o.nswp) break;
      }
      y[i].b.reset(c, cry.size());                                         // :396
      copy_f64(c, cry.size(), cry.p(), y[i].p());
      if (dir > 0) ++swp;
      fill_f64(c, 1, 0.0, sc.p() + 1);
      dir = -dir;
    } else {
      i += dir;
    }
  }
  y[d - 1].b.reset(c, cry.size());                                         // :408
  copy_f64(c, cry.size(), cry.p(), y[d - 1].p());
  std::vector<double> hn(d);                                               // :414-419
  read_scalars(c, nrms.p(), hn.data(), int(d));
  double ls = 0.0;
  for (double v : hn) ls += std::log(v);
  const double nrm = std::exp(ls / double(d));
  auto pack = [&](std::vector<Buf>& t, const std::vector<int64_t>& r, double s) {
    auto* h = new ttg_tt_s();
    h->ctx = c;
    h->d = d;
    h->is_matrix = false;
    h->n = n;
    h->r = r;
    h->ps.assign(d + 1, 0);
    for (int64_t k = 0; k < d; ++k) h->ps[k + 1] = h->ps[k] + r[k] * n[k] * r[k + 1];
    h->numel = h->ps[d];
    h->core = static_cast<double*>(c->alloc->get(sizeof(double) * h->numel));
    for (int64_t k = 0; k < d; ++k)
      axpby_f64(c, h->ps[k + 1] - h->ps[k], s, t[k].p(), 0.0, h->core + h->ps[k]);
    return h;
  };
  ttg_tt_s* yo = pack(y, ry, nrm);
  ttg_tt_s* zo = (use_z && z_out) ? pack(z, rz, 1.0) : nullptr;
  try {
    check_factorizations(c);
  } catch (...) {
    ttg_tt_free(yo);
    if (zo) ttg_tt_free(zo);
    throw;
  }
  *y_out = yo;
  if (z_out) *z_out = zo;
  if (sweeps_out) *sweeps_out = sweeps;
  TTG_API_END
}

}  // extern "C"
