// AMEn approximation of linear combinations of TT tensors on the device.
//
// Restates core/amen_sum.m:1-483 on its default option path for TT inputs
// (can false, renorm 'direct', fkick false, kickrank2 0, multrank false):
// y(:, m) ~ sum_j X{j} c(j, m) for m = 1..M is one TT whose current core
// carries the output index m.  Every core is in turn the projection of the
// sum onto the interfaces of the other cores of y (proj_sum, :647-684),
// truncated by an SVD to tol ||s|| / sqrt(d) and, in the backward
// half-sweeps, enriched by the projected residual of a rank-kickrank TT z.
// Cores and interfaces stay on the device; the host reads the singular
// values for the rank decisions and one number per sweep.
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

// Interface of bra `a` [ra1, n, ra2] and ket `b` [rb1, n, rb2]
// (compute_next_Phi of amen_sum.m:557-627, one summand):
//   'lr': prev [ra1, rb1] -> out [ra2, rb2];  'rl': prev [rb2, ra2] -> out [rb1, ra1].
void phi_pair(Context* c, int dir, int64_t ra1, int64_t n, int64_t ra2, int64_t rb1, int64_t rb2,
              const double* prev, const double* a, const double* b, Buf& out) {
  out.b.reset(c, dir == 0 ? ra2 * rb2 : rb1 * ra1);
  next_phi_f64(c, dir, ra1, n, ra2, rb1, rb2, 1, 1, prev, a, nullptr, b, out.p());
}

}  // namespace

extern "C" {

int ttg_amen_sum_opts_default(ttg_amen_sum_opts* o) {
  if (!o) return TTG_ERR_INVALID;
  *o = ttg_amen_sum_opts{};
  o->nswp = 20;      // amen_sum.m:56
  o->kickrank = 4;   // :57
  o->init_qr = 1;    // :63
  o->rmax = 0;       // :67 (Inf)
  o->seed = 0x5eed5eedull;
  return TTG_OK;
}

int ttg_amen_sum(int64_t count, const ttg_tt* X, const double* coef, int64_t M, double tol,
                 const ttg_amen_sum_opts* opts, ttg_tt y0, ttg_tt z0, ttg_tt* y_out,
                 ttg_tt* z_out, int64_t* sweeps_out) {
  TTG_API_BEGIN
  TTG_REQUIRE(X && coef && y_out, "NULL argument");
  *y_out = nullptr;
  if (z_out) *z_out = nullptr;
  TTG_REQUIRE(count >= 1 && M >= 1, "count and M must be >= 1");
  TTG_REQUIRE(std::isfinite(tol) && tol > 0, "tol must be > 0");
  for (int64_t j = 0; j < count * M; ++j)
    TTG_REQUIRE(std::isfinite(coef[j]), "coefficient %lld is not finite", (long long)j);
  ttg_amen_sum_opts o;
  if (opts)
    o = *opts;
  else
    ttg_amen_sum_opts_default(&o);
  TTG_REQUIRE(o.nswp >= 1 && o.kickrank >= 0, "invalid options");
  const int64_t N = count;
  for (int64_t j = 0; j < N; ++j) TTG_REQUIRE(X[j], "X[%lld] is NULL", (long long)j);
  Context* c = X[0]->ctx;
  const int64_t d = X[0]->d;
  TTG_REQUIRE(d >= 2, "amen_sum needs d >= 2");
  const std::vector<int64_t> n = X[0]->n;
  for (int64_t j = 0; j < N; ++j) {
    TTG_REQUIRE(X[j]->ctx == c && !X[j]->is_matrix && X[j]->d == d,
                "X[%lld]: TT tensors of one context with equal d are required", (long long)j);
    for (int64_t k = 0; k < d; ++k)
      TTG_REQUIRE(X[j]->n[k] == n[k], "X[%lld]: mode size mismatch at core %lld", (long long)j,
                  (long long)k);
    TTG_REQUIRE(X[j]->r[0] == 1 && X[j]->r[d] == 1, "X[%lld]: border ranks must be 1",
                (long long)j);
  }
  TTG_CUDA(cudaSetDevice(c->device));
  for (int64_t j = 0; j < N; ++j) require_finite(X[j], "X");
  require_finite(y0, "y0");
  require_finite(z0, "z0");
  TTG_CUDA(cudaMemsetAsync(c->d_err, 0, 8 * sizeof(int), c->stream));
  const bool kick = o.kickrank > 0;
  const int64_t rmax = o.rmax > 0 ? o.rmax : INT64_MAX;
  auto Xk = [&](int64_t i, int64_t j) { return X[j]->core + X[j]->ps[i]; };
  auto rxj = [&](int64_t i, int64_t j) { return X[j]->r[i]; };

  // Initial guesses (:152-187).  Given ones are orthogonalised from the
  // left (init_qr); missing ones are right-orthogonal random TTs of this
  // library's generator, orthogonalised the same way.
  ttg_tt_s* y0own = nullptr;
  ttg_tt_s* z0own = nullptr;
  if (!y0) y0 = y0own = tt_rand_device(c, n, 2, o.seed);
  if (kick && !z0) z0 = z0own = tt_rand_device(c, n, o.kickrank, o.seed ^ 0x9e3779b9ull);
  struct Own {
    ttg_tt_s *a, *b;
    ~Own() {
      if (a) ttg_tt_free(a);
      if (b) ttg_tt_free(b);
    }
  } own{y0own, z0own};
  const bool init_qr = o.init_qr != 0 || y0own != nullptr;
  TTG_REQUIRE(y0->ctx == c && !y0->is_matrix && y0->d == d && y0->r[0] == 1,
              "y0 shape mismatch");
  if (kick)
    TTG_REQUIRE(z0->ctx == c && !z0->is_matrix && z0->d == d && z0->r[0] == 1 && z0->r[d] == 1,
                "z0 shape mismatch");
  for (int64_t k = 0; k < d; ++k) {
    TTG_REQUIRE(y0->n[k] == n[k], "y0 mode size mismatch");
    if (kick) TTG_REQUIRE(z0->n[k] == n[k], "z0 mode size mismatch");
  }
  std::vector<int64_t> ry = y0->r, rz;
  std::vector<Buf> y(d), z(d);
  for (int64_t k = 0; k < d; ++k) {
    const int64_t sz = y0->ps[k + 1] - y0->ps[k];
    y[k].b.reset(c, sz);
    copy_f64(c, sz, y0->core + y0->ps[k], y[k].p());
  }
  if (kick) {
    rz = z0->r;
    for (int64_t k = 0; k < d; ++k) {
      const int64_t sz = z0->ps[k + 1] - z0->ps[k];
      z[k].b.reset(c, sz);
      copy_f64(c, sz, z0->core + z0->ps[k], z[k].p());
    }
  }
  DBuf<double> C(c, N * M);
  TTG_CUDA(cudaMemcpyAsync(C.p(), coef, sizeof(double) * N * M, cudaMemcpyHostToDevice,
                           c->stream));

  // Interfaces (:188-196): phiyx{i, j} 'lr' [ry, rx_j], 'rl' [rx_j, ry];
  // phizx likewise with z; phizy 'lr' [rz, ry], 'rl' [ry, rz].
  std::vector<std::vector<Buf>> phiyx(d + 1), phizx(d + 1);
  for (int64_t k = 0; k <= d; ++k) {
    phiyx[k].resize(N);
    phizx[k].resize(N);
  }
  std::vector<Buf> phizy(d + 1);
  for (int64_t k : {int64_t(0), d}) {
    for (int64_t j = 0; j < N; ++j) {
      phiyx[k][j].b.reset(c, 1);
      fill_f64(c, 1, 1.0, phiyx[k][j].p());
      phizx[k][j].b.reset(c, 1);
      fill_f64(c, 1, 1.0, phizx[k][j].p());
    }
    phizy[k].b.reset(c, 1);
    fill_f64(c, 1, 1.0, phizy[k].p());
  }
  // nrms (:129): scale of y carried outside its cores; sc[0] dx, sc[1]
  // max_dx, sc[2..2+N) interface norms.
  DBuf<double> nrms(c, d), sc(c, 2 + N);
  fill_f64(c, d, 1.0, nrms.p());

  // Y'X interfaces with the largest norm taken out (:580-588).
  auto y_lr = [&](int64_t i) {
    for (int64_t j = 0; j < N; ++j) {
      phi_pair(c, 0, ry[i], n[i], ry[i + 1], rxj(i, j), rxj(i + 1, j), phiyx[i][j].p(), y[i].p(),
               Xk(i, j), phiyx[i + 1][j]);
      dot_f64(c, ry[i + 1] * rxj(i + 1, j), phiyx[i + 1][j].p(), nullptr, sc.p() + 2 + j, true);
    }
    fill_f64(c, 1, 0.0, nrms.p() + i);
    for (int64_t j = 0; j < N; ++j) scalar_op(c, SC_MAXUPD, nrms.p() + i, sc.p() + 2 + j);
    scalar_op(c, SC_ONE_IF_ZERO, nrms.p() + i, nrms.p() + i);
    for (int64_t j = 0; j < N; ++j)
      scale_dev_f64(c, ry[i + 1] * rxj(i + 1, j), phiyx[i + 1][j].p(), phiyx[i + 1][j].p(),
                    nullptr, nrms.p() + i);
  };
  auto y_rl = [&](int64_t i) {
    for (int64_t j = 0; j < N; ++j) {
      phi_pair(c, 1, ry[i], n[i], ry[i + 1], rxj(i, j), rxj(i + 1, j), phiyx[i + 1][j].p(),
               y[i].p(), Xk(i, j), phiyx[i][j]);
      dot_f64(c, rxj(i, j) * ry[i], phiyx[i][j].p(), nullptr, sc.p() + 2 + j, true);
    }
    fill_f64(c, 1, 0.0, nrms.p() + i);
    for (int64_t j = 0; j < N; ++j) scalar_op(c, SC_MAXUPD, nrms.p() + i, sc.p() + 2 + j);
    scalar_op(c, SC_ONE_IF_ZERO, nrms.p() + i, nrms.p() + i);
    for (int64_t j = 0; j < N; ++j)
      scale_dev_f64(c, rxj(i, j) * ry[i], phiyx[i][j].p(), phiyx[i][j].p(), nullptr,
                    nrms.p() + i);
  };
  // Z'X divided by the Y'X norm, Z'Y as is (:216-222, :354-360, :435-441).
  auto z_lr = [&](int64_t i) {
    for (int64_t j = 0; j < N; ++j) {
      phi_pair(c, 0, rz[i], n[i], rz[i + 1], rxj(i, j), rxj(i + 1, j), phizx[i][j].p(), z[i].p(),
               Xk(i, j), phizx[i + 1][j]);
      scale_dev_f64(c, rz[i + 1] * rxj(i + 1, j), phizx[i + 1][j].p(), phizx[i + 1][j].p(),
                    nullptr, nrms.p() + i);
    }
    phi_pair(c, 0, rz[i], n[i], rz[i + 1], ry[i], ry[i + 1], phizy[i].p(), z[i].p(), y[i].p(),
             phizy[i + 1]);
  };
  auto z_rl = [&](int64_t i) {
    for (int64_t j = 0; j < N; ++j) {
      phi_pair(c, 1, rz[i], n[i], rz[i + 1], rxj(i, j), rxj(i + 1, j), phizx[i + 1][j].p(),
               z[i].p(), Xk(i, j), phizx[i][j]);
      scale_dev_f64(c, rxj(i, j) * rz[i], phizx[i][j].p(), phizx[i][j].p(), nullptr,
                    nrms.p() + i);
    }
    phi_pair(c, 1, rz[i], n[i], rz[i + 1], ry[i], ry[i + 1], phizy[i + 1].p(), z[i].p(),
             y[i].p(), phizy[i]);
  };
  // proj_sum (:647-684): out (ra1 n ra2 x M) = sum_j vec(Phi1_j X_j Phi2_j) c(j, :)
  // with Phi1_j [ra1, rx_j] and Phi2_j [rx_j, ra2].
  auto proj_sum = [&](const std::vector<Buf>& P1, int64_t ra1, int64_t i,
                      const std::vector<Buf>& P2, int64_t ra2, DBuf<double>& out) {
    const int64_t L = ra1 * n[i] * ra2;
    DBuf<double> T(c, L * N);
    for (int64_t j = 0; j < N; ++j) {
      const int64_t r1 = rxj(i, j), r2 = rxj(i + 1, j);
      DBuf<double> t1(c, ra1 * n[i] * r2);
      gemm_f64(c, false, false, ra1, n[i] * r2, r1, 1.0, P1[j].p(), ra1, 0, Xk(i, j), r1, 0, 0.0,
               t1.p(), ra1, 0, 1);
      gemm_f64(c, false, false, ra1 * n[i], ra2, r2, 1.0, t1.p(), ra1 * n[i], 0, P2[j].p(), r2,
               0, 0.0, T.p() + L * j, ra1 * n[i], 0, 1);
    }
    out.reset(c, L * M);
    gemm_f64(c, false, false, L, M, N, 1.0, T.p(), L, 0, C.p(), N, 0, 0.0, out.p(), L, 0, 1);
  };
  // QR of the left-unfolded core i, R/||R||_F pushed into core i+1 (:196-210).
  auto orth_left = [&](std::vector<Buf>& t, std::vector<int64_t>& r, int64_t i) {
    const int64_t m = r[i] * n[i], cols = r[i + 1], k = std::min(m, cols);
    DBuf<double> Q(c, m * k), R(c, k * cols), nr(c, 1);
    qr_f64(c, m, cols, t[i].p(), Q.p(), R.p());
    dot_f64(c, k * cols, R.p(), nullptr, nr.p(), true);
    normalize_by_dev(c, k * cols, R.p(), nr.p());
    const int64_t nc = n[i + 1] * r[i + 2];
    DBuf<double> nx(c, k * nc);
    gemm_f64(c, false, false, k, nc, cols, 1.0, R.p(), k, 0, t[i + 1].p(), cols, 0, 0.0, nx.p(),
             k, 0, 1);
    r[i + 1] = k;
    t[i].b = std::move(Q);
    t[i + 1].b = std::move(nx);
  };
  auto svd_rank = [&](const DBuf<double>& S, int64_t K) {
    std::vector<double> hs(K);
    read_scalars(c, S.p(), hs.data(), int(K));
    double ns = 0.0;
    for (double v : hs) ns += v * v;
    const int64_t r = my_chop2(hs.data(), K, tol * std::sqrt(ns) / std::sqrt(double(d)));
    return std::min(r, rmax);                                               // :288-289
  };

  for (int64_t i = 0; i + 1 < d; ++i) {                                     // :194-241
    if (init_qr) orth_left(y, ry, i);
    y_lr(i);
    if (kick) {
      orth_left(z, rz, i);
      z_lr(i);
    }
  }
  // The last core carries the output index (:247-251): [ry, n, 1, M], its
  // first min(ry_d, M) columns kept, zero-padded to M.
  {
    const int64_t rows = ry[d - 1] * n[d - 1], k = std::min(ry[d], M);
    DBuf<double> last(c, rows * M);
    fill_f64(c, rows * M, 0.0, last.p());
    copy_f64(c, rows * k, y[d - 1].p(), last.p());
    y[d - 1].b = std::move(last);
    ry[d] = 1;
  }

  int64_t i = d - 1, dir = -1, swp = 1, sweeps = 0;                         // :253
  fill_f64(c, 1, 0.0, sc.p() + 1);
  DBuf<double> cry;
  while (swp <= o.nswp) {
    proj_sum(phiyx[i], ry[i], i, phiyx[i + 1], ry[i + 1], cry);            // :255
    const int64_t L = ry[i] * n[i] * ry[i + 1];
    dot_f64(c, L * M, cry.p(), nullptr, nrms.p() + i, true);               // :256-263
    normalize_by_dev(c, L * M, cry.p(), nrms.p() + i);
    // dx = ||cry - y_i|| / ||cry|| (||cry|| = 1 unless cry = 0)  (:265-269)
    diffnrm_f64(c, L * M, cry.p(), y[i].p(), sc.p(), true);
    scalar_op(c, SC_MAXUPD, sc.p() + 1, sc.p());
    const int64_t ni = n[i];
    if (dir > 0 && i < d - 1) {                                             // :271
      const int64_t Mr = ry[i] * ni, Cc = ry[i + 1] * M, K = std::min(Mr, Cc);
      DBuf<double> U(c, Mr * K), S(c, K), VT(c, K * Cc);
      svd_f64(c, Mr, Cc, cry.p(), U.p(), S.p(), VT.p());
      const int64_t r = svd_rank(S, K);
      DBuf<double> u(c, Mr * r), vt(c, Cc * r), v(c, Cc * r);
      copy_f64(c, Mr * r, U.p(), u.p());
      transpose_f64(c, r, Cc, VT.p(), K, vt.p(), Cc);
      copy2d_f64(c, Cc, r, vt.p(), Cc, v.p(), Cc, S.p());                  // :291 V s
      DBuf<double> crz;
      int64_t kz = 0;
      if (kick) {                                                           // :301-327
        // cry2 = u v' as (ry n ry2) x M
        DBuf<double> cry2(c, Mr * Cc);
        gemm_f64(c, false, true, Mr, Cc, r, 1.0, u.p(), Mr, 0, v.p(), Cc, 0, 0.0, cry2.p(), Mr,
                 0, 1);
        // crys = reshape(cry2.', M ry n, ry2) * phizy{i+1}  -> (M ry n) x rz2
        DBuf<double> c2t(c, L * M), crys(c, M * Mr * rz[i + 1]);
        transpose_f64(c, L, M, cry2.p(), L, c2t.p(), M);
        gemm_f64(c, false, false, M * Mr, rz[i + 1], ry[i + 1], 1.0, c2t.p(), M * Mr, 0,
                 phizy[i + 1].p(), ry[i + 1], 0, 0.0, crys.p(), M * Mr, 0, 1);
        // crys = reshape(crys, M, ry n rz2).'  -> (ry n rz2) x M
        DBuf<double> cs(c, Mr * rz[i + 1] * M);
        transpose_f64(c, M, Mr * rz[i + 1], crys.p(), M, cs.p(), Mr * rz[i + 1]);
        // cryz = phizy{i} * reshape(crys, ry, n rz2 M) -> (rz n rz2) x M
        const int64_t Lz = rz[i] * ni * rz[i + 1];
        DBuf<double> cryz(c, Lz * M);
        gemm_f64(c, false, false, rz[i], ni * rz[i + 1] * M, ry[i], 1.0, phizy[i].p(), rz[i], 0,
                 cs.p(), ry[i], 0, 0.0, cryz.p(), rz[i], 0, 1);
        // crz = proj_sum(phizx) / nrms(i) - cryz
        proj_sum(phizx[i], rz[i], i, phizx[i + 1], rz[i + 1], crz);
        scale_dev_f64(c, Lz * M, crz.p(), crz.p(), nullptr, nrms.p() + i);
        axpby_f64(c, Lz * M, -1.0, cryz.p(), 1.0, crz.p());
        // left singular vectors of (rz n) x (rz2 M), first kickrank of them
        const int64_t zm = rz[i] * ni, zc = rz[i + 1] * M, zk = std::min(zm, zc);
        DBuf<double> Uz(c, zm * zk), Sz(c, zk), VTz(c, zk * zc);
        svd_f64(c, zm, zc, crz.p(), Uz.p(), Sz.p(), VTz.p());
        kz = std::min(zk, o.kickrank);
        crz.reset(c, zm * kz);
        copy_f64(c, zm * kz, Uz.p(), crz.p());
      }
      y[i].b = std::move(u);                                                // :342
      // cr2 = reshape(v, ry2, M r).' * y{i+1}  -> (M r) x (n2 ry3), then
      // reshape(., M, r n2 ry3).'  -> [r, n2, ry3, M]  (:344-348)
      const int64_t nc = n[i + 1] * ry[i + 2];
      DBuf<double> t(c, M * r * nc), nx(c, r * nc * M);
      gemm_f64(c, true, false, M * r, nc, ry[i + 1], 1.0, v.p(), ry[i + 1], 0, y[i + 1].p(),
               ry[i + 1], 0, 0.0, t.p(), M * r, 0, 1);
      transpose_f64(c, M, r * nc, t.p(), M, nx.p(), r * nc);
      y[i + 1].b = std::move(nx);
      ry[i + 1] = r;
      y_lr(i);                                                              // :352
      if (kick) {                                                           // :354-360
        rz[i + 1] = kz;
        z[i].b = std::move(crz);
        z_lr(i);
      }
    } else if (dir < 0 && i > 0) {                                          // :361
      // SVD of reshape(cry.', M ry, n ry2)
      const int64_t Mr = M * ry[i], Cc = ni * ry[i + 1], K = std::min(Mr, Cc);
      DBuf<double> cT(c, L * M);
      transpose_f64(c, L, M, cry.p(), L, cT.p(), M);
      DBuf<double> U(c, Mr * K), S(c, K), VT(c, K * Cc);
      svd_f64(c, Mr, Cc, cT.p(), U.p(), S.p(), VT.p());
      int64_t r = svd_rank(S, K);
      DBuf<double> u(c, Mr * r), v(c, Cc * r);
      copy2d_f64(c, Mr, r, U.p(), Mr, u.p(), Mr, S.p());                   // u s
      transpose_f64(c, r, Cc, VT.p(), K, v.p(), Cc);                       // V(:, 1:r)
      DBuf<double> crz;
      int64_t kz = 0;
      if (kick) {                                                           // :382-420
        // cry2 = reshape(u v', M, ry n ry2)
        DBuf<double> cry2(c, Mr * Cc);
        gemm_f64(c, false, true, Mr, Cc, r, 1.0, u.p(), Mr, 0, v.p(), Cc, 0, 0.0, cry2.p(), Mr,
                 0, 1);
        // crys = phizy{i} * reshape(cry2.', ry, n ry2 M) -> (rz n ry2) x M
        DBuf<double> c2t(c, L * M), crys(c, rz[i] * ni * ry[i + 1] * M);
        transpose_f64(c, M, L, cry2.p(), M, c2t.p(), L);
        gemm_f64(c, false, false, rz[i], ni * ry[i + 1] * M, ry[i], 1.0, phizy[i].p(), rz[i], 0,
                 c2t.p(), ry[i], 0, 0.0, crys.p(), rz[i], 0, 1);
        // cryz = reshape(crys.', M rz n, ry2) * phizy{i+1}, then transposed
        const int64_t Lz = rz[i] * ni * rz[i + 1], Ls = rz[i] * ni * ry[i + 1];
        DBuf<double> cst(c, Ls * M), cz(c, M * rz[i] * ni * rz[i + 1]), cryz(c, Lz * M);
        transpose_f64(c, Ls, M, crys.p(), Ls, cst.p(), M);
        gemm_f64(c, false, false, M * rz[i] * ni, rz[i + 1], ry[i + 1], 1.0, cst.p(),
                 M * rz[i] * ni, 0, phizy[i + 1].p(), ry[i + 1], 0, 0.0, cz.p(),
                 M * rz[i] * ni, 0, 1);
        transpose_f64(c, M, Lz, cz.p(), M, cryz.p(), Lz);
        // crz = proj_sum(phizx, phizx) / nrms(i) - cryz; rows of V' (kickrank)
        proj_sum(phizx[i], rz[i], i, phizx[i + 1], rz[i + 1], crz);
        scale_dev_f64(c, Lz * M, crz.p(), crz.p(), nullptr, nrms.p() + i);
        axpby_f64(c, Lz * M, -1.0, cryz.p(), 1.0, crz.p());
        {
          const int64_t zm = M * rz[i], zc = ni * rz[i + 1], zk = std::min(zm, zc);
          DBuf<double> zt(c, Lz * M), Uz(c, zm * zk), Sz(c, zk), VTz(c, zk * zc);
          transpose_f64(c, Lz, M, crz.p(), Lz, zt.p(), M);
          svd_f64(c, zm, zc, zt.p(), Uz.p(), Sz.p(), VTz.p());
          kz = std::min(zk, o.kickrank);
          crz.reset(c, kz * zc);                                          // (kz, n rz2)
          copy2d_f64(c, kz, zc, VTz.p(), zk, crz.p(), kz);
        }
        // crs = proj_sum(phizx{i}, phiyx{i+1}) / nrms(i) - crys; rows of V'
        DBuf<double> crs;
        proj_sum(phizx[i], rz[i], i, phiyx[i + 1], ry[i + 1], crs);
        scale_dev_f64(c, Ls * M, crs.p(), crs.p(), nullptr, nrms.p() + i);
        axpby_f64(c, Ls * M, -1.0, crys.p(), 1.0, crs.p());
        int64_t ks = 0;
        DBuf<double> crsT;  // (n ry2) x ks
        {
          const int64_t sm = M * rz[i], scn = ni * ry[i + 1], sk = std::min(sm, scn);
          DBuf<double> st(c, Ls * M), Us(c, sm * sk), Ss(c, sk), VTs(c, sk * scn);
          transpose_f64(c, Ls, M, crs.p(), Ls, st.p(), M);
          svd_f64(c, sm, scn, st.p(), Us.p(), Ss.p(), VTs.p());
          ks = std::min(sk, o.kickrank);
          crsT.reset(c, scn * ks);
          transpose_f64(c, ks, scn, VTs.p(), sk, crsT.p(), scn);
        }
        // [v, R] = qr([v, crs]); u = [u, 0] * R.'  (:412-418)
        const int64_t w = r + ks;
        DBuf<double> vv(c, Cc * w);
        copy_f64(c, Cc * r, v.p(), vv.p());
        copy_f64(c, Cc * ks, crsT.p(), vv.p() + Cc * r);
        const int64_t k2 = std::min(Cc, w);
        DBuf<double> Q(c, Cc * k2), R(c, k2 * w), un(c, Mr * k2);
        qr_f64(c, Cc, w, vv.p(), Q.p(), R.p());
        gemm_f64(c, false, true, Mr, k2, r, 1.0, u.p(), Mr, 0, R.p(), k2, 0, 0.0, un.p(), Mr, 0,
                 1);
        u = std::move(un);
        v = std::move(Q);
        r = k2;
      }
      // y{i} = v.' [r, n, ry2]; y{i-1} = y{i-1} * uu  [ry0, n0, r, M]  (:421-429)
      DBuf<double> yi(c, r * Cc);
      transpose_f64(c, Cc, r, v.p(), Cc, yi.p(), r);
      // uu = reshape(reshape(u, M, ry r).', ry, r M)
      DBuf<double> uu(c, Mr * r);
      transpose_f64(c, M, ry[i] * r, u.p(), M, uu.p(), ry[i] * r);
      const int64_t mp = ry[i - 1] * n[i - 1];
      DBuf<double> prev(c, mp * r * M);
      gemm_f64(c, false, false, mp, r * M, ry[i], 1.0, y[i - 1].p(), mp, 0, uu.p(), ry[i], 0,
               0.0, prev.p(), mp, 0, 1);
      y[i].b = std::move(yi);
      y[i - 1].b = std::move(prev);
      ry[i] = r;
      y_rl(i);                                                              // :433
      if (kick) {                                                           // :435-441
        rz[i] = kz;
        z[i].b = std::move(crz);
        z_rl(i);
      }
    }
    // At the turning cores y{i} keeps its value (:442-444); the last
    // projection becomes y{d} after the sweeps (:466).
    if ((dir > 0 && i == d - 1) || (dir < 0 && i == 0)) {                   // :451-463
      if (dir > 0) {
        sweeps = swp;
        double mdx = 0.0;
        read_scalars(c, sc.p() + 1, &mdx, 1);
        if (o.verb > 0)
          fprintf(stderr, "amen_sum: swp=%lld, max_dx=%3.3e, max_r=%lld\n", (long long)swp, mdx,
                  (long long)*std::max_element(ry.begin(), ry.end()));
        if (mdx < tol || swp == o.nswp) break;
      }
      fill_f64(c, 1, 0.0, sc.p() + 1);
      if (dir > 0) ++swp;
      dir = -dir;
    } else {
      i += dir;
    }
  }
  // y{d} = cry as [ry, n, M] (:466): the output rank M is the last TT rank.
  const int64_t Ld = ry[d - 1] * n[d - 1];
  y[d - 1].b.reset(c, Ld * M);
  copy_f64(c, Ld * M, cry.p(), y[d - 1].p());
  ry[d] = M;
  std::vector<double> hn(d);                                                // :469-473
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
  ttg_tt_s* zo = (kick && z_out) ? pack(z, rz, 1.0) : nullptr;
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
