// TT rounding on the device (FP64): restates @tt_tensor/round.m:20-108.
//
// Cores stay on the device; the host only sees the R-factor norms and the
// singular values it needs for the rank decision (my_chop2,
// core/my_chop2.m:18-35).
#include <cmath>
#include <vector>

#include "linalg.h"
#include "mixed_ops.h"
#include "round.h"

namespace ttg {

int64_t my_chop2(const double* sv, int64_t n, double eps) {
  double nrm = 0.0;
  for (int64_t i = 0; i < n; ++i) nrm += sv[i] * sv[i];
  if (std::sqrt(nrm) == 0.0) return 1;  // my_chop2.m:18-21
  if (eps <= 0) return n;               // my_chop2.m:23-26
  // sv0 = cumsum(sv(end:-1:1).^2); ff = find(sv0 < eps^2); r = n - ff(end)
  double acc = 0.0;
  int64_t last = -1;  // 0-based index into the reversed cumulative sums
  for (int64_t k = 0; k < n; ++k) {
    acc += sv[n - 1 - k] * sv[n - 1 - k];
    if (acc < eps * eps) last = k;
  }
  if (last < 0) return n;
  return n - (last + 1);
}

namespace {
struct Timer {
  Context* c;
  cudaEvent_t a, b;
  explicit Timer(Context* cc) : c(cc) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, c->stream);
  }
  double stop() {
    cudaEventRecord(b, c->stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};
}  // namespace

ttg_tt_s* round_tt(ttg_tt_s* in, double eps, const std::vector<int64_t>& rmax_in, int precision,
                   ttg_round_stats* stats) {
  Context* c = in->ctx;
  TTG_REQUIRE(!in->is_matrix, "round: TT matrices are rounded through their tensor form");
  TTG_REQUIRE(precision == TTG_FP64 || precision == TTG_MIXED, "round: unknown precision %d",
              precision);
  require_finite(in, "the input tensor");
  const int64_t d = in->d;
  std::vector<int64_t> n = in->n, r = in->r;
  std::vector<int64_t> rmax(d + 1, INT64_MAX);
  if (rmax_in.size() == 1)
    for (auto& v : rmax) v = rmax_in[0];
  else if (rmax_in.size() == size_t(d + 1))
    rmax = rmax_in;
  Timer t_all(c);
  // Working copies of the cores (capacity: the input sizes bound every
  // intermediate core since QR/SVD never increase a rank).
  std::vector<DBuf<double>> cr(d);
  for (int64_t k = 0; k < d; ++k) {
    cr[k].reset(c, in->ps[k + 1] - in->ps[k]);
    copy_f64(c, in->ps[k + 1] - in->ps[k], in->core + in->ps[k], cr[k].p());
  }
  std::vector<double> nrm(d, 0.0);
  double ms_qr = 0, ms_svd = 0;
  int64_t fallbacks = 0;
  {
    Timer tq(c);
    // Left-to-right QR sweep (round.m:39-53).
    for (int64_t i = 0; i + 1 < d; ++i) {
      const int64_t m = r[i] * n[i], cols = r[i + 1];
      const int64_t k = std::min(m, cols);
      DBuf<double> Q(c, m * k), R(c, k * cols);
      qr_f64(c, m, cols, cr[i].p(), Q.p(), R.p());
      nrm[i + 1] = nrm2_host(c, k * cols, R.p());                     // round.m:41
      if (nrm[i + 1] != 0.0) axpby_f64(c, k * cols, 1.0 / nrm[i + 1], R.p(), 0.0, R.p());
      const int64_t nc = n[i + 1] * r[i + 2];
      DBuf<double> c1(c, k * nc);
      if (precision == TTG_MIXED)                                       // round.m:47
        gemm_bf16(c, false, false, k, nc, cols, R.p(), k, cr[i + 1].p(), cols, c1.p(), k);
      else
        gemm_f64(c, false, false, k, nc, cols, 1.0, R.p(), k, 0, cr[i + 1].p(), cols, 0, 0.0,
                 c1.p(), k, 0, 1);
      r[i + 1] = k;                                                     // round.m:48
      cr[i] = std::move(Q);
      cr[i + 1] = std::move(c1);
    }
    ms_qr = tq.stop();
  }
  const double ep = d > 1 ? eps / std::sqrt(double(d - 1)) : eps;       // round.m:56
  {
    Timer ts(c);
    std::vector<double> hs;
    // Right-to-left SVD sweep (round.m:59-89).
    for (int64_t i = d - 1; i >= 1; --i) {
      const int64_t rows = r[i], cols = n[i] * r[i + 1];
      const int64_t K = std::min(rows, cols);
      DBuf<double> U(c, rows * K), S(c, K), VT(c, K * cols);
      TTG_CUDA(cudaMemsetAsync(c->d_err + 3, 0, sizeof(int), c->stream));
      svd_f64(c, rows, cols, cr[i].p(), U.p(), S.p(), VT.p());          // round.m:65
      hs.resize(K);
      int sweep_cap = 0;
      TTG_CUDA(cudaMemcpyAsync(&sweep_cap, c->d_err + 3, sizeof(int), cudaMemcpyDeviceToHost,
                               c->stream));
      sync(c);
      if (sweep_cap) {  // the Jacobi SVD did not converge: round.m:64-74's fallback
        TTG_CUDA(cudaMemsetAsync(c->d_err + 3, 0, sizeof(int), c->stream));
        svd_f64_fallback(c, rows, cols, cr[i].p(), U.p(), S.p(), VT.p());
        fallbacks++;
      }
      TTG_CUDA(cudaMemcpyAsync(hs.data(), S.p(), sizeof(double) * K, cudaMemcpyDeviceToHost,
                               c->stream));
      sync(c);
      double ns = 0.0;
      for (double v : hs) ns += v * v;
      int64_t r1 = my_chop2(hs.data(), K, std::sqrt(ns) * ep);         // round.m:77
      r1 = std::min(r1, rmax[i]);                                        // round.m:78
      if (r1 < 1) r1 = 1;
      // core_{i-1} = core_{i-1} * (U(:,1:r1) diag(s))  (round.m:80-83)
      DBuf<double> US(c, rows * r1);
      copy2d_f64(c, rows, r1, U.p(), rows, US.p(), rows, S.p());
      const int64_t m1 = r[i - 1] * n[i - 1];
      DBuf<double> c1(c, m1 * r1);
      if (precision == TTG_MIXED)                                       // round.m:83
        gemm_bf16(c, false, false, m1, r1, rows, cr[i - 1].p(), m1, US.p(), rows, c1.p(), m1);
      else
        gemm_f64(c, false, false, m1, r1, rows, 1.0, cr[i - 1].p(), m1, 0, US.p(), rows, 0, 0.0,
                 c1.p(), m1, 0, 1);
      // core_i = VT(1:r1, :)  (round.m:84)
      DBuf<double> c0(c, r1 * cols);
      copy2d_f64(c, r1, cols, VT.p(), K, c0.p(), r1);
      r[i] = r1;
      cr[i] = std::move(c0);
      cr[i - 1] = std::move(c1);
    }
    ms_svd = ts.stop();
  }
  // Norm balancing (round.m:94-107).
  const int64_t s0 = r[0] * n[0] * r[1];
  nrm[0] = nrm2_host(c, s0, cr[0].p());
  if (nrm[0] != 0.0) axpby_f64(c, s0, 1.0 / nrm[0], cr[0].p(), 0.0, cr[0].p());
  double lsum = 0.0;
  for (double v : nrm) lsum += std::log(std::fabs(v));
  const double nrm0 = std::exp(lsum / double(d));
  auto* out = new ttg_tt_s();
  out->ctx = c;
  out->d = d;
  out->is_matrix = false;
  out->n = n;
  out->r = r;
  out->ps.assign(d + 1, 0);
  for (int64_t k = 0; k < d; ++k) out->ps[k + 1] = out->ps[k] + r[k] * n[k] * r[k + 1];
  out->numel = out->ps[d];
  out->core = static_cast<double*>(c->alloc->get(sizeof(double) * out->numel));
  for (int64_t k = 0; k < d; ++k)
    axpby_f64(c, out->ps[k + 1] - out->ps[k], nrm0, cr[k].p(), 0.0, out->core + out->ps[k]);
  const double ms_all = t_all.stop();
  if (stats) {
    stats->ms_total = ms_all;
    stats->ms_qr_sweep = ms_qr;
    stats->ms_svd_sweep = ms_svd;
    int64_t mr = 0;
    for (auto v : r) mr = std::max(mr, v);
    stats->max_rank = mr;
    stats->svd_fallbacks = fallbacks;
  }
  return out;
}

}  // namespace ttg
