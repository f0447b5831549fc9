// extern "C" entry points of the hot path (include/ttgpu.h).
#include <atomic>
#include <cmath>
#include <thread>

#include "amen.h"
#include "group.cuh"
#include "grad.h"
#include "linalg.h"
#include "round.h"
#include "mixed_ops.h"

using namespace ttg;

namespace {

// Shared checks of the gradient entries: same context, a device output.
ttg::Context* grad_ctx(ttg_tt x, ttg_tt other, double* grad) {
  TTG_REQUIRE(x && grad, "NULL argument");
  if (other) TTG_REQUIRE(other->ctx == x->ctx, "operands belong to different contexts");
  TTG_CUDA(cudaSetDevice(x->ctx->device));
  return x->ctx;
}

// Error slots start clear for every call that reads them at its end, so a
// failed call cannot leak its flags into the next one.
void clear_error_slots(ttg::Context* c) {
  TTG_CUDA(cudaMemsetAsync(c->d_err, 0, 8 * sizeof(int), c->stream));
}

void grad_value_out(ttg::Context* c, const double* dval, double* value) {
  if (value) ttg::read_scalars(c, dval, value, 1);
}

// Checks shared by the batched entries; clears the outputs.
void check_batch(Context* owner, int64_t count, const ttg_tt* A, const ttg_tt* y,
                 const double* tol, const ttg_tt* x0, const ttg_tt* z0, ttg_tt* x_out,
                 ttg_amen_stats* stats, int32_t* status) {
  TTG_REQUIRE(A && y && tol, "NULL argument");
  for (int64_t i = 0; i < count; ++i) {
    x_out[i] = nullptr;
    if (status) status[i] = TTG_OK;
    if (stats) stats[i] = ttg_amen_stats{};
    TTG_REQUIRE(A[i] && y[i], "system %lld: NULL handle", (long long)i);
    TTG_REQUIRE(A[i]->ctx == owner && y[i]->ctx == owner,
                "system %lld: handles belong to another context", (long long)i);
    if (x0 && x0[i]) TTG_REQUIRE(x0[i]->ctx == owner, "system %lld: x0 context", (long long)i);
    if (z0 && z0[i]) TTG_REQUIRE(z0[i]->ctx == owner, "system %lld: z0 context", (long long)i);
    TTG_REQUIRE(std::isfinite(tol[i]) && tol[i] > 0, "system %lld: tol must be > 0",
                (long long)i);
  }
}

}  // namespace

extern "C" {

void ttg_amen_opts_default(ttg_amen_opts* o) {
  if (!o) return;
  o->nswp = 50;            // amen_solve2.m:79
  o->rmax = 1000;          // :87
  o->max_full_size = 50;   // :75
  o->local_restart = 40;   // :80
  o->local_iters = 2;      // :81
  o->kickrank = 4;         // :102
  o->resid_damp = 2.0;     // :77
  o->tol_exit = 0.0;       // :92, :156-158
  o->trunc_norm = 1;       // :88-89
  o->local_prec = 0;       // :83-84
  o->precision = TTG_FP64;
  o->verb = 0;
  o->seed = 0x243F6A8885A308D3ull;
  o->timing = 0;
  o->reserved = 0;
  o->trace = nullptr;
  o->trace_cap = 0;
}

int ttg_context_set_option(ttg_context ctx, int32_t key, int64_t value) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx, "NULL argument");
  switch (key) {
    case TTG_OPT_JACOBI_MAX_SWEEPS:
      TTG_REQUIRE(value >= 1 && value <= 1000, "Jacobi sweep limit %lld out of [1, 1000]",
                  (long long)value);
      ctx->c.jacobi_max_sweeps = int(value);
      break;
    case TTG_OPT_GROUP_SMS:
      TTG_REQUIRE(value >= 0 && value <= 4096, "SM count %lld out of [0, 4096]",
                  (long long)value);
      ctx->c.group_sms = int(value);
      break;
    default:
      fail(TTG_ERR_INVALID, "unknown context option %d", int(key));
  }
  TTG_API_END
}

int ttg_selftest_wait(ttg_context ctx, int32_t which) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx, "NULL argument");
  TTG_REQUIRE(which >= 0 && which <= 3, "unknown wait %d", int(which));
  Context* c = &ctx->c;
  TTG_CUDA(cudaSetDevice(c->device));
  DBuf<int> flag(c, 1);
  TTG_CUDA(cudaMemsetAsync(flag.p(), 0, sizeof(int), c->stream));
  const long long limit = 1 << 14;
  switch (which) {
    case 0: selftest_wait_gmres(c, flag.p(), limit); break;
    case 1: selftest_wait_mbarrier(c, flag.p(), limit); break;
    case 2: selftest_wait_jacobi(c, flag.p(), limit); break;
    default: selftest_wait_arnoldi(c, flag.p(), limit); break;
  }
  int h = 0;
  TTG_CUDA(cudaMemcpyAsync(&h, flag.p(), sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  if (h) fail(TTG_ERR_TIMEOUT, "bounded device wait %d gave up (code %d)", int(which), h);
  TTG_API_END
}

int ttg_round(ttg_tt in, double eps, const int64_t* rmax, int64_t nrmax, int32_t precision,
              ttg_tt* out, ttg_round_stats* stats) {
  TTG_API_BEGIN
  TTG_REQUIRE(in && out, "NULL argument");
  TTG_REQUIRE(std::isfinite(eps) && eps >= 0, "eps must be finite and >= 0");
  TTG_REQUIRE(rmax == nullptr || nrmax == 1 || nrmax == in->d + 1,
              "rmax must have 1 or d+1 entries");
  TTG_CUDA(cudaSetDevice(in->ctx->device));
  clear_error_slots(in->ctx);
  std::vector<int64_t> rm;
  if (rmax) {
    rm.assign(rmax, rmax + nrmax);
    for (auto v : rm) TTG_REQUIRE(v >= 1, "rmax entries must be >= 1");
  }
  *out = round_tt(in, eps, rm, precision, stats);
  check_factorizations(in->ctx);
  TTG_API_END
}

int ttg_amen_solve(ttg_tt A, ttg_tt y, double tol, const ttg_amen_opts* opts, ttg_tt x0,
                   ttg_tt z0, ttg_tt* x_out, ttg_amen_stats* stats) {
  TTG_API_BEGIN
  TTG_REQUIRE(A && y && x_out, "NULL argument");
  TTG_REQUIRE(std::isfinite(tol) && tol > 0, "tol must be > 0");
  ttg_amen_opts o;
  if (opts)
    o = *opts;
  else
    ttg_amen_opts_default(&o);
  if (stats) *stats = ttg_amen_stats{};
  TTG_CUDA(cudaSetDevice(A->ctx->device));
  if (x0) TTG_REQUIRE(x0->ctx == A->ctx, "x0 belongs to another context");
  if (z0) TTG_REQUIRE(z0->ctx == A->ctx, "z0 belongs to another context");
  *x_out = amen_solve(A->ctx, A, y, tol, o, x0, z0, stats);
  TTG_API_END
}

void ttg_alstpz_opts_default(ttg_amen_opts* o) {
  if (!o) return;
  ttg_amen_opts_default(o);
  o->nswp = 10;           // alstpz_solve.m:61
  o->max_full_size = 50;  // :56
  o->kickrank = 4;        // :67
}

int ttg_alstpz_solve(ttg_tt A, ttg_tt y, double tol, const ttg_amen_opts* opts, ttg_tt x0,
                     ttg_tt* x_out, ttg_amen_stats* stats) {
  TTG_API_BEGIN
  TTG_REQUIRE(A && y && x_out, "NULL argument");
  TTG_REQUIRE(std::isfinite(tol) && tol > 0, "tol must be > 0");
  ttg_amen_opts o;
  if (opts)
    o = *opts;
  else
    ttg_alstpz_opts_default(&o);
  if (stats) *stats = ttg_amen_stats{};
  TTG_CUDA(cudaSetDevice(A->ctx->device));
  if (x0) TTG_REQUIRE(x0->ctx == A->ctx, "x0 belongs to another context");
  *x_out = alstpz_solve(A->ctx, A, y, tol, o, x0, stats);
  TTG_API_END
}

int ttg_local_matvec(ttg_context ctx, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1,
                     int64_t ra2, const double* Phi1, const double* A, const double* Phi2,
                     const double* x, double* y, int32_t precision) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && Phi1 && A && Phi2 && x && y, "NULL argument");
  TTG_REQUIRE(rx1 >= 1 && n >= 1 && rx2 >= 1 && ra1 >= 1 && ra2 >= 1, "sizes must be >= 1");
  TTG_REQUIRE(precision == TTG_FP64 || precision == TTG_MIXED,
              "ttg_local_matvec: unknown precision %d", precision);
  Context* c = &ctx->c;
  TTG_CUDA(cudaSetDevice(c->device));
  MvDims d{rx1, rx1, ra1, n, n, rx2, ra2, rx2};
  if (precision == TTG_FP64) {
    local_matvec_f64(c, d, Phi1, A, Phi2, x, y);
  } else {
    // BF16 tensor-core path; vectors go through the reversed FP32 layout.
    const int64_t sz = d.in_size();
    MixedOp op;
    op.prepare(c, d, Phi1, A, Phi2);
    DBuf<float> xr(c, sz), yr(c, sz);
    TTG_CUDA(cudaMemsetAsync(c->d_err + 1, 0, sizeof(int), c->stream));
    nat_to_rev(c, rx1, n, rx2, x, xr.p(), 1.0);
    op.apply(c, xr.p(), yr.p());
    fill_f64(c, sz, 0.0, y);
    rev_to_nat_add(c, rx1, n, rx2, yr.p(), y, 1.0);
  }
  sync(c);
  if (precision == TTG_MIXED) {
    int herr = 0;
    TTG_CUDA(cudaMemcpy(&herr, c->d_err + 1, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) fail(TTG_ERR_TIMEOUT, "tensor-core matvec: a bounded wait timed out");
  }
  TTG_API_END
}

int ttg_next_phi(ttg_context ctx, int32_t dir, int64_t rx1, int64_t n, int64_t rx2, int64_t ry1,
                 int64_t ry2, int64_t ra1, int64_t ra2, const double* Phi_prev, const double* x,
                 const double* A, const double* y, double* Phi_out, double* nrm_out) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && Phi_prev && x && y && Phi_out, "NULL argument");
  TTG_REQUIRE(dir == 0 || dir == 1, "dir must be 0 ('lr') or 1 ('rl')");
  TTG_REQUIRE(rx1 >= 1 && n >= 1 && rx2 >= 1 && ry1 >= 1 && ry2 >= 1, "sizes must be >= 1");
  if (A) TTG_REQUIRE(ra1 >= 1 && ra2 >= 1, "ra sizes must be >= 1");
  Context* c = &ctx->c;
  TTG_CUDA(cudaSetDevice(c->device));
  const int64_t cnt =
      next_phi_f64(c, dir, rx1, n, rx2, ry1, ry2, ra1, ra2, Phi_prev, x, A, y, Phi_out);
  if (nrm_out) {
    double nrm = nrm2_host(c, cnt, Phi_out);
    if (nrm > 0)
      axpby_f64(c, cnt, 1.0 / nrm, Phi_out, 0.0, Phi_out);
    else
      nrm = 1.0;
    *nrm_out = nrm;
  }
  sync(c);
  TTG_API_END
}

int ttg_dense_qr(ttg_context ctx, int64_t m, int64_t n, const double* A, double* Q, double* R) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && A && Q && R, "NULL argument");
  TTG_REQUIRE(m >= 1 && n >= 1, "sizes must be >= 1");
  Context* c = &ctx->c;
  TTG_CUDA(cudaSetDevice(c->device));
  clear_error_slots(c);
  qr_f64(c, m, n, A, Q, R, true);
  check_factorizations(c);
  TTG_API_END
}

int ttg_dense_svd(ttg_context ctx, int64_t m, int64_t n, const double* A, double* U, double* S,
                  double* VT) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && A && U && S && VT, "NULL argument");
  TTG_REQUIRE(m >= 1 && n >= 1, "sizes must be >= 1");
  Context* c = &ctx->c;
  TTG_CUDA(cudaSetDevice(c->device));
  clear_error_slots(c);
  TTG_CUDA(cudaMemsetAsync(c->d_err + 3, 0, sizeof(int), c->stream));
  svd_f64(c, m, n, A, U, S, VT);
  int herr = 0;
  TTG_CUDA(cudaMemcpyAsync(&herr, c->d_err + 3, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  if (herr) fail(TTG_ERR_NOCONV, "Jacobi SVD reached its sweep limit");
  check_factorizations(c);
  TTG_API_END
}

int ttg_local_solve(ttg_context ctx, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1,
                    int64_t ra2, const double* Phi1, const double* A, const double* Phi2,
                    const double* rhs, double tol, int32_t trunc_norm, const double* sol_prev,
                    int32_t prec, int64_t nrestart, int64_t niters, double* sol_out,
                    int32_t precision, int64_t* iters_out) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && Phi1 && A && Phi2 && rhs && sol_prev && sol_out, "NULL argument");
  TTG_REQUIRE(rx1 >= 1 && n >= 1 && rx2 >= 1 && ra1 >= 1 && ra2 >= 1, "sizes must be >= 1");
  TTG_REQUIRE(trunc_norm == 1, "only the residual branch (trunc_norm = 1) is implemented");
  TTG_REQUIRE(prec >= 0 && prec <= 3,
              "prec %d is unknown (0 none, 1 'cjacobi', 2 'ljacobi', 3 'rjacobi')", int(prec));
  TTG_REQUIRE(nrestart >= 1 && niters >= 1, "nrestart and niters must be >= 1");
  TTG_REQUIRE(std::isfinite(tol) && tol > 0, "tol must be > 0");
  Context* c = &ctx->c;
  TTG_CUDA(cudaSetDevice(c->device));
  MvDims d{rx1, rx1, ra1, n, n, rx2, ra2, rx2};
  TTG_CUDA(cudaMemsetAsync(c->d_err, 0, 8 * sizeof(int), c->stream));
  LocalSolveResult r =
      local_solve(c, d, Phi1, A, Phi2, rhs, tol, sol_prev, nrestart, niters, sol_out, precision,
                  prec);
  int herr[8];
  TTG_CUDA(cudaMemcpyAsync(herr, c->d_err, sizeof(herr), cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  if (herr[0] || herr[1] || herr[2] || herr[4]) clear_error_slots(c);
  if (herr[0] || herr[1] || herr[2])
    fail(TTG_ERR_TIMEOUT, "a bounded device-side wait timed out in the local solve");
  if (herr[4]) fail(TTG_ERR_SOLVER, "a singular preconditioner block or factorization");
  if (iters_out) *iters_out = r.iters;
  TTG_API_END
}

int ttg_grad_xAx(ttg_tt x, ttg_tt A, double* grad, double* value) {
  TTG_API_BEGIN
  TTG_REQUIRE(A, "NULL argument");
  Context* c = grad_ctx(x, A, grad);
  DBuf<double> v(c, 1);
  grad_xAx(c, x, A, grad, v.p());
  grad_value_out(c, v.p(), value);
  sync(c);
  TTG_API_END
}

int ttg_grad_xb(ttg_tt x, ttg_tt b, double* grad, double* value) {
  TTG_API_BEGIN
  TTG_REQUIRE(b, "NULL argument");
  Context* c = grad_ctx(x, b, grad);
  DBuf<double> v(c, 1);
  grad_xb(c, x, b, grad, v.p());
  grad_value_out(c, v.p(), value);
  sync(c);
  TTG_API_END
}

int ttg_grad_sampled(ttg_tt x, int64_t nsamples, const int32_t* idx, const double* y,
                     double* grad, double* value) {
  TTG_API_BEGIN
  Context* c = grad_ctx(x, nullptr, grad);
  TTG_REQUIRE(nsamples >= 0, "nsamples must be >= 0");
  DBuf<double> v(c, 1);
  grad_sampled(c, x, nsamples, idx, y, grad, v.p());
  grad_value_out(c, v.p(), value);
  sync(c);
  TTG_API_END
}


int ttg_amen_solve_grouped(ttg_context ctx, int64_t count, const ttg_tt* A, const ttg_tt* y,
                           const double* tol, const ttg_amen_opts* opts, const ttg_tt* x0,
                           const ttg_tt* z0, int32_t width, ttg_tt* x_out,
                           ttg_amen_stats* stats, int32_t* status,
                           ttg_group_stats* group_stats) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && x_out, "NULL argument");
  TTG_REQUIRE(count >= 0, "count must be >= 0");
  if (group_stats) *group_stats = ttg_group_stats{};
  if (count == 0) return TTG_OK;
  Context* owner = &ctx->c;
  TTG_CUDA(cudaSetDevice(owner->device));
  check_batch(owner, count, A, y, tol, x0, z0, x_out, stats, status);
  int64_t w = width > 0 ? width : count;
  w = std::max<int64_t>(1, std::min<int64_t>({w, count, 1024}));
  ttg_amen_opts dflt;
  ttg_amen_opts_default(&dflt);
  std::mutex emu;
  int64_t first_bad = -1;
  int first_code = TTG_OK;
  std::string first_msg;
  auto record = [&](int64_t i, int code, const char* msg) {
    if (status) status[i] = code;
    std::lock_guard<std::mutex> lock(emu);
    if (first_bad < 0 || i < first_bad) {
      first_bad = i;
      first_code = code;
      first_msg = msg;
    }
  };
  auto body = [&](int64_t i, Context* c) {
    try {
      ttg_amen_opts o = opts ? opts[i] : dflt;
      o.timing = 0;  // no event timing inside a grouped batch
      x_out[i] = amen_solve(c, A[i], y[i], tol[i], o, x0 ? x0[i] : nullptr,
                            z0 ? z0[i] : nullptr, stats ? &stats[i] : nullptr, owner);
    } catch (const Error& e) {
      record(i, e.code, e.msg.c_str());
    } catch (const std::exception& e) {
      record(i, TTG_ERR_INVALID, e.what());
    }
  };
  run_grouped(owner, int(w), count, body, group_stats);
  if (first_bad >= 0)
    fail(first_code, "system %lld: %s", (long long)first_bad, first_msg.c_str());
  TTG_API_END
}

int ttg_amen_solve_batch(ttg_context ctx, int64_t count, const ttg_tt* A, const ttg_tt* y,
                         const double* tol, const ttg_amen_opts* opts, const ttg_tt* x0,
                         const ttg_tt* z0, int32_t workers, ttg_tt* x_out,
                         ttg_amen_stats* stats, int32_t* status) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && x_out, "NULL argument");
  TTG_REQUIRE(count >= 0, "count must be >= 0");
  if (count == 0) return TTG_OK;
  Context* owner = &ctx->c;
  TTG_CUDA(cudaSetDevice(owner->device));
  check_batch(owner, count, A, y, tol, x0, z0, x_out, stats, status);
  int64_t nw = workers > 0 ? workers : 8;
  nw = std::max<int64_t>(1, std::min<int64_t>({nw, count, 64}));
  // Inputs uploaded on the owner's stream are complete before other streams
  // read them, and no block of the owner's allocator is still in flight.
  sync(owner);
  std::vector<Context*> w(nw);
  {
    std::lock_guard<std::mutex> lock(ctx->mu);
    while (int64_t(ctx->workers.size()) < nw) {
      std::unique_ptr<Context> c(new Context());
      try {
        context_init(*c, owner->device);
      } catch (...) {
        context_release(*c);
        throw;
      }
      ctx->workers.push_back(std::move(c));
    }
    const int share = std::max(4, owner->num_sms / int(nw));
    for (int64_t k = 0; k < nw; ++k) {
      w[k] = ctx->workers[k].get();
      // Cooperative Krylov grids are sized from num_sms: a share of the SMs
      // per worker lets the workers' grids be resident together.
      w[k]->num_sms = share;
      w[k]->jacobi_max_sweeps = owner->jacobi_max_sweeps;
    }
  }
  ttg_amen_opts dflt;
  ttg_amen_opts_default(&dflt);
  std::atomic<int64_t> next{0};
  std::mutex emu;
  int64_t first_bad = -1;
  int first_code = TTG_OK;
  std::string first_msg;
  auto record = [&](int64_t i, int code, const char* msg) {
    if (status) status[i] = code;
    std::lock_guard<std::mutex> lock(emu);
    if (first_bad < 0 || i < first_bad) {
      first_bad = i;
      first_code = code;
      first_msg = msg;
    }
  };
  auto run = [&](Context* c) {
    cudaSetDevice(c->device);
    for (;;) {
      const int64_t i = next.fetch_add(1);
      if (i >= count) break;
      try {
        x_out[i] = amen_solve(c, A[i], y[i], tol[i], opts ? opts[i] : dflt,
                              x0 ? x0[i] : nullptr, z0 ? z0[i] : nullptr,
                              stats ? &stats[i] : nullptr, owner);
      } catch (const Error& e) {
        record(i, e.code, e.msg.c_str());
      } catch (const std::exception& e) {
        record(i, TTG_ERR_INVALID, e.what());
      }
    }
  };
  std::vector<std::thread> th;
  for (int64_t k = 1; k < nw; ++k) th.emplace_back(run, w[k]);
  run(w[0]);
  for (auto& t : th) t.join();
  for (int64_t k = 0; k < nw; ++k) w[k]->num_sms = owner->num_sms;
  if (first_bad >= 0)
    fail(first_code, "system %lld: %s", (long long)first_bad, first_msg.c_str());
  TTG_API_END
}

}  // extern "C"
