// Caller-side TT algebra around the hot path, on device-resident handles:
// the exact TT-matrix-by-TT-tensor product, linear combinations, the
// QR-based norm and the inner product -- what the true residual
// ||A x - y|| / ||y|| of a solve needs, and what round's callers feed it.
//
//   matvec : @tt_matrix/mtimes.m:38-65   C_k[(al,a), i, (be,b)] =
//            sum_j A_k[al,i,j,be] x_k[a,j,b]  (ranks multiply, al fastest)
//   axpby  : @tt_tensor/plus.m:40-86      rank concatenation: first core
//            [a x_1, b y_1], middle cores block-diagonal, last [x_d; y_d]
//   norm   : @tt_tensor/norm.m:16-42      left-to-right QR sweep; the norm
//            is the product of the R-factor norms and the last core's
//   dot    : @tt_tensor/dot.m:92-111      interface-matrix sweep
#include <cmath>
#include <vector>

#include "internal.h"
#include "kernels.h"
#include "linalg.h"

using namespace ttg;

namespace {

int grid_for(Context* c, int64_t n) {
  int64_t b = (n + 255) / 256;
  const int64_t cap = int64_t(c->num_sms) * 8;
  if (b > cap) b = cap;
  return int(b < 1 ? 1 : b);
}

// One core of the exact product (one thread per output entry).
__global__ void k_mv_core(int64_t ra1, int64_t n, int64_t m, int64_t ra2, int64_t rx1,
                          int64_t rx2, const double* __restrict__ A,
                          const double* __restrict__ x, double* __restrict__ out) {
  const int64_t r1 = ra1 * rx1, total = r1 * n * ra2 * rx2;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    int64_t t = e;
    const int64_t al = t % ra1;
    t /= ra1;
    const int64_t a = t % rx1;
    t /= rx1;
    const int64_t i = t % n;
    t /= n;
    const int64_t be = t % ra2;
    const int64_t b = t / ra2;
    const double* Ap = A + al + ra1 * i + ra1 * n * m * be;  // A[al, i, j, be], stride ra1 n in j
    const double* xp = x + a + rx1 * m * b;                  // x[a, j, b], stride rx1 in j
    double s = 0.0;
    for (int64_t j = 0; j < m; ++j) s += Ap[ra1 * n * j] * xp[rx1 * j];
    out[e] = s;
  }
}

// out[r1o, n, r2o] zero-filled beforehand; copy s * in[r1, n, r2] into the
// block starting at (o1, *, o2).
__global__ void k_place_block(int64_t r1, int64_t n, int64_t r2, double s,
                              const double* __restrict__ in, int64_t r1o, int64_t n_o,
                              int64_t o1, int64_t o2, double* __restrict__ out) {
  const int64_t total = r1 * n * r2;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t a = e % r1, i = (e / r1) % n, b = e / (r1 * n);
    out[(o1 + a) + r1o * (i + n_o * (o2 + b))] = s * in[e];
  }
}

ttg_tt_s* new_tensor(Context* c, const std::vector<int64_t>& n, const std::vector<int64_t>& r) {
  auto* t = new ttg_tt_s();
  t->ctx = c;
  t->d = int64_t(n.size());
  t->is_matrix = false;
  t->n = n;
  t->r = r;
  t->ps.assign(t->d + 1, 0);
  for (int64_t k = 0; k < t->d; ++k) t->ps[k + 1] = t->ps[k] + r[k] * n[k] * r[k + 1];
  t->numel = t->ps[t->d];
  t->core = static_cast<double*>(c->alloc->get(sizeof(double) * std::max<int64_t>(t->numel, 1)));
  return t;
}

void check_vector(const ttg_tt_s* x, const char* what) {
  TTG_REQUIRE(x && !x->is_matrix, "%s must be a TT tensor", what);
}

// QR-based norm (norm.m:16-42) on device; returns the host value.
double tt_norm_dev(Context* c, const ttg_tt_s* x) {
  const int64_t d = x->d;
  std::vector<int64_t> r = x->r;
  DBuf<double> cur(c, r[0] * x->n[0] * r[1]);
  copy_f64(c, cur.size(), x->core, cur.p());
  DBuf<double> nr(c, d);
  for (int64_t i = 0; i < d - 1; ++i) {
    const int64_t m = r[i] * x->n[i], cols = r[i + 1];
    const int64_t k = std::min(m, cols);
    DBuf<double> Q(c, m * k), R(c, k * cols);
    qr_f64(c, m, cols, cur.p(), Q.p(), R.p());                  // :27
    dot_f64(c, k * cols, R.p(), nullptr, nr.p() + i, true);     // :27 norm(ru,'fro')
    scalar_op(c, SC_MAX_CONST, nr.p() + i, nr.p() + i, nullptr, nullptr, 1e-308);  // :28
    const int64_t nc = x->n[i + 1] * r[i + 2];
    DBuf<double> next(c, k * nc);
    // ru ./ nrm(i) * core_{i+1}   (:29-32)
    gemm_f64(c, false, false, k, nc, cols, 1.0, R.p(), k, 0, x->core + x->ps[i + 1], cols, 0,
             0.0, next.p(), k, 0, 1);
    scale_dev_f64(c, k * nc, next.p(), next.p(), nullptr, nr.p() + i);
    r[i + 1] = k;                                                // :33
    cur = std::move(next);
  }
  dot_f64(c, cur.size(), cur.p(), nullptr, nr.p() + d - 1, true);  // :40
  std::vector<double> h(d);
  read_scalars(c, nr.p(), h.data(), int(d));
  double p = 1.0;
  for (double v : h) p *= v;                                     // :41
  return p;
}

}  // namespace

extern "C" {

int ttg_tt_matvec(ttg_tt A, ttg_tt x, ttg_tt* out) {
  TTG_API_BEGIN
  TTG_REQUIRE(A && x && out, "NULL argument");
  TTG_REQUIRE(A->is_matrix, "A must be a TT matrix");
  check_vector(x, "x");
  TTG_REQUIRE(A->ctx == x->ctx, "operands belong to different contexts");
  TTG_REQUIRE(A->d == x->d, "A has %lld cores, x has %lld", (long long)A->d, (long long)x->d);
  for (int64_t k = 0; k < A->d; ++k)
    TTG_REQUIRE(A->m[k] == x->n[k], "core %lld: A has %lld columns, x mode size %lld",
                (long long)k, (long long)A->m[k], (long long)x->n[k]);
  Context* c = A->ctx;
  TTG_CUDA(cudaSetDevice(c->device));
  const int64_t d = A->d;
  std::vector<int64_t> r(d + 1);
  for (int64_t k = 0; k <= d; ++k) r[k] = A->r[k] * x->r[k];    // mtimes.m:42
  ttg_tt_s* t = new_tensor(c, A->n, r);
  for (int64_t k = 0; k < d; ++k) {
    const int64_t total = r[k] * A->n[k] * r[k + 1];
    k_mv_core<<<grid_for(c, total), 256, 0, c->stream>>>(A->r[k], A->n[k], A->m[k], A->r[k + 1],
                                                          x->r[k], x->r[k + 1],
                                                          A->core + A->ps[k],
                                                          x->core + x->ps[k], t->core + t->ps[k]);
    c->launches += 1;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ttg_tt_free(t);
    fail(TTG_ERR_CUDA, "matvec launch: %s", cudaGetErrorString(e));
  }
  sync(c);
  *out = t;
  TTG_API_END
}

int ttg_tt_axpby(double a, ttg_tt x, double b, ttg_tt y, ttg_tt* out) {
  TTG_API_BEGIN
  TTG_REQUIRE(x && y && out, "NULL argument");
  check_vector(x, "x");
  check_vector(y, "y");
  TTG_REQUIRE(x->ctx == y->ctx, "operands belong to different contexts");
  TTG_REQUIRE(x->d == y->d, "x has %lld cores, y has %lld", (long long)x->d, (long long)y->d);
  const int64_t d = x->d;
  for (int64_t k = 0; k < d; ++k)
    TTG_REQUIRE(x->n[k] == y->n[k], "core %lld: mode sizes %lld and %lld", (long long)k,
                (long long)x->n[k], (long long)y->n[k]);
  TTG_REQUIRE(x->r[0] == y->r[0] && x->r[d] == y->r[d], "boundary ranks differ");
  Context* c = x->ctx;
  TTG_CUDA(cudaSetDevice(c->device));
  std::vector<int64_t> r(d + 1);
  r[0] = x->r[0];
  r[d] = x->r[d];
  for (int64_t k = 1; k < d; ++k) r[k] = x->r[k] + y->r[k];     // plus.m:49-52
  if (d == 1) r[1] = x->r[1];
  ttg_tt_s* t = new_tensor(c, x->n, r);
  fill_f64(c, t->numel, 0.0, t->core);
  for (int64_t k = 0; k < d; ++k) {
    const int64_t n = x->n[k];
    // x block at (0, 0); y block after x's ranks except on the border
    const int64_t oy1 = (k == 0) ? 0 : x->r[k];
    const int64_t oy2 = (k == d - 1) ? 0 : x->r[k + 1];
    const double sx = (k == 0) ? a : 1.0, sy = (k == 0) ? b : 1.0;
    if (d == 1) {  // one core: a x + b y elementwise
      axpby_f64(c, t->numel, a, x->core, 0.0, t->core);
      axpby_f64(c, t->numel, b, y->core, 1.0, t->core);
      break;
    }
    const int64_t tx = x->r[k] * n * x->r[k + 1], ty = y->r[k] * n * y->r[k + 1];
    k_place_block<<<grid_for(c, tx), 256, 0, c->stream>>>(x->r[k], n, x->r[k + 1], sx,
                                                           x->core + x->ps[k], r[k], n, 0, 0,
                                                           t->core + t->ps[k]);
    k_place_block<<<grid_for(c, ty), 256, 0, c->stream>>>(y->r[k], n, y->r[k + 1], sy,
                                                           y->core + y->ps[k], r[k], n, oy1, oy2,
                                                           t->core + t->ps[k]);
    c->launches += 2;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ttg_tt_free(t);
    fail(TTG_ERR_CUDA, "axpby launch: %s", cudaGetErrorString(e));
  }
  sync(c);
  *out = t;
  TTG_API_END
}

int ttg_tt_norm(ttg_tt x, double* nrm) {
  TTG_API_BEGIN
  TTG_REQUIRE(x && nrm, "NULL argument");
  check_vector(x, "x");
  Context* c = x->ctx;
  TTG_CUDA(cudaSetDevice(c->device));
  TTG_CUDA(cudaMemsetAsync(c->d_err, 0, 8 * sizeof(int), c->stream));
  *nrm = tt_norm_dev(c, x);
  check_factorizations(c);
  TTG_API_END
}

int ttg_tt_dot(ttg_tt x, ttg_tt y, double* val) {
  TTG_API_BEGIN
  TTG_REQUIRE(x && y && val, "NULL argument");
  check_vector(x, "x");
  check_vector(y, "y");
  TTG_REQUIRE(x->ctx == y->ctx, "operands belong to different contexts");
  TTG_REQUIRE(x->d == y->d, "x has %lld cores, y has %lld", (long long)x->d, (long long)y->d);
  const int64_t d = x->d;
  for (int64_t k = 0; k < d; ++k)
    TTG_REQUIRE(x->n[k] == y->n[k], "core %lld: mode sizes differ", (long long)k);
  Context* c = x->ctx;
  TTG_CUDA(cudaSetDevice(c->device));
  // p [rx_k, ry_k] (dot.m:92-111 with r1(1) = r2(1) = 1 folded in):
  //   p <- x_k' (p y_k), contracted over (rx_k, n_k)
  TTG_REQUIRE(x->r[0] == 1 && y->r[0] == 1 && x->r[d] == 1 && y->r[d] == 1,
              "dot: boundary ranks must be 1");
  DBuf<double> p(c, 1);
  fill_f64(c, 1, 1.0, p.p());
  for (int64_t k = 0; k < d; ++k) {
    const int64_t rx1 = x->r[k], rx2 = x->r[k + 1], ry1 = y->r[k], ry2 = y->r[k + 1];
    const int64_t n = x->n[k];
    DBuf<double> t(c, rx1 * n * ry2), pn(c, rx2 * ry2);
    // t[a, (i, q)] = p[a, p'] y_k[p', (i, q)]
    gemm_f64(c, false, false, rx1, n * ry2, ry1, 1.0, p.p(), rx1, 0, y->core + y->ps[k], ry1, 0,
             0.0, t.p(), rx1, 0, 1);
    // pn[c, q] = sum_{(a, i)} x_k[(a, i), c] t[(a, i), q]
    gemm_f64(c, true, false, rx2, ry2, rx1 * n, 1.0, x->core + x->ps[k], rx1 * n, 0, t.p(),
             rx1 * n, 0, 0.0, pn.p(), rx2, 0, 1);
    p = std::move(pn);
  }
  read_scalars(c, p.p(), val, 1);
  TTG_API_END
}

}  // extern "C"
