// FP64 QR / SVD / LU on the device: the library's own one-CTA and blocked
// factorizations, with cuSOLVER only for the shapes they do not cover.
#include <map>
#include <mutex>

#include "group.cuh"
#include "linalg.h"
#include "small_dense.h"

namespace ttg {

namespace {

TTG_BODY(k_triu)(TTG_BLOCK, int64_t k, int64_t n, const double* __restrict__ A, int64_t lda,
                       double* __restrict__ R) {
  pdl_begin();
  const int64_t total = k * n;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e % k, j = e / k;
    R[e] = (i <= j) ? A[i + j * lda] : 0.0;
  }
}
TTG_KERNEL(k_triu, 0);

// A non-zero info is folded into the context error slot 4 on the device (no
// host round trip); callers check the slot once their sequence is done.
void check_info(Context* c, const int* dinfo, const char* /*what*/) {
  accumulate_info(c, dinfo, c->d_err + 4);
}

int as_int(int64_t v, const char* what) {
  TTG_REQUIRE(v >= 0 && v <= 0x7fffffff, "%s = %lld exceeds the 32-bit solver range", what,
              (long long)v);
  return int(v);
}

}  // namespace

// cuSOLVER workspace queries need a handle; a context of a grouped batch
// has none (its library calls are recorded and issued with the executor's),
// so queries then go through one shared handle per device.
template <class F>
void with_query_handle(Context* c, F f) {
  if (c->solver) {
    f(c->solver);
    return;
  }
  static std::mutex mu;
  static std::map<int, cusolverDnHandle_t> handles;
  std::lock_guard<std::mutex> lock(mu);
  cusolverDnHandle_t& h = handles[c->device];
  if (!h) TTG_SOLVER(cusolverDnCreate(&h));
  f(h);
}

void check_factorizations(Context* c) {
  int h[5] = {0, 0, 0, 0, 0};
  read_device(c, h, c->d_err, sizeof(h));
  if (h[0] || h[1] || h[2] || h[4]) {
    memset_async(c, c->d_err, 0, 5 * sizeof(int));
    if (h[0] || h[1] || h[2])
      fail(TTG_ERR_TIMEOUT, "a bounded device-side wait timed out in a factorization");
    fail(TTG_ERR_SOLVER, "a device factorization reported a non-zero LAPACK info");
  }
}

void extract_triu_f64(Context* c, int64_t k, int64_t n, const double* A, int64_t lda, double* R) {
  if (k <= 0 || n <= 0) return;
  int64_t blocks = (k * n + 255) / 256;
  if (blocks > int64_t(c->num_sms) * 8) blocks = int64_t(c->num_sms) * 8;
  launch(c, k_triu, unsigned(blocks), 256, 0, k, n, A, lda, R);
  TTG_CHECK_LAUNCH();
}

namespace {

// Columns per diagonal block of the blocked Cholesky (one-CTA factor +
// inverse of each block, chol_inv_f64).
constexpr int64_t CHB = 96;

// diag(G) += factor * trace(G), one CTA (the shift of the first pass).
TTG_BODY(k_add_trace_shift)(TTG_BLOCK, int64_t n, double* __restrict__ G, int64_t ldg, double factor) {
  pdl_begin();
  __shared__ double red[32];
  double t = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) t += G[i + i * ldg];
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  const double s = factor * red[0];
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) G[i + i * ldg] += s;
}
TTG_KERNEL(k_add_trace_shift, 0);

// Blocked right-looking Cholesky R' R = G of an n x n SPD matrix (G is
// overwritten by its Schur complements).  Each diagonal block of at most
// CHB columns is factored in one CTA together with its inverse; the panel
// below it is L_ik = G_ik R_kk^{-1} and the trailing matrix loses L_ik L_jk'.
// R: n x n upper (ld n); Rinv_d: the inverses of the diagonal blocks, block
// k (bk x bk, ld bk) at offset k0 * CHB.
void chol_blocked_f64(Context* c, int64_t n, double* G, double* R, double* Rinv_d, int* flag) {
  fill_f64(c, n * n, 0.0, R);
  DBuf<double> Rkk(c, CHB * CHB), P(c, n * CHB);
  for (int64_t k0 = 0; k0 < n; k0 += CHB) {
    const int64_t bk = std::min(CHB, n - k0), rest = n - k0 - bk;
    double* Rinv_k = Rinv_d + k0 * CHB;
    chol_inv_f64(c, bk, G + k0 + k0 * n, n, 0.0, Rkk.p(), Rinv_k, flag);
    copy2d_f64(c, bk, bk, Rkk.p(), bk, R + k0 + k0 * n, n);
    if (rest == 0) break;
    const int64_t r0 = k0 + bk;
    gemm_f64(c, false, false, rest, bk, bk, 1.0, G + r0 + k0 * n, n, 0, Rinv_k, bk, 0, 0.0,
             P.p(), rest, 0, 1);                                       // L_ik
    transpose_f64(c, rest, bk, P.p(), rest, R + k0 + r0 * n, n);       // R_ki = L_ik'
    gemm_f64(c, false, true, rest, rest, bk, -1.0, P.p(), rest, 0, P.p(), rest, 0, 1.0,
             G + r0 + r0 * n, n, 0, 1);                                // Schur complement
  }
}

// dst = src R^{-1} by block forward substitution over the column blocks:
// dst_k = (src_k - dst_{<k} R_{<k,k}) R_kk^{-1}.  src, dst: m x n (ld m).
void solve_blocked_f64(Context* c, int64_t m, int64_t n, const double* src, const double* R,
                       const double* Rinv_d, double* dst) {
  DBuf<double> W(c, m * CHB);
  for (int64_t k0 = 0; k0 < n; k0 += CHB) {
    const int64_t bk = std::min(CHB, n - k0);
    copy_f64(c, m * bk, src + k0 * m, W.p());
    if (k0 > 0)
      gemm_f64(c, false, false, m, bk, k0, -1.0, dst, m, 0, R + k0 * n, n, 0, 1.0, W.p(), m, 0,
               1);
    gemm_f64(c, false, false, m, bk, bk, 1.0, W.p(), m, 0, Rinv_d + k0 * CHB, bk, 0, 0.0,
             dst + k0 * m, m, 0, 1);
  }
}

// Shifted Cholesky QR, three passes (sCholeskyQR3: Fukaya, Kannan,
// Nakatsukasa, Yamamoto, Yanagisawa, SIAM J. Sci. Comput. 42 (2020)
// A477-A503).  Pass 1 factors the Gram matrix shifted by
// s = 11 (m n + n (n + 1)) u ||A||_F^2, which keeps it positive definite for
// any A (rank-deficient included) and leaves Q1 = A R1^{-1} with condition
// number O(u^{-1/2}); two plain Cholesky QR passes then restore
// orthogonality to O(u).  R = R3 R2 R1 (positive diagonal).  Every step is a
// GEMM (split-K for the m-long Gram products) or one small one-CTA kernel.
// Returns false (outputs unusable) when the input was too close to rank
// deficient for the unshifted passes.
bool scholqr3_f64(Context* c, int64_t m, int64_t n, const double* A, double* Q, double* R) {
  DBuf<double> G(c, n * n), Ri(c, n * n), Rinv(c, n * n), Racc(c, n * n), T(c, n * n),
      W(c, m * n);
  const bool blocked = n > CHB;  // beyond one CTA: blocked Cholesky and solve
  DBuf<int> flag(c, 1);
  memset_async(c, flag.p(), 0, sizeof(int));
  const double u = 1.1102230246251565e-16;
  const double shift = 11.0 * (double(m) * n + double(n) * (n + 1)) * u;
  const double* src = A;
  for (int pass = 0; pass < 3; ++pass) {
    double* dst = (pass == 1) ? W.p() : Q;  // Q1 -> Q, Q2 -> W, Q3 -> Q
    gemm_f64(c, true, false, n, n, m, 1.0, src, m, 0, src, m, 0, 0.0, G.p(), n, 0, 1);
    if (blocked) {
      if (pass == 0) {
        launch(c, k_add_trace_shift, 1, 256, 0, n, G.p(), n, shift);
        TTG_CHECK_LAUNCH();
      }
      chol_blocked_f64(c, n, G.p(), Ri.p(), Rinv.p(), flag.p());
      solve_blocked_f64(c, m, n, src, Ri.p(), Rinv.p(), dst);
    } else {
      chol_inv_f64(c, n, G.p(), n, pass == 0 ? shift : 0.0, Ri.p(), Rinv.p(), flag.p());
      gemm_f64(c, false, false, m, n, n, 1.0, src, m, 0, Rinv.p(), n, 0, 0.0, dst, m, 0, 1);
    }
    if (pass == 0) {
      copy_f64(c, n * n, Ri.p(), Racc.p());
    } else {  // Racc = Ri * Racc
      gemm_f64(c, false, false, n, n, n, 1.0, Ri.p(), n, 0, Racc.p(), n, 0, 0.0, T.p(), n, 0, 1);
      copy_f64(c, n * n, T.p(), Racc.p());
    }
    src = dst;
  }
  copy_f64(c, n * n, Racc.p(), R);
  // Exactly rank-deficient inputs break the unshifted passes (singular Gram
  // matrices): check Q's orthogonality and report; the caller then takes
  // the Householder path.  One host read per factorization.
  gemm_f64(c, true, false, n, n, m, 1.0, Q, m, 0, Q, m, 0, 0.0, G.p(), n, 0, 1);
  orth_check(c, n, G.p(), 1e-12, flag.p());
  int h = 0;
  read_device(c, &h, flag.p(), sizeof(int));
  return h == 0;
}

bool scholqr_ok(int64_t m, int64_t n) {
  return n >= 8 && n <= 1024 && m >= 4 * n && chol_inv_fits(std::min(n, CHB));
}

}  // namespace

int64_t qr_f64(Context* c, int64_t m, int64_t n, const double* A, double* Q, double* R,
               bool lapack_signs) {
  const int64_t k = std::min(m, n);
  if (small_qr_fits(m, n)) {
    small_qr_f64(c, m, n, A, m, Q, R);
    return k;
  }
  if (skinny_qr_fits(m, n)) {  // a few columns, too tall for shared memory
    skinny_qr_f64(c, m, n, A, m, Q, R);
    return k;
  }
  if (!lapack_signs && scholqr_ok(m, n) && scholqr3_f64(c, m, n, A, Q, R)) return k;
  const int mi = as_int(m, "m"), ni = as_int(n, "n"), ki = as_int(k, "k");
  DBuf<double> work(c, m * n), tau(c, k > 0 ? k : 1);
  DBuf<int> info(c, 1);
  copy_f64(c, m * n, A, work.p());
  int lw1 = 0, lw2 = 0;
  double* wp = work.p();
  double* tp = tau.p();
  int* ip = info.p();
  with_query_handle(c, [&](cusolverDnHandle_t h) {
    TTG_SOLVER(cusolverDnDgeqrf_bufferSize(h, mi, ni, wp, mi, &lw1));
    TTG_SOLVER(cusolverDnDorgqr_bufferSize(h, mi, ki, ki, wp, mi, tp, &lw2));
  });
  DBuf<double> ws(c, std::max(std::max(lw1, lw2), 1));
  double* sp = ws.p();
  solver_call(c, [=](cudaStream_t, cusolverDnHandle_t h) {
    TTG_SOLVER(cusolverDnDgeqrf(h, mi, ni, wp, mi, tp, sp, lw1, ip));
  });
  extract_triu_f64(c, k, n, work.p(), m, R);
  solver_call(c, [=](cudaStream_t, cusolverDnHandle_t h) {
    TTG_SOLVER(cusolverDnDorgqr(h, mi, ki, ki, wp, mi, tp, sp, lw2, ip));
  });
  copy_f64(c, m * k, work.p(), Q);
  check_info(c, info.p(), "geqrf/orgqr");
  return k;
}

namespace {
// Economy SVD of a tall m x n (m >= n) matrix: QR, then one-sided Jacobi SVD
// of the n x n triangular factor R (small_dense.cu) run on the rows of R
// (the columns of R^T), U = Q Ur; up to 8 columns, one-sided Jacobi on A
// itself in one CTA.
void svd_tall(Context* c, int64_t m, int64_t n, const double* A, double* U, double* S,
              double* VT) {
  if (svd_tall_small_fits(m, n)) {  // few columns: rotate A itself, one launch
    svd_tall_small_f64(c, m, n, A, m, U, S, VT);
    return;
  }
  if (m == n) {
    jacobi_svd_f64(c, n, A, m, U, S, VT);
    return;
  }
  DBuf<double> Q(c, m * n), R(c, n * n), Ur(c, n * n);
  qr_f64(c, m, n, A, Q.p(), R.p());
  jacobi_svd_f64(c, n, R.p(), n, Ur.p(), S, VT, true);
  gemm_f64(c, false, false, m, n, n, 1.0, Q.p(), m, 0, Ur.p(), n, 0, 0.0, U, m, 0, 1);
}
}  // namespace

int64_t svd_f64(Context* c, int64_t m, int64_t n, const double* A, double* U, double* S,
                double* VT) {
  const int64_t k = std::min(m, n);
  if (k <= 0) return 0;
  if (m >= n) {
    svd_tall(c, m, n, A, U, S, VT);
  } else {
    // A^T (n x m) = U' S V'^T  ->  A = V' S U'^T : U = V' = (VT')^T, VT = U'^T
    DBuf<double> At(c, n * m), Up(c, n * m), VTp(c, m * m);
    transpose_f64(c, m, n, A, m, At.p(), n);
    svd_tall(c, n, m, At.p(), Up.p(), S, VTp.p());
    transpose_f64(c, m, m, VTp.p(), m, U, m);     // U (m x m) = VT'^T
    transpose_f64(c, n, m, Up.p(), n, VT, m);     // VT (m x n) = U'^T
  }
  return k;
}

namespace {
// Economy SVD of a tall m x n (m >= n) matrix by cuSOLVER's bidiagonal QR
// (gesvd): the fallback when the Jacobi SVD reaches its sweep limit.
void svd_gesvd_tall(Context* c, int64_t m, int64_t n, const double* A, double* U, double* S,
                    double* VT) {
  const int mi = as_int(m, "m"), ni = as_int(n, "n");
  DBuf<double> W(c, m * n), rw(c, std::max<int64_t>(n, 1));
  DBuf<int> info(c, 1);
  copy_f64(c, m * n, A, W.p());
  int lwork = 0;
  with_query_handle(c, [&](cusolverDnHandle_t h) {
    TTG_SOLVER(cusolverDnDgesvd_bufferSize(h, mi, ni, &lwork));
  });
  DBuf<double> ws(c, std::max(lwork, 1));
  double* wp = W.p();
  double* sp = ws.p();
  double* rp = rw.p();
  int* ip = info.p();
  solver_call(c, [=](cudaStream_t, cusolverDnHandle_t h) {
    TTG_SOLVER(cusolverDnDgesvd(h, 'S', 'S', mi, ni, wp, mi, S, U, mi, VT, ni, sp, lwork, rp,
                                ip));
  });
  check_info(c, info.p(), "gesvd");
}
}  // namespace

int64_t svd_f64_fallback(Context* c, int64_t m, int64_t n, const double* A, double* U, double* S,
                         double* VT) {
  const int64_t k = std::min(m, n);
  if (k <= 0) return 0;
  if (m >= n) {
    svd_gesvd_tall(c, m, n, A, U, S, VT);
  } else {
    DBuf<double> At(c, n * m), Up(c, n * m), VTp(c, m * m);
    transpose_f64(c, m, n, A, m, At.p(), n);
    svd_gesvd_tall(c, n, m, At.p(), Up.p(), S, VTp.p());
    transpose_f64(c, m, m, VTp.p(), m, U, m);
    transpose_f64(c, n, m, Up.p(), n, VT, m);
  }
  return k;
}

void lu_solve_f64(Context* c, int64_t N, const double* B, double* rhs, int64_t nrhs) {
  if (lu_small_fits(N, nrhs)) {  // the dense local systems (N < max_full_size)
    lu_small_f64(c, N, B, rhs, nrhs);
    return;
  }
  const int Ni = as_int(N, "N"), nr = as_int(nrhs, "nrhs");
  DBuf<double> W(c, N * N);
  DBuf<int> piv(c, std::max<int64_t>(N, 1)), info(c, 1);
  copy_f64(c, N * N, B, W.p());
  int lwork = 0;
  double* wp = W.p();
  with_query_handle(c, [&](cusolverDnHandle_t h) {
    TTG_SOLVER(cusolverDnDgetrf_bufferSize(h, Ni, Ni, wp, Ni, &lwork));
  });
  DBuf<double> ws(c, std::max(lwork, 1));
  double* sp = ws.p();
  int* pp = piv.p();
  int* ip = info.p();
  solver_call(c, [=](cudaStream_t, cusolverDnHandle_t h) {
    TTG_SOLVER(cusolverDnDgetrf(h, Ni, Ni, wp, Ni, sp, pp, ip));
    TTG_SOLVER(cusolverDnDgetrs(h, CUBLAS_OP_N, Ni, nr, wp, Ni, pp, rhs, Ni, ip));
  });
  check_info(c, info.p(), "getrf/getrs");
}

}  // namespace ttg
