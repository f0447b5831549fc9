// FP64 QR / SVD / LU on the device through cuSOLVER (library factorizations;
// the contractions around them are this library's own kernels).
#include "linalg.h"
#include "small_dense.h"

namespace ttg {

namespace {

__global__ void k_triu(int64_t k, int64_t n, const double* __restrict__ A, int64_t lda,
                       double* __restrict__ R) {
  const int64_t total = k * n;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e % k, j = e / k;
    R[e] = (i <= j) ? A[i + j * lda] : 0.0;
  }
}

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

void check_factorizations(Context* c) {
  int h = 0;
  TTG_CUDA(cudaMemcpyAsync(&h, c->d_err + 4, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  if (h) {
    TTG_CUDA(cudaMemsetAsync(c->d_err + 4, 0, sizeof(int), c->stream));
    fail(TTG_ERR_SOLVER, "a device factorization reported a non-zero LAPACK info");
  }
}

void extract_triu_f64(Context* c, int64_t k, int64_t n, const double* A, int64_t lda, double* R) {
  if (k <= 0 || n <= 0) return;
  int64_t blocks = (k * n + 255) / 256;
  if (blocks > int64_t(c->num_sms) * 8) blocks = int64_t(c->num_sms) * 8;
  k_triu<<<unsigned(blocks), 256, 0, c->stream>>>(k, n, A, lda, R);
  c->launches += 1;
  TTG_CHECK_LAUNCH();
}

namespace {

// Row r of an m-row matrix -> row of the padded (p x Lr)-row layout in which
// the first `rem` blocks hold Lr rows and the others Lr - 1 (zero-filled).
__device__ __forceinline__ int64_t padded_row(int64_t r, int64_t Lr, int64_t rem) {
  if (r < rem * Lr) return r;
  const int64_t q = r - rem * Lr;
  return (rem + q / (Lr - 1)) * Lr + q % (Lr - 1);
}

// dir 0: out[padded_row(r), c] = in[r, c];  dir 1: out[r, c] = in[padded_row(r), c].
__global__ void k_pad_rows(int64_t m, int64_t n, int64_t Lr, int64_t rem, const double* in,
                           int64_t ldi, double* out, int64_t ldo, int dir) {
  const int64_t total = m * n;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e % m, col = e / m;
    const int64_t pr = padded_row(r, Lr, rem);
    if (dir == 0)
      out[pr + col * ldo] = in[r + col * ldi];
    else
      out[r + col * ldo] = in[pr + col * ldi];
  }
}

void pad_rows(Context* c, int64_t m, int64_t n, int64_t Lr, int64_t rem, const double* in,
              int64_t ldi, double* out, int64_t ldo, int dir) {
  int64_t blocks = (m * n + 255) / 256;
  if (blocks > int64_t(c->num_sms) * 8) blocks = int64_t(c->num_sms) * 8;
  k_pad_rows<<<unsigned(blocks), 256, 0, c->stream>>>(m, n, Lr, rem, in, ldi, out, ldo, dir);
  c->launches += 1;
  TTG_CHECK_LAUNCH();
}

// TSQR: one-CTA Householder QRs of row blocks (one batched launch), the
// stacked n x n R factors factored again (recursively), and Q assembled as
// Q_b = Q_leaf_b * Q_top[b] by one batched GEMM per level.  Blocks hold
// Lr or Lr - 1 rows (>= n), stored Lr apart with zero rows at the end of the
// short ones: zero rows leave the reflectors, and so R, unchanged and give
// zero rows of Q.  Q: m x n (ld m), R: n x n (ld n); requires m >= 2n.
void tsqr_f64(Context* c, int64_t m, int64_t n, const double* A, int64_t lda, double* Q,
              double* R) {
  if (small_qr_fits(m, n)) {
    small_qr_f64(c, m, n, A, lda, Q, R);
    return;
  }
  const int64_t L = small_qr_max_rows(n);
  const int64_t p = (m + L - 1) / L;
  const int64_t Lr = (m + p - 1) / p;
  const int64_t rem = m - p * (Lr - 1);  // blocks with Lr rows (1..p)
  const int64_t P = p * Lr;
  TTG_REQUIRE(Lr - 1 >= n, "tsqr: blocks of %lld rows for %lld columns", (long long)Lr,
              (long long)n);
  const double* Al = A;
  int64_t ldl = lda;
  DBuf<double> Apad, Qp;
  if (P != m || lda != m) {
    Apad.reset(c, P * n);
    if (P != m) fill_f64(c, P * n, 0.0, Apad.p());
    pad_rows(c, m, n, Lr, rem, A, lda, Apad.p(), P, 0);
    Al = Apad.p();
    ldl = P;
  }
  DBuf<double> Q0(c, P * n), S(c, p * n * n), Qt(c, p * n * n);
  small_qr_batched_f64(c, p, Lr, n, Al, ldl, Lr, Q0.p(), Lr * n, S.p(), p * n, n);
  tsqr_f64(c, p * n, n, S.p(), p * n, Qt.p(), R);
  double* Qo = Q;
  if (P != m) {
    Qp.reset(c, P * n);
    Qo = Qp.p();
  }
  gemm_f64(c, false, false, Lr, n, n, 1.0, Q0.p(), Lr, Lr * n, Qt.p(), p * n, n, 0.0, Qo, P, Lr,
           p);
  if (P != m) pad_rows(c, m, n, Lr, rem, Qp.p(), P, Q, m, 1);
}

bool tsqr_ok(int64_t m, int64_t n) {
  return n >= 1 && n <= 96 && m >= 2 * n && small_qr_max_rows(n) >= 2 * n + 2 &&
         m <= (int64_t(1) << 31);
}

}  // namespace

int64_t qr_f64(Context* c, int64_t m, int64_t n, const double* A, double* Q, double* R,
               bool lapack_signs) {
  const int64_t k = std::min(m, n);
  if (small_qr_fits(m, n)) {
    small_qr_f64(c, m, n, A, m, Q, R);
    return k;
  }
  if (!lapack_signs && tsqr_ok(m, n)) {
    tsqr_f64(c, m, n, A, m, Q, R);
    return k;
  }
  const int mi = as_int(m, "m"), ni = as_int(n, "n"), ki = as_int(k, "k");
  DBuf<double> work(c, m * n), tau(c, k > 0 ? k : 1);
  DBuf<int> info(c, 1);
  copy_f64(c, m * n, A, work.p());
  int lw1 = 0, lw2 = 0;
  TTG_SOLVER(cusolverDnDgeqrf_bufferSize(c->solver, mi, ni, work.p(), mi, &lw1));
  TTG_SOLVER(cusolverDnDorgqr_bufferSize(c->solver, mi, ki, ki, work.p(), mi, tau.p(), &lw2));
  DBuf<double> ws(c, std::max(std::max(lw1, lw2), 1));
  TTG_SOLVER(cusolverDnDgeqrf(c->solver, mi, ni, work.p(), mi, tau.p(), ws.p(), lw1, info.p()));
  extract_triu_f64(c, k, n, work.p(), m, R);
  TTG_SOLVER(cusolverDnDorgqr(c->solver, mi, ki, ki, work.p(), mi, tau.p(), ws.p(), lw2, info.p()));
  copy_f64(c, m * k, work.p(), Q);
  check_info(c, info.p(), "geqrf/orgqr");
  return k;
}

namespace {
// Economy SVD of a tall m x n (m >= n) matrix: QR, then one-sided Jacobi SVD
// of the n x n triangular factor (small_dense.cu), U = Q Ur.
void svd_tall(Context* c, int64_t m, int64_t n, const double* A, double* U, double* S,
              double* VT) {
  if (m == n) {
    jacobi_svd_f64(c, n, A, m, U, S, VT);
    return;
  }
  DBuf<double> Q(c, m * n), R(c, n * n), Ur(c, n * n);
  qr_f64(c, m, n, A, Q.p(), R.p());
  jacobi_svd_f64(c, n, R.p(), n, Ur.p(), S, VT);
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

void lu_solve_f64(Context* c, int64_t N, const double* B, double* rhs, int64_t nrhs) {
  const int Ni = as_int(N, "N"), nr = as_int(nrhs, "nrhs");
  DBuf<double> W(c, N * N);
  DBuf<int> piv(c, std::max<int64_t>(N, 1)), info(c, 1);
  copy_f64(c, N * N, B, W.p());
  int lwork = 0;
  TTG_SOLVER(cusolverDnDgetrf_bufferSize(c->solver, Ni, Ni, W.p(), Ni, &lwork));
  DBuf<double> ws(c, std::max(lwork, 1));
  TTG_SOLVER(cusolverDnDgetrf(c->solver, Ni, Ni, W.p(), Ni, ws.p(), piv.p(), info.p()));
  TTG_SOLVER(cusolverDnDgetrs(c->solver, CUBLAS_OP_N, Ni, nr, W.p(), Ni, piv.p(), rhs, Ni, info.p()));
  check_info(c, info.p(), "getrf/getrs");
}

}  // namespace ttg
