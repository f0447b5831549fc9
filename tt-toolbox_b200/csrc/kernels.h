// Launchers of the device kernels used by the host drivers.
#pragma once

#include <initializer_list>
#include <utility>
#include "internal.h"

namespace ttg {

// C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b], column-major, FP64.
//   op(A) is M x K: tA=false -> A(m,k) = A[m + k*lda];  tA=true -> A[k + m*lda]
//   op(B) is K x N: tB=false -> B(k,n) = B[k + n*ldb];  tB=true -> B[n + k*ldb]
// Batch b uses A + b*sA, B + b*sB, C + b*sC.  FP64 tensor-core (DMMA) tiles.
void gemm_f64(Context* c, bool tA, bool tB, int64_t M, int64_t N, int64_t K, double alpha,
              const double* A, int64_t lda, int64_t sA, const double* B, int64_t ldb,
              int64_t sB, double beta, double* C, int64_t ldc, int64_t sC, int64_t batch = 1);

// out = sum(x.*y) (or sum(x.^2) when y == nullptr) into a device scalar;
// deterministic one-launch reduction (block partials summed in block order
// by the last block).  If do_sqrt, stores sqrt of the sum.
void dot_f64(Context* c, int64_t n, const double* x, const double* y, double* out,
             bool do_sqrt = false);
// Frobenius norm to host (synchronises).
double nrm2_host(Context* c, int64_t n, const double* x);
// Squared distance ||x - y||^2 into device scalar (sqrt if requested).
void diffnrm_f64(Context* c, int64_t n, const double* x, const double* y, double* out,
                 bool do_sqrt = true);

// Number of NaN / Inf entries of x (synchronises): the input checks of the
// API entries.
int64_t count_nonfinite_f64(Context* c, int64_t n, const double* x);
// Fails with TTG_ERR_INVALID when a core of t holds NaN or Inf (one device
// pass and one read-back); name is the argument name in the message.
void require_finite(const ttg_tt_s* t, const char* name);
// The same for several tensors on context c, with one host read.
void require_finite(Context* c, std::initializer_list<std::pair<const ttg_tt_s*, const char*>> ts);

// Self-tests of the bounded device waits (ttg_selftest_wait): each runs the
// wait helper of one kernel family with a small poll limit on a condition
// that nothing satisfies, so that *flag (device int, zeroed by the caller)
// ends up non-zero; synchronises.
void selftest_wait_gmres(Context* c, int* flag, long long limit);
void selftest_wait_mbarrier(Context* c, int* flag, long long limit);
void selftest_wait_jacobi(Context* c, int* flag, long long limit);
void selftest_wait_arnoldi(Context* c, int* flag, long long limit);

// y = a*x + b*y ; with a, b host scalars.
void axpby_f64(Context* c, int64_t n, double a, const double* x, double b, double* y);
// y = x * s[0] / s[1] style scaling with device scalars: y = x * (num ? *num : 1) / (den ? *den : 1)
void scale_dev_f64(Context* c, int64_t n, const double* x, double* y, const double* num,
                   const double* den);
void fill_f64(Context* c, int64_t n, double v, double* y);
void copy_f64(Context* c, int64_t n, const double* x, double* y);

// out (cols x rows) = in(rows x cols)^T, column-major, batched with strides.
void transpose_f64(Context* c, int64_t rows, int64_t cols, const double* in, int64_t ldi,
                   double* out, int64_t ldo, int64_t batch = 1, int64_t si = 0, int64_t so = 0);

// Copy a sub-matrix: out[i + j*ldo] = in[i + j*ldi] * (scale_col ? scale_col[j] : 1)
void copy2d_f64(Context* c, int64_t rows, int64_t cols, const double* in, int64_t ldi,
                double* out, int64_t ldo, const double* scale_col = nullptr);

// Right-orthogonal random core generator input: N(0,1) entries from a
// counter-based hash (seed, offset).
void randn_f64(Context* c, int64_t n, uint64_t seed, uint64_t offset, double* y);

// ---- device-resident scalar bookkeeping (no host round trip) -------------
// x /= *nrm in place (nothing when *nrm == 0, and *nrm is then set to 1) --
// the normalisation of compute_next_Phi with nargout > 1.
void normalize_by_dev(Context* c, int64_t n, double* x, double* nrm);
// y = a*x + (*b)*y with a host scalar a and a device scalar b.
void axpby_dev(Context* c, int64_t n, double a, const double* x, const double* b, double* y);
// Scalar program on device memory (one thread): see ScalOp.
enum ScalOp : int {
  SC_DIV = 0,        // out = p0 / p1
  SC_MAXUPD = 1,     // out = max(out, p0)
  SC_NRMSC_DIV = 2,  // out /= (p0 / (p1 * p2))      (amen_solve2.m:327,737)
  SC_NRMSC_MUL = 3,  // out *= (p0 / (p1 * p2))      (amen_solve2.m:372,754)
  SC_MUL = 4,        // out *= p0
  SC_MAX_CONST = 5,  // out = max(p0, host constant)
  SC_DIV_NZ = 6,     // out = p1 > 0 ? p0 / p1 : 0
  SC_ONE_IF_ZERO = 7,  // out = p0 == 0 ? 1 : p0
};
void scalar_op(Context* c, int op, double* out, const double* p0, const double* p1 = nullptr,
               const double* p2 = nullptr, double k = 0.0);
// *out = first b < nb with cand[b] / *den > *thr, or -1 (one thread).
void first_exceeding(Context* c, int64_t nb, const double* cand, const double* den,
                     const double* thr, double* out);
// *keep = 1 when every column j of a projected block kept more than tau of
// its norm (G1[j,j] > tau^2 G0[j,j]; G0, G1 Gram matrices before / after).
void collapse_flag(Context* c, int64_t k, const double* G0, int64_t ld0, const double* G1,
                   int64_t ld1, double tau, int* keep);
// *flag |= 1 when max |G - I| > tol (G: n x n, ld n) or G has a NaN.
void orth_check(Context* c, int64_t n, const double* G, double tol, int* flag);
// err_slot |= (*info != 0): LAPACK-style status accumulated without a host sync.
void accumulate_info(Context* c, const int* info, int* err_slot);

}  // namespace ttg
