// Centre block-Jacobi local preconditioner ('cjacobi', MEX prec = 1).
//
// Restates solve/solve3d_2ml.m:50-67 (generation) and :138-146 (application),
// the MATLAB twin of the MEX path's djac_gen/djac_apply (fmex/solve3d_2.c:
// 212-231,272-274; readable C in fmex/solve3d.c:47-128): for every rank
// pair (i, k) the n x n diagonal block of the local matrix
//   J_ik = sum_{al,be} Phi1[i,i,al] A[al,:,:,be] Phi2[k,be,k]
// is inverted, and P x applies the inverses block by block.
//
// Generation: two small GEMMs (diagonal of Phi1 against A, then against the
// diagonal of Phi2) give all blocks at once; one CTA per block inverts it by
// Gauss-Jordan elimination with partial (row) pivoting in shared memory --
// the pivot is the first entry of largest magnitude, LAPACK's choice, and
// the row interchanges are undone as column interchanges at the end.
// Application is HBM-bound: every inverse entry is read once per apply.
#include "group.cuh"
#include "jacobi.h"
#include "linalg.h"

#include <cmath>

namespace ttg {

namespace {

constexpr int GJ_THREADS = 256;

TTG_BODY(k_diag_phi1)(TTG_BLOCK, int64_t rx1, int64_t ra1, const double* __restrict__ Phi1,
                            double* __restrict__ d1) {
  pdl_begin();
  const int64_t total = rx1 * ra1;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e % rx1, a = e / rx1;
    d1[e] = Phi1[i + rx1 * i + rx1 * rx1 * a];  // d1[i, a] = Phi1[i, i, a]
  }
}
TTG_KERNEL(k_diag_phi1, 0);

TTG_BODY(k_diag_phi2)(TTG_BLOCK, int64_t rx2, int64_t ra2, const double* __restrict__ Phi2,
                            double* __restrict__ d2) {
  pdl_begin();
  const int64_t total = ra2 * rx2;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e % ra2, k = e / ra2;
    d2[e] = Phi2[k + rx2 * b + rx2 * ra2 * k];  // d2[b, k] = Phi2[k, b, k]
  }
}
TTG_KERNEL(k_diag_phi2, 0);

// One CTA per block (i, k), blockIdx.x = i + rx1 k; the block's entry (j, m)
// lives at J[i + rx1 (j + n m) + rx1 n n k].  In place.
TTG_BODY(k_block_inv)(TTG_BLOCK, int64_t rx1, int n,
                                                          double* __restrict__ J,
                                                          int* __restrict__ err) {
  pdl_begin();
  extern __shared__ double a[];  // n x n, a[r + n c]
  __shared__ double f[JAC_MAX_N], g[JAC_MAX_N];
  __shared__ int piv[JAC_MAX_N];
  __shared__ int s_q;
  __shared__ double s_max;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t b = blockIdx.x;
  const int64_t i = b % rx1, k = b / rx1;
  double* blk = J + i + rx1 * int64_t(n) * n * k;
  for (int e = tid; e < n * n; e += GJ_THREADS) a[e] = blk[rx1 * int64_t(e)];
  __syncthreads();
  bool singular = false;
  for (int p = 0; p < n; ++p) {
    if (warp == 0) {
      double best = -1.0;
      int bi = p;
      for (int r = p + lane; r < n; r += 32) {
        const double v = fabs(a[r + n * p]);
        if (v > best) {
          best = v;
          bi = r;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (lane == 0) {
        s_q = bi;
        s_max = best;
        piv[p] = bi;
      }
    }
    __syncthreads();
    if (!(s_max > 0.0)) {  // exactly singular (or NaN) block
      singular = true;
      break;
    }
    const int q = s_q;
    if (q != p)
      for (int col = tid; col < n; col += GJ_THREADS) {
        const double t = a[p + n * col];
        a[p + n * col] = a[q + n * col];
        a[q + n * col] = t;
      }
    __syncthreads();
    const double pinv = 1.0 / a[p + n * p];
    for (int t = tid; t < n; t += GJ_THREADS) {
      g[t] = (t == p ? 1.0 : a[p + n * t]) * pinv;  // scaled pivot row
      f[t] = (t == p ? 0.0 : a[t + n * p]);         // multipliers of the other rows
    }
    __syncthreads();
    for (int e = tid; e < n * n; e += GJ_THREADS) {
      const int r = e % n, col = e / n;
      if (r == p)
        a[e] = g[col];
      else
        a[e] = (col == p ? 0.0 : a[e]) - f[r] * g[col];
    }
    __syncthreads();
  }
  if (singular) {
    if (tid == 0) atomicOr(err, 1);
    for (int e = tid; e < n * n; e += GJ_THREADS) blk[rx1 * int64_t(e)] = nan("");
    return;
  }
  // inv(A) = inv(P A) P: undo the row interchanges as column interchanges
  for (int p = n - 1; p >= 0; --p) {
    const int q = piv[p];
    if (q != p)
      for (int r = tid; r < n; r += GJ_THREADS) {
        const double t = a[r + n * p];
        a[r + n * p] = a[r + n * q];
        a[r + n * q] = t;
      }
    __syncthreads();
  }
  for (int e = tid; e < n * n; e += GJ_THREADS) blk[rx1 * int64_t(e)] = a[e];
}
TTG_KERNEL(k_block_inv, GJ_THREADS);

// y[i, j, k] = sum_m J[i, j, m, k] x[i, m, k]; threads over (i, j, k), i fastest.
TTG_BODY(k_jac_apply_c)(TTG_BLOCK, int64_t rx1, int64_t n, int64_t rx2, const double* __restrict__ J,
                              const double* __restrict__ x, double* __restrict__ y) {
  pdl_begin();
  const int64_t total = rx1 * n * rx2;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e % rx1, j = (e / rx1) % n, k = e / (rx1 * n);
    const double* Jr = J + i + rx1 * j + rx1 * n * n * k;
    const double* xr = x + i + rx1 * n * k;
    double s = 0.0;
    for (int64_t m = 0; m < n; ++m) s += Jr[rx1 * n * m] * xr[rx1 * m];
    y[e] = s;
  }
}
TTG_KERNEL(k_jac_apply_c, 0);

// Left block-Jacobi ('ljacobi'): J[(i + rx1 j) + B (a + rx1 m) + B^2 k] =
// sum_al Phi1[i, a, al] AK[al, j, m, k], B = rx1 n, with
// AK[al, j, m, k] = sum_be A[al, j, m, be] Phi2[k, be, k].
TTG_BODY(k_jac_build_l)(TTG_BLOCK, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1,
                              const double* __restrict__ Phi1, const double* __restrict__ AK,
                              double* __restrict__ J) {
  pdl_begin();
  const int64_t B = rx1 * n, total = B * B * rx2;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t row = e % B, col = (e / B) % B, k = e / (B * B);
    const int64_t i = row % rx1, j = row / rx1, a = col % rx1, m = col / rx1;
    double s = 0.0;
    for (int64_t al = 0; al < ra1; ++al)
      s += Phi1[i + rx1 * a + rx1 * rx1 * al] * AK[al + ra1 * (j + n * m) + ra1 * n * n * k];
    J[e] = s;
  }
}
TTG_KERNEL(k_jac_build_l, 0);

// Right block-Jacobi ('rjacobi'): J[(j + n k) + B (m + n q) + B^2 i] =
// sum_be G[i, j, m, be] Phi2[q, be, k], B = n rx2, with
// G[i, j, m, be] = sum_al Phi1[i, i, al] A[al, j, m, be].
TTG_BODY(k_jac_build_r)(TTG_BLOCK, int64_t rx1, int64_t n, int64_t rx2, int64_t ra2,
                              const double* __restrict__ G, const double* __restrict__ Phi2,
                              double* __restrict__ J) {
  pdl_begin();
  const int64_t B = n * rx2, total = B * B * rx1;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t row = e % B, col = (e / B) % B, i = e / (B * B);
    const int64_t j = row % n, k = row / n, m = col % n, q = col / n;
    double s = 0.0;
    for (int64_t be = 0; be < ra2; ++be)
      s += G[i + rx1 * (j + n * m + n * n * be)] * Phi2[q + rx2 * be + rx2 * ra2 * k];
    J[e] = s;
  }
}
TTG_KERNEL(k_jac_build_r, 0);

// blk = I (B x B, column-major)
TTG_BODY(k_set_identity)(TTG_BLOCK, int64_t B, double* __restrict__ blk) {
  pdl_begin();
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < B * B;
       e += int64_t(gridDim.x) * blockDim.x)
    blk[e] = (e % B == e / B) ? 1.0 : 0.0;
}
TTG_KERNEL(k_set_identity, 0);

int blocks_for(Context* c, int64_t n) {
  int64_t b = (n + 255) / 256;
  const int64_t cap = int64_t(c->num_sms) * 8;
  if (b > cap) b = cap;
  return int(b < 1 ? 1 : b);
}

}  // namespace

void jac_gen_c_f64(Context* c, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1, int64_t ra2,
                   const double* Phi1, const double* A, const double* Phi2, double* J) {
  TTG_REQUIRE(n >= 1 && n <= JAC_MAX_N, "cjacobi: mode size %lld above %lld", (long long)n,
              (long long)JAC_MAX_N);
  TTG_REQUIRE(rx1 * rx2 <= int64_t(0x7fffffff), "cjacobi: too many blocks");
  DBuf<double> d1(c, rx1 * ra1), d2(c, ra2 * rx2), G(c, rx1 * n * n * ra2);
  launch(c, k_diag_phi1, blocks_for(c, rx1 * ra1), 256, 0, rx1, ra1, Phi1, d1.p());
  launch(c, k_diag_phi2, blocks_for(c, ra2 * rx2), 256, 0, rx2, ra2, Phi2, d2.p());
  TTG_CHECK_LAUNCH();
  // G[i, (j, m, be)] = sum_al d1[i, al] A[al, (j, m, be)]
  gemm_f64(c, false, false, rx1, n * n * ra2, ra1, 1.0, d1.p(), rx1, 0, A, ra1, 0, 0.0, G.p(),
           rx1, 0, 1);
  // J[(i, j, m), k] = sum_be G[(i, j, m), be] d2[be, k]
  gemm_f64(c, false, false, rx1 * n * n, rx2, ra2, 1.0, G.p(), rx1 * n * n, 0, d2.p(), ra2, 0,
           0.0, J, rx1 * n * n, 0, 1);
  const size_t smem = sizeof(double) * size_t(n) * size_t(n);
  ensure_smem_attr(k_block_inv.fn(), c->device, int(smem));
  launch(c, k_block_inv, unsigned(rx1 * rx2), GJ_THREADS, smem, rx1, int(n), J, c->d_err + 4);
  TTG_CHECK_LAUNCH();
}

void jac_apply_c_f64(Context* c, int64_t rx1, int64_t n, int64_t rx2, const double* J,
                     const double* x, double* y) {
  launch(c, k_jac_apply_c, blocks_for(c, rx1 * n * rx2), 256, 0, rx1, n, rx2, J, x, y);
  TTG_CHECK_LAUNCH();
}

void inv_blocks_f64(Context* c, int64_t B, int64_t nblocks, double* J) {
  if (B <= JAC_MAX_N) {  // one CTA per block, Gauss-Jordan in shared memory
    TTG_REQUIRE(nblocks <= int64_t(0x7fffffff), "too many blocks");
    const size_t smem = sizeof(double) * size_t(B) * size_t(B);
    ensure_smem_attr(k_block_inv.fn(), c->device, int(smem));
    launch(c, k_block_inv, unsigned(nblocks), GJ_THREADS, smem, int64_t(1), int(B), J,
           c->d_err + 4);
    TTG_CHECK_LAUNCH();
    return;
  }
  // Larger blocks: LU with partial pivoting and B X = I per block.
  DBuf<double> W(c, B * B);
  for (int64_t k = 0; k < nblocks; ++k) {
    double* blk = J + B * B * k;
    copy_f64(c, B * B, blk, W.p());
    launch(c, k_set_identity, blocks_for(c, B * B), 256, 0, B, blk);
    TTG_CHECK_LAUNCH();
    lu_solve_f64(c, B, W.p(), blk, B);
  }
}

int64_t jac_size(int prec, int64_t rx1, int64_t n, int64_t rx2) {
  if (prec == 1) return rx1 * n * n * rx2;
  if (prec == 2) return (rx1 * n) * (rx1 * n) * rx2;
  return (n * rx2) * (n * rx2) * rx1;
}

void jac_gen_f64(Context* c, int prec, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1,
                 int64_t ra2, const double* Phi1, const double* A, const double* Phi2,
                 double* J) {
  if (prec == 1) {
    jac_gen_c_f64(c, rx1, n, rx2, ra1, ra2, Phi1, A, Phi2, J);
    return;
  }
  TTG_REQUIRE(prec == 2 || prec == 3, "unknown local preconditioner %d", prec);
  TTG_REQUIRE(jac_size(prec, rx1, n, rx2) <= JAC_MAX_ELEMS,
              "%s: the inverse blocks need %lld doubles, above the limit of %lld",
              prec == 2 ? "ljacobi" : "rjacobi", (long long)jac_size(prec, rx1, n, rx2),
              (long long)JAC_MAX_ELEMS);
  if (prec == 2) {  // solve/solve3d_2ml.m:33-48
    DBuf<double> d2(c, ra2 * rx2), AK(c, ra1 * n * n * rx2);
    launch(c, k_diag_phi2, blocks_for(c, ra2 * rx2), 256, 0, rx2, ra2, Phi2, d2.p());
    TTG_CHECK_LAUNCH();
    gemm_f64(c, false, false, ra1 * n * n, rx2, ra2, 1.0, A, ra1 * n * n, 0, d2.p(), ra2, 0, 0.0,
             AK.p(), ra1 * n * n, 0, 1);
    const int64_t B = rx1 * n;
    launch(c, k_jac_build_l, blocks_for(c, B * B * rx2), 256, 0, rx1, n, rx2, ra1, Phi1, AK.p(),
           J);
    TTG_CHECK_LAUNCH();
    inv_blocks_f64(c, B, rx2, J);
  } else {          // solve/solve3d_2ml.m:21-32
    DBuf<double> d1(c, rx1 * ra1), G(c, rx1 * n * n * ra2);
    launch(c, k_diag_phi1, blocks_for(c, rx1 * ra1), 256, 0, rx1, ra1, Phi1, d1.p());
    TTG_CHECK_LAUNCH();
    gemm_f64(c, false, false, rx1, n * n * ra2, ra1, 1.0, d1.p(), rx1, 0, A, ra1, 0, 0.0, G.p(),
             rx1, 0, 1);
    const int64_t B = n * rx2;
    launch(c, k_jac_build_r, blocks_for(c, B * B * rx1), 256, 0, rx1, n, rx2, ra2, G.p(), Phi2,
           J);
    TTG_CHECK_LAUNCH();
    inv_blocks_f64(c, B, rx1, J);
  }
}

void jac_apply_f64(Context* c, int prec, int64_t rx1, int64_t n, int64_t rx2, const double* J,
                   const double* x, double* y, double* scratch) {
  if (prec == 1) {
    jac_apply_c_f64(c, rx1, n, rx2, J, x, y);
  } else if (prec == 2) {  // y(:, k) = J_k x(:, k), x as (rx1 n) x rx2 (solve3d_2ml.m:130-137)
    const int64_t B = rx1 * n;
    gemm_f64(c, false, false, B, 1, B, 1.0, J, B, B * B, x, B, B, 0.0, y, B, B, rx2);
  } else {                 // per i over (j, k)  (solve3d_2ml.m:120-129)
    const int64_t B = n * rx2;
    double* xt = scratch;
    double* yt = scratch + B * rx1;
    transpose_f64(c, rx1, B, x, rx1, xt, B);
    gemm_f64(c, false, false, B, 1, B, 1.0, J, B, B * B, xt, B, B, 0.0, yt, B, B, rx1);
    transpose_f64(c, B, rx1, yt, B, y, rx1);
  }
}

}  // namespace ttg
