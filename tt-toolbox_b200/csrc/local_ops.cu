// FP64 local matvec (bfun3) and interface update (compute_next_Phi).
//
// Both are three contractions.  The intermediate layouts are chosen so that
// every contraction is a plain (batched) column-major GEMM on the DMMA engine
// with no permutation pass in between -- the reference interleaves its three
// GEMMs with two explicit transposes (amen_solve2.m:937-950, :857-905).
#include <algorithm>

#include "group.cuh"
#include "local_ops.h"

namespace ttg {

void local_matvec_f64(Context* c, const MvDims& d, const double* Phi1, const double* A,
                      const double* Phi2, const double* x, double* y, double* t1, double* t2) {
  MvTiming timing(c, 0);
  // (1) T1[(a,m),(be,k)] = x[(a,m), b] * Phi2[b, (be,k)]
  gemm_f64(c, false, false, d.rx1 * d.m, d.ra2 * d.ry2, d.rx2, 1.0, x, d.rx1 * d.m, 0, Phi2,
           d.rx2, 0, 0.0, t1, d.rx1 * d.m, 0, 1);
  // (2) for each k: T2_k[a,(al,j)] = T1_k[a,(m,be)] * A[(al,j),(m,be)]^T
  gemm_f64(c, false, true, d.rx1, d.ra1 * d.n, d.m * d.ra2, 1.0, t1, d.rx1,
           d.rx1 * d.m * d.ra2, A, d.ra1 * d.n, 0, 0.0, t2, d.rx1, d.rx1 * d.ra1 * d.n, d.ry2);
  // (3) y[i,(j,k)] = Phi1[i,(a,al)] * T2[(a,al),(j,k)]
  gemm_f64(c, false, false, d.ry1, d.n * d.ry2, d.rx1 * d.ra1, 1.0, Phi1, d.ry1, 0, t2,
           d.rx1 * d.ra1, 0, 0.0, y, d.ry1, 0, 1);
  c->matvecs += 1;
  c->matvec_flops += int64_t(d.flops());
  c->mv_count[0] += 1;
  c->mv_flops[0] += d.flops();
}

void local_matvec_f64(Context* c, const MvDims& d, const double* Phi1, const double* A,
                      const double* Phi2, const double* x, double* y) {
  DBuf<double> t1(c, d.t1_size()), t2(c, d.t2_size());
  local_matvec_f64(c, d, Phi1, A, Phi2, x, y, t1.p(), t2.p());
}

int64_t next_phi_f64(Context* c, int dir, int64_t rx1, int64_t n, int64_t rx2, int64_t ry1,
                     int64_t ry2, int64_t ra1, int64_t ra2, const double* Phi_prev,
                     const double* x, const double* A, const double* y, double* out) {
  const int64_t m = n;
  if (!A) ra1 = ra2 = 1;
  if (dir == 0) {
    // 'lr': out[c, e, be] = sum x[a,j,c] Phi[a,y1,al] A[al,j,mm,be] y[y1,mm,e]
    DBuf<double> w1(c, ry1 * ra1 * n * rx2);
    // (1) W1[(y1,al),(j,c)] = Phi^T[(y1,al), a] * x[a,(j,c)]
    gemm_f64(c, true, false, ry1 * ra1, n * rx2, rx1, 1.0, Phi_prev, rx1, 0, x, rx1, 0, 0.0,
             w1.p(), ry1 * ra1, 0, 1);
    if (A) {
      DBuf<double> w2(c, ry1 * m * ra2 * rx2);
      // (2) for each c: W2_c[y1,(mm,be)] = W1_c[y1,(al,j)] * A[(al,j),(mm,be)]
      gemm_f64(c, false, false, ry1, m * ra2, ra1 * n, 1.0, w1.p(), ry1, ry1 * ra1 * n, A,
               ra1 * n, 0, 0.0, w2.p(), ry1, ry1 * m * ra2, rx2);
      // (3) for each be: out_be[c, e] = W2[(y1,mm), be, c]^T * y[(y1,mm), e]
      gemm_f64(c, true, false, rx2, ry2, ry1 * m, 1.0, w2.p(), ry1 * m * ra2, ry1 * m, y,
               ry1 * m, 0, 0.0, out, rx2, rx2 * ry2, ra2);
    } else {
      // out[c, e] = W1[(y1,j), c]^T * y[(y1,j), e]
      gemm_f64(c, true, false, rx2, ry2, ry1 * n, 1.0, w1.p(), ry1 * n, 0, y, ry1 * m, 0, 0.0,
               out, rx2, 0, 1);
    }
    return rx2 * ry2 * ra2;
  } else {
    // 'rl': out[y1, al, a] = sum y[y1,mm,e] Phi[e,be,c] A[al,j,mm,be] x[a,j,c]
    DBuf<double> z1(c, ry1 * m * ra2 * rx2);
    // (1) Z1[(y1,mm),(be,c)] = y[(y1,mm), e] * Phi[e,(be,c)]
    gemm_f64(c, false, false, ry1 * m, ra2 * rx2, ry2, 1.0, y, ry1 * m, 0, Phi_prev, ry2, 0, 0.0,
             z1.p(), ry1 * m, 0, 1);
    if (A) {
      DBuf<double> z2(c, ry1 * ra1 * n * rx2);
      // (2) for each c: Z2_c[y1,(al,j)] = Z1_c[y1,(mm,be)] * A[(al,j),(mm,be)]^T
      gemm_f64(c, false, true, ry1, ra1 * n, m * ra2, 1.0, z1.p(), ry1, ry1 * m * ra2, A,
               ra1 * n, 0, 0.0, z2.p(), ry1, ry1 * ra1 * n, rx2);
      // (3) out[(y1,al), a] = Z2[(y1,al),(j,c)] * x[a,(j,c)]^T
      gemm_f64(c, false, true, ry1 * ra1, rx1, n * rx2, 1.0, z2.p(), ry1 * ra1, 0, x, rx1, 0,
               0.0, out, ry1 * ra1, 0, 1);
    } else {
      // out[y1, a] = Z1[y1,(j,c)] * x[a,(j,c)]^T
      gemm_f64(c, false, true, ry1, rx1, n * rx2, 1.0, z1.p(), ry1, 0, x, rx1, 0, 0.0, out, ry1,
               0, 1);
    }
    return ry1 * ra1 * rx1;
  }
}

namespace {
TTG_BODY(k_assemble)(TTG_BLOCK, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1, int64_t ra2,
                           const double* __restrict__ Phi1, const double* __restrict__ A,
                           const double* __restrict__ Phi2, double* __restrict__ B) {
  pdl_begin();
  const int64_t N = rx1 * n * rx2;
  const int64_t total = N * N;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t row = e % N, col = e / N;
    const int64_t i = row % rx1, j = (row / rx1) % n, k = row / (rx1 * n);
    const int64_t a = col % rx1, mm = (col / rx1) % n, b = col / (rx1 * n);
    double s = 0.0;
    for (int64_t be = 0; be < ra2; ++be) {
      const double p2 = Phi2[b + rx2 * (be + ra2 * k)];
      double t = 0.0;
      for (int64_t al = 0; al < ra1; ++al)
        t += Phi1[i + rx1 * (a + rx1 * al)] * A[al + ra1 * (j + n * (mm + n * be))];
      s += t * p2;
    }
    B[e] = s;
  }
}
TTG_KERNEL(k_assemble, 0);
}  // namespace

void assemble_local_f64(Context* c, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1,
                        int64_t ra2, const double* Phi1, const double* A, const double* Phi2,
                        double* B) {
  const int64_t N = rx1 * n * rx2;
  int64_t blocks = (N * N + 255) / 256;
  if (blocks > int64_t(c->num_sms) * 8) blocks = int64_t(c->num_sms) * 8;
  if (blocks < 1) blocks = 1;
  launch(c, k_assemble, unsigned(blocks), 256, 0, rx1, n, rx2, ra1, ra2, Phi1, A, Phi2, B);
  TTG_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Candidate residuals of the truncation loop (amen_solve2.m:539-551)
// ---------------------------------------------------------------------------

void rank1_images_f64(Context* c, const MvDims& d, const double* Phi1, const double* A,
                      const double* Phi2, const double* U, int64_t ldu, const double* VT,
                      int64_t ldvt, const double* s, int64_t k0, int64_t cnt, double* W,
                      double* scratch) {
  const int64_t r1 = d.rx1, n = d.n, r2 = d.rx2, a1 = d.ra1, a2 = d.ra2;
  const int64_t N = d.out_size();
  double* Q = scratch;                       // [(be,c), t]   a2*r2*cnt
  double* Qs = Q + a2 * r2 * cnt;            // scaled by s_k
  double* Z = Qs + a2 * r2 * cnt;            // [a, al, j, be, t]  r1*a1*n*a2*cnt
  double* P = Z + r1 * a1 * n * a2 * cnt;    // [i, j, be, t]      r1*n*a2*cnt
  // Q[(be,c), t] = sum_b Phi2[b, (be,c)] V[b, k0+t]
  gemm_f64(c, true, true, a2 * r2, cnt, r2, 1.0, Phi2, r2, 0, VT + k0, ldvt, 0, 0.0, Q, a2 * r2,
           0, 1);
  copy2d_f64(c, a2 * r2, cnt, Q, a2 * r2, Qs, a2 * r2, s + k0);
  // Z[a, (al,j), be, t] = sum_m U[(a,m), k0+t] A[al, j, m, be]
  for (int64_t be = 0; be < a2; ++be)
    gemm_f64(c, false, true, r1, a1 * n, n, 1.0, U + k0 * ldu, r1, ldu, A + be * a1 * n * n,
             a1 * n, 0, 0.0, Z + be * r1 * a1 * n, r1, r1 * a1 * n * a2, cnt);
  // P[i, (j, be, t)] = sum_{a,al} Phi1[i, (a,al)] Z[(a,al), (j, be, t)]
  gemm_f64(c, false, false, r1, n * a2 * cnt, r1 * a1, 1.0, Phi1, r1, 0, Z, r1 * a1, 0, 0.0, P,
           r1, 0, 1);
  // W_t[(i,j), c] = sum_be P_t[(i,j), be] Qs_t[be, c]
  gemm_f64(c, false, false, r1 * n, r2, a2, 1.0, P, r1 * n, r1 * n * a2, Qs, a2, a2 * r2, 0.0,
           W, r1 * n, N, cnt);
}

int64_t rank1_scratch_size(const MvDims& d, int64_t cnt) {
  return cnt * (2 * d.ra2 * d.rx2 + d.rx1 * d.ra1 * d.n * d.ra2 + d.rx1 * d.n * d.ra2);
}

namespace {

constexpr int CN_THREADS = 256;

// part[blk * MAXC + b] = sum over this block's i of (R[i] + sum_{t >= cnt-1-b} W[i + N t])^2
TTG_BODY(k_cumnorm)(TTG_BLOCK, int64_t N, int cnt,
                                                         double* __restrict__ R,
                                                         const double* __restrict__ W,
                                                         double* __restrict__ part) {
  pdl_begin();
  double acc2[CUMNORM_MAXC];
#pragma unroll
  for (int b = 0; b < CUMNORM_MAXC; ++b) acc2[b] = 0.0;
  for (int64_t i = blockIdx.x * int64_t(CN_THREADS) + threadIdx.x; i < N;
       i += int64_t(gridDim.x) * CN_THREADS) {
    double v = R[i];
#pragma unroll
    for (int b = 0; b < CUMNORM_MAXC; ++b) {
      if (b < cnt) {
        v += W[i + N * int64_t(cnt - 1 - b)];
        acc2[b] += v * v;
      }
    }
    R[i] = v;
  }
  __shared__ double sh[CN_THREADS / 32][CUMNORM_MAXC];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int b = 0; b < CUMNORM_MAXC; ++b) {
    double x = acc2[b];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh[w][b] = x;
  }
  __syncthreads();
  if (threadIdx.x < CUMNORM_MAXC) {
    double x = 0.0;
    for (int k = 0; k < CN_THREADS / 32; ++k) x += sh[k][threadIdx.x];
    part[int64_t(blockIdx.x) * CUMNORM_MAXC + threadIdx.x] = x;
  }
}
TTG_KERNEL(k_cumnorm, CN_THREADS);

// One warp per candidate: lanes stride over the block partials, then a fixed
// shuffle tree (deterministic).
TTG_BODY(k_cumnorm_final)(TTG_BLOCK, int nblk, int cnt, const double* __restrict__ part,
                                double* __restrict__ out) {
  pdl_begin();
  const int b = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (b >= cnt) return;
  double x = 0.0;
  for (int k = lane; k < nblk; k += 32) x += part[int64_t(k) * CUMNORM_MAXC + b];
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  if (lane == 0) out[b] = sqrt(x);
}
TTG_KERNEL(k_cumnorm_final, 0);

}  // namespace

void cumulative_norms_f64(Context* c, int64_t N, int64_t cnt, double* R, const double* W,
                          double* part, double* out) {
  TTG_REQUIRE(cnt >= 1 && cnt <= CUMNORM_MAXC, "cumulative_norms: cnt %lld", (long long)cnt);
  int64_t nb = (N + CN_THREADS - 1) / CN_THREADS;
  nb = std::max<int64_t>(1, std::min<int64_t>(nb, int64_t(c->num_sms) * 4));
  launch(c, k_cumnorm, unsigned(nb), CN_THREADS, 0, N, int(cnt), R, W, part);
  launch(c, k_cumnorm_final, 1, 32 * CUMNORM_MAXC, 0, int(nb), int(cnt), part, out);
  TTG_CHECK_LAUNCH();
}

int64_t cumulative_norms_part_size(Context* c) { return int64_t(c->num_sms) * 4 * CUMNORM_MAXC; }

}  // namespace ttg
