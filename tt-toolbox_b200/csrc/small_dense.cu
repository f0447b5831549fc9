// Single-CTA FP64 dense factorizations for the small matrices of the AMEn
// and rounding sweeps (replacing library calls whose host-side sequencing
// cost milliseconds on 64x64 inputs):
//
//   k_jacobi_svd : one-sided (Hestenes) Jacobi SVD of a square n x n matrix,
//                  round-robin pairing, one warp per column pair, the matrix
//                  held in shared memory (global memory above ~160 columns),
//                  V accumulated in global memory.  Singular values sorted
//                  descending.  One launch, no host round trip.
//   k_house_qr   : Householder QR (LAPACK sign convention: beta =
//                  -sign(alpha) ||x||, as geqrf/orgqr and MATLAB's qr(A,0))
//                  of an m x n matrix that fits in shared memory; forms the
//                  thin Q and R.
#include <cmath>
#include <cstdlib>

#include <map>
#include <mutex>

#include <cooperative_groups.h>

#include "group.cuh"
#include "small_dense.h"

namespace ttg {

namespace {

constexpr int SD_THREADS = 1024;
constexpr int SD_WARPS = SD_THREADS / 32;
constexpr size_t SMEM_LIMIT = 200 * 1024;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Column index of slot k in round r of a round-robin tournament on ne (even)
// players: slot 0 is fixed, the others rotate.  k - 1 + r < 2 (ne - 1), so a
// conditional subtraction replaces the modulo.
__device__ __forceinline__ int rr_player(int k, int r, int ne) {
  int x = k - 1 + r;
  if (x >= ne - 1) x -= ne - 1;
  return k == 0 ? 0 : 1 + x;
}

// Sum over the G lanes of a warp (G = 32) or half-warp (G = 16); all 32
// lanes take part in every shuffle.
template <int G>
__device__ __forceinline__ double gsum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One Jacobi rotation of the column pair p < q of A (n x n, ld n) and of V,
// on the G lanes gl = 0..G-1 of a warp or half-warp.  live = false keeps the
// group in the shuffles and touches nothing.  Returns max(off, ga^2/(al be))
// when the pair is rotated, else off.
template <int G>
__device__ __forceinline__ double jacobi_pair(double* A, double* V, int n, int p, int q, int gl,
                                              bool live, double tol2, double off) {
  double* ap = A + int64_t(p) * n;
  double* aq = A + int64_t(q) * n;
  double al = 0.0, be = 0.0, ga = 0.0;
  if (live) {
    for (int i = gl; i < n; i += G) {
      const double x = ap[i], y = aq[i];
      al += x * x;
      be += y * y;
      ga += x * y;
    }
  }
  al = gsum<G>(al);
  be = gsum<G>(be);
  ga = gsum<G>(ga);
  // |ga| <= tol sqrt(al be), compared in squares (no square root on the
  // path of a pair that needs no rotation)
  const double ab = al * be, g2 = ga * ga;
  if (!live || ab == 0.0 || g2 <= tol2 * ab) return off;
  off = fmax(off, g2 / ab);
  // t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), zeta = (be - al) / (2 ga),
  // written with one division: t = sign(zeta) |g| / (|dd| + hypot(dd, g))
  // for dd = be - al, g = 2 ga (sign(zeta) = +1 when dd = 0).
  const double dd = be - al, gg = 2.0 * ga;
  const double sg = ((dd >= 0.0) == (gg > 0.0) || dd == 0.0) ? 1.0 : -1.0;
  const double t = sg * fabs(gg) / (fabs(dd) + sqrt(dd * dd + gg * gg));
  const double c = rsqrt(1.0 + t * t), s = c * t;
  double* vp = V + int64_t(p) * n;
  double* vq = V + int64_t(q) * n;
  for (int i = gl; i < n; i += G) {
    const double x = ap[i], y = aq[i];
    ap[i] = c * x - s * y;
    aq[i] = s * x + c * y;
    const double vx = vp[i], vy = vq[i];
    vp[i] = c * vx - s * vy;
    vq[i] = s * vx + c * vy;
  }
  return off;
}

// Singular values = column norms of the rotated A, ranked descending
// (stable on index); U = A diag(1/s), VT = V^T in that order.  With trans the
// rotated matrix is the transpose of the input (X = In^T = Ux S Vx^T), so the
// input's factors swap: U = Vx, VT = Ux^T.  One CTA of SD_THREADS; sig: 2n
// doubles of scratch.
__device__ void jacobi_finish(int n, const double* A, const double* V, double* __restrict__ U,
                              double* __restrict__ S, double* __restrict__ VT, double* sig,
                              int trans) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j = warp; j < n; j += SD_WARPS) {
    const double* aj = A + int64_t(j) * n;
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += aj[i] * aj[i];
    s = wsum(s);
    if (lane == 0) sig[j] = sqrt(s);
  }
  __syncthreads();
  for (int j = tid; j < n; j += SD_THREADS) {
    const double sj = sig[j];
    int pos = 0;
    for (int k = 0; k < n; ++k) {
      const double sk = sig[k];
      pos += (sk > sj) || (sk == sj && k < j);
    }
    S[pos] = sj;
    sig[n + j] = double(pos);
  }
  __syncthreads();
  for (int e = tid; e < n * n; e += SD_THREADS) {
    const int i = e % n, j = e / n;
    const int pos = int(sig[n + j]);
    const double sj = sig[j];
    const double ua = sj > 0.0 ? A[e] / sj : (i == pos ? 1.0 : 0.0);
    if (!trans) {
      U[i + int64_t(pos) * n] = ua;
      VT[pos + int64_t(i) * n] = V[e];
    } else {
      U[i + int64_t(pos) * n] = V[e];
      VT[pos + int64_t(i) * n] = ua;
    }
  }
}

// A: n x n (column-major, lda) input; U (n x n, ld n), S (n), VT (n x n, ld n)
// outputs.  work: n*n doubles of global scratch used when A does not fit in
// shared memory.  Status: *err = 5 if the sweep limit is reached.
TTG_BODY(k_jacobi_svd)(TTG_BLOCK, int n, const double* __restrict__ Ain,
                                                          int lda, double* __restrict__ U,
                                                          double* __restrict__ S,
                                                          double* __restrict__ VT,
                                                          double* __restrict__ Vg,
                                                          double* __restrict__ work, int in_smem,
                                                          int trans, int* err, int max_sweeps) {
  pdl_begin();
  extern __shared__ double sm[];
  __shared__ double s_off[SD_WARPS];
  __shared__ int s_done;
  // in_smem: 0 = A and V in global memory, 1 = A in shared memory,
  // 2 = A and V in shared memory.
  double* A = in_smem ? sm : work;
  double* V = in_smem == 2 ? sm + int64_t(n) * n : Vg;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < n * n; e += SD_THREADS) {
    const int i = e % n, j = e / n;
    A[e] = trans ? Ain[j + int64_t(i) * lda] : Ain[i + int64_t(j) * lda];
    V[e] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int ne = (n + 1) & ~1;  // even number of players (dummy column n if odd)
  const double tol = 4.0 * 2.220446049250313e-16, tol2 = tol * tol;
  int sweep = 0;
  for (sweep = 0; sweep < max_sweeps; ++sweep) {
    double off = 0.0;
    for (int r = 0; r < ne - 1; ++r) {
      if (ne / 2 > SD_WARPS && ne / 2 <= 2 * SD_WARPS) {
        // 32 < pairs <= 64: one half-warp per pair, the whole round at once
        // (a warp per pair would take two pairs in turn on most warps).
        const int pr = tid >> 4;
        int p = 0, q = 0;
        bool live = false;
        if (pr < ne / 2) {
          p = rr_player(pr, r, ne);
          q = rr_player(ne - 1 - pr, r, ne);
          if (p > q) {
            const int t = p;
            p = q;
            q = t;
          }
          live = q < n;  // else a dummy player
          if (!live) p = q = 0;
        }
        off = jacobi_pair<16>(A, V, n, p, q, lane & 15, live, tol2, off);
      } else {
        for (int pr = warp; pr < ne / 2; pr += SD_WARPS) {
          int p = rr_player(pr, r, ne), q = rr_player(ne - 1 - pr, r, ne);
          if (p > q) {
            const int t = p;
            p = q;
            q = t;
          }
          if (q >= n) continue;  // dummy player
          off = jacobi_pair<32>(A, V, n, p, q, lane, true, tol2, off);
        }
      }
      __syncthreads();
    }
    off = fmax(off, __shfl_xor_sync(0xffffffffu, off, 16));  // both half-warps
    if (lane == 0) s_off[warp] = off;
    __syncthreads();
    if (tid == 0) {
      double m = 0.0;
      for (int w = 0; w < SD_WARPS; ++w) m = fmax(m, s_off[w]);
      s_done = (m <= tol2) ? 1 : 0;
    }
    __syncthreads();
    if (s_done) break;
  }
  if (tid == 0 && sweep >= max_sweeps) atomicExch(err, 5);
  jacobi_finish(n, A, V, U, S, VT, work + int64_t(n) * n, trans);
}
TTG_KERNEL(k_jacobi_svd, SD_THREADS);


// ---------------------------------------------------------------------------
// Grid-wide one-sided Jacobi SVD for matrices too large for one CTA's shared
// memory: one CTA per column pair of a round-robin round, a bounded grid
// barrier between rounds (cooperative launch), the same rotation and
// stopping rule as k_jacobi_svd.
// ---------------------------------------------------------------------------

constexpr int JC_THREADS = 256;
constexpr long long JC_SPIN_LIMIT = 1LL << 24;

__device__ void jc_barrier(TTG_BLOCK, unsigned* bar, int* err, long long limit = JC_SPIN_LIMIT) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = bar + 1;
    volatile int* verr = err;
    const unsigned gen = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long spins = 0;
      while (*vgen == gen) {
        if (*verr) break;
        if (++spins > limit) {
          atomicExch(err, 6);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// A (n x n work copy, ld n) and V (n x n) in global memory; offmax: three
// u64 slots holding the per-sweep maximum off-diagonal measure (bit pattern
// of a non-negative double).  *sweeps_out = sweeps run.
TTG_BODY(k_jacobi_coop)(TTG_BLOCK, int n, const double* __restrict__ Ain,
                                                           int lda, double* A, double* V,
                                                           unsigned* bar,
                                                           unsigned long long* offmax, int* err,
                                                           int* sweep_err, int trans,
                                                           int max_sweeps) {
  __shared__ double red[3][JC_THREADS / 32];
  __shared__ double s_rot[2];
  __shared__ int s_skip;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t nn = int64_t(n) * n;
  for (int64_t e = blockIdx.x * int64_t(JC_THREADS) + tid; e < nn;
       e += int64_t(gridDim.x) * JC_THREADS) {
    const int64_t i = e % n, j = e / n;
    A[e] = trans ? Ain[j + i * lda] : Ain[i + j * lda];
    V[e] = (i == j) ? 1.0 : 0.0;
  }
  if (blockIdx.x == 0 && tid < 3) offmax[tid] = 0ull;
  jc_barrier(blockIdx, gridDim, bar, err);
  const int ne = (n + 1) & ~1;
  const double tol = 4.0 * 2.220446049250313e-16;
  int sweep = 0;
  for (sweep = 0; sweep < max_sweeps; ++sweep) {
    const int slot = sweep % 3;
    if (blockIdx.x == 0 && tid == 0) offmax[(sweep + 1) % 3] = 0ull;
    double off = 0.0;
    for (int r = 0; r < ne - 1; ++r) {
      for (int pr = blockIdx.x; pr < ne / 2; pr += gridDim.x) {
        int p = rr_player(pr, r, ne), q = rr_player(ne - 1 - pr, r, ne);
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        if (q >= n) continue;  // dummy player (uniform in the CTA)
        double* ap = A + int64_t(p) * n;
        double* aq = A + int64_t(q) * n;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i = tid; i < n; i += JC_THREADS) {
          const double x = ap[i], y = aq[i];
          al += x * x;
          be += y * y;
          ga += x * y;
        }
        al = wsum(al);
        be = wsum(be);
        ga = wsum(ga);
        if (lane == 0) {
          red[0][warp] = al;
          red[1][warp] = be;
          red[2][warp] = ga;
        }
        __syncthreads();
        if (tid == 0) {
          double a2 = 0.0, b2 = 0.0, g2 = 0.0;
          for (int w = 0; w < JC_THREADS / 32; ++w) {
            a2 += red[0][w];
            b2 += red[1][w];
            g2 += red[2][w];
          }
          const double nrm = sqrt(a2 * b2);
          if (nrm == 0.0 || fabs(g2) <= tol * nrm) {
            s_skip = 1;
          } else {
            s_skip = 0;
            off = fmax(off, fabs(g2) / nrm);
            const double zeta = (b2 - a2) / (2.0 * g2);
            const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            const double cc = 1.0 / sqrt(1.0 + t * t);
            s_rot[0] = cc;
            s_rot[1] = cc * t;
          }
        }
        __syncthreads();
        if (!s_skip) {
          const double cc = s_rot[0], sn = s_rot[1];
          double* vp = V + int64_t(p) * n;
          double* vq = V + int64_t(q) * n;
          for (int i = tid; i < n; i += JC_THREADS) {
            const double x = ap[i], y = aq[i];
            ap[i] = cc * x - sn * y;
            aq[i] = sn * x + cc * y;
            const double vx = vp[i], vy = vq[i];
            vp[i] = cc * vx - sn * vy;
            vq[i] = sn * vx + cc * vy;
          }
        }
        __syncthreads();
      }
      jc_barrier(blockIdx, gridDim, bar, err);
    }
    if (tid == 0) atomicMax(offmax + slot, (unsigned long long)__double_as_longlong(off));
    jc_barrier(blockIdx, gridDim, bar, err);
    const double m = __longlong_as_double((long long)(*(volatile unsigned long long*)(offmax + slot)));
    if (m <= tol) break;
    if (*(volatile int*)err) break;
  }
  if (blockIdx.x == 0 && tid == 0 && sweep >= max_sweeps) atomicExch(sweep_err, 5);
}
TTG_COOP_KERNEL(k_jacobi_coop, JC_THREADS);

// ---------------------------------------------------------------------------
// Cluster Jacobi SVD for 113 < n <= 256 (the 256 x 256 R factors of the
// rounding sweeps): one thread-block cluster of JK_CS CTAs holds A and V in
// distributed shared memory, JK cols = ceil(n / JK_CS) columns per CTA, one
// warp per column.  Columns never move: in each round of the round-robin
// tournament the owners of a pair (P, Q) both read the two columns (one
// local, one remote over DSMEM), compute the same rotation from the same
// values in the same order, and each writes its own rotated column into the
// other of two buffers.  One hardware cluster barrier per round replaces the
// software grid barrier of k_jacobi_coop (the SVD is bound by the latency of
// its ~2300 rounds, not by arithmetic): 0.27 us per cluster barrier against
// several us per grid barrier, while reading the partner's two 256-entry
// columns over DSMEM costs about 2.4 us per round (measured: per-thread
// ld.shared::cluster; bulk shared::cta -> shared::cluster pushes of the
// column blocks completing on the partner's mbarrier measured slower still,
// and so did a row-partitioned form that sends only the partial inner
// products and the rotations across the cluster, with two barriers per
// round: 235 against 195 ms for the SVD sweep of rounding a d = 20, n = 16
// sum of four rank-64 TTs).  Same rotation formula and stopping
// rule as k_jacobi_svd; the rotated A and V go to global memory for
// k_jacobi_finish.  All CTAs of a cluster are co-resident by construction,
// and every CTA takes the same number of rounds (the stopping decision is
// read by all from the same published values): the barriers cannot wait
// for a CTA that is not running.
// ---------------------------------------------------------------------------

constexpr int JK_CS = 16;
constexpr int JK_MAX_N = 256;
constexpr int JK_MAX_COLS = JK_MAX_N / JK_CS;
constexpr int JK_THREADS = 32 * JK_MAX_COLS;
constexpr int JK_MAXR = JK_MAX_N / 32;  // column entries per lane

// Partner of player p in round r of a circle-method tournament on ne (even)
// players: player ne - 1 is fixed and meets r; the others pair as
// p + q = 2 r (mod ne - 1).  Every pair meets once in ne - 1 rounds.
__device__ __forceinline__ int jk_partner(int p, int r, int ne) {
  const int m = ne - 1;
  if (p == m) return r;
  if (p == r) return m;
  int q = 2 * r - p;
  if (q < 0)
    q += m;
  else if (q >= m)
    q -= m;
  return q;
}

// Load of a double from the shared memory of a CTA of the cluster (address
// from mapa: the partner's column, which may sit in this CTA too).
__device__ __forceinline__ double ld_dsmem(uint32_t addr) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr));
  return v;
}

__global__ void __launch_bounds__(JK_THREADS, 1)
    k_jacobi_cluster(int n, const double* __restrict__ Ain, int lda, int trans,
                     double* __restrict__ Aout, double* __restrict__ Vout, int* err,
                     int max_sweeps) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ double sm[];  // A[2][cpc][n], then V[2][cpc][n]
  __shared__ double s_off[2][JK_CS];  // rank 0: per-CTA sweep maxima, by sweep parity
  __shared__ double s_woff[JK_MAX_COLS];
  const int rank = int(cl.block_rank());
  const int ne = (n + 1) & ~1, cpc = (ne + JK_CS - 1) / JK_CS;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int64_t cn = int64_t(cpc) * n;
  for (int64_t e = tid; e < cn; e += blockDim.x) {
    const int j = int(e / n), i = int(e % n), p = rank * cpc + j;
    if (p < n) {
      sm[e] = trans ? Ain[p + int64_t(i) * lda] : Ain[i + int64_t(p) * lda];
      sm[2 * cn + e] = (i == p) ? 1.0 : 0.0;
    }
  }
  cl.sync();
  const double tol = 4.0 * 2.220446049250313e-16, tol2 = tol * tol;
  const int p = rank * cpc + w;
  const bool own = w < cpc && p < n;
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(sm));
  int cur = 0, sweep = 0;
  for (sweep = 0; sweep < max_sweeps; ++sweep) {
    double off = 0.0;
    for (int r = 0; r < ne - 1; ++r) {
      if (own) {
        const int q = jk_partner(p, r, ne);
        const double* ap = sm + cur * cn + int64_t(w) * n;
        const double* vp = ap + 2 * cn;
        double* na = sm + (cur ^ 1) * cn + int64_t(w) * n;
        double* nv = na + 2 * cn;
        if (q >= n) {  // dummy partner (odd n): the column stays
          for (int i = lane; i < n; i += 32) {
            na[i] = ap[i];
            nv[i] = vp[i];
          }
        } else {
          const int rq = q / cpc, jq = q - rq * cpc;
          uint32_t rb;
          asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(rb) : "r"(sbase), "r"(rq));
          const uint32_t aq = rb + uint32_t(8 * (cur * cn + int64_t(jq) * n));
          const uint32_t vq = aq + uint32_t(16 * cn);
          // own column o (local), partner column t (over DSMEM)
          double o[JK_MAXR], t[JK_MAXR], vo[JK_MAXR], vt[JK_MAXR];
#pragma unroll
          for (int k = 0; k < JK_MAXR; ++k) {
            const int i = lane + 32 * k;
            const bool in = i < n;
            t[k] = in ? ld_dsmem(aq + 8 * i) : 0.0;
            vt[k] = in ? ld_dsmem(vq + 8 * i) : 0.0;
            o[k] = in ? ap[i] : 0.0;
            vo[k] = in ? vp[i] : 0.0;
          }
          // al = |a_P|^2, be = |a_Q|^2, ga = <a_P, a_Q> for P < Q: both
          // owners of the pair form the same sums in the same order.
          const bool low = p < q;
          double sp = 0.0, sq = 0.0, ga = 0.0;
#pragma unroll
          for (int k = 0; k < JK_MAXR; ++k) {
            sp = fma(o[k], o[k], sp);
            sq = fma(t[k], t[k], sq);
            ga = low ? fma(o[k], t[k], ga) : fma(t[k], o[k], ga);
          }
          sp = wsum(sp);
          sq = wsum(sq);
          ga = wsum(ga);
          const double al = low ? sp : sq, be = low ? sq : sp;
          const double ab = al * be, g2 = ga * ga;
          if (ab == 0.0 || g2 <= tol2 * ab) {
#pragma unroll
            for (int k = 0; k < JK_MAXR; ++k) {
              const int i = lane + 32 * k;
              if (i < n) {
                na[i] = o[k];
                nv[i] = vo[k];
              }
            }
          } else {
            off = fmax(off, g2 / ab);
            const double dd = be - al, gg = 2.0 * ga;
            const double sg = ((dd >= 0.0) == (gg > 0.0) || dd == 0.0) ? 1.0 : -1.0;
            const double tt = sg * fabs(gg) / (fabs(dd) + sqrt(fma(dd, dd, gg * gg)));
            const double c = rsqrt(fma(tt, tt, 1.0)), sn = c * tt;
            // P' = c P - s Q, Q' = s P + c Q
            if (low) {
#pragma unroll
              for (int k = 0; k < JK_MAXR; ++k) {
                const int i = lane + 32 * k;
                if (i < n) {
                  na[i] = fma(c, o[k], -(sn * t[k]));
                  nv[i] = fma(c, vo[k], -(sn * vt[k]));
                }
              }
            } else {
#pragma unroll
              for (int k = 0; k < JK_MAXR; ++k) {
                const int i = lane + 32 * k;
                if (i < n) {
                  na[i] = fma(sn, t[k], c * o[k]);
                  nv[i] = fma(sn, vt[k], c * vo[k]);
                }
              }
            }
          }
        }
      }
      if (r == ne - 2) {  // last round of the sweep: publish this CTA's maximum
        if (lane == 0 && w < JK_MAX_COLS) s_woff[w] = own ? off : 0.0;
        __syncthreads();
        if (tid == 0) {
          double m = 0.0;
          for (int j = 0; j < cpc; ++j) m = fmax(m, s_woff[j]);
          double* so = cl.map_shared_rank(&s_off[sweep & 1][0], 0);
          so[rank] = m;
        }
      }
      cl.sync();
      cur ^= 1;
    }
    const double* so = cl.map_shared_rank(&s_off[sweep & 1][0], 0);
    double m = 0.0;
    for (int k = 0; k < JK_CS; ++k) m = fmax(m, so[k]);
    if (m <= tol2) break;
  }
  if (rank == 0 && tid == 0 && sweep >= max_sweeps) atomicExch(err, 5);
  for (int64_t e = tid; e < cn; e += blockDim.x) {
    const int j = int(e / n), i = int(e % n), pc = rank * cpc + j;
    if (pc < n) {
      Aout[i + int64_t(pc) * n] = sm[cur * cn + e];
      Vout[i + int64_t(pc) * n] = sm[(2 + cur) * cn + e];
    }
  }
  cl.sync();  // rank 0's published maxima are read until here
}

// ---------------------------------------------------------------------------
// Block-cyclic form of the grid-wide Jacobi SVD: the n columns fall into
// blocks of JB_W; each round of a round-robin tournament on the blocks
// gives every CTA one block pair, whose 2 JB_W columns of A and of V it
// loads into shared memory and rotates through one full inner sweep of
// one-sided Jacobi (every pair of its columns) before writing them back.
// One grid barrier per block round instead of one per column round (31
// instead of 255 barriers per sweep at n = 256); the rotations and the
// stopping rule are those of k_jacobi_coop.
// ---------------------------------------------------------------------------

constexpr int JB_W = 8;
constexpr int JB_THREADS = 256;
constexpr int JB_WARPS = JB_THREADS / 32;

TTG_BODY(k_jacobi_block)(TTG_BLOCK, int n, const double* __restrict__ Ain,
                                                            int lda, double* A, double* V,
                                                            unsigned* bar,
                                                            unsigned long long* offmax, int* err,
                                                            int* sweep_err, int trans,
                                                            int max_sweeps) {
  extern __shared__ double sjb[];  // [2 JB_W][n] columns of A, then of V
  __shared__ int s_col[2 * JB_W];
  __shared__ double s_off[JB_WARPS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t nn = int64_t(n) * n;
  for (int64_t e = blockIdx.x * int64_t(JB_THREADS) + tid; e < nn;
       e += int64_t(gridDim.x) * JB_THREADS) {
    const int64_t i = e % n, j = e / n;
    A[e] = trans ? Ain[j + i * lda] : Ain[i + j * lda];
    V[e] = (i == j) ? 1.0 : 0.0;
  }
  if (blockIdx.x == 0 && tid < 3) offmax[tid] = 0ull;
  jc_barrier(blockIdx, gridDim, bar, err);
  double* sA = sjb;
  double* sV = sjb + int64_t(2 * JB_W) * n;
  const int nb = (n + JB_W - 1) / JB_W;
  const int nbe = (nb + 1) & ~1;  // even number of block players (dummy block if odd)
  const double tol = 4.0 * 2.220446049250313e-16;
  int sweep = 0;
  for (sweep = 0; sweep < max_sweeps; ++sweep) {
    const int slot = sweep % 3;
    if (blockIdx.x == 0 && tid == 0) offmax[(sweep + 1) % 3] = 0ull;
    double off = 0.0;  // per warp
    for (int r = 0; r < nbe - 1; ++r) {
      for (int pr = blockIdx.x; pr < nbe / 2; pr += gridDim.x) {
        const int P = rr_player(pr, r, nbe), Q = rr_player(nbe - 1 - pr, r, nbe);
        // the block pair's columns (a dummy block contributes none)
        int nc = 0;
        if (tid == 0) {
          for (int b : {P, Q})
            for (int c = b * JB_W; c < (b + 1) * JB_W && c < n && b < nb; ++c) s_col[nc++] = c;
          for (int k = nc; k < 2 * JB_W; ++k) s_col[k] = -1;
        }
        __syncthreads();
        nc = 0;
        for (int k = 0; k < 2 * JB_W; ++k) nc += s_col[k] >= 0;
        for (int64_t e = tid; e < int64_t(nc) * n; e += JB_THREADS) {
          const int k = int(e / n);
          const int64_t i = e % n;
          sA[e] = A[i + int64_t(s_col[k]) * n];
          sV[e] = V[i + int64_t(s_col[k]) * n];
        }
        __syncthreads();
        // one inner sweep over all column pairs of the block pair
        const int ne = (nc + 1) & ~1;
        for (int ir = 0; ir < ne - 1; ++ir) {
          for (int ip = warp; ip < ne / 2; ip += JB_WARPS) {
            int p = rr_player(ip, ir, ne), q = rr_player(ne - 1 - ip, ir, ne);
            if (p > q) {
              const int t = p;
              p = q;
              q = t;
            }
            if (q >= nc) continue;  // dummy
            double* ap = sA + int64_t(p) * n;
            double* aq = sA + int64_t(q) * n;
            double al = 0.0, be = 0.0, ga = 0.0;
            for (int i = lane; i < n; i += 32) {
              const double x = ap[i], y = aq[i];
              al += x * x;
              be += y * y;
              ga += x * y;
            }
            al = wsum(al);
            be = wsum(be);
            ga = wsum(ga);
            const double nrm = sqrt(al * be);
            if (nrm == 0.0 || fabs(ga) <= tol * nrm) continue;  // uniform in the warp
            off = fmax(off, fabs(ga) / nrm);
            const double zeta = (be - al) / (2.0 * ga);
            const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            const double cc = 1.0 / sqrt(1.0 + t * t), sn = cc * t;
            double* vp = sV + int64_t(p) * n;
            double* vq = sV + int64_t(q) * n;
            for (int i = lane; i < n; i += 32) {
              const double x = ap[i], y = aq[i];
              ap[i] = cc * x - sn * y;
              aq[i] = sn * x + cc * y;
              const double vx = vp[i], vy = vq[i];
              vp[i] = cc * vx - sn * vy;
              vq[i] = sn * vx + cc * vy;
            }
          }
          __syncthreads();
        }
        for (int64_t e = tid; e < int64_t(nc) * n; e += JB_THREADS) {
          const int k = int(e / n);
          const int64_t i = e % n;
          A[i + int64_t(s_col[k]) * n] = sA[e];
          V[i + int64_t(s_col[k]) * n] = sV[e];
        }
        __syncthreads();
      }
      jc_barrier(blockIdx, gridDim, bar, err);
    }
    if (lane == 0) s_off[warp] = off;
    __syncthreads();
    if (tid == 0) {
      double m = 0.0;
      for (int w = 0; w < JB_WARPS; ++w) m = fmax(m, s_off[w]);
      atomicMax(offmax + slot, (unsigned long long)__double_as_longlong(m));
    }
    jc_barrier(blockIdx, gridDim, bar, err);
    const double m = __longlong_as_double((long long)(*(volatile unsigned long long*)(offmax + slot)));
    if (m <= tol) break;
    if (*(volatile int*)err) break;
  }
  if (blockIdx.x == 0 && tid == 0 && sweep >= max_sweeps) atomicExch(sweep_err, 5);
}
TTG_COOP_KERNEL(k_jacobi_block, JB_THREADS);

TTG_BODY(k_jacobi_finish)(TTG_BLOCK, int n, const double* A,
                                                             const double* V, double* U,
                                                             double* S, double* VT, double* sig,
                                                             int trans) {
  pdl_begin();
  jacobi_finish(n, A, V, U, S, VT, sig, trans);
}
TTG_KERNEL(k_jacobi_finish, SD_THREADS);

// Householder QR of the m x n matrix A (column-major, lda) held in shared
// memory: Q (m x k, ld m), R (k x n, ld k), k = min(m, n).
TTG_BODY(k_house_qr)(TTG_BLOCK, int m, int n, const double* __restrict__ Ain,
                                                        int lda, double* __restrict__ Q,
                                                        double* __restrict__ R,
                                                        const int* skip) {
  pdl_begin();
  if (skip && *skip) return;  // conditional factorization (Context::skip)
  const int ldr = m < n ? m : n;
  extern __shared__ double sm[];
  double* A = sm;                 // m x n
  double* tau = sm + int64_t(m) * n;  // k
  __shared__ double red[SD_WARPS];
  __shared__ double bcast[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k = m < n ? m : n;
  for (int e = tid; e < m * n; e += SD_THREADS) A[e] = Ain[(e % m) + int64_t(e / m) * lda];
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    double* aj = A + int64_t(j) * m;
    // ||x(2:end)||^2
    double s = 0.0;
    for (int i = j + 1 + tid; i < m; i += SD_THREADS) s += aj[i] * aj[i];
    s = wsum(s);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < SD_WARPS; ++w) t += red[w];
      const double alpha = aj[j];
      double beta, tj, scal;
      if (t == 0.0) {
        beta = alpha;
        tj = 0.0;
        scal = 0.0;
      } else {
        beta = -copysign(sqrt(alpha * alpha + t), alpha);
        tj = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      tau[j] = tj;
      aj[j] = beta;
      bcast[0] = scal;
    }
    __syncthreads();
    const double scal = bcast[0];
    for (int i = j + 1 + tid; i < m; i += SD_THREADS) aj[i] *= scal;  // v(2:end), v(1) = 1
    __syncthreads();
    const double tj = tau[j];
    if (tj != 0.0) {
      for (int c = j + 1 + warp; c < n; c += SD_WARPS) {
        double* ac = A + int64_t(c) * m;
        double w = 0.0;
        for (int i = j + lane; i < m; i += 32) w += (i == j ? 1.0 : aj[i]) * ac[i];
        w = wsum(w) * tj;
        for (int i = j + lane; i < m; i += 32) ac[i] -= w * (i == j ? 1.0 : aj[i]);
      }
    }
    __syncthreads();
  }
  // R
  for (int e = tid; e < k * n; e += SD_THREADS) {
    const int i = e % k, c = e / k;
    R[i + int64_t(c) * ldr] = (i <= c) ? A[i + int64_t(c) * m] : 0.0;
  }
  __syncthreads();
  // Q = H_0 H_1 ... H_{k-1} I(:, 0:k), applied right to left in place of the
  // reflectors (LAPACK dorg2r's scheme): when H_j is applied, columns c > j
  // of A already hold Q's columns (zero in rows <= j, as I's are), so H_j
  // updates them, and then column j becomes H_j e_j = e_j - tau_j v_j, with
  // its rows above j cleared.  The arithmetic is that of applying H_j to I's
  // column j (w = tau_j exactly), so Q matches a product formed on I.
  for (int j = k - 1; j >= 0; --j) {
    const double tj = tau[j];
    double* v = A + int64_t(j) * m;
    if (tj != 0.0) {
      for (int c = j + 1 + warp; c < k; c += SD_WARPS) {
        double* qc = A + int64_t(c) * m;
        double w = 0.0;
        for (int i = j + lane; i < m; i += 32) w += (i == j ? 1.0 : v[i]) * qc[i];
        w = wsum(w) * tj;
        for (int i = j + lane; i < m; i += 32) qc[i] -= w * (i == j ? 1.0 : v[i]);
      }
    }
    __syncthreads();
    for (int i = tid; i < m; i += SD_THREADS)
      v[i] = i < j ? 0.0 : (i == j ? 1.0 - tj : 0.0 - tj * v[i]);
    __syncthreads();
  }
  for (int e = tid; e < m * k; e += SD_THREADS) Q[e] = A[e];
}
TTG_KERNEL(k_house_qr, SD_THREADS);


// ---------------------------------------------------------------------------
// Householder QR of a skinny m x n matrix (n <= SK_MAX_N) too tall for shared
// memory: the work copy W lives in global memory (L2), every thread owns the
// rows i = tid (mod SD_THREADS), and each reflector needs two block-wide
// reductions -- the column norm, then the n - j - 1 inner products of all
// trailing columns at once -- instead of one warp per column.  Same
// reflectors and signs as k_house_qr (LAPACK's dlarfg convention).
// ---------------------------------------------------------------------------

constexpr int SK_MAX_N = 8;

// Block-wide sums of cnt <= SK_MAX_N values per thread; every thread gets
// the totals in out[0..cnt).  scratch: SD_WARPS * SK_MAX_N doubles (shared).
__device__ void block_sums(const double* v, int cnt, double* scratch, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = 0; q < cnt; ++q) {
    const double s = wsum(v[q]);
    if (lane == 0) scratch[warp * SK_MAX_N + q] = s;
  }
  __syncthreads();
  if (threadIdx.x < cnt) {
    double t = 0.0;
    for (int w = 0; w < SD_WARPS; ++w) t += scratch[w * SK_MAX_N + threadIdx.x];
    scratch[SD_WARPS * SK_MAX_N + threadIdx.x] = t;
  }
  __syncthreads();
  for (int q = 0; q < cnt; ++q) out[q] = scratch[SD_WARPS * SK_MAX_N + q];
  __syncthreads();
}

TTG_BODY(k_house_qr_skinny)(TTG_BLOCK, int64_t m, int n,
                                                               const double* __restrict__ Ain,
                                                               int64_t lda, double* __restrict__ W,
                                                               double* __restrict__ Q,
                                                               double* __restrict__ R) {
  pdl_begin();
  __shared__ double scratch[(SD_WARPS + 1) * SK_MAX_N];
  __shared__ double tau[SK_MAX_N];
  const int tid = threadIdx.x;
  const int k = int(m < n ? m : n);
  for (int64_t e = tid; e < m * n; e += SD_THREADS) W[e] = Ain[(e % m) + (e / m) * lda];
  __syncthreads();
  double part[SK_MAX_N], tot[SK_MAX_N];
  for (int j = 0; j < k; ++j) {
    double* wj = W + int64_t(j) * m;
    double s = 0.0;
    for (int64_t i = j + 1 + tid; i < m; i += SD_THREADS) s += wj[i] * wj[i];
    part[0] = s;
    block_sums(part, 1, scratch, tot);
    const double alpha = wj[j];
    __syncthreads();  // every thread has read alpha before wj[j] changes
    double beta, tj, scal;
    if (tot[0] == 0.0) {
      beta = alpha;
      tj = 0.0;
      scal = 0.0;
    } else {
      beta = -copysign(sqrt(alpha * alpha + tot[0]), alpha);
      tj = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    for (int64_t i = j + 1 + tid; i < m; i += SD_THREADS) wj[i] *= scal;  // v, v(j) = 1
    if (tid == 0) {
      tau[j] = tj;
      wj[j] = beta;
    }
    __syncthreads();
    const int nc = n - j - 1;
    if (tj != 0.0 && nc > 0) {
      for (int q = 0; q < nc; ++q) part[q] = 0.0;
      for (int64_t i = j + 1 + tid; i < m; i += SD_THREADS) {
        const double vi = wj[i];
        for (int q = 0; q < nc; ++q) part[q] += vi * W[i + int64_t(j + 1 + q) * m];
      }
      block_sums(part, nc, scratch, tot);
      for (int q = 0; q < nc; ++q) tot[q] = tj * (tot[q] + W[j + int64_t(j + 1 + q) * m]);
      __syncthreads();  // row j read by all before it changes
      for (int q = 0; q < nc; ++q) {
        double* wc = W + int64_t(j + 1 + q) * m;
        for (int64_t i = j + 1 + tid; i < m; i += SD_THREADS) wc[i] -= tot[q] * wj[i];
        if (tid == 0) wc[j] -= tot[q];
      }
      __syncthreads();
    }
  }
  for (int e = tid; e < k * n; e += SD_THREADS) {
    const int i = e % k, c = e / k;
    R[i + int64_t(c) * k] = (i <= c) ? W[i + int64_t(c) * m] : 0.0;
  }
  // Q = H_0 ... H_{k-1} I(:, 0:k), right to left.
  for (int64_t e = tid; e < m * k; e += SD_THREADS) Q[e] = ((e % m) == (e / m)) ? 1.0 : 0.0;
  __syncthreads();
  for (int j = k - 1; j >= 0; --j) {
    const double tj = tau[j];
    if (tj == 0.0) continue;  // uniform
    const double* v = W + int64_t(j) * m;
    const int nc = k - j;
    for (int q = 0; q < nc; ++q) part[q] = 0.0;
    for (int64_t i = j + 1 + tid; i < m; i += SD_THREADS) {
      const double vi = v[i];
      for (int q = 0; q < nc; ++q) part[q] += vi * Q[i + int64_t(j + q) * m];
    }
    block_sums(part, nc, scratch, tot);
    for (int q = 0; q < nc; ++q) tot[q] = tj * (tot[q] + Q[j + int64_t(j + q) * m]);
    __syncthreads();  // row j read by all before it changes
    for (int q = 0; q < nc; ++q) {
      double* qc = Q + int64_t(j + q) * m;
      for (int64_t i = j + 1 + tid; i < m; i += SD_THREADS) qc[i] -= tot[q] * v[i];
      if (tid == 0) qc[j] -= tot[q];
    }
    __syncthreads();
  }
}
TTG_KERNEL(k_house_qr_skinny, SD_THREADS);

// ---------------------------------------------------------------------------
// Cholesky factor and its inverse for shifted Cholesky QR
// ---------------------------------------------------------------------------

// G (n x n SPD Gram matrix, ldg) -> R = chol(G + shift I) upper (R' R = G +
// shift I) and Rinv = R^{-1}, both n x n with leading dimension n.  shift =
// shift_factor * trace(G).  err_slot |= 1 if a pivot is not positive.
TTG_BODY(k_chol_inv)(TTG_BLOCK, int n, const double* __restrict__ G,
                                                        int ldg, double shift_factor,
                                                        double* __restrict__ R,
                                                        double* __restrict__ Rinv, int* err) {
  pdl_begin();
  extern __shared__ double sm[];
  double* L = sm;                  // n x n, lower triangle = Cholesky factor
  double* X = sm + int64_t(n) * n; // n x n, L^{-1}
  __shared__ double s_shift;
  __shared__ int s_bad;
  const int tid = threadIdx.x;
  for (int e = tid; e < n * n; e += SD_THREADS) L[e] = G[(e % n) + int64_t(e / n) * ldg];
  __syncthreads();
  if (tid == 0) {
    double tr = 0.0;
    for (int i = 0; i < n; ++i) tr += L[i + n * i];
    s_shift = shift_factor * tr;
    s_bad = 0;
  }
  __syncthreads();
  for (int i = tid; i < n; i += SD_THREADS) L[i + n * i] += s_shift;
  for (int e = tid; e < n * n; e += SD_THREADS) {
    const int r = e % n, c = e / n;
    X[e] = (r == c) ? 1.0 : 0.0;
    if (r > c) {  // strictly lower parts of the triangular outputs
      R[e] = 0.0;
      Rinv[e] = 0.0;
    }
  }
  __syncthreads();
  // Right-looking Cholesky G = L L', with the forward elimination L X = I
  // applied to X = I in the same steps (X = L^{-1} at the end).  Step j
  // reads column j of L and row j of X unscaled (nothing writes them in
  // that step), removes column j from the trailing lower triangle and row j
  // from the rows of X below it (with the pivot's reciprocal squared), and
  // writes row j of R = L' and column j of Rinv = X' scaled: one barrier
  // per column.  The step's n columns -- trailing columns k of L (rows k..n)
  // and columns cc <= j of X (rows j+1..n) -- go one per warp, lanes down
  // the rows, so no thread divides an index or idles on the upper triangle;
  // every element takes the same products in the same order as an
  // element-per-thread loop.
  const int lane = tid & 31, warp = tid >> 5;
  for (int j = 0; j < n; ++j) {
    const double d = L[j + n * j];
    const double dj = d > 0.0 ? sqrt(d) : 1.0;
    if (tid == 0 && !(d > 0.0)) s_bad = 1;
    const double inv = 1.0 / dj, inv2 = inv * inv;
    const int m = n - j - 1;
    const double* lj = L + n * j;
    for (int u = warp; u < n; u += SD_WARPS) {
      if (u < m) {
        const int k = j + 1 + u;
        const double lk = lj[k];
        double* col = L + n * k;
        for (int i = k + lane; i < n; i += 32) col[i] -= lj[i] * lk * inv2;
      } else {
        double* col = X + n * (u - m);
        const double xj = col[j];
        for (int i = j + 1 + lane; i < n; i += 32) col[i] -= lj[i] * xj * inv2;
      }
    }
    for (int i = j + tid; i < n; i += SD_THREADS)
      R[j + int64_t(n) * i] = (i == j) ? dj : L[i + n * j] * inv;
    for (int cc = tid; cc <= j; cc += SD_THREADS) Rinv[cc + int64_t(n) * j] = X[j + n * cc] * inv;
    __syncthreads();
  }
  if (tid == 0 && s_bad) atomicOr(err, 1);
}
TTG_KERNEL(k_chol_inv, SD_THREADS);


// ---------------------------------------------------------------------------
// One-sided Jacobi SVD of a tall m x n matrix with few columns (n <=
// TS_MAX_N, m >= n), held in shared memory and rotated directly (no QR
// first): one warp per column pair of a round-robin round, the rotation and
// stopping rule of k_jacobi_svd.  U = A V diag(1/s) (m x n, ld m); columns of
// exactly zero norm are completed to an orthonormal set (Gram-Schmidt of unit
// vectors against the other columns), so U always has orthonormal columns.
// S descending, VT (n x n, ld n).  One launch replaces QR + square SVD +
// U = Q Ur for the small SVDs of the sweeps (Z updates, early truncations).
// ---------------------------------------------------------------------------

constexpr int TS_THREADS = 256;
constexpr int TS_WARPS = TS_THREADS / 32;
constexpr int TS_MAX_N = 8;

TTG_BODY(k_svd_tall_small)(TTG_BLOCK, int m, int n,
                                                              const double* __restrict__ Ain,
                                                              int lda, double* __restrict__ U,
                                                              double* __restrict__ S,
                                                              double* __restrict__ VT,
                                                              int* err, int max_sweeps) {
  pdl_begin();
  extern __shared__ double A[];  // m x n
  __shared__ double V[TS_MAX_N * TS_MAX_N];
  __shared__ double sig[TS_MAX_N];
  __shared__ int pos[TS_MAX_N];
  __shared__ double s_off[TS_WARPS];
  __shared__ int s_done;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < m * n; e += TS_THREADS) {
    const int i = e % m, j = e / m;
    A[e] = Ain[i + int64_t(j) * lda];
  }
  for (int e = tid; e < n * n; e += TS_THREADS) V[e] = (e % n == e / n) ? 1.0 : 0.0;
  __syncthreads();
  const int ne = (n + 1) & ~1;
  const double tol = 4.0 * 2.220446049250313e-16, tol2 = tol * tol;
  int sweep = 0;
  for (sweep = 0; sweep < max_sweeps; ++sweep) {
    double off = 0.0;
    for (int r = 0; r < ne - 1; ++r) {
      for (int pr = warp; pr < ne / 2; pr += TS_WARPS) {
        int p = rr_player(pr, r, ne), q = rr_player(ne - 1 - pr, r, ne);
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        if (q >= n) continue;  // dummy player
        double* ap = A + int64_t(p) * m;
        double* aq = A + int64_t(q) * m;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i = lane; i < m; i += 32) {
          const double x = ap[i], y = aq[i];
          al += x * x;
          be += y * y;
          ga += x * y;
        }
        al = wsum(al);
        be = wsum(be);
        ga = wsum(ga);
        const double ab = al * be, g2 = ga * ga;
        if (ab == 0.0 || g2 <= tol2 * ab) continue;
        off = fmax(off, g2 / ab);
        const double dd = be - al, gg = 2.0 * ga;
        const double sg = ((dd >= 0.0) == (gg > 0.0) || dd == 0.0) ? 1.0 : -1.0;
        const double t = sg * fabs(gg) / (fabs(dd) + sqrt(dd * dd + gg * gg));
        const double c = rsqrt(1.0 + t * t), s = c * t;
        for (int i = lane; i < m; i += 32) {
          const double x = ap[i], y = aq[i];
          ap[i] = c * x - s * y;
          aq[i] = s * x + c * y;
        }
        if (lane < n) {
          const double vx = V[lane + p * n], vy = V[lane + q * n];
          V[lane + p * n] = c * vx - s * vy;
          V[lane + q * n] = s * vx + c * vy;
        }
      }
      __syncthreads();
    }
    if (lane == 0) s_off[warp] = off;
    __syncthreads();
    if (tid == 0) {
      double mx = 0.0;
      for (int w = 0; w < TS_WARPS; ++w) mx = fmax(mx, s_off[w]);
      s_done = (mx <= tol2) ? 1 : 0;
    }
    __syncthreads();
    if (s_done) break;
  }
  if (tid == 0 && sweep >= max_sweeps) atomicExch(err, 5);
  // singular values = column norms, ranked descending (stable on index)
  if (warp < n) {
    const double* aj = A + int64_t(warp) * m;
    double s = 0.0;
    for (int i = lane; i < m; i += 32) s += aj[i] * aj[i];
    s = wsum(s);
    if (lane == 0) sig[warp] = sqrt(s);
  }
  __syncthreads();
  if (tid < n) {
    const double sj = sig[tid];
    int p = 0;
    for (int k = 0; k < n; ++k) p += (sig[k] > sj) || (sig[k] == sj && k < tid);
    pos[tid] = p;
  }
  for (int e = tid; e < m * n; e += TS_THREADS) {
    const double sj = sig[e / m];
    if (sj > 0.0) A[e] /= sj;
  }
  __syncthreads();
  // complete zero columns: e_k minus its projections on the columns kept so
  // far (twice), accepted when at least 0.3 of it is left (the mean left
  // over all k is at least 1 - (n - 1) / m >= 1 / n)
  if (warp == 0) {
    for (int j = 0; j < n; ++j) {
      if (sig[j] > 0.0) continue;
      double* aj = A + int64_t(j) * m;
      for (int k = 0; k < m; ++k) {
        for (int i = lane; i < m; i += 32) aj[i] = (i == k) ? 1.0 : 0.0;
        __syncwarp();
        for (int pass = 0; pass < 2; ++pass) {
          for (int q = 0; q < n; ++q) {
            if (q == j || (sig[q] == 0.0 && q > j)) continue;
            const double* aq = A + int64_t(q) * m;
            double d = 0.0;
            for (int i = lane; i < m; i += 32) d += aq[i] * aj[i];
            d = wsum(d);
            for (int i = lane; i < m; i += 32) aj[i] -= d * aq[i];
            __syncwarp();
          }
        }
        double nr = 0.0;
        for (int i = lane; i < m; i += 32) nr += aj[i] * aj[i];
        nr = sqrt(wsum(nr));
        if (nr > 0.3) {
          for (int i = lane; i < m; i += 32) aj[i] /= nr;
          __syncwarp();
          break;
        }
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < m * n; e += TS_THREADS) {
    const int i = e % m, j = e / m;
    U[i + int64_t(pos[j]) * m] = A[e];
  }
  for (int e = tid; e < n * n; e += TS_THREADS) {
    const int i = e % n, j = e / n;
    VT[pos[j] + i * n] = V[e];
  }
  if (tid < n) S[pos[tid]] = sig[tid];
}
TTG_KERNEL(k_svd_tall_small, TS_THREADS);

// ---------------------------------------------------------------------------
// LU with partial pivoting and the two triangular solves (LAPACK getf2 +
// getrs, unblocked) of an n x n matrix held in shared memory, for the dense
// local systems of AMEn (n < max_full_size): X <- B^{-1} X for nrhs
// right-hand sides.  The pivot is the first entry of largest magnitude in
// its column (idamax); the multipliers are formed with the pivot's
// reciprocal; the row swaps and the unit-lower elimination are applied to X
// as the factorization proceeds, then X is solved with the upper factor
// column by column.  *err |= 1 on an exactly zero pivot (getrf's info > 0).
// ---------------------------------------------------------------------------

TTG_BODY(k_lu_small)(TTG_BLOCK, int n, const double* __restrict__ B, int nrhs,
                     double* __restrict__ X, int* err) {
  pdl_begin();
  extern __shared__ double slu[];
  double* a = slu;             // n x n, column-major
  double* x = slu + n * n;     // n x nrhs
  __shared__ int s_piv, s_bad;
  const int tid = threadIdx.x;
  for (int e = tid; e < n * n; e += blockDim.x) a[e] = B[e];
  for (int e = tid; e < n * nrhs; e += blockDim.x) x[e] = X[e];
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (tid < 32) {  // idamax over rows k..n-1 of column k
      double best = -1.0;
      int bi = k;
      for (int i = k + tid; i < n; i += 32) {
        const double v = fabs(a[i + n * k]);
        if (v > best) {
          best = v;
          bi = i;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (tid == 0) {
        s_piv = bi;
        if (!(best > 0.0)) s_bad = 1;
      }
    }
    __syncthreads();
    const int p = s_piv;
    if (p != k) {
      for (int j = tid; j < n; j += blockDim.x) {
        const double t = a[k + n * j];
        a[k + n * j] = a[p + n * j];
        a[p + n * j] = t;
      }
      for (int r = tid; r < nrhs; r += blockDim.x) {
        const double t = x[k + n * r];
        x[k + n * r] = x[p + n * r];
        x[p + n * r] = t;
      }
    }
    __syncthreads();
    const double piv = a[k + n * k];
    if (piv != 0.0) {
      const double rinv = 1.0 / piv;
      for (int i = k + 1 + tid; i < n; i += blockDim.x) a[i + n * k] *= rinv;
    }
    __syncthreads();
    const int rows = n - k - 1;
    if (rows > 0) {
      const int tot = rows * (n - k - 1 + nrhs);
      for (int e = tid; e < tot; e += blockDim.x) {
        const int i = k + 1 + e % rows, c = e / rows;
        const double l = a[i + n * k];
        if (c < n - k - 1) {
          const int j = k + 1 + c;
          a[i + n * j] -= l * a[k + n * j];
        } else {
          const int r = c - (n - k - 1);
          x[i + n * r] -= l * x[k + n * r];
        }
      }
    }
    __syncthreads();
  }
  for (int k = n - 1; k >= 0; --k) {
    for (int r = tid; r < nrhs; r += blockDim.x) x[k + n * r] /= a[k + n * k];
    __syncthreads();
    for (int e = tid; e < k * nrhs; e += blockDim.x) {
      const int i = e % k, r = e / k;
      x[i + n * r] -= x[k + n * r] * a[i + n * k];
    }
    __syncthreads();
  }
  for (int e = tid; e < n * nrhs; e += blockDim.x) X[e] = x[e];
  if (tid == 0 && s_bad) atomicOr(err, 1);
}
TTG_KERNEL(k_lu_small, SD_THREADS);

}  // namespace

bool lu_small_fits(int64_t n, int64_t nrhs) {
  return n >= 1 && nrhs >= 1 && sizeof(double) * size_t(n) * size_t(n + nrhs) <= SMEM_LIMIT;
}

void lu_small_f64(Context* c, int64_t n, const double* B, double* X, int64_t nrhs) {
  TTG_REQUIRE(lu_small_fits(n, nrhs), "lu_small: n = %lld, nrhs = %lld out of range",
              (long long)n, (long long)nrhs);
  const size_t smem = sizeof(double) * size_t(n) * size_t(n + nrhs);
  ensure_smem_attr(k_lu_small.fn(), c->device, int(SMEM_LIMIT + 1024));
  launch(c, k_lu_small, 1, SD_THREADS, smem, int(n), B, int(nrhs), X, c->d_err + 4);
  TTG_CHECK_LAUNCH();
}

bool chol_inv_fits(int64_t n) { return 2 * n * n * int64_t(sizeof(double)) <= int64_t(SMEM_LIMIT); }

void chol_inv_f64(Context* c, int64_t n, const double* G, int64_t ldg, double shift_factor,
                  double* R, double* Rinv, int* flag) {
  TTG_REQUIRE(chol_inv_fits(n), "chol_inv: n = %lld too large", (long long)n);
  const size_t smem = 2 * sizeof(double) * size_t(n * n);
  ensure_smem_attr(k_chol_inv.fn(), c->device, int(SMEM_LIMIT + 1024));
  launch(c, k_chol_inv, 1, SD_THREADS, smem, int(n), G, int(ldg), shift_factor, R, Rinv,
         flag ? flag : c->d_err + 4);
  TTG_CHECK_LAUNCH();
}

bool skinny_qr_fits(int64_t m, int64_t n) { return n >= 1 && n <= SK_MAX_N && m >= n; }

void skinny_qr_f64(Context* c, int64_t m, int64_t n, const double* A, int64_t lda, double* Q,
                   double* R) {
  TTG_REQUIRE(skinny_qr_fits(m, n), "skinny QR: %lld x %lld out of range", (long long)m,
              (long long)n);
  DBuf<double> W(c, m * n);
  launch(c, k_house_qr_skinny, 1, SD_THREADS, 0, m, int(n), A, lda, W.p(), Q, R);
  TTG_CHECK_LAUNCH();
}

bool small_qr_fits(int64_t m, int64_t n) {
  return m * n + std::min(m, n) <= int64_t(SMEM_LIMIT / sizeof(double)) && m <= 0x7fffffff;
}

void small_qr_f64(Context* c, int64_t m, int64_t n, const double* A, int64_t lda, double* Q,
                  double* R) {
  const size_t smem = sizeof(double) * size_t(m * n + std::min(m, n));
  ensure_smem_attr(k_house_qr.fn(), c->device, int(SMEM_LIMIT + 1024));
  launch(c, k_house_qr, 1, SD_THREADS, smem, int(m), int(n), A, int(lda), Q, R, c->skip);
  TTG_CHECK_LAUNCH();
}


bool svd_tall_small_fits(int64_t m, int64_t n) {
  return n >= 1 && n <= TS_MAX_N && m >= n && m * n * int64_t(sizeof(double)) <= int64_t(128 * 1024);
}

void svd_tall_small_f64(Context* c, int64_t m, int64_t n, const double* A, int64_t lda, double* U,
                        double* S, double* VT) {
  TTG_REQUIRE(svd_tall_small_fits(m, n), "svd_tall_small: %lld x %lld out of range",
              (long long)m, (long long)n);
  const size_t smem = sizeof(double) * size_t(m * n);
  ensure_smem_attr(k_svd_tall_small.fn(), c->device,
                   int(128 * 1024 + 1024));
  launch(c, k_svd_tall_small, 1, TS_THREADS, smem, int(m), int(n), A, int(lda), U, S, VT,
         c->d_err + 3, c->jacobi_max_sweeps);
  TTG_CHECK_LAUNCH();
}

// TTG_JACOBI_BLOCK=1 selects the block-cyclic grid-wide Jacobi SVD; the
// default is the one-pair-per-CTA rounds (measured no slower in rounding and
// a little more accurate at n >= 256).
static bool getenv_flag_on(const char* name) {
  const char* e = getenv(name);
  return e && e[0] == '1';
}

// The block-pair columns of A and V (4 JB_W n doubles) fit in shared memory.
static bool jacobi_block_fits(int64_t n) {
  return n >= 4 * JB_W && sizeof(double) * 4 * JB_W * size_t(n) <= SMEM_LIMIT &&
         getenv_flag_on("TTG_JACOBI_BLOCK");
}

size_t jacobi_cluster_smem(int64_t n) {
  const int64_t cpc = (((n + 1) & ~int64_t(1)) + JK_CS - 1) / JK_CS;
  return sizeof(double) * 4 * size_t(cpc) * size_t(n);
}

// The cluster form runs where one CTA's shared memory cannot hold both A
// and V (n > 113) up to JK_MAX_N (measured 2.1x the grid-wide form's speed
// at n = 120 and 144, 1.2x at 256), unless TTG_JACOBI_CLUSTER=0, when the device
// can place a 16-CTA cluster with that shared memory (checked once per
// device and size class: attributes set, cudaOccupancyMaxActiveClusters).
// Outside a grouped batch it also takes the sizes from
// TTG_JACOBI_CLUSTER_MIN_N (default 48) up, which the one-CTA kernel could
// hold: a lone solve waits on each SVD (whole SVD of a Gaussian n x n matrix,
// cluster against one CTA: 2.0 against 5.7 ms at n = 113, 0.89 against 1.39
// at 64, 0.68 against 0.84 at 48, even at 32), while a grouped batch fills
// the GPU with concurrent systems and wants the one-CTA kernel's single SM.
int64_t jacobi_cluster_min_n() {
  static const int64_t v = [] {
    const char* e = getenv("TTG_JACOBI_CLUSTER_MIN_N");
    const long long x = e ? atoll(e) : 0;
    return int64_t(x >= 2 ? x : 48);
  }();
  return v;
}

bool jacobi_cluster_ok(Context* c, int64_t n) {
  static const bool on = [] {
    const char* e = getenv("TTG_JACOBI_CLUSTER");
    return !(e && e[0] == '0');
  }();
  if (!on || n > JK_MAX_N || n < 2) return false;
  const size_t smem = jacobi_cluster_smem(n);
  static std::mutex mu;
  static std::map<std::pair<int, size_t>, bool> seen;
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_pair(c->device, smem);
  auto it = seen.find(key);
  if (it != seen.end()) return it->second;
  // The attribute is set once to the largest size any n takes (setting it
  // per size would lower it below a size already admitted).
  bool ok = cudaFuncSetAttribute(k_jacobi_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed,
                                 1) == cudaSuccess &&
            cudaFuncSetAttribute(k_jacobi_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(jacobi_cluster_smem(JK_MAX_N))) == cudaSuccess;
  if (ok) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(JK_CS);
    cfg.blockDim = dim3(JK_THREADS);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = JK_CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    ok = cudaOccupancyMaxActiveClusters(&clusters, k_jacobi_cluster, &cfg) == cudaSuccess &&
         clusters >= 1;
  }
  cudaGetLastError();  // a refused attribute or query leaves no sticky state
  seen[key] = ok;
  return ok;
}

void jacobi_svd_f64(Context* c, int64_t n, const double* A, int64_t lda, double* U, double* S,
                    double* VT, bool via_transpose) {
  int trans = via_transpose ? 1 : 0;
  TTG_REQUIRE(n >= 1 && n <= 4096, "jacobi_svd: n = %lld out of range", (long long)n);
  const size_t mat = size_t(n * n) * sizeof(double);
  const int mode = 2 * mat <= SMEM_LIMIT ? 2 : (mat <= SMEM_LIMIT ? 1 : 0);
  DBuf<double> V(c, n * n), work(c, n * n + 2 * n);
  if (mode == 0 && jacobi_block_fits(n)) {
    // Block-cyclic grid-wide rounds: one CTA per block pair.
    const size_t bsm = sizeof(double) * 4 * JB_W * size_t(n);
    ensure_smem_attr(k_jacobi_block.fn(), c->device, int(bsm));
    int occ = 0;
    TTG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_jacobi_block.plain(),
                                                           JB_THREADS, bsm));
    const int64_t bpairs = ((n + JB_W - 1) / JB_W + 1) / 2;
    const int blocks = int(std::max<int64_t>(
        1, std::min<int64_t>(bpairs, int64_t(c->num_sms) * std::max(occ, 1))));
    DBuf<unsigned> bar(c, 2);
    DBuf<unsigned long long> offmax(c, 3);
    memset_async(c, bar.p(), 0, 2 * sizeof(unsigned));
    launch(c, k_jacobi_block, blocks, JB_THREADS, bsm, int(n), A, int(lda), work.p(), V.p(),
           bar.p(), offmax.p(), c->d_err + 0, c->d_err + 3, trans, c->jacobi_max_sweeps);
    launch(c, k_jacobi_finish, 1, SD_THREADS, 0, int(n), work.p(), V.p(), U, S, VT,
           work.p() + int64_t(n) * n, trans);
    TTG_CHECK_LAUNCH();
    return;
  }
  if ((mode == 0 || mode == 1 || (!c->rec && n >= jacobi_cluster_min_n())) &&
      jacobi_cluster_ok(c, n)) {
    // One 16-CTA cluster, A and V in distributed shared memory.
    const size_t jsm = jacobi_cluster_smem(n);
    const int ns = int(n), ilda = int(lda), sweeps = c->jacobi_max_sweeps;
    double* Aw = work.p();
    double* Vw = V.p();
    int* err = c->d_err + 3;
    auto issue = [=](cudaStream_t s) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(JK_CS);
      cfg.blockDim = dim3(JK_THREADS);
      cfg.dynamicSmemBytes = jsm;
      cfg.stream = s;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = JK_CS;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      TTG_CUDA(cudaLaunchKernelEx(&cfg, k_jacobi_cluster, ns, A, ilda, trans, Aw, Vw, err,
                                  sweeps));
    };
    if (c->rec) {
      rec_op(c->rec, [issue](cudaStream_t s, cusolverDnHandle_t) { issue(s); });
    } else {
      issue(c->stream);
    }
    c->launches += 1;
    launch(c, k_jacobi_finish, 1, SD_THREADS, 0, int(n), work.p(), V.p(), U, S, VT,
           work.p() + int64_t(n) * n, trans);
    TTG_CHECK_LAUNCH();
    return;
  }
  if (mode != 2) {
    // Grid-wide rounds: one CTA per column pair (up to what fits at once).
    int occ = 0;
    TTG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_jacobi_coop.plain(),
                                                           JC_THREADS, 0));
    const int64_t pairs = (n + 1) / 2;
    const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(pairs,
                                                                  int64_t(c->num_sms) * occ)));
    DBuf<unsigned> bar(c, 2);
    DBuf<unsigned long long> offmax(c, 3);
    memset_async(c, bar.p(), 0, 2 * sizeof(unsigned));
    launch(c, k_jacobi_coop, blocks, JC_THREADS, 0, int(n), A, int(lda), work.p(), V.p(),
           bar.p(), offmax.p(), c->d_err + 0, c->d_err + 3, trans, c->jacobi_max_sweeps);
    launch(c, k_jacobi_finish, 1, SD_THREADS, 0, int(n), work.p(), V.p(), U, S, VT,
           work.p() + int64_t(n) * n, trans);
    TTG_CHECK_LAUNCH();
    return;
  }
  ensure_smem_attr(k_jacobi_svd.fn(), c->device,
                   int(SMEM_LIMIT + 1024));
  const size_t smem = size_t(mode) * mat;
  launch(c, k_jacobi_svd, 1, SD_THREADS, smem, int(n), A, int(lda), U, S, VT, V.p(), work.p(),
         mode, trans, c->d_err + 3, c->jacobi_max_sweeps);
  TTG_CHECK_LAUNCH();
}

namespace {
__global__ void k_selftest_jc_barrier(unsigned* bar, int* flag, long long limit) {
  if (blockIdx.x != 0) return;
  jc_barrier(blockIdx, gridDim, bar, flag, limit);
}
}  // namespace

// Self-test of the bounded barrier of the cooperative Jacobi SVD: block 1
// never arrives; block 0 gives up after `limit` polls and raises *flag.
void selftest_wait_jacobi(Context* c, int* flag, long long limit) {
  DBuf<unsigned> bar(c, 2);
  TTG_CUDA(cudaMemsetAsync(bar.p(), 0, 2 * sizeof(unsigned), c->stream));
  k_selftest_jc_barrier<<<2, 32, 0, c->stream>>>(bar.p(), flag, limit);
  TTG_CHECK_LAUNCH();
  sync(c);
}

}  // namespace ttg
