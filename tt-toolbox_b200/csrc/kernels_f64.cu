// FP64 kernels: DMMA-tiled batched GEMM, deterministic reductions,
// transposes and elementwise helpers.
//
// The GEMM is the contraction engine of the FP64 (parity) path: every local
// matvec (bfun3) and every interface update (compute_next_Phi) is written as
// three batched column-major GEMMs whose operand layouts need no explicit
// permutations (see local_ops.cu).  Tiles: 64x64x16 per CTA, 4 warps of
// 32x32, each warp issuing mma.sync.m8n8k4 f64 (the FP64 tensor path; tcgen05
// has no FP64 kind).  Global->shared staging with cp.async (8-byte granules so
// any leading dimension works), double buffered.
#include "group.cuh"
#include "kernels.h"
#include "dmma.cuh"

namespace ttg {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, PADS = 8;
// Split-K partial values one CTA may sum in the GEMM kernel itself.
constexpr int64_t SPLITK_INKERNEL_MAX = 4096;

struct GemmP {
  int64_t M, N, K;
  const double* A;
  int64_t lda, sA;
  const double* B;
  int64_t ldb, sB;
  double* C;
  int64_t ldc, sC;
  double alpha, beta;
  const int* skip;  // optional: return at once when *skip != 0
  // Split-K: nsplit > 1 slices of kc columns of K per batch item, blockIdx.z =
  // item * nsplit + slice.  Each slice writes its partial tile to `part`
  // ([item][slice] blocks of M x N, ld M).  With `cnt` (one arrival counter
  // per tile and item) the slice that arrives last at its tile adds the
  // partials in slice order (deterministic), applies alpha/beta, writes C and
  // resets the counter; without it k_splitk_reduce does the same afterwards.
  int64_t nsplit, kc;
  double* part;
  unsigned* cnt;
};

template <bool TA, bool TB>
TTG_BODY(k_gemm_f64)(TTG_BLOCK, GemmP p) {
  pdl_begin();
  __shared__ double As[2][BK][BM + PADS];
  __shared__ double Bs[2][BK][BN + PADS];
  if (p.skip && *p.skip) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool split = p.nsplit > 1;
  const int64_t item = split ? blockIdx.z / p.nsplit : blockIdx.z;
  const int64_t slice = split ? blockIdx.z % p.nsplit : 0;
  const int64_t kb0 = slice * p.kc;
  const double* __restrict__ A = p.A + item * p.sA + (TA ? kb0 : kb0 * p.lda);
  const double* __restrict__ B = p.B + item * p.sB + (TB ? kb0 * p.ldb : kb0);
  const int64_t K = split ? min(p.K - kb0, p.kc) : p.K;
  const int64_t m0 = int64_t(blockIdx.x) * BM, n0 = int64_t(blockIdx.y) * BN;
  const int64_t M = p.M, N = p.N;

  auto load_tile = [&](int64_t k0, int buf) {
    if (!TA) {  // m contiguous
      const int m = tid & 63, kb = tid >> 6;
      const int64_t gm = m0 + m;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = kb + 2 * i;
        const int64_t gk = k0 + k;
        const bool ok = gm < M && gk < K;
        cp_async8(&As[buf][k][m], ok ? A + gm + gk * p.lda : A, ok);
      }
    } else {  // k contiguous: A(m,k) = A[k + m*lda]
      const int k = tid & 15, mb = tid >> 4;
      const int64_t gk = k0 + k;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int m = mb + 8 * i;
        const int64_t gm = m0 + m;
        const bool ok = gm < M && gk < K;
        cp_async8(&As[buf][k][m], ok ? A + gk + gm * p.lda : A, ok);
      }
    }
    if (!TB) {  // k contiguous: B(k,n) = B[k + n*ldb]
      const int k = tid & 15, nb = tid >> 4;
      const int64_t gk = k0 + k;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int n = nb + 8 * i;
        const int64_t gn = n0 + n;
        const bool ok = gn < N && gk < K;
        cp_async8(&Bs[buf][k][n], ok ? B + gk + gn * p.ldb : B, ok);
      }
    } else {  // n contiguous: B(k,n) = B[n + k*ldb]
      const int n = tid & 63, kb = tid >> 6;
      const int64_t gn = n0 + n;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = kb + 2 * i;
        const int64_t gk = k0 + k;
        const bool ok = gn < N && gk < K;
        cp_async8(&Bs[buf][k][n], ok ? B + gn + gk * p.ldb : B, ok);
      }
    }
    cp_async_commit();
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  const int64_t ktiles = (K + BK - 1) / BK;
  if (ktiles > 0) load_tile(0, 0);
  for (int64_t kt = 0; kt < ktiles; ++kt) {
    const int buf = int(kt & 1);
    if (kt + 1 < ktiles) {
      load_tile((kt + 1) * BK, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK / 4; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[buf][kk * 4 + t][wm + i * 8 + g];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk * 4 + t][wn + j * 8 + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
  }

  double* __restrict__ C = p.C + item * p.sC;
  if (!split) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t row = m0 + wm + i * 8 + g;
      if (row >= M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int64_t col = n0 + wn + j * 8 + 2 * t + e;
          if (col < N) {
            double* dst = C + row + col * p.ldc;
            double v = p.alpha * acc[i][j][e];
            if (p.beta != 0.0) v += p.beta * *dst;
            *dst = v;
          }
        }
      }
    }
    return;
  }

  // Split-K: publish this slice's partial tile, then the last slice to
  // arrive reduces the tile.
  const int64_t MN = M * N;
  double* Pme = p.part + blockIdx.z * MN;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t row = m0 + wm + i * 8 + g;
    if (row >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t col = n0 + wn + j * 8 + 2 * t + e;
        if (col < N) Pme[row + col * M] = acc[i][j][e];
      }
    }
  }
  if (!p.cnt) return;
  __threadfence();
  __syncthreads();
  __shared__ int s_last;
  if (tid == 0) {
    unsigned* ctr = p.cnt + item * (int64_t(gridDim.x) * gridDim.y) + blockIdx.x +
                    int64_t(gridDim.x) * blockIdx.y;
    const unsigned prev = atomicAdd(ctr, 1u);
    s_last = prev == unsigned(p.nsplit - 1);
    if (s_last) *ctr = 0u;  // every slice has arrived: ready for the next launch
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const double* P0 = p.part + item * p.nsplit * MN;
  for (int e = tid; e < BM * BN; e += 128) {
    const int64_t row = m0 + (e % BM), col = n0 + (e / BM);
    if (row >= M || col >= N) continue;
    const int64_t off = row + col * M;
    double acc2 = 0.0;
    for (int64_t z = 0; z < p.nsplit; ++z) acc2 += __ldcg(P0 + z * MN + off);
    double* dst = C + row + col * p.ldc;
    double v = p.alpha * acc2;
    if (p.beta != 0.0) v += p.beta * *dst;
    *dst = v;
  }
}
template <bool TA, bool TB>
TTG_KERNEL_T(k_gemm_f64, 128, TA, TB);

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------

constexpr int RED_THREADS = 256;
constexpr int RED_MAX_BLOCKS = 1024;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
    r = warp_sum(r);
  }
  return r;  // valid in thread 0
}

// mode 0: sum x*y ; mode 1: sum x^2 ; mode 2: sum (x-y)^2.
// Per-block partial sums; the last block to finish adds the partials in
// block order (deterministic) and writes the result: one launch.  `counter` is a
// device int that is zero between reductions (reset by the last block).
TTG_BODY(k_reduce_fused)(TTG_BLOCK, int64_t n, const double* __restrict__ x,
                               const double* __restrict__ y, int mode, double* __restrict__ part,
                               unsigned* counter, double* out, int do_sqrt) {
  pdl_begin();
  __shared__ double sh[32];
  __shared__ bool last;
  double s = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double a = x[i];
    if (mode == 0)
      s += a * y[i];
    else if (mode == 1)
      s += a * a;
    else {
      const double dlt = a - y[i];
      s += dlt * dlt;
    }
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (int i = threadIdx.x; i < int(gridDim.x); i += blockDim.x)
    t += reinterpret_cast<volatile const double*>(part)[i];
  t = block_sum(t, sh);
  if (threadIdx.x == 0) {
    *out = do_sqrt ? sqrt(t) : t;
    *counter = 0u;
  }
}
TTG_KERNEL(k_reduce_fused, 0);

void reduce_launch(Context* c, int64_t n, const double* x, const double* y, int mode,
                   double* out, bool do_sqrt) {
  int nb = int(std::min<int64_t>((n + RED_THREADS * 4 - 1) / (RED_THREADS * 4), RED_MAX_BLOCKS));
  if (nb < 1) nb = 1;
  DBuf<double> part(c, nb);
  launch(c, k_reduce_fused, nb, RED_THREADS, 0, n, x, y, mode, part.p(),
         reinterpret_cast<unsigned*>(c->d_err + 63), out, do_sqrt ? 1 : 0);
  TTG_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Elementwise
// ---------------------------------------------------------------------------

TTG_BODY(k_count_nonfinite)(TTG_BLOCK, int64_t n, const double* __restrict__ x,
                                  unsigned long long* __restrict__ out) {
  pdl_begin();
  unsigned long long cnt = 0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    cnt += isfinite(x[i]) ? 0ull : 1ull;
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, cnt);
}
TTG_KERNEL(k_count_nonfinite, 0);

TTG_BODY(k_axpby)(TTG_BLOCK, int64_t n, double a, const double* __restrict__ x, double b,
                        double* __restrict__ y) {
  pdl_begin();
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    y[i] = (b == 0.0 ? 0.0 : b * y[i]) + a * x[i];
}
TTG_KERNEL(k_axpby, 0);

TTG_BODY(k_scale_dev)(TTG_BLOCK, int64_t n, const double* __restrict__ x, double* __restrict__ y,
                            const double* num, const double* den) {
  pdl_begin();
  const double s = (num ? *num : 1.0) / (den ? *den : 1.0);
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    y[i] = x[i] * s;
}
TTG_KERNEL(k_scale_dev, 0);

TTG_BODY(k_copy)(TTG_BLOCK, int64_t n, const double* __restrict__ x, double* __restrict__ y) {
  pdl_begin();
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    y[i] = x[i];
}
TTG_KERNEL(k_copy, 0);

TTG_BODY(k_fill)(TTG_BLOCK, int64_t n, double v, double* y) {
  pdl_begin();
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    y[i] = v;
}
TTG_KERNEL(k_fill, 0);

TTG_BODY(k_transpose)(TTG_BLOCK, int64_t rows, int64_t cols, const double* __restrict__ in,
                            int64_t ldi, int64_t si, double* __restrict__ out, int64_t ldo,
                            int64_t so) {
  pdl_begin();
  __shared__ double tile[32][33];
  const int64_t b = blockIdx.z;
  in += b * si;
  out += b * so;
  const int64_t r0 = int64_t(blockIdx.x) * 32, c0 = int64_t(blockIdx.y) * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int64_t r = r0 + threadIdx.x, cc = c0 + j;
    if (r < rows && cc < cols) tile[j][threadIdx.x] = in[r + cc * ldi];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int64_t cc = c0 + threadIdx.x, r = r0 + j;
    if (r < rows && cc < cols) out[cc + r * ldo] = tile[threadIdx.x][j];
  }
}
TTG_KERNEL(k_transpose, 0);

TTG_BODY(k_copy2d)(TTG_BLOCK, int64_t rows, int64_t cols, const double* __restrict__ in, int64_t ldi,
                         double* __restrict__ out, int64_t ldo, const double* scale_col) {
  pdl_begin();
  const int64_t total = rows * cols;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = i % rows, cidx = i / rows;
    double v = in[r + cidx * ldi];
    if (scale_col) v *= scale_col[cidx];
    out[r + cidx * ldo] = v;
  }
}
TTG_KERNEL(k_copy2d, 0);

// splitmix64-based counter hash -> two uniforms -> Box-Muller normal.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

TTG_BODY(k_randn)(TTG_BLOCK, int64_t n, uint64_t seed, uint64_t offset, double* y) {
  pdl_begin();
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t h1 = mix64(seed ^ mix64(2 * (offset + i)));
    const uint64_t h2 = mix64(seed ^ mix64(2 * (offset + i) + 1));
    const double u1 = (double((h1 >> 11) + 1)) * (1.0 / 9007199254740993.0);
    const double u2 = double(h2 >> 11) * (1.0 / 9007199254740992.0);
    y[i] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
}
TTG_KERNEL(k_randn, 0);

TTG_BODY(k_normalize_by)(TTG_BLOCK, int64_t n, double* __restrict__ x, double* nrm) {
  pdl_begin();
  const double v = *nrm;
  const double s = v > 0.0 ? 1.0 / v : 1.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    x[i] *= s;
  // Every block has read *nrm above; a zero norm is reported as 1.
  if (blockIdx.x == 0 && threadIdx.x == 0 && !(v > 0.0)) *nrm = 1.0;
}
TTG_KERNEL(k_normalize_by, 0);

TTG_BODY(k_axpby_dev)(TTG_BLOCK, int64_t n, double a, const double* __restrict__ x,
                            const double* __restrict__ b, double* __restrict__ y) {
  pdl_begin();
  const double bv = *b;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    y[i] = bv * y[i] + a * x[i];
}
TTG_KERNEL(k_axpby_dev, 0);

TTG_BODY(k_scalar_op)(TTG_BLOCK, int op, double* out, const double* p0, const double* p1,
                            const double* p2, double k) {
  pdl_begin();
  switch (op) {
    case 0: *out = *p0 / *p1; break;
    case 1: *out = fmax(*out, *p0); break;
    case 2: *out = *out / (*p0 / (*p1 * *p2)); break;
    case 3: *out = *out * (*p0 / (*p1 * *p2)); break;
    case 4: *out = *out * *p0; break;
    case 5: *out = fmax(*p0, k); break;
    case 6: *out = (*p1 > 0.0) ? *p0 / *p1 : 0.0; break;
    case 7: *out = (*p0 == 0.0) ? 1.0 : *p0; break;
    default: break;
  }
}
TTG_KERNEL(k_scalar_op, 0);

TTG_BODY(k_first_exceeding)(TTG_BLOCK, int64_t nb, const double* cand, const double* den,
                                  const double* thr, double* out) {
  pdl_begin();
  double r = -1.0;
  for (int64_t b = 0; b < nb; ++b) {
    if (cand[b] / *den > *thr) {
      r = double(b);
      break;
    }
  }
  *out = r;
}
TTG_KERNEL(k_first_exceeding, 0);

// C_b = alpha * sum_z part[b][z] + beta * C_b over the split-K slices, in
// slice order (deterministic).  part: batch x s blocks of M x N (ld M).
TTG_BODY(k_splitk_reduce)(TTG_BLOCK, int64_t M, int64_t N, int64_t s, int64_t batch,
                                const double* __restrict__ part, double alpha, double beta,
                                double* __restrict__ C, int64_t ldc, int64_t sC,
                                const int* skip) {
  pdl_begin();
  if (skip && *skip) return;
  const int64_t MN = M * N;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < MN * batch;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e / MN, r = e % MN;
    const double* src = part + b * s * MN + r;
    double acc = 0.0;
    for (int64_t z = 0; z < s; ++z) acc += src[z * MN];
    const int64_t m = r % M, n = r / M;
    double* dst = C + b * sC + m + n * ldc;
    double v = alpha * acc;
    if (beta != 0.0) v += beta * *dst;
    *dst = v;
  }
}
TTG_KERNEL(k_splitk_reduce, 0);

// *keep = 1 when every column j kept G1[j,j] > tau^2 G0[j,j] (one thread).
TTG_BODY(k_collapse_flag)(TTG_BLOCK, int64_t k, const double* G0, int64_t ld0, const double* G1,
                                int64_t ld1, double tau, int* keep) {
  pdl_begin();
  int ok = 1;
  for (int64_t j = 0; j < k; ++j)
    if (!(G1[j + j * ld1] > tau * tau * G0[j + j * ld0])) ok = 0;
  *keep = ok;
}
TTG_KERNEL(k_collapse_flag, 0);

// *flag |= 1 when max |G - I| > tol (G: n x n Gram matrix of a basis).
TTG_BODY(k_orth_check)(TTG_BLOCK, int64_t n, const double* G, double tol, int* flag) {
  pdl_begin();
  int bad = 0;
  for (int64_t e = threadIdx.x; e < n * n; e += blockDim.x) {
    const double v = G[e] - ((e % n) == (e / n) ? 1.0 : 0.0);
    if (!(fabs(v) <= tol)) bad = 1;
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}
TTG_KERNEL(k_orth_check, 0);

TTG_BODY(k_accumulate_info)(TTG_BLOCK, const int* info, int* err_slot) {
  pdl_begin();
  if (*info != 0) atomicOr(err_slot, 1);
}
TTG_KERNEL(k_accumulate_info, 0);

int grid_for(Context* c, int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  int64_t cap = int64_t(c->num_sms) * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return int(b);
}

}  // namespace

void gemm_f64(Context* c, bool tA, bool tB, int64_t M, int64_t N, int64_t K, double alpha,
              const double* A, int64_t lda, int64_t sA, const double* B, int64_t ldb, int64_t sB,
              double beta, double* C, int64_t ldc, int64_t sC, int64_t batch) {
  if (M <= 0 || N <= 0 || batch <= 0) return;
  if (K <= 0) {
    // C = beta*C
    for (int64_t b = 0; b < batch; ++b) {
      if (beta == 0.0) {
        for (int64_t j = 0; j < N; ++j) fill_f64(c, M, 0.0, C + b * sC + j * ldc);
      } else if (beta != 1.0) {
        for (int64_t j = 0; j < N; ++j) axpby_f64(c, M, 0.0, C + b * sC + j * ldc, beta, C + b * sC + j * ldc);
      }
    }
    return;
  }
  TTG_REQUIRE(batch <= 65535, "gemm batch %lld too large", (long long)batch);
  const int64_t gx = (M + BM - 1) / BM, gy = (N + BN - 1) / BN;
  TTG_REQUIRE(gy <= 65535 && gx <= 0x7fffffff, "gemm too large");
  GemmP p{M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, alpha, beta, c->skip, 1, 0, nullptr,
          nullptr};
  dim3 grid{unsigned(gx), unsigned(gy), unsigned(batch)};
  // Split-K when the output tiles (times the batch) cannot fill the SMs and
  // K is long: one CTA's FP64 DMMA rate is a small share of the device's, so
  // a few long-K CTAs (inner products of tall matrices: interface updates,
  // Gram matrices, projections) would run for about K x 30 ns each.  K is cut
  // into slices of at least 4 k-tiles so that about two CTAs per SM run.  The
  // slices of a tile are summed in slice order: by the last slice to finish
  // when the partials are few (no second launch), else by a reduction kernel
  // spread over the device (one CTA reading many partials is latency-bound).
  DBuf<double> part;
  const int64_t ctas = gx * gy * batch;
  const int64_t ktiles = (K + BK - 1) / BK;
  // (A context without an allocator -- the caller-scratch entry point -- runs
  // every product unsplit.)
  if (c->alloc && c->d_tile_cnt && ctas < c->num_sms && ktiles >= 8 &&
      ctas <= GEMM_TILE_COUNTERS) {
    int64_t s = std::min<int64_t>((2 * c->num_sms + ctas - 1) / ctas, ktiles / 4);
    if (s * batch > 65535) s = 65535 / batch;
    if (s >= 2) {
      const int64_t kc = (ktiles + s - 1) / s * BK;
      s = (K + kc - 1) / kc;
      if (s >= 2) {
        part.reset(c, batch * s * M * N);
        p.nsplit = s;
        p.kc = kc;
        p.part = part.p();
        const int64_t tile_elems = std::min<int64_t>(M, BM) * std::min<int64_t>(N, BN);
        if (s * tile_elems <= SPLITK_INKERNEL_MAX) p.cnt = c->d_tile_cnt;
        grid.z = unsigned(batch * s);
      }
    }
  }
  if (!tA && !tB)
    launch(c, k_gemm_f64<false, false>, grid, 128, 0, p);
  else if (!tA && tB)
    launch(c, k_gemm_f64<false, true>, grid, 128, 0, p);
  else if (tA && !tB)
    launch(c, k_gemm_f64<true, false>, grid, 128, 0, p);
  else
    launch(c, k_gemm_f64<true, true>, grid, 128, 0, p);
  TTG_CHECK_LAUNCH();
  if (p.nsplit > 1 && !p.cnt) {
    launch(c, k_splitk_reduce, grid_for(c, M * N * batch), 256, 0, M, N, p.nsplit, batch,
           part.p(), alpha, beta, C, ldc, sC, c->skip);
    TTG_CHECK_LAUNCH();
  }
}

void dot_f64(Context* c, int64_t n, const double* x, const double* y, double* out, bool do_sqrt) {
  reduce_launch(c, n, x, y, y ? 0 : 1, out, do_sqrt);
}

void diffnrm_f64(Context* c, int64_t n, const double* x, const double* y, double* out,
                 bool do_sqrt) {
  reduce_launch(c, n, x, y, 2, out, do_sqrt);
}

double nrm2_host(Context* c, int64_t n, const double* x) {
  DBuf<double> s(c, 1);
  dot_f64(c, n, x, nullptr, s.p(), true);
  double h = 0.0;
  read_scalars(c, s.p(), &h, 1);
  return h;
}

int64_t count_nonfinite_f64(Context* c, int64_t n, const double* x) {
  if (n <= 0) return 0;
  DBuf<unsigned long long> cnt(c, 1);
  memset_async(c, cnt.p(), 0, sizeof(unsigned long long));
  launch(c, k_count_nonfinite, grid_for(c, n), 256, 0, n, x, cnt.p());
  TTG_CHECK_LAUNCH();
  unsigned long long h = 0;
  read_device(c, &h, cnt.p(), sizeof(h));
  return int64_t(h);
}

void require_finite(const ttg_tt_s* t, const char* name) {
  if (!t) return;
  require_finite(t->ctx, {{t, name}});
}

void require_finite(Context* c, std::initializer_list<std::pair<const ttg_tt_s*, const char*>> ts) {
  const int64_t k = int64_t(ts.size());
  DBuf<unsigned long long> cnt(c, k);
  memset_async(c, cnt.p(), 0, sizeof(unsigned long long) * k);
  int64_t j = 0;
  for (const auto& t : ts) {
    if (t.first && t.first->numel > 0)
      launch(c, k_count_nonfinite, grid_for(c, t.first->numel), 256, 0, t.first->numel,
             t.first->core, cnt.p() + j);
    ++j;
  }
  TTG_CHECK_LAUNCH();
  unsigned long long h[16] = {};
  TTG_REQUIRE(k <= 16, "require_finite: too many tensors");
  read_device(c, h, cnt.p(), sizeof(unsigned long long) * k);  // one read for all
  j = 0;
  for (const auto& t : ts) {
    TTG_REQUIRE(h[j] == 0, "%s holds %lld non-finite entries (NaN or Inf)", t.second,
                (long long)h[j]);
    ++j;
  }
}

void axpby_f64(Context* c, int64_t n, double a, const double* x, double b, double* y) {
  if (n <= 0) return;
  launch(c, k_axpby, grid_for(c, n), 256, 0, n, a, x, b, y);
  TTG_CHECK_LAUNCH();
}

void scale_dev_f64(Context* c, int64_t n, const double* x, double* y, const double* num,
                   const double* den) {
  if (n <= 0) return;
  launch(c, k_scale_dev, grid_for(c, n), 256, 0, n, x, y, num, den);
  TTG_CHECK_LAUNCH();
}

void fill_f64(Context* c, int64_t n, double v, double* y) {
  if (n <= 0) return;
  launch(c, k_fill, grid_for(c, n), 256, 0, n, v, y);
  TTG_CHECK_LAUNCH();
}

void copy_f64(Context* c, int64_t n, const double* x, double* y) {
  if (n <= 0 || x == y) return;
  // a kernel rather than a memcpy node, so that it chains with its
  // neighbours as a programmatic dependent launch
  launch(c, k_copy, grid_for(c, n), 256, 0, n, x, y);
  TTG_CHECK_LAUNCH();
}

void transpose_f64(Context* c, int64_t rows, int64_t cols, const double* in, int64_t ldi,
                   double* out, int64_t ldo, int64_t batch, int64_t si, int64_t so) {
  if (rows <= 0 || cols <= 0 || batch <= 0) return;
  TTG_REQUIRE((cols + 31) / 32 <= 65535 && batch <= 65535, "transpose too large");
  dim3 grid{unsigned((rows + 31) / 32), unsigned((cols + 31) / 32), unsigned(batch)};
  launch(c, k_transpose, grid, dim3(32, 8), 0, rows, cols, in, ldi, si, out, ldo, so);
  TTG_CHECK_LAUNCH();
}

void copy2d_f64(Context* c, int64_t rows, int64_t cols, const double* in, int64_t ldi,
                double* out, int64_t ldo, const double* scale_col) {
  if (rows <= 0 || cols <= 0) return;
  launch(c, k_copy2d, grid_for(c, rows * cols), 256, 0, rows, cols, in, ldi, out, ldo,
         scale_col);
  TTG_CHECK_LAUNCH();
}

void normalize_by_dev(Context* c, int64_t n, double* x, double* nrm) {
  if (n <= 0) return;
  launch(c, k_normalize_by, grid_for(c, n), 256, 0, n, x, nrm);
  TTG_CHECK_LAUNCH();
}

void axpby_dev(Context* c, int64_t n, double a, const double* x, const double* b, double* y) {
  if (n <= 0) return;
  launch(c, k_axpby_dev, grid_for(c, n), 256, 0, n, a, x, b, y);
  TTG_CHECK_LAUNCH();
}

void scalar_op(Context* c, int op, double* out, const double* p0, const double* p1,
               const double* p2, double k) {
  launch(c, k_scalar_op, 1, 1, 0, op, out, p0, p1, p2, k);
  TTG_CHECK_LAUNCH();
}

void first_exceeding(Context* c, int64_t nb, const double* cand, const double* den,
                     const double* thr, double* out) {
  launch(c, k_first_exceeding, 1, 1, 0, nb, cand, den, thr, out);
  TTG_CHECK_LAUNCH();
}

void collapse_flag(Context* c, int64_t k, const double* G0, int64_t ld0, const double* G1,
                   int64_t ld1, double tau, int* keep) {
  launch(c, k_collapse_flag, 1, 1, 0, k, G0, ld0, G1, ld1, tau, keep);
  TTG_CHECK_LAUNCH();
}

void orth_check(Context* c, int64_t n, const double* G, double tol, int* flag) {
  launch(c, k_orth_check, 1, 256, 0, n, G, tol, flag);
  TTG_CHECK_LAUNCH();
}

void accumulate_info(Context* c, const int* info, int* err_slot) {
  launch(c, k_accumulate_info, 1, 1, 0, info, err_slot);
  TTG_CHECK_LAUNCH();
}

void randn_f64(Context* c, int64_t n, uint64_t seed, uint64_t offset, double* y) {
  if (n <= 0) return;
  launch(c, k_randn, grid_for(c, n), 256, 0, n, seed, offset, y);
  TTG_CHECK_LAUNCH();
}

}  // namespace ttg
