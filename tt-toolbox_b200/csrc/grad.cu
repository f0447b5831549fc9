// Gradients of three TT functionals with respect to every core (FP64).
//
// TT-Toolbox has no derivative code.  The forward maps are its own:
//   <x, A x>  : @tt_matrix/mtimes.m:38-65 (A x) and @tt_tensor/dot.m:92-111
//   <x, b>    : @tt_tensor/dot.m:92-111 (left-to-right interface sweep)
//   X[idx_s]  : @tt_tensor/subsref.m:93-123 (an entry is the product of the
//               core slices x_k(:, i_k, :))
// A TT functional is multilinear in the cores, so the gradient with respect
// to core k is the functional with core k removed: the interfaces left and
// right of k contracted with everything that touched core k.
//
// <x, A x>: the interfaces are those of AMEn's local system (compute_next_Phi,
//   solve/amen_solve2.m:834-920, without its normalisation).  With the left
//   interface L_k [bra, ket, ra] and the right interface R_k [ket, ra, bra],
//   the derivative through the bra copy of x_k is the local matvec bfun3
//   (solve/amen_solve2.m:924-951) L_k x A_k x R_{k+1} applied to x_k, and the
//   derivative through the ket copy is the same with bra and ket exchanged
//   (transposed interfaces and A_k^T).  Both run on the DMMA GEMMs of the
//   local matvec.
// <x, b>:   two interface sweeps Psi_L [rx, rb], Psi_R [rx, rb]; three GEMMs
//   per core.
// sum_s (X[idx_s] - y_s)^2: per sample s, the row vector l_k(s) = product of
//   the slices left of k and the column vector rho_k(s) = 2 e_s times the
//   product of the slices right of k, e_s = X[idx_s] - y_s.  The gradient of
//   core k at slice j is sum over samples with i_k = j of l_k(s)^T rho_k(s)^T.
//   Samples are bucketed by i_k (stable counting sort, deterministic), and
//   every product becomes a gathered GEMM on the FP64 tensor cores: the CTA
//   owns 64 samples of one bucket, stages their vectors (gathered rows) and
//   the bucket's slice in shared memory and multiplies with mma.m8n8k4.  The
//   gradient is a split-K GEMM per bucket (512 samples per CTA) whose
//   partials are summed in a fixed order, so results are bitwise repeatable.
#include "grad.h"
#include "dmma.cuh"
#include "kernels.h"
#include "local_ops.h"

namespace ttg {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, PADS = 8;
constexpr int PT = 64;           // samples per propagation tile
constexpr int GT = 512;          // samples per gradient (split-K) tile
constexpr int SORT_CHUNK = 1024; // samples per sorting warp
constexpr int64_t MAX_BUCKETS = 8192;

int blocks_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  return int(b < 1 ? 1 : (b > 65535 * 16 ? 65535 * 16 : b));
}

// ---------------------------------------------------------------------------
// 4-D permutation: out[sum_a i_a * ostride_a] = in[i0 + d0*(i1 + d1*(i2 + d2*i3))]
// ---------------------------------------------------------------------------
struct Perm4 {
  int64_t d0, d1, d2, d3;
  int64_t o0, o1, o2, o3;
};

__global__ void k_permute4(Perm4 p, const double* __restrict__ in, double* __restrict__ out) {
  const int64_t total = p.d0 * p.d1 * p.d2 * p.d3;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
       t += int64_t(gridDim.x) * blockDim.x) {
    int64_t r = t;
    const int64_t i0 = r % p.d0;
    r /= p.d0;
    const int64_t i1 = r % p.d1;
    r /= p.d1;
    const int64_t i2 = r % p.d2;
    const int64_t i3 = r / p.d2;
    out[i0 * p.o0 + i1 * p.o1 + i2 * p.o2 + i3 * p.o3] = in[t];
  }
}

void permute4(Context* c, const Perm4& p, const double* in, double* out) {
  const int64_t total = p.d0 * p.d1 * p.d2 * p.d3;
  if (total <= 0) return;
  k_permute4<<<blocks_for(total), 256, 0, c->stream>>>(p, in, out);
  c->launches += 1;
  TTG_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Sample bucketing (stable counting sort of one index column)
// ---------------------------------------------------------------------------

// err |= 1 when some idx[s + k*S] is outside [0, n_k).
__global__ void k_check_idx(int64_t S, int d, const int* __restrict__ idx,
                            const int64_t* __restrict__ nk, int* err) {
  const int64_t total = S * d;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
       t += int64_t(gridDim.x) * blockDim.x) {
    const int v = idx[t];
    if (v < 0 || v >= nk[t / S]) atomicOr(err, 1);
  }
}

__device__ __forceinline__ int clamp_bucket(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

// counts[j * nblk + b] = #samples of chunk b with idx = j.  One warp per chunk.
__global__ void k_bucket_count(int64_t S, const int* __restrict__ col, int n, int nblk,
                               int* __restrict__ counts) {
  extern __shared__ int sh_cnt[];
  for (int j = threadIdx.x; j < n; j += 32) sh_cnt[j] = 0;
  __syncwarp();
  const int64_t s0 = int64_t(blockIdx.x) * SORT_CHUNK;
  const int64_t s1 = min(S, s0 + SORT_CHUNK);
  for (int64_t s = s0 + threadIdx.x; s < s1; s += 32) atomicAdd(&sh_cnt[clamp_bucket(col[s], n)], 1);
  __syncwarp();
  for (int j = threadIdx.x; j < n; j += 32) counts[int64_t(j) * nblk + blockIdx.x] = sh_cnt[j];
}

// Exclusive scan of counts[j * nblk + (0..nblk-1)] in place; total[j].
__global__ void k_bucket_scan(int nblk, int* __restrict__ counts, int* __restrict__ total) {
  __shared__ int sh[256];
  __shared__ int carry;
  int* row = counts + int64_t(blockIdx.x) * nblk;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nblk; base += 256) {
    const int i = base + threadIdx.x;
    const int v = i < nblk ? row[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {  // Hillis-Steele inclusive scan
      const int add = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < nblk) row[i] = carry + sh[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 255) carry += sh[255];
    __syncthreads();
  }
  if (threadIdx.x == 0) total[blockIdx.x] = carry;
}

// Bucket starts and the tile tables of both tilings (one thread; n is small).
//   meta[0 .. n]            bucket start (meta[n] = S)
//   meta[n+1 .. 2n+1]       first propagation tile of each bucket (+ total)
//   meta[2n+2 .. 3n+2]      first gradient tile of each bucket (+ total)
__global__ void k_bucket_base(int n, const int* __restrict__ total, int* __restrict__ meta) {
  int s = 0, tp = 0, tg = 0;
  for (int j = 0; j < n; ++j) {
    meta[j] = s;
    meta[n + 1 + j] = tp;
    meta[2 * n + 2 + j] = tg;
    const int cnt = total[j];
    s += cnt;
    tp += (cnt + PT - 1) / PT;
    tg += (cnt + GT - 1) / GT;
  }
  meta[n] = s;
  meta[2 * n + 1] = tp;
  meta[3 * n + 2] = tg;
}

// perm[bucket_start[j] + offs[j*nblk+b] + rank] = s, stable within buckets.
__global__ void k_bucket_scatter(int64_t S, const int* __restrict__ col, int n, int nblk,
                                 const int* __restrict__ offs, const int* __restrict__ meta,
                                 int* __restrict__ perm) {
  extern __shared__ int sh_cnt[];
  for (int j = threadIdx.x; j < n; j += 32) sh_cnt[j] = 0;
  __syncwarp();
  const int lane = threadIdx.x;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t s0 = int64_t(blockIdx.x) * SORT_CHUNK;
  const int64_t s1 = min(S, s0 + SORT_CHUNK);
  for (int64_t sb = s0; sb < s1; sb += 32) {
    const int64_t s = sb + lane;
    const bool valid = s < s1;
    const int v = valid ? clamp_bucket(col[s], n) : n + lane;  // invalid lanes: own groups
    const unsigned same = __match_any_sync(0xffffffffu, v);
    const int rank = __popc(same & lt);
    const int before = valid ? sh_cnt[v] : 0;
    __syncwarp();
    if (valid) {
      perm[int64_t(meta[v]) + offs[int64_t(v) * nblk + blockIdx.x] + before + rank] = int(s);
      if (rank == 0) sh_cnt[v] = before + __popc(same);
    }
    __syncwarp();
  }
}

// Bucket j of tile t: the largest j with start[j] <= t (start has n+1 entries).
__device__ __forceinline__ int find_bucket(const int* __restrict__ start, int n, int t) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= t)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// Gathered propagation GEMM
//   forward  (BWD=false): vout[s, c] = sum_a vin[s, a] * x_k[a, j, c]
//   backward (BWD=true):  vout[s, a] = sum_c x_k[a, j, c] * vin[s, c]
// for every sample s of bucket j (i_k(s) = j).  Sample vectors are rows:
// v[s * ld + a].  CTA = 64 samples x 64 outputs, K in steps of 16.
// ---------------------------------------------------------------------------
struct PropP {
  const double* vin;
  int64_t ldi;
  double* vout;
  int64_t ldo;
  const double* core;
  int64_t r1, n, r2;
  int64_t K, N;
  const int* perm;
  const int* meta;  // bucket table (k_bucket_base layout)
};

template <bool BWD>
__global__ void __launch_bounds__(128) k_prop(PropP p) {
  __shared__ double As[2][BK][BM + PADS];
  __shared__ double Bs[2][BK][BN + PADS];
  __shared__ int64_t rowoff[BM];
  const int nb = int(p.n);
  const int* bstart = p.meta;
  const int* tstart = p.meta + nb + 1;
  const int t = blockIdx.x;
  if (t >= tstart[nb]) return;
  const int j = find_bucket(tstart, nb, t);
  const int64_t s0 = int64_t(bstart[j]) + int64_t(t - tstart[j]) * PT;
  const int64_t cnt = min(int64_t(PT), int64_t(bstart[j + 1]) - s0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < BM) rowoff[tid] = tid < cnt ? int64_t(p.perm[s0 + tid]) : -1;
  __syncthreads();
  const double* __restrict__ W = p.core + p.r1 * j;
  const int64_t ldw = p.r1 * p.n;
  const int64_t n0 = int64_t(blockIdx.y) * BN;
  const int64_t K = p.K, N = p.N;

  auto load_tile = [&](int64_t k0, int buf) {
    {  // A(m, k) = vin[rowoff[m] * ldi + k]   (k contiguous)
      const int k = tid & 15, mb = tid >> 4;
      const int64_t gk = k0 + k;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int m = mb + 8 * i;
        const int64_t ro = rowoff[m];
        const bool ok = ro >= 0 && gk < K;
        cp_async8(&As[buf][k][m], ok ? p.vin + ro * p.ldi + gk : p.vin, ok);
      }
    }
    if (!BWD) {  // B(k=a, n=c) = W[a + c*ldw]   (k contiguous)
      const int k = tid & 15, nb2 = tid >> 4;
      const int64_t gk = k0 + k;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int nn = nb2 + 8 * i;
        const int64_t gn = n0 + nn;
        const bool ok = gn < N && gk < K;
        cp_async8(&Bs[buf][k][nn], ok ? W + gk + gn * ldw : W, ok);
      }
    } else {  // B(k=c, n=a) = W[a + c*ldw]   (n contiguous)
      const int nn = tid & 63, kb = tid >> 6;
      const int64_t gn = n0 + nn;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = kb + 2 * i;
        const int64_t gk = k0 + k;
        const bool ok = gn < N && gk < K;
        cp_async8(&Bs[buf][k][nn], ok ? W + gn + gk * ldw : W, ok);
      }
    }
    cp_async_commit();
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) acc[i][jj][0] = acc[i][jj][1] = 0.0;

  const int g = lane >> 2, tq = lane & 3;
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
      for (int i = 0; i < 4; ++i) a[i] = As[buf][kk * 4 + tq][wm + i * 8 + g];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) b[jj] = Bs[buf][kk * 4 + tq][wn + jj * 8 + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) dmma(acc[i][jj][0], acc[i][jj][1], a[i], b[jj]);
    }
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = wm + i * 8 + g;
    const int64_t ro = rowoff[m];
    if (ro < 0) continue;
    double* dst = p.vout + ro * p.ldo;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t col = n0 + wn + jj * 8 + 2 * tq + e;
        if (col < N) dst[col] = acc[i][jj][e];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Gradient partials: part[t][a + r1*c] = sum over the <= 512 samples s of
// gradient tile t of L[s, a] * P[s, c]   (M = r1, N = r2, K = samples)
// ---------------------------------------------------------------------------
struct GradP {
  const double* L;
  int64_t ldl;
  const double* P;
  int64_t ldp;
  double* part;
  int64_t r1, n, r2;
  const int* perm;
  const int* meta;
};

__global__ void __launch_bounds__(128) k_grad_tiles(GradP p) {
  __shared__ double As[2][BK][BM + PADS];
  __shared__ double Bs[2][BK][BN + PADS];
  __shared__ int64_t rowoff[GT];
  const int nb = int(p.n);
  const int* bstart = p.meta;
  const int* gstart = p.meta + 2 * nb + 2;
  const int t = blockIdx.x;
  if (t >= gstart[nb]) return;
  const int j = find_bucket(gstart, nb, t);
  const int64_t s0 = int64_t(bstart[j]) + int64_t(t - gstart[j]) * GT;
  const int64_t cnt = min(int64_t(GT), int64_t(bstart[j + 1]) - s0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < GT; i += 128) rowoff[i] = i < cnt ? int64_t(p.perm[s0 + i]) : -1;
  __syncthreads();
  const int64_t m0 = int64_t(blockIdx.y) * BM, n0 = int64_t(blockIdx.z) * BN;
  const int64_t M = p.r1, N = p.r2, K = cnt;

  auto load_tile = [&](int64_t k0, int buf) {
    const int x = tid & 63, kb = tid >> 6;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = kb + 2 * i;
      const int64_t gk = k0 + k;
      const int64_t ro = gk < K ? rowoff[gk] : -1;
      const int64_t gm = m0 + x, gn = n0 + x;
      const bool oka = ro >= 0 && gm < M;
      const bool okb = ro >= 0 && gn < N;
      cp_async8(&As[buf][k][x], oka ? p.L + ro * p.ldl + gm : p.L, oka);
      cp_async8(&Bs[buf][k][x], okb ? p.P + ro * p.ldp + gn : p.P, okb);
    }
    cp_async_commit();
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) acc[i][jj][0] = acc[i][jj][1] = 0.0;

  const int g = lane >> 2, tq = lane & 3;
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
      for (int i = 0; i < 4; ++i) a[i] = As[buf][kk * 4 + tq][wm + i * 8 + g];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) b[jj] = Bs[buf][kk * 4 + tq][wn + jj * 8 + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) dmma(acc[i][jj][0], acc[i][jj][1], a[i], b[jj]);
    }
    __syncthreads();
  }

  double* dst = p.part + int64_t(t) * (p.r1 * p.r2);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t row = m0 + wm + i * 8 + g;
    if (row >= M) continue;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t col = n0 + wn + jj * 8 + 2 * tq + e;
        if (col < N) dst[row + col * M] = acc[i][jj][e];
      }
    }
  }
}

// grad[a + r1*j + r1*n*c] = sum_{t in gradient tiles of bucket j} part[t][a + r1*c]
// (fixed order; empty buckets give zero slices).
__global__ void k_grad_reduce(int64_t r1, int64_t n, int64_t r2, const double* __restrict__ part,
                              const int* __restrict__ meta, double* __restrict__ grad) {
  const int64_t total = r1 * r2 * n;
  const int* gstart = meta + 2 * n + 2;
  const int64_t R = r1 * r2;
  for (int64_t id = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; id < total;
       id += int64_t(gridDim.x) * blockDim.x) {
    const int64_t ac = id % R;
    const int64_t j = id / R;
    const int64_t a = ac % r1, c = ac / r1;
    double s = 0.0;
    for (int t = gstart[j]; t < gstart[j + 1]; ++t) s += part[int64_t(t) * R + ac];
    grad[a + r1 * j + r1 * n * c] = s;
  }
}

// e = v - y; rho = 2 e.
__global__ void k_sample_residual(int64_t S, const double* __restrict__ v,
                                  const double* __restrict__ y, double* __restrict__ e,
                                  double* __restrict__ rho) {
  for (int64_t s = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; s < S;
       s += int64_t(gridDim.x) * blockDim.x) {
    const double r = v[s] - y[s];
    e[s] = r;
    rho[s] = 2.0 * r;
  }
}

void check_tt_vector(const ttg_tt_s* x, const char* what) {
  TTG_REQUIRE(x && !x->is_matrix, "%s must be a TT tensor", what);
  TTG_REQUIRE(x->r[0] == 1 && x->r[x->d] == 1, "%s: boundary ranks must be 1", what);
}

}  // namespace

// ---------------------------------------------------------------------------
// <x, A x>
// ---------------------------------------------------------------------------
void grad_xAx(Context* c, const ttg_tt_s* x, const ttg_tt_s* A, double* grad, double* value) {
  check_tt_vector(x, "x");
  TTG_REQUIRE(A && A->is_matrix, "A must be a TT matrix");
  const int64_t d = x->d;
  TTG_REQUIRE(A->d == d, "A has %lld cores, x has %lld", (long long)A->d, (long long)d);
  TTG_REQUIRE(A->r[0] == 1 && A->r[d] == 1, "A: boundary ranks must be 1");
  for (int64_t k = 0; k < d; ++k)
    TTG_REQUIRE(A->n[k] == x->n[k] && A->m[k] == x->n[k],
                "core %lld: A is %lldx%lld, x has mode size %lld", (long long)k,
                (long long)A->n[k], (long long)A->m[k], (long long)x->n[k]);
  const auto& r = x->r;
  const auto& ra = A->r;
  // Interfaces: L[k] [r_k, r_k, ra_k] (k = 0..d), R[k] [r_k, ra_k, r_k].
  std::vector<int64_t> off(d + 2, 0);
  for (int64_t k = 0; k <= d; ++k) off[k + 1] = off[k] + r[k] * r[k] * ra[k];
  DBuf<double> L(c, off[d + 1]), R(c, off[d + 1]);
  fill_f64(c, 1, 1.0, L.p());
  fill_f64(c, 1, 1.0, R.p() + off[d]);
  for (int64_t k = 0; k < d; ++k) {
    const double* xk = x->core + x->ps[k];
    next_phi_f64(c, 0, r[k], x->n[k], r[k + 1], r[k], r[k + 1], ra[k], ra[k + 1], L.p() + off[k],
                 xk, A->core + A->ps[k], xk, L.p() + off[k + 1]);
  }
  for (int64_t k = d - 1; k >= 0; --k) {
    const double* xk = x->core + x->ps[k];
    next_phi_f64(c, 1, r[k], x->n[k], r[k + 1], r[k], r[k + 1], ra[k], ra[k + 1],
                 R.p() + off[k + 1], xk, A->core + A->ps[k], xk, R.p() + off[k]);
  }
  if (value) copy_f64(c, 1, L.p() + off[d], value);
  // Scratch for the two local matvecs of the largest core.
  int64_t t1 = 0, t2 = 0, nx = 0, nphi = 0, na = 0;
  for (int64_t k = 0; k < d; ++k) {
    MvDims dm{r[k], r[k], ra[k], x->n[k], x->n[k], r[k + 1], ra[k + 1], r[k + 1]};
    t1 = std::max(t1, dm.t1_size());
    t2 = std::max(t2, dm.t2_size());
    nx = std::max(nx, dm.out_size());
    nphi = std::max(nphi, std::max(r[k] * r[k] * ra[k], r[k + 1] * r[k + 1] * ra[k + 1]));
    na = std::max(na, ra[k] * x->n[k] * x->n[k] * ra[k + 1]);
  }
  DBuf<double> T1(c, t1), T2(c, t2), G2(c, nx), Ls(c, nphi), Rs(c, nphi), At(c, na);
  for (int64_t k = 0; k < d; ++k) {
    const int64_t r1 = r[k], r2 = r[k + 1], a1 = ra[k], a2 = ra[k + 1], n = x->n[k];
    MvDims dm{r1, r1, a1, n, n, r2, a2, r2};
    const double* xk = x->core + x->ps[k];
    const double* Ak = A->core + A->ps[k];
    double* gk = grad + x->ps[k];
    // through the bra copy: (L_k x A_k x R_{k+1}) x_k
    local_matvec_f64(c, dm, L.p() + off[k], Ak, R.p() + off[k + 1], xk, gk, T1.p(), T2.p());
    // through the ket copy: bra and ket exchanged
    permute4(c, Perm4{r1, r1, a1, 1, r1, 1, r1 * r1, 0}, L.p() + off[k], Ls.p());
    permute4(c, Perm4{r2, a2, r2, 1, r2 * a2, r2, 1, 0}, R.p() + off[k + 1], Rs.p());
    permute4(c, Perm4{a1, n, n, a2, 1, a1 * n, a1, a1 * n * n}, Ak, At.p());
    local_matvec_f64(c, dm, Ls.p(), At.p(), Rs.p(), xk, G2.p(), T1.p(), T2.p());
    axpby_f64(c, dm.out_size(), 1.0, G2.p(), 1.0, gk);
  }
}

// ---------------------------------------------------------------------------
// <x, b>
// ---------------------------------------------------------------------------
void grad_xb(Context* c, const ttg_tt_s* x, const ttg_tt_s* b, double* grad, double* value) {
  check_tt_vector(x, "x");
  check_tt_vector(b, "b");
  const int64_t d = x->d;
  TTG_REQUIRE(b->d == d, "b has %lld cores, x has %lld", (long long)b->d, (long long)d);
  for (int64_t k = 0; k < d; ++k)
    TTG_REQUIRE(b->n[k] == x->n[k], "core %lld: mode sizes differ (%lld vs %lld)", (long long)k,
                (long long)b->n[k], (long long)x->n[k]);
  const auto& r = x->r;
  const auto& rb = b->r;
  std::vector<int64_t> poff(d + 2, 0), toff(d + 1, 0);
  for (int64_t k = 0; k <= d; ++k) poff[k + 1] = poff[k] + r[k] * rb[k];
  for (int64_t k = 0; k < d; ++k) toff[k + 1] = toff[k] + r[k] * x->n[k] * rb[k + 1];
  DBuf<double> PL(c, poff[d + 1]), PR(c, poff[d + 1]), T(c, toff[d]);
  int64_t umax = 1;
  for (int64_t k = 0; k < d; ++k) umax = std::max(umax, rb[k] * x->n[k] * r[k + 1]);
  DBuf<double> U(c, umax);
  fill_f64(c, 1, 1.0, PL.p());
  fill_f64(c, 1, 1.0, PR.p() + poff[d]);
  for (int64_t k = 0; k < d; ++k) {
    const int64_t r1 = r[k], r2 = r[k + 1], q1 = rb[k], q2 = rb[k + 1], n = x->n[k];
    const double* xk = x->core + x->ps[k];
    const double* bk = b->core + b->ps[k];
    double* Tk = T.p() + toff[k];
    // T[a, (i,q)] = Psi_L[a, p] b_k[p, (i,q)]
    gemm_f64(c, false, false, r1, n * q2, q1, 1.0, PL.p() + poff[k], r1, 0, bk, q1, 0, 0.0, Tk,
             r1, 0);
    // Psi_L[k+1][c, q] = sum_{(a,i)} x_k[(a,i), c] T[(a,i), q]
    gemm_f64(c, true, false, r2, q2, r1 * n, 1.0, xk, r1 * n, 0, Tk, r1 * n, 0, 0.0,
             PL.p() + poff[k + 1], r2, 0);
  }
  for (int64_t k = d - 1; k >= 0; --k) {
    const int64_t r1 = r[k], r2 = r[k + 1], q1 = rb[k], q2 = rb[k + 1], n = x->n[k];
    const double* xk = x->core + x->ps[k];
    const double* bk = b->core + b->ps[k];
    const double* PRn = PR.p() + poff[k + 1];
    // gradient: G[(a,i), c] = sum_q T[(a,i), q] Psi_R[k+1][c, q]
    gemm_f64(c, false, true, r1 * n, r2, q2, 1.0, T.p() + toff[k], r1 * n, 0, PRn, r2, 0, 0.0,
             grad + x->ps[k], r1 * n, 0);
    if (k == 0) break;
    // U[(p,i), c] = sum_q b_k[(p,i), q] Psi_R[k+1][c, q]
    gemm_f64(c, false, true, q1 * n, r2, q2, 1.0, bk, q1 * n, 0, PRn, r2, 0, 0.0, U.p(), q1 * n,
             0);
    // Psi_R[k][a, p] = sum_{(i,c)} x_k[a, (i,c)] U[p, (i,c)]
    gemm_f64(c, false, true, r1, q1, n * r2, 1.0, xk, r1, 0, U.p(), q1, 0, 0.0,
             PR.p() + poff[k], r1, 0);
  }
  if (value) copy_f64(c, 1, PL.p() + poff[d], value);
}

// ---------------------------------------------------------------------------
// sum_s (X[idx_s] - y_s)^2
// ---------------------------------------------------------------------------
void grad_sampled(Context* c, const ttg_tt_s* x, int64_t S, const int* idx, const double* y,
                  double* grad, double* value) {
  check_tt_vector(x, "x");
  const int64_t d = x->d;
  const auto& r = x->r;
  TTG_REQUIRE(S >= 0 && S <= int64_t(0x7fffffff) - 1, "sample count %lld out of range",
              (long long)S);
  for (int64_t k = 0; k < d; ++k)
    TTG_REQUIRE(x->n[k] <= MAX_BUCKETS, "mode size %lld above %lld", (long long)x->n[k],
                (long long)MAX_BUCKETS);
  if (S == 0) {
    fill_f64(c, x->numel, 0.0, grad);
    if (value) fill_f64(c, 1, 0.0, value);
    return;
  }
  TTG_REQUIRE(idx && y, "NULL sample arrays");
  // Index range check (one read-back; the sort below clamps as well).
  {
    DBuf<int64_t> nk(c, d);
    DBuf<int> err(c, 1);
    TTG_CUDA(cudaMemcpyAsync(nk.p(), x->n.data(), d * sizeof(int64_t), cudaMemcpyHostToDevice,
                             c->stream));
    TTG_CUDA(cudaMemsetAsync(err.p(), 0, sizeof(int), c->stream));
    k_check_idx<<<blocks_for(S * d), 256, 0, c->stream>>>(S, int(d), idx, nk.p(), err.p());
    c->launches += 1;
    TTG_CHECK_LAUNCH();
    int h = 0;
    TTG_CUDA(cudaMemcpyAsync(&h, err.p(), sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    TTG_CUDA(cudaStreamSynchronize(c->stream));
    TTG_REQUIRE(h == 0, "sample index out of range (idx is 0-based, column k in [0, n_k))");
  }
  // Bucketing of every index column.
  const int nblk = int((S + SORT_CHUNK - 1) / SORT_CHUNK);
  int64_t nmax = 1;
  std::vector<int64_t> moff(d + 1, 0);
  for (int64_t k = 0; k < d; ++k) {
    nmax = std::max(nmax, x->n[k]);
    moff[k + 1] = moff[k] + 3 * x->n[k] + 3;
  }
  DBuf<int> perm(c, size_t(S) * d), meta(c, moff[d]), counts(c, size_t(nmax) * nblk),
      total(c, nmax);
  std::vector<int> hmeta(moff[d]);
  for (int64_t k = 0; k < d; ++k) {
    const int n = int(x->n[k]);
    const int* col = idx + k * S;
    k_bucket_count<<<nblk, 32, n * sizeof(int), c->stream>>>(S, col, n, nblk, counts.p());
    k_bucket_scan<<<n, 256, 0, c->stream>>>(nblk, counts.p(), total.p());
    k_bucket_base<<<1, 1, 0, c->stream>>>(n, total.p(), meta.p() + moff[k]);
    k_bucket_scatter<<<nblk, 32, n * sizeof(int), c->stream>>>(S, col, n, nblk, counts.p(),
                                                                meta.p() + moff[k],
                                                                perm.p() + k * S);
    c->launches += 4;
    TTG_CHECK_LAUNCH();
  }
  // Tile counts per core sized the grids; read them once.
  TTG_CUDA(cudaMemcpyAsync(hmeta.data(), meta.p(), moff[d] * sizeof(int), cudaMemcpyDeviceToHost,
                           c->stream));
  TTG_CUDA(cudaStreamSynchronize(c->stream));
  // Left vectors l_k [S x r_k], k = 0..d (l_0 = 1, l_d = the sampled entries).
  std::vector<int64_t> loff(d + 2, 0);
  int64_t rmax = 1;
  for (int64_t k = 0; k <= d; ++k) {
    loff[k + 1] = loff[k] + S * r[k];
    rmax = std::max(rmax, r[k]);
  }
  int64_t partmax = 1;
  for (int64_t k = 0; k < d; ++k) {
    const int n = int(x->n[k]);
    partmax = std::max(partmax, int64_t(hmeta[moff[k] + 3 * n + 2]) * r[k] * r[k + 1]);
  }
  DBuf<double> Lv(c, loff[d + 1]), rho0(c, S * rmax), rho1(c, S * rmax), e(c, S),
      part(c, partmax);
  fill_f64(c, S, 1.0, Lv.p());
  for (int64_t k = 0; k < d; ++k) {
    const int n = int(x->n[k]);
    const int ntiles = hmeta[moff[k] + 2 * n + 1];
    if (ntiles == 0) continue;
    PropP p{Lv.p() + loff[k], r[k], Lv.p() + loff[k + 1], r[k + 1], x->core + x->ps[k],
            r[k], x->n[k], r[k + 1], r[k], r[k + 1], perm.p() + k * S, meta.p() + moff[k]};
    dim3 grid{unsigned(ntiles), unsigned((r[k + 1] + BN - 1) / BN), 1};
    k_prop<false><<<grid, 128, 0, c->stream>>>(p);
    c->launches += 1;
    TTG_CHECK_LAUNCH();
  }
  double* rho = rho0.p();
  double* rho_next = rho1.p();
  k_sample_residual<<<blocks_for(S), 256, 0, c->stream>>>(S, Lv.p() + loff[d], y, e.p(), rho);
  c->launches += 1;
  TTG_CHECK_LAUNCH();
  if (value) dot_f64(c, S, e.p(), nullptr, value);
  for (int64_t k = d - 1; k >= 0; --k) {
    const int n = int(x->n[k]);
    const int ngt = hmeta[moff[k] + 3 * n + 2];
    const int64_t r1 = r[k], r2 = r[k + 1];
    GradP gp{Lv.p() + loff[k], r1, rho, r2, part.p(), r1, x->n[k], r2, perm.p() + k * S,
             meta.p() + moff[k]};
    dim3 gg{unsigned(ngt), unsigned((r1 + BM - 1) / BM), unsigned((r2 + BN - 1) / BN)};
    k_grad_tiles<<<gg, 128, 0, c->stream>>>(gp);
    k_grad_reduce<<<blocks_for(r1 * r2 * x->n[k]), 256, 0, c->stream>>>(
        r1, x->n[k], r2, part.p(), meta.p() + moff[k], grad + x->ps[k]);
    c->launches += 2;
    TTG_CHECK_LAUNCH();
    if (k == 0) break;
    const int ntiles = hmeta[moff[k] + 2 * n + 1];
    PropP p{rho, r2, rho_next, r1, x->core + x->ps[k], r1, x->n[k], r2, r2, r1,
            perm.p() + k * S, meta.p() + moff[k]};
    dim3 grid{unsigned(ntiles), unsigned((r1 + BN - 1) / BN), 1};
    k_prop<true><<<grid, 128, 0, c->stream>>>(p);
    c->launches += 1;
    TTG_CHECK_LAUNCH();
    std::swap(rho, rho_next);
  }
}

}  // namespace ttg
