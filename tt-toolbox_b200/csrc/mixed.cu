// Mixed-precision local solve: FP64 iterative refinement around an FP32
// GMRES whose matvecs run on BF16 tensor cores (mixed_ops.cu).
//
// Same contract as the MEX local solver (fmex/solve3d_2.c:254-279): start
// from sol_prev and stop once ||rhs - B sol|| <= tol ||rhs||, with the true
// residual always evaluated by the FP64 matvec.  Each refinement step solves
// B dx = r approximately in low precision (relative tolerance 1e-3 or the
// remaining target, whichever is looser), then sol += dx and r is recomputed
// in FP64.  The inner Krylov solver is GMRES(restart) with classical
// Gram-Schmidt applied twice (CGS2): one cooperative kernel per Arnoldi step
// performs both projections, the normalisation and the Givens update of the
// least-squares residual; partial sums are reduced in a fixed order.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "group.cuh"
#include "jacobi.h"
#include "mixed.h"
#include "mixed_ops.h"

namespace ttg {

namespace {

constexpr int AR_THREADS = 256;
constexpr int AR_WARPS = AR_THREADS / 32;
constexpr long long AR_SPIN_LIMIT = 1LL << 24;
constexpr int MAX_OUTER = 8;
constexpr double INNER_TOL = 1e-3;

struct ArArgs {
  int64_t sz;
  int m;           // restart length
  float* V;        // sz x (m+1)
  float* w;        // matvec output, orthogonalised in place
  double* H;       // (m+1) x m, column-major
  double* cs;      // m
  double* sn;      // m
  double* g;       // m+1
  double* scal;    // [0] |g_{j+1}|  [1] norm of the new Arnoldi vector  [2] beta
                   // [3] norm of the solve's right-hand side  [4] stop threshold
  double* part;    // 2 * (m+1) * gridDim.x
  unsigned* bar;   // [0] count [1] generation
  int* err;
  int* stop;       // [0] converged flag, [1] step at which it converged (-1: at start)
  double reltol;   // stop once |g_{j+1}| <= reltol * scal[3]
  // BF16 operand of the next local matvec, written with each new basis
  // vector: X[b + ldx * row] = bf16(V[b + rx2 * row]) (padding b >= rx2 stays
  // zero), so the matvec needs no conversion launch.
  __nv_bfloat16* X;
  int rx2;
  int ldx;
};

__device__ __forceinline__ void put_x(const ArArgs& a, int64_t i, float v) {
  if (!a.X) return;  // preconditioned solve: the operand is P v, written apart
  const int64_t row = i / a.rx2, b = i - row * a.rx2;
  a.X[b + int64_t(a.ldx) * row] = __float2bfloat16_rn(v);
}

__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sumd(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ void ar_barrier(TTG_BLOCK, unsigned* bar, int* err, long long limit = AR_SPIN_LIMIT) {
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
          atomicExch(err, 4);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

#define AR_LOOP(idx, n)                                                             \
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < (n);    \
       idx += int64_t(gridDim.x) * blockDim.x)

// part[c*nb + block] = block partial of V(:,c)'w, c < ncol.  red: AR_WARPS*(m+1) floats.
// Columns go in groups of AR_COLS per pass over w, so that each thread has
// AR_COLS independent loads in flight instead of one memory latency per
// column; every column's sum is formed in the same order as one column per
// pass would form it.
constexpr int AR_COLS = 8;
__device__ void partial_dots(TTG_BLOCK, const ArArgs& a, int ncol, double* part, float* red) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c0 = 0; c0 < ncol; c0 += AR_COLS) {
    const int nc = ncol - c0 < AR_COLS ? ncol - c0 : AR_COLS;
    float s[AR_COLS];
#pragma unroll
    for (int k = 0; k < AR_COLS; ++k) s[k] = 0.f;
    AR_LOOP(i, a.sz) {
      const float wi = a.w[i];
#pragma unroll
      for (int k = 0; k < AR_COLS; ++k)
        if (k < nc) s[k] += a.V[int64_t(c0 + k) * a.sz + i] * wi;
    }
#pragma unroll
    for (int k = 0; k < AR_COLS; ++k) {
      if (k < nc) {
        const float t = warp_sumf(s[k]);
        if (lane == 0) red[warp * (a.m + 1) + c0 + k] = t;
      }
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < AR_WARPS; ++q) s += double(red[q * (a.m + 1) + c]);
    part[int64_t(c) * gridDim.x + blockIdx.x] = s;
  }
}

// Sum the block partials of ncol columns (same fixed order in every block).
__device__ void reduce_parts(TTG_BLOCK, const double* part, int ncol, double* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c = warp; c < ncol; c += AR_WARPS) {
    double s = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) s += __ldcg(part + int64_t(c) * gridDim.x + b);
    s = warp_sumd(s);
    if (lane == 0) out[c] = s;
  }
  __syncthreads();
}

// Shared memory of k_arnoldi: hp (m+1 doubles), ht (m+2), red (AR_WARPS
// (m+1) floats), then 2 m doubles for the rotations of the Givens update,
// 8-byte aligned.
__device__ __forceinline__ double* red_d(double* shd, int m) {
  const size_t off = sizeof(double) * 2 * (m + 2) + sizeof(float) * AR_WARPS * (m + 1);
  return reinterpret_cast<double*>(reinterpret_cast<char*>(shd) + ((off + 7) & ~size_t(7)));
}

// One Arnoldi step for column j: w -= V h twice (CGS2), normalise into
// V(:, j+1), Givens update of H(:, j) and g; scal[0] = |g_{j+1}|.
TTG_BODY(k_arnoldi)(TTG_BLOCK, ArArgs a, int j) {
  if (*(volatile int*)a.stop) return;  // queued after convergence
  extern __shared__ double shd[];
  double* hp = shd;                 // m+1 : this pass's coefficients
  double* ht = shd + (a.m + 1);     // m+2 : accumulated coefficients
  float* red = reinterpret_cast<float*>(shd + 2 * (a.m + 2));
  const int ncol = j + 1;
  double* part0 = a.part;
  double* part1 = a.part + int64_t(a.m + 1) * gridDim.x;
  for (int c = threadIdx.x; c <= ncol; c += blockDim.x) ht[c] = 0.0;
  for (int pass = 0; pass < 2; ++pass) {
    double* part = pass ? part1 : part0;
    partial_dots(blockIdx, gridDim, a, ncol, part, red);
    ar_barrier(blockIdx, gridDim, a.bar, a.err);
    reduce_parts(blockIdx, gridDim, part, ncol, hp);
    AR_LOOP(i, a.sz) {
      float s = 0.f;
      for (int c = 0; c < ncol; ++c) s += a.V[int64_t(c) * a.sz + i] * float(hp[c]);
      a.w[i] -= s;
    }
    for (int c = threadIdx.x; c < ncol; c += blockDim.x) ht[c] += hp[c];
    __syncthreads();
  }
  // norm of w (reuses part0: every block finished reading it before the
  // second pass's barrier)
  {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float s = 0.f;
    AR_LOOP(i, a.sz) s += a.w[i] * a.w[i];
    s = warp_sumf(s);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < AR_WARPS; ++q) t += double(red[q]);
      part0[blockIdx.x] = t;
    }
    ar_barrier(blockIdx, gridDim, a.bar, a.err);
    reduce_parts(blockIdx, gridDim, part0, 1, hp);
  }
  const double nrm = sqrt(hp[0]);
  float* Vn = a.V + int64_t(j + 1) * a.sz;
  const float inv = nrm > 0.0 ? float(1.0 / nrm) : 0.f;
  AR_LOOP(i, a.sz) {
    const float v = a.w[i] * inv;
    Vn[i] = v;
    put_x(a, i, v);
  }
  if (blockIdx.x == 0) {
    // The Givens update runs on one thread over a shared-memory copy of the
    // column (ht) and of the previous rotations: a chain of dependent
    // shared-memory accesses instead of global ones.  Same operations in the
    // same order as on the global arrays.
    double* cl = red_d(shd, a.m);
    double* sl = cl + a.m;
    for (int i = threadIdx.x; i < j; i += blockDim.x) {
      cl[i] = a.cs[i];
      sl[i] = a.sn[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      ht[j + 1] = nrm;
      for (int i = 0; i < j; ++i) {  // previous rotations
        const double x = ht[i], y = ht[i + 1];
        ht[i] = cl[i] * x + sl[i] * y;
        ht[i + 1] = -sl[i] * x + cl[i] * y;
      }
      const double x = ht[j], y = ht[j + 1];
      const double rho = sqrt(x * x + y * y);
      const double c0 = rho > 0.0 ? x / rho : 1.0, s0 = rho > 0.0 ? y / rho : 0.0;
      a.cs[j] = c0;
      a.sn[j] = s0;
      ht[j] = rho;
      ht[j + 1] = 0.0;
      a.g[j + 1] = -s0 * a.g[j];
      a.g[j] = c0 * a.g[j];
      a.scal[0] = fabs(a.g[j + 1]);
      a.scal[1] = nrm;
      if (a.scal[0] <= a.scal[4]) {
        a.stop[1] = j;
        __threadfence();
        a.stop[0] = 1;
      }
    }
    __syncthreads();
    double* Hj = a.H + int64_t(a.m + 1) * j;
    for (int c = threadIdx.x; c <= j + 1; c += blockDim.x) Hj[c] = ht[c];
  }
}
TTG_COOP_KERNEL(k_arnoldi, AR_THREADS);

// V(:,0) = r / ||r||, g = [||r||, 0, ...]; scal[2] = ||r||.  On the first
// restart (first != 0) r is the right-hand side: scal[3] = ||r||.  The stop
// threshold reltol * scal[3] goes to scal[4]; a residual already below it
// (or zero) raises the stop flag with step -1, so the queued steps return at
// once and the host learns it at its next read of the flags.
TTG_BODY(k_ar_init)(TTG_BLOCK, ArArgs a, const float* r, int first) {
  __shared__ float red[AR_WARPS];
  __shared__ double tot[1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float s = 0.f;
  AR_LOOP(i, a.sz) s += r[i] * r[i];
  s = warp_sumf(s);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < AR_WARPS; ++q) t += double(red[q]);
    a.part[blockIdx.x] = t;
  }
  ar_barrier(blockIdx, gridDim, a.bar, a.err);
  reduce_parts(blockIdx, gridDim, a.part, 1, tot);
  const double beta = sqrt(tot[0]);
  const float inv = beta > 0.0 ? float(1.0 / beta) : 0.f;
  AR_LOOP(i, a.sz) {
    const float v = r[i] * inv;
    a.V[i] = v;
    put_x(a, i, v);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int k = 0; k <= a.m; ++k) a.g[k] = 0.0;
    a.g[0] = beta;
    a.scal[2] = beta;
    a.scal[0] = beta;
    if (first) a.scal[3] = beta;
    const double thr = a.reltol * a.scal[3];
    a.scal[4] = thr;
    if (beta <= thr || beta == 0.0) {
      a.stop[1] = -1;
      __threadfence();
      a.stop[0] = 1;
    }
  }
}
TTG_COOP_KERNEL(k_ar_init, AR_THREADS);

// x += V(:, 0:k) y with H(0:k,0:k) y = g(0:k) (upper triangular after Givens).
TTG_BODY(k_ar_update)(TTG_BLOCK, ArArgs a, int k, float* x) {
  pdl_begin();
  // y (m+1), then H's leading k x k block (ld k) and g (k), copied in
  // parallel so that the back-substitution on one thread reads shared memory.
  extern __shared__ double y[];
  double* Hs = y + (a.m + 1);
  double* gs = Hs + int64_t(k) * k;
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
    const int row = e % k, col = e / k;
    Hs[e] = a.H[row + int64_t(a.m + 1) * col];
  }
  for (int e = threadIdx.x; e < k; e += blockDim.x) gs[e] = a.g[e];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int row = k - 1; row >= 0; --row) {
      double v = gs[row];
      for (int col = row + 1; col < k; ++col) v -= Hs[row + k * col] * y[col];
      const double d = Hs[row + k * row];
      y[row] = d != 0.0 ? v / d : 0.0;
    }
  }
  __syncthreads();
  AR_LOOP(i, a.sz) {
    float s = 0.f;
    for (int c = 0; c < k; ++c) s += a.V[int64_t(c) * a.sz + i] * float(y[c]);
    x[i] += s;
  }
}
TTG_KERNEL(k_ar_update, 0);

// Centre block-Jacobi on vectors in the reversed layout v[k + rx2 (j + n i)]:
// out[k, j, i] = sum_m J[i, j, m, k] v[k, m, i] with the FP64 blocks J of
// jac_gen_c_f64 (natural layout J[i + rx1 (j + n (m + n k))]).  To BF16 in
// the matvec's K-major operand layout (xb, ld ldx) or to FP32 (xf).
TTG_BODY(k_prec_rev)(TTG_BLOCK, int64_t rx1, int64_t n, int64_t rx2, const double* __restrict__ J,
                           const float* __restrict__ v, __nv_bfloat16* __restrict__ xb,
                           int64_t ldx, float* __restrict__ xf, const int* skip) {
  pdl_begin();
  if (skip && *skip) return;
  const int64_t total = rx1 * n * rx2;
  AR_LOOP(e, total) {
    const int64_t k = e % rx2, j = (e / rx2) % n, i = e / (rx2 * n);
    const double* Jr = J + i + rx1 * j + rx1 * n * n * k;
    const float* vr = v + k + rx2 * n * i;
    double s = 0.0;
    for (int64_t m = 0; m < n; ++m) s += Jr[rx1 * n * m] * double(vr[rx2 * m]);
    if (xb)
      xb[k + ldx * (j + n * i)] = __float2bfloat16_rn(float(s));
    else
      xf[e] = float(s);
  }
}
TTG_KERNEL(k_prec_rev, 0);

// r = b - y (FP32)
TTG_BODY(k_sub_f32)(TTG_BLOCK, int64_t n, const float* b, const float* y, float* r) {
  pdl_begin();
  AR_LOOP(i, n) r[i] = b[i] - y[i];
}
TTG_KERNEL(k_sub_f32, 0);

struct Gmres32 {
  Context* c;
  int64_t sz;
  int m;
  int blocks;
  DBuf<float> V, w, r;
  DBuf<double> small, part;
  DBuf<unsigned> bar;
  DBuf<int> stop;
  ArArgs a{};

  Gmres32(Context* cc, int64_t n, int restart) : c(cc), sz(n), m(restart) {
    V.reset(c, size_t(sz) * (m + 1));
    w.reset(c, sz);
    r.reset(c, sz);
    small.reset(c, size_t(m + 1) * m + 2 * m + (m + 1) + 8);
    int occ = 0;
    occ = max_active_blocks(k_arnoldi.fn(), AR_THREADS, arnoldi_smem());
    if (occ < 1) occ = 1;
    int64_t want = (sz + AR_THREADS * 4 - 1) / (AR_THREADS * 4);
    const int64_t cap = int64_t(c->num_sms) * std::min(occ, 2);
    blocks = int(std::max<int64_t>(1, std::min(want, cap)));
    part.reset(c, size_t(2) * (m + 1) * blocks);
    bar.reset(c, 4);
    memset_async(c, bar.p(), 0, 4 * sizeof(unsigned));
    a.sz = sz;
    a.m = m;
    a.V = V.p();
    a.w = w.p();
    a.H = small.p();
    a.cs = a.H + size_t(m + 1) * m;
    a.sn = a.cs + m;
    a.g = a.sn + m;
    a.scal = a.g + (m + 1);
    a.part = part.p();
    a.bar = bar.p();
    a.err = c->d_err + 2;
    stop.reset(c, 4);
    a.stop = stop.p();
    a.reltol = 0.0;
    a.X = nullptr;
  }

  size_t arnoldi_smem() const {
    return sizeof(double) * (2 * (m + 2)) + sizeof(float) * AR_WARPS * (m + 1) + 8 +
           sizeof(double) * 2 * m + 16;
  }


  // Right-preconditioned operand: X = bf16(P v) for the centre block-Jacobi
  // blocks J (FP64, natural layout), v in the reversed layout.
  void prec_x(MixedOp& op, const double* J, const float* v) {
    launch(c, k_prec_rev, blocks, AR_THREADS, 0, op.d.rx1, op.d.n, op.d.rx2, J, v, op.X.p(),
           op.ldx, static_cast<float*>(nullptr), c->skip);
    TTG_CHECK_LAUNCH();
  }

  // Solve B x = b approximately (B P y = b, x = y, when J is given: the
  // caller applies P to x); x (FP32, zeroed here); returns Krylov steps.
  int64_t solve(MixedOp& op, const float* b, float* x, double reltol, int64_t max_restarts,
                const double* J = nullptr) {
    int64_t steps = 0;
    a.X = J ? nullptr : op.X.p();
    a.rx2 = int(op.d.rx2);
    a.ldx = int(op.ldx);
    a.reltol = reltol;
    memset_async(c, x, 0, sizeof(float) * sz);
    for (int64_t it = 0; it < max_restarts; ++it) {
      const float* rr = b;
      if (it > 0) {
        if (J) {
          prec_x(op, J, x);
          op.apply_converted(c, w.p());
        } else {
          op.apply(c, x, w.p());
        }
        launch(c, k_sub_f32, blocks, AR_THREADS, 0, sz, b, w.p(), r.p());
        rr = r.p();
      }
      memset_async(c, stop.p(), 0, 2 * sizeof(int));
      const int first = it == 0 ? 1 : 0;
      launch(c, k_ar_init, blocks, AR_THREADS, 0, a, rr, first);
      // Steps queued in chunks; k_arnoldi (or k_ar_init, for a residual
      // already below the threshold) raises the stop flag and later queued
      // kernels return at once (see gmres.cu).  The first chunk is the step
      // count of the context's previous inner solve, later ones half of it,
      // so that most solves need one or two reads of the flags.  Matvecs
      // queued past the converged step are taken out of the counters and
      // timings afterwards.
      int j = 0, queued = 0;
      const int hint = std::max(3, c->krylov_hint);
      int chunk = std::min(m, hint);
      bool conv = false, at_start = false;
      std::vector<uint64_t> seqs;
      SkipGuard guard(c, stop.p());
      while (j < m) {
        const int jend = std::min(m, j + chunk);
        for (int jj = j; jj < jend; ++jj) {
          const int jv = jj;
          seqs.push_back(c->ev_seq);
          if (J) prec_x(op, J, V.p() + int64_t(jj) * sz);  // X = bf16(P V(:, jv))
          op.apply_converted(c, w.p());  // X holds V(:, jv) (k_ar_init / k_arnoldi)
          launch(c, k_arnoldi, blocks, AR_THREADS, arnoldi_smem(), a, jv);
        }
        queued = jend;
        int flag[2];
        read_device(c, flag, stop.p(), sizeof(flag));
        if (flag[0]) {
          if (flag[1] < 0) {
            at_start = true;
          } else {
            conv = true;
            j = flag[1];
          }
          break;
        }
        j = jend;
        chunk = std::max(3, hint / 2);
      }
      guard.release();
      {
        const int done = at_start ? 0 : (conv ? j + 1 : m);
        const int skipped = queued - done;
        if (skipped > 0) {
          const double fl = op.d.flops();
          c->matvecs -= skipped;
          c->matvec_flops -= int64_t(fl) * skipped;
          c->mv_count[1] -= skipped;
          c->mv_flops[1] -= fl * skipped;
          c->mv_bytes_lp -= op.bytes_per_matvec() * skipped;
          // three recorded GEMMs per queued matvec (grouped: three-launch form)
          if (c->rec) rec_retract_flop(c->rec, fl * skipped, 3 * int64_t(skipped));
          if (c->time_matvec) c->ev_void(seqs[done], c->ev_seq);
        }
      }
      if (at_start) break;  // nothing left to reduce: x stays as it is
      const int k = conv ? j + 1 : m;
      steps += k;
      c->krylov_hint = k;
      launch(c, k_ar_update, blocks, AR_THREADS,
             sizeof(double) * (size_t(m + 1) + size_t(k) * k + size_t(k)), a, k, x);
      TTG_CHECK_LAUNCH();
      if (conv) break;
    }
    return steps;
  }
};

}  // namespace

LocalSolveResult local_solve_mixed(Context* c, const MvDims& d, const double* Phi1,
                                   const double* A, const double* Phi2, const double* rhs,
                                   const double* dres, double nres, double nrhs, double tol,
                                   const double* sol_prev, int64_t nrestart, int64_t niters,
                                   double* sol, double* bsol_out, int prec) {
  LocalSolveResult out;
  const int64_t sz = d.in_size();
  TTG_REQUIRE(prec == 0 || prec == 1,
              "the mixed-precision local solve has the 'cjacobi' preconditioner only");
  // Centre block-Jacobi blocks (FP64) for the right preconditioning of the
  // low-precision Krylov solves and of the FP64 fallback.
  DBuf<double> J, pw;
  if (prec == 1) {
    J.reset(c, jac_size(1, d.rx1, d.n, d.rx2));
    pw.reset(c, sz);
    jac_gen_c_f64(c, d.rx1, d.n, d.rx2, d.ra1, d.ra2, Phi1, A, Phi2, J.p());
  }
  if (nrestart > sz) nrestart = sz;
  TTG_REQUIRE(nrestart <= 1024, "mixed solve: restart length %lld too large", (long long)nrestart);
  MixedOp op;
  op.prepare(c, d, Phi1, A, Phi2);
  Gmres32 gm(c, sz, int(nrestart));
  DBuf<double> t1(c, d.t1_size()), t2(c, d.t2_size()), r64(c, sz), prev(c, sz), s(c, 2);
  DBuf<float> rrev(c, sz), dx(c, sz), dxp;
  if (prec == 1) dxp.reset(c, sz);
  copy_f64(c, sz, sol_prev, sol);
  auto residual = [&]() -> double {
    if (bsol_out) {
      local_matvec_f64(c, d, Phi1, A, Phi2, sol, bsol_out, t1.p(), t2.p());
      copy_f64(c, sz, bsol_out, r64.p());
    } else {
      local_matvec_f64(c, d, Phi1, A, Phi2, sol, r64.p(), t1.p(), t2.p());
    }
    out.matvecs_fp64++;
    axpby_f64(c, sz, 1.0, rhs, -1.0, r64.p());
    dot_f64(c, sz, r64.p(), nullptr, s.p(), true);
    double h;
    read_scalars(c, s.p(), &h, 1);
    return h;
  };
  const double target = tol * nrhs;
  copy_f64(c, sz, dres, r64.p());
  double nr = nres;
  bool r64_valid = true;  // r64 = rhs - B sol for the current sol
  for (int outer = 0; outer < MAX_OUTER; ++outer) {
    if (!(nr > target)) break;
    nat_to_rev(c, d.rx1, d.n, d.rx2, r64.p(), rrev.p(), 1.0 / nr);
    const double reltol = std::max(target / nr, INNER_TOL);
    out.iters += gm.solve(op, rrev.p(), dx.p(), reltol, niters, prec ? J.p() : nullptr);
    copy_f64(c, sz, sol, prev.p());
    if (prec) {  // the correction is P y
      launch(c, k_prec_rev, gm.blocks, AR_THREADS, 0, d.rx1, d.n, d.rx2, J.p(), dx.p(),
             static_cast<__nv_bfloat16*>(nullptr), int64_t(0), dxp.p(),
             static_cast<const int*>(nullptr));
      TTG_CHECK_LAUNCH();
      rev_to_nat_add(c, d.rx1, d.n, d.rx2, dxp.p(), sol, nr);
    } else {
      rev_to_nat_add(c, d.rx1, d.n, d.rx2, dx.p(), sol, nr);
    }
    const double nr_new = residual();
    out.have_bsol = bsol_out != nullptr;
    if (!(nr_new < nr)) {  // no progress: keep the better iterate and stop
      copy_f64(c, sz, prev.p(), sol);
      out.have_bsol = false;
      r64_valid = false;
      break;
    }
    const bool stagnating = nr_new > 0.5 * nr;
    nr = nr_new;
    if (stagnating) break;
  }
  if (nr > target) {
    // The low-precision corrections stopped paying (the local operator is
    // too ill-conditioned for BF16 products): finish with the FP64
    // Householder GMRES of the FP64 path on the remaining residual, so the
    // local solve meets the same tolerance as there.
    if (!r64_valid) nr = residual();
    if (nr > target) {
      DBuf<double> dsol(c, sz);
      auto mv = [&](const double* x, double* y) {
        if (prec == 1) {  // B P x
          jac_apply_c_f64(c, d.rx1, d.n, d.rx2, J.p(), x, pw.p());
          local_matvec_f64(c, d, Phi1, A, Phi2, pw.p(), y, t1.p(), t2.p());
        } else {
          local_matvec_f64(c, d, Phi1, A, Phi2, x, y, t1.p(), t2.p());
        }
      };
      GmresResult g = gmres_hh_f64(c, mv, r64.p(), sz, nrestart, target / nr, niters, dsol.p());
      if (prec == 1) {
        jac_apply_c_f64(c, d.rx1, d.n, d.rx2, J.p(), dsol.p(), pw.p());
        copy_f64(c, sz, pw.p(), dsol.p());
      }
      axpby_f64(c, sz, 1.0, dsol.p(), 1.0, sol);
      out.iters += g.iters;
      out.matvecs_fp64 += g.matvecs;
      out.have_bsol = false;
      c->mixed_fallbacks += 1;
    }
  }
  // Bounded-wait timeouts are reported through the context error slots 1-2,
  // checked by the caller once its sequence is done.
  out.matvecs = out.iters;
  return out;
}

namespace {
__global__ void k_selftest_ar_barrier(unsigned* bar, int* flag, long long limit) {
  if (blockIdx.x != 0) return;
  ar_barrier(blockIdx, gridDim, bar, flag, limit);
}
}  // namespace

// Self-test of the bounded barrier of the Arnoldi kernels: block 1 never
// arrives; block 0 gives up after `limit` polls and raises *flag.
void selftest_wait_arnoldi(Context* c, int* flag, long long limit) {
  DBuf<unsigned> bar(c, 2);
  TTG_CUDA(cudaMemsetAsync(bar.p(), 0, 2 * sizeof(unsigned), c->stream));
  k_selftest_ar_barrier<<<2, 32, 0, c->stream>>>(bar.p(), flag, limit);
  TTG_CHECK_LAUNCH();
  sync(c);
}

}  // namespace ttg
