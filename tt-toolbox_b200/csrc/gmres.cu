// Device GMRES with Householder orthogonalisation (FP64).
//
// Restates dgmresr_hh (fmex/solve3d.c:339-518).  The Arnoldi work outside
// the matvec is done by three cooperative kernels, each one launch covering
// a whole sequence of reflector applications:
//   hh_build  : v_j = P_0 ... P_{j-1} (P_j e_j), normalised       (:396-406)
//   hh_tail   : w = P_j ... P_0 (B v_j), next reflector, Givens     (:421-473)
//   hh_correct: upper-triangular solve and the correction x += Q y  (:487-507)
// plus hh_init for the restart vector (:376-392).  Each reflector needs a
// global dot product before its update, so the blocks meet at a grid barrier
// per reflector; the partial sums are reduced in a fixed order, so results
// are deterministic run to run.  Every barrier wait is bounded: on timeout
// the kernel raises the context error flag and runs to completion, and the
// host returns TTG_ERR_TIMEOUT.
#include <cmath>
#include <cstring>

#include "gmres.h"
#include "group.cuh"

namespace ttg {

namespace {

constexpr int HH_THREADS = 256;
constexpr long long BAR_SPIN_LIMIT = 1LL << 24;

// Restart lengths up to which k_hh_tail / k_hh_correct stage their serial
// sections in shared memory (3 nrestart + 1, nrestart^2 + 2 nrestart doubles).
constexpr int64_t HH_STAGE_MAX = 1024;
constexpr int64_t HH_CORRECT_STAGE_MAX = 64;

size_t hh_tail_smem(int64_t nrestart) {
  return nrestart <= HH_STAGE_MAX ? sizeof(double) * size_t(3 * nrestart + 1) : 0;
}
size_t hh_correct_smem(int64_t nrestart) {
  return sizeof(double) * size_t(nrestart + (nrestart <= HH_CORRECT_STAGE_MAX
                                                 ? nrestart * nrestart + nrestart : 0));
}

struct HhArgs {
  int64_t sz;
  int64_t nrestart;
  double* U;  // sz x (nrestart+1)
  double* w;
  double* w2;
  double* sol;
  const double* rhs;
  double* tau;   // nrestart+1
  double* J;     // 2 x nrestart
  double* R;     // nrestart x nrestart
  double* scal;  // [0] nrmrhs [1] curres [2] nrmr [3] exact-flag [4] w[j+1]
  double* part;  // 2 * gridDim.x
  unsigned* bar; // [0] count [1] generation [2] reduction parity
  int* err;
  int* stop;     // [0] converged flag, [1] step at which it converged
  double tol;    // relative stopping tolerance of the current solve
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum, result broadcast to every thread.
__device__ double block_sum_all(double v) {
  __shared__ double sh[33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double r = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
    r = warp_sum(r);
    if (threadIdx.x == 0) sh[32] = r;
  }
  __syncthreads();
  return sh[32];
}

__device__ void grid_barrier(TTG_BLOCK, unsigned* bar, int* err,
                             long long limit = BAR_SPIN_LIMIT) {
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
          atomicExch(err, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// Grid-wide deterministic sum; every thread of every block gets the result.
// Partial buffers alternate so one barrier per reduction suffices.
__device__ double grid_sum(TTG_BLOCK, double v, const HhArgs& a, unsigned& parity) {
  v = block_sum_all(v);
  double* part = a.part + (parity & 1u) * gridDim.x;
  if (threadIdx.x == 0) part[blockIdx.x] = v;
  grid_barrier(blockIdx, gridDim, a.bar, a.err);
  double s = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += __ldcg(part + i);
  s = block_sum_all(s);
  parity ^= 1u;
  return s;
}

#define GRID_LOOP(idx, n)                                                           \
  for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < (n);    \
       idx += int64_t(gridDim.x) * blockDim.x)

// w = rhs - w2 ; U_0 = Householder vector of w ; tau_0 = -beta  (:376-392)
TTG_BODY(k_hh_init)(TTG_BLOCK, HhArgs a, int it) {
  unsigned parity = 0;
  const int64_t sz = a.sz;
  double s = 0.0;
  GRID_LOOP(i, sz) {
    const double v = a.rhs[i] - a.w2[i];
    a.w[i] = v;
    s += v * v;
  }
  const double nrmr = sqrt(grid_sum(blockIdx, gridDim, s, a, parity));
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (it == 0) a.scal[0] = nrmr;
    a.scal[2] = nrmr;
    a.scal[3] = (nrmr == 0.0) ? 1.0 : 0.0;
  }
  if (nrmr == 0.0) return;
  const double w0 = __ldcg(a.w);
  const double beta = (w0 < 0.0) ? -nrmr : nrmr;
  const double nu = sqrt(2.0 * nrmr * nrmr + 2.0 * beta * w0);
  GRID_LOOP(i, sz) {
    const double v = (i == 0) ? (a.w[i] + beta) : a.w[i];
    a.U[i] = v / nu;
  }
  if (blockIdx.x == 0) {
    for (int64_t k = threadIdx.x; k <= a.nrestart; k += blockDim.x) a.tau[k] = 0.0;
    __syncthreads();
    if (threadIdx.x == 0) a.tau[0] = -beta;
  }
}
TTG_COOP_KERNEL(k_hh_init, HH_THREADS);

// v_j = P_0 ... P_{j-1} (P_j e_j), normalised, into w  (:396-406)
TTG_BODY(k_hh_build)(TTG_BLOCK, HhArgs a, int64_t j) {
  if (*(volatile int*)a.stop) return;  // queued after convergence
  unsigned parity = 0;
  const int64_t sz = a.sz;
  const double* Uj = a.U + j * sz;
  const double ujj = __ldcg(Uj + j);
  GRID_LOOP(i, sz) { a.w[i] = -2.0 * ujj * Uj[i] + (i == j ? 1.0 : 0.0); }
  for (int64_t r = j - 1; r >= 0; --r) {
    const double* Ur = a.U + r * sz;
    double s = 0.0;
    GRID_LOOP(i, sz) s += Ur[i] * a.w[i];
    const double dot = grid_sum(blockIdx, gridDim, s, a, parity);
    GRID_LOOP(i, sz) a.w[i] -= 2.0 * dot * Ur[i];
  }
  double s = 0.0;
  GRID_LOOP(i, sz) s += a.w[i] * a.w[i];
  const double inv = 1.0 / sqrt(grid_sum(blockIdx, gridDim, s, a, parity));
  GRID_LOOP(i, sz) a.w[i] *= inv;
}
TTG_COOP_KERNEL(k_hh_build, HH_THREADS);

// w2 = P_j ... P_0 w2 ; new reflector U_{j+1} ; Givens ; R(:,j) ; residual (:421-473)
TTG_BODY(k_hh_tail)(TTG_BLOCK, HhArgs a, int64_t j) {
  if (*(volatile int*)a.stop) return;  // queued after convergence
  unsigned parity = 0;
  const int64_t sz = a.sz;
  double* w = a.w2;
  for (int64_t r = 0; r <= j; ++r) {
    const double* Ur = a.U + r * sz;
    double s = 0.0;
    GRID_LOOP(i, sz) s += Ur[i] * w[i];
    const double dot = grid_sum(blockIdx, gridDim, s, a, parity);
    GRID_LOOP(i, sz) w[i] -= 2.0 * dot * Ur[i];
  }
  if (j < sz - 1) {
    // The owner of w[j+1] publishes it before the barrier: after the barrier
    // it rewrites w[j+1], so other blocks must not read w itself.
    double s = 0.0;
    GRID_LOOP(i, sz) {
      if (i > j) s += w[i] * w[i];
      if (i == j + 1) a.scal[4] = w[i];
    }
    double alpha = sqrt(grid_sum(blockIdx, gridDim, s, a, parity));
    const double wj1 = __ldcg(a.scal + 4);
    double* Un = a.U + (j + 1) * sz;
    if (alpha != 0.0) {
      if (wj1 < 0.0) alpha = -alpha;
      const double nu = sqrt(2.0 * alpha * alpha + 2.0 * alpha * wj1);
      GRID_LOOP(i, sz) {
        double u;
        if (i <= j)
          u = 0.0;
        else if (i == j + 1)
          u = (w[i] + alpha) / nu;
        else
          u = w[i] / nu;
        Un[i] = u;
        if (i == j + 1)
          w[i] = -alpha;
        else if (i > j + 1)
          w[i] = 0.0;
      }
    } else {
      GRID_LOOP(i, sz) Un[i] = (i <= j) ? 0.0 : w[i];
    }
  }
  grid_barrier(blockIdx, gridDim, a.bar, a.err);
  if (blockIdx.x == 0) {
    // Givens rotations to the top of w (:445-449) on one thread.  With
    // staging (restart length up to HH_STAGE_MAX) the chain of dependent
    // accesses runs on shared-memory copies of w's top entries and of the
    // rotators, copied in and out by the block; the same operations in the
    // same order as on the global arrays.
    extern __shared__ double tsm[];
    const bool staged = a.nrestart <= HH_STAGE_MAX;
    const int64_t top = a.nrestart + 1 < sz ? a.nrestart + 1 : sz;
    double* wl = staged ? tsm : w;
    double* Jl = staged ? tsm + (a.nrestart + 1) : a.J;
    if (staged) {
      for (int64_t e = threadIdx.x; e < top; e += blockDim.x) wl[e] = __ldcg(w + e);
      for (int64_t e = threadIdx.x; e < 2 * j; e += blockDim.x) Jl[e] = a.J[e];
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      for (int64_t i = 0; i < j; ++i) {
        const double b = staged ? wl[i] : __ldcg(w + i);
        const double b1 = staged ? wl[i + 1] : __ldcg(w + i + 1);
        const double c0 = Jl[2 * i], c1 = Jl[2 * i + 1];
        wl[i] = c0 * b + c1 * b1;
        wl[i + 1] = -c1 * b + c0 * b1;
      }
      if (j < sz - 1) {  // new rotator (:454-465)
        const double wj = staged ? wl[j] : __ldcg(w + j);
        const double wj1 = staged ? wl[j + 1] : __ldcg(w + j + 1);
        const double rho = sqrt(wj * wj + wj1 * wj1);
        const double c0 = wj / rho, c1 = wj1 / rho;
        a.J[2 * j] = c0;
        a.J[2 * j + 1] = c1;
        a.tau[j + 1] = -c1 * a.tau[j];
        a.tau[j] = c0 * a.tau[j];
        wl[j] = rho;
        wl[j + 1] = 0.0;
      }
      if (!staged)
        for (int64_t k = 0; k < a.nrestart; ++k)
          a.R[k + j * a.nrestart] = (k < sz) ? __ldcg(w + k) : 0.0;
      const double curres = fabs(a.tau[j + 1]) / a.scal[0];
      a.scal[1] = curres;
      if (curres < a.tol) {  // (:476) later queued steps see the flag and return
        a.stop[1] = int(j);
        __threadfence();
        a.stop[0] = 1;
      }
    }
    if (staged) {
      __syncthreads();
      for (int64_t k = threadIdx.x; k < a.nrestart; k += blockDim.x)
        a.R[k + j * a.nrestart] = (k < sz) ? wl[k] : 0.0;
      for (int64_t e = threadIdx.x; e < top; e += blockDim.x) w[e] = wl[e];
    }
  }
}
TTG_COOP_KERNEL(k_hh_tail, HH_THREADS);

// Triangular solve + correction sol += P_0..P_j (sum y_i e_i)  (:487-507)
TTG_BODY(k_hh_correct)(TTG_BLOCK, HhArgs a, int64_t j, int64_t ni) {
  // y (nrestart); with staging also R's leading ni x ni block (ld ni) and
  // tau, copied by the block so that the back-substitution on one thread
  // reads shared memory (same operations, same order).
  extern __shared__ double y[];
  unsigned parity = 0;
  const int64_t sz = a.sz;
  const bool staged = a.nrestart <= HH_CORRECT_STAGE_MAX;
  double* Rs = y + a.nrestart;
  double* ts = Rs + ni * ni;
  if (staged) {
    for (int64_t e = threadIdx.x; e < ni * ni; e += blockDim.x)
      Rs[e] = a.R[(e % ni) + (e / ni) * a.nrestart];
    for (int64_t e = threadIdx.x; e < ni; e += blockDim.x) ts[e] = a.tau[e];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int64_t row = ni - 1; row >= 0; --row) {
      double v = staged ? ts[row] : a.tau[row];
      for (int64_t col = row + 1; col < ni; ++col)
        v -= (staged ? Rs[row + col * ni] : a.R[row + col * a.nrestart]) * y[col];
      y[row] = v / (staged ? Rs[row + row * ni] : a.R[row + row * a.nrestart]);
    }
  }
  __syncthreads();
  const double* Uj = a.U + j * sz;
  const double ujj = __ldcg(Uj + j);
  const double yj = y[j];
  GRID_LOOP(i, sz) a.w[i] = -2.0 * ujj * yj * Uj[i] + (i == j ? yj : 0.0);
  for (int64_t r = j - 1; r >= 0; --r) {
    const double* Ur = a.U + r * sz;
    double s = 0.0;
    GRID_LOOP(i, sz) {
      if (i == r) a.w[i] += y[r];
      s += Ur[i] * a.w[i];
    }
    const double dot = grid_sum(blockIdx, gridDim, s, a, parity);
    GRID_LOOP(i, sz) a.w[i] -= 2.0 * dot * Ur[i];
  }
  GRID_LOOP(i, sz) a.sol[i] += a.w[i];
}
TTG_COOP_KERNEL(k_hh_correct, HH_THREADS);

int coop_blocks(Context* c, const void* kernel, size_t smem, int64_t sz) {
  int occ = 0;
  occ = max_active_blocks(kernel, HH_THREADS, smem);
  if (occ < 1) occ = 1;
  int64_t want = (sz + HH_THREADS * 4 - 1) / (HH_THREADS * 4);
  int64_t cap = int64_t(c->num_sms) * std::min(occ, 2);
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  return int(want);
}


}  // namespace

GmresResult gmres_hh_f64(Context* c, const ApplyFn& apply, const double* rhs, int64_t sz,
                         int64_t nrestart, double tol, int64_t niters, double* sol) {
  GmresResult res;
  TTG_REQUIRE(nrestart >= 1 && nrestart <= 4096, "nrestart %lld out of range",
              (long long)nrestart);
  DBuf<double> U(c, size_t(sz) * (nrestart + 1)), w(c, sz), w2(c, sz);
  DBuf<double> small(c, (nrestart + 1) + 2 * nrestart + nrestart * nrestart + 8);
  const int blocks = std::min(
      std::min(coop_blocks(c, k_hh_init.fn(), 0, sz), coop_blocks(c, k_hh_build.fn(), 0, sz)),
      std::min(coop_blocks(c, k_hh_tail.fn(), hh_tail_smem(nrestart), sz),
               coop_blocks(c, k_hh_correct.fn(), hh_correct_smem(nrestart), sz)));
  DBuf<double> part(c, 2 * blocks);
  DBuf<unsigned> bar(c, 4);
  DBuf<int> stop(c, 4);
  memset_async(c, bar.p(), 0, 4 * sizeof(unsigned));
  memset_async(c, c->d_err, 0, sizeof(int));

  HhArgs a;
  a.sz = sz;
  a.nrestart = nrestart;
  a.U = U.p();
  a.w = w.p();
  a.w2 = w2.p();
  a.sol = sol;
  a.rhs = rhs;
  a.tau = small.p();
  a.J = a.tau + (nrestart + 1);
  a.R = a.J + 2 * nrestart;
  a.scal = a.R + nrestart * nrestart;
  a.part = part.p();
  a.bar = bar.p();
  a.err = c->d_err;
  a.stop = stop.p();
  a.tol = tol;
  fill_f64(c, sz, 0.0, sol);

  // Arnoldi steps are queued in chunks of growing length without a host
  // round trip per step; k_hh_tail raises a device flag on convergence and
  // every kernel queued after it (reflector kernels and the matvec GEMMs,
  // through Context::skip) returns at once.  The host reads the flag, the
  // converged step and the residual estimate once per chunk.
  struct Probe {
    int flag[2];
    double curres;
  };
  auto probe = [&](Probe& p) {
    double* stage = c->h_scal;
    const int* sp = stop.p();
    const double* cp = a.scal + 1;
    if (c->rec) {
      rec_read(c, 0, sp, 2 * sizeof(int));
      rec_read(c, sizeof(double), cp, sizeof(double));
      rec_wait(c->rec);
    } else {
      TTG_CUDA(cudaMemcpyAsync(stage, sp, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      TTG_CUDA(
          cudaMemcpyAsync(stage + 1, cp, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      sync(c);
    }
    memcpy(p.flag, stage, 2 * sizeof(int));
    p.curres = stage[1];
  };
  double curres = INFINITY;
  for (int64_t it = 0; it < niters; ++it) {
    apply(sol, w2.p());
    res.matvecs++;
    launch(c, k_hh_init, blocks, HH_THREADS, 0, a, int(it));
    memset_async(c, stop.p(), 0, 2 * sizeof(int));
    double hs[4];
    read_scalars(c, a.scal, hs, 4);
    if (hs[3] != 0.0) {  // exact solution: nothing to correct
      curres = 0.0;
      break;
    }
    bool broke = false;
    int64_t j = 0, chunk = 3;
    SkipGuard guard(c, stop.p());
    while (j < nrestart) {
      const int64_t jend = std::min(nrestart, j + chunk);
      for (int64_t jj = j; jj < jend; ++jj) {
        launch(c, k_hh_build, blocks, HH_THREADS, 0, a, jj);
        apply(w.p(), w2.p());
        launch(c, k_hh_tail, blocks, HH_THREADS, hh_tail_smem(nrestart), a, jj);
      }
      Probe p;
      probe(p);
      curres = p.curres;
      if (p.flag[0]) {
        broke = true;
        j = p.flag[1];
        break;
      }
      j = jend;
      chunk *= 2;
    }
    guard.release();
    const int64_t steps = broke ? j + 1 : nrestart;
    res.iters += steps;
    res.matvecs += steps;
    int64_t ni;
    if (!broke) {
      j = nrestart - 1;
      ni = nrestart;
    } else {
      ni = j + 1;
    }
    launch(c, k_hh_correct, blocks, HH_THREADS, hh_correct_smem(nrestart), a, j, ni);
    if (curres < tol) break;
  }
  res.relres = curres;
  return res;
}

// Self-test of the bounded grid barrier: block 1 never arrives, so block 0
// waits until its (small) poll limit runs out and raises *flag.
__global__ void k_selftest_grid_barrier(unsigned* bar, int* flag, long long limit) {
  if (blockIdx.x != 0) return;
  grid_barrier(blockIdx, gridDim, bar, flag, limit);
}

void selftest_wait_gmres(Context* c, int* flag, long long limit) {
  DBuf<unsigned> bar(c, 2);
  TTG_CUDA(cudaMemsetAsync(bar.p(), 0, 2 * sizeof(unsigned), c->stream));
  k_selftest_grid_barrier<<<2, 32, 0, c->stream>>>(bar.p(), flag, limit);
  TTG_CHECK_LAUNCH();
  sync(c);
}

}  // namespace ttg
