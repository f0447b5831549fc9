// BF16 tensor-core (tcgen05) local matvec for the mixed-precision path.
//
// y = (Phi1 x A x Phi2) x is three GEMMs (see local_ops.cu).  Here every
// operand is stored K-major in BF16 so that each stage is one tcgen05 GEMM
// fed by TMA (128-byte swizzle), accumulating in FP32 in tensor memory.  The
// layouts of the two intermediates are chosen by the epilogue of the stage
// that produces them, so no permutation pass runs between the stages:
//
//   vector layout ("reversed"): v[k + rx2*(j + n*i)]      (i: rx1, j: n, k: rx2)
//   stage 1  T1[(m,a),(be,k)] = X[(m,a), b] * Phi2[b,(be,k)]        K = rx2
//            X  = v as bf16 rows (m,a), K-major, ld ldx
//            T1 stored [(m,be) | ld1][a][k]  (K-major operand of stage 2)
//   stage 2  per k: T2_k[a,(al,j)] = T1_k[a,(m,be)] * AT[(al,j),(m,be)]  K = n*ra2
//            T2 stored [(a,al) | ld2][k][j]  (K-major operand of stage 3)
//   stage 3  y[(k,j), i] = T2[(k,j),(a,al)] * Phi1T[i,(a,al)]        K = rx1*ra1
//            written straight into the reversed vector layout (FP32).
//
// One CTA computes a 128 x BN tile: warp 0 issues TMA loads into a 3-stage
// shared-memory ring, one thread of warp 1 issues tcgen05.mma (M=128, N=BN,
// K=16) and commits to mbarriers, and all four warps drain the FP32
// accumulator from tensor memory (tcgen05.ld) in the epilogue.  All waits
// are bounded; a timeout sets the context error flag.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cstdlib>
#include <map>
#include <mutex>

#include "group.cuh"
#include "mixed_ops.h"
#include "umma.cuh"

namespace ttg {

namespace {

constexpr int UM_STAGES = 3;
constexpr int UM_BM = 128;
constexpr int UM_BK = 64;
constexpr int UM_A_BYTES = UM_BM * UM_BK * 2;

struct OutMap {
  void* base;
  int64_t M, N;            // valid extents per batch
  int64_t r_s1, r_t1, r_t2;
  int64_t c_s1, c_t1, c_t2;
  int64_t batch_stride;    // elements
};

__device__ __forceinline__ int64_t map2(int64_t i, int64_t s1, int64_t t1, int64_t t2) {
  return (i % s1) * t1 + (i / s1) * t2;
}

template <int BN>
constexpr size_t umma_smem_bytes() {
  return 1024 + size_t(UM_STAGES) * (UM_A_BYTES + BN * UM_BK * 2) + (2 * UM_STAGES + 1) * 8 + 16;
}

// Body of the BF16 GEMM tile kernel; the tensor maps are passed by address
// (kernel parameters of the plain launch, argument packs in global memory
// in a grouped launch).
template <int BN, bool OUT_BF16>
__device__ __forceinline__ void umma_body(TTG_BLOCK, const CUtensorMap* tmA,
                                          const CUtensorMap* tmB, int K, int a_rows_pb,
                                          int b_rows_pb, const OutMap& om, int* err,
                                          const int* skip) {
  pdl_begin();
  using namespace umma;
  if (skip && *skip) return;  // queued Krylov step after convergence
  constexpr int B_BYTES = BN * UM_BK * 2;
  constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + UM_STAGES * UM_A_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + UM_STAGES * B_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * UM_STAGES + 1);
  const uint32_t bar_full = smem_u32(bars);
  const uint32_t bar_empty = smem_u32(bars + UM_STAGES);
  const uint32_t bar_done = smem_u32(bars + 2 * UM_STAGES);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * UM_BM, n0 = blockIdx.y * BN, bz = blockIdx.z;
  const int nk = (K + UM_BK - 1) / UM_BK;

  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_slot), TMEM_COLS);
    tmem_relinquish();
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < UM_STAGES; ++s) {
      mbar_init(bar_full + 8 * s, 1);
      mbar_init(bar_empty + 8 * s, 1);
    }
    mbar_init(bar_done, 1);
    fence_barrier_init();
    fence_proxy_async();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // TMA producer.
    const int arow = bz * a_rows_pb + m0, brow = bz * b_rows_pb + n0;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % UM_STAGES;
      if (kb >= UM_STAGES) {
        if (!mbar_wait(bar_empty + 8 * s, ((kb / UM_STAGES) - 1) & 1, err)) break;
      }
      mbar_expect_tx(bar_full + 8 * s, UM_A_BYTES + B_BYTES);
      tma_load_2d(smem_u32(sA + s * UM_A_BYTES), tmA, kb * UM_BK, arow, bar_full + 8 * s);
      tma_load_2d(smem_u32(sB + s * B_BYTES), tmB, kb * UM_BK, brow, bar_full + 8 * s);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer.
    const uint32_t idesc = idesc_bf16_f32(UM_BM, BN);
    bool ok = true;
    for (int kb = 0; kb < nk && ok; ++kb) {
      const int s = kb % UM_STAGES;
      ok = mbar_wait(bar_full + 8 * s, (kb / UM_STAGES) & 1, err);
      if (!ok) break;
      tc_fence_after();
      const uint32_t a0 = smem_u32(sA + s * UM_A_BYTES), b0 = smem_u32(sB + s * B_BYTES);
#pragma unroll
      for (int kk = 0; kk < UM_BK / 16; ++kk) {
        mma_bf16(tmem, desc_k_sw128(a0 + kk * 32), desc_k_sw128(b0 + kk * 32), idesc,
                 (kb > 0 || kk > 0) ? 1u : 0u);
      }
      mma_commit(bar_empty + 8 * s);
    }
    mma_commit(bar_done);
  }
  __syncwarp();

  // Epilogue: warp w owns accumulator rows (TMEM lanes) 32w .. 32w+31.
  const bool ok = mbar_wait(bar_done, 0, err);
  tc_fence_after();
  if (ok) {
    const int row = warp * 32 + lane;
    const int64_t m = int64_t(m0) + row;
    const bool row_ok = m < om.M;
    const int64_t roff = row_ok ? map2(m, om.r_s1, om.r_t1, om.r_t2) : 0;
    const int64_t boff = int64_t(bz) * om.batch_stride;
    // Column offsets advance incrementally: (n % c_s1, n / c_s1) -> no
    // division per element.
    int64_t cq = (int64_t(n0)) / om.c_s1, cr = (int64_t(n0)) % om.c_s1;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      if (n0 + c0 >= om.N) break;  // uniform across the CTA
      float v[16];
      tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), v);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int64_t n = int64_t(n0) + c0 + j;
        if (row_ok && n < om.N) {
          const int64_t off = boff + roff + cr * om.c_t1 + cq * om.c_t2;
          if (OUT_BF16)
            static_cast<__nv_bfloat16*>(om.base)[off] = __float2bfloat16_rn(v[j]);
          else
            static_cast<float*>(om.base)[off] = v[j];
        }
        if (++cr == om.c_s1) {
          cr = 0;
          ++cq;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

template <int BN, bool OUT_BF16>
__global__ void __launch_bounds__(128, 1)
    k_umma_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                int K, int a_rows_pb, int b_rows_pb, OutMap om, int* err, const int* skip) {
  umma_body<BN, OUT_BF16>(blockIdx, gridDim, &tmA, &tmB, K, a_rows_pb, b_rows_pb, om, err,
                          skip);
}

// Grouped form: the argument packs (tensor maps first, 64-byte aligned) sit
// in global memory, written by the host-to-device copy before the launch.
using UmmaPack = Pack<CUtensorMap, CUtensorMap, int, int, int, OutMap, int*, const int*>;

template <int BN, bool OUT_BF16>
__global__ void __launch_bounds__(128, 1) k_umma_group(GroupArgs g) {
  uint3 b;
  dim3 gd;
  const uint32_t r = group_locate(g, b, gd);
  UmmaPack& p = *reinterpret_cast<UmmaPack*>(const_cast<char*>(g.packs) + size_t(r) * g.stride);
  // The staging buffer is reused flush after flush: take the maps as they
  // are now, not as the tensor-map proxy may have cached them earlier.
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&pk<0>(p))
               : "memory");
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&pk<1>(p))
               : "memory");
  umma_body<BN, OUT_BF16>(b, gd, &pk<0>(p), &pk<1>(p), pk<2>(p), pk<3>(p), pk<4>(p), pk<5>(p),
                          pk<6>(p), pk<7>(p));
}

template <int BN, bool OUT_BF16>
void umma_issue(const void* pack, dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl) {
  issue_plain<false, CUtensorMap, CUtensorMap, int, int, int, OutMap, int*, const int*>(
      reinterpret_cast<const void*>(&k_umma_gemm<BN, OUT_BF16>), pack, grid, block, smem, s,
      pdl);
}

template <int BN, bool OUT_BF16>
const GroupInfo* umma_info() {
  static const GroupInfo gi{reinterpret_cast<const void*>(&k_umma_gemm<BN, OUT_BF16>),
                            reinterpret_cast<const void*>(&k_umma_group<BN, OUT_BF16>), false,
                            uint32_t(sizeof(UmmaPack)), uint32_t(alignof(UmmaPack)),
                            &umma_issue<BN, OUT_BF16>};
  return &gi;
}

// ---------------------------------------------------------------------------
// Fused local matvec: the three GEMM stages in ONE persistent launch.
//
// One CTA per SM (cooperative launch, so all CTAs are resident) walks the
// output tiles of stage 1, then -- after a grid-wide barrier that makes the
// stage's T1 writes visible -- those of stage 2, then of stage 3.  T1 and T2
// (a few MB) are written by one stage and read by the next inside the same
// launch, so they stay in L2: DRAM sees the operands and y only.  Roles:
// warp 0 issues TMA loads into a FU_STAGES-deep shared-memory ring (across
// tile and stage boundaries), one thread of warp 1 issues tcgen05.mma into
// one of two TMEM accumulators, warps 2-9 drain the other accumulator
// (tcgen05.ld) and store it in the next stage's K-major layout.  Two CTAs
// fit on an SM (shared memory and TMEM).  Every wait
// is bounded: a timeout raises the error flag and every role winds down.
// ---------------------------------------------------------------------------

constexpr int FU_STAGES = 3;
constexpr int FU_BN_MAX = 128;
// warp 0 TMA, warp 1 MMA, warps 2-9 drain the accumulator: two warps per
// TMEM lane quarter, each taking every other 16-column chunk.
constexpr int FU_THREADS = 320;
constexpr int FU_EPI_WARPS = 8;
constexpr int FU_B_BYTES = FU_BN_MAX * UM_BK * 2;
constexpr uint32_t FU_TMEM_COLS = 2 * FU_BN_MAX;
constexpr long long FU_BAR_SPIN_LIMIT = 1LL << 24;

constexpr size_t fused_smem_bytes() {
  return 1024 + size_t(FU_STAGES) * (UM_A_BYTES + FU_B_BYTES) + (2 * FU_STAGES + 4) * 8 + 64;
}

struct FusedStage {
  OutMap om;
  int K, a_rows_pb, b_rows_pb;
  int mt, nt, batch;  // tiles: M tiles of 128 rows, N tiles of bn columns, batches
  int bn;             // 64 or 128
  int out_bf16;
};

struct FusedArgs {
  FusedStage st[3];
  unsigned* bar;      // grid barrier: arrival counter, generation
  int* err;
  const int* skip;
};

// Generation barrier over the grid (all CTAs resident: cooperative launch);
// bounded, the waiting thread gives up and raises *err.
__device__ void fu_grid_barrier(unsigned* bar, int* err) {
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
        if (++spins > FU_BAR_SPIN_LIMIT) {
          atomicExch(err, 7);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
}

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__global__ void __launch_bounds__(FU_THREADS, 2)
    k_mv_fused(const __grid_constant__ CUtensorMap tA1, const __grid_constant__ CUtensorMap tB1,
               const __grid_constant__ CUtensorMap tA2, const __grid_constant__ CUtensorMap tB2,
               const __grid_constant__ CUtensorMap tA3, const __grid_constant__ CUtensorMap tB3,
               const __grid_constant__ FusedArgs fa) {
  using namespace umma;
  if (fa.skip && *fa.skip) return;  // queued Krylov step after convergence (uniform)
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + FU_STAGES * UM_A_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + FU_STAGES * FU_B_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * FU_STAGES + 4);
  uint32_t* consumed_slot = tmem_slot + 1;
  const uint32_t bar_full = smem_u32(bars);
  const uint32_t bar_empty = smem_u32(bars + FU_STAGES);
  const uint32_t bar_accf = smem_u32(bars + 2 * FU_STAGES);      // 2: accumulator ready
  const uint32_t bar_acce = smem_u32(bars + 2 * FU_STAGES + 2);  // 2: accumulator drained
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* err = fa.err;

  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_slot), FU_TMEM_COLS);
    tmem_relinquish();
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < FU_STAGES; ++s) {
      mbar_init(bar_full + 8 * s, 1);
      mbar_init(bar_empty + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(bar_accf + 8 * b, 1);
      mbar_init(bar_acce + 8 * b, FU_EPI_WARPS);  // one arrival per epilogue warp
    }
    fence_barrier_init();
    fence_proxy_async();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // Counters advance identically in the roles that share a barrier ring.
  uint32_t kb_cnt = 0;    // K-blocks issued (producer) / consumed (MMA)
  uint32_t tile_cnt = 0;  // tiles accumulated (MMA) / drained (epilogue)
  for (int s = 0; s < 3; ++s) {
    const FusedStage& S = fa.st[s];
    const CUtensorMap* tA = s == 0 ? &tA1 : (s == 1 ? &tA2 : &tA3);
    const CUtensorMap* tB = s == 0 ? &tB1 : (s == 1 ? &tB2 : &tB3);
    const int ntiles = S.mt * S.nt * S.batch;
    const int nk = (S.K + UM_BK - 1) / UM_BK;
    const uint32_t b_bytes = uint32_t(S.bn) * UM_BK * 2;
    if (warp == 0) {
      if (lane == 0) {  // TMA producer
        if (s > 0) fence_proxy_async_global();  // the previous stage's stores, seen by TMA
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
          const int mi = t % S.mt, rest = t / S.mt, ni = rest % S.nt, bz = rest / S.nt;
          const int arow = bz * S.a_rows_pb + mi * UM_BM, brow = bz * S.b_rows_pb + ni * S.bn;
          for (int kb = 0; kb < nk; ++kb, ++kb_cnt) {
            const uint32_t slot = kb_cnt % FU_STAGES;
            if (kb_cnt >= FU_STAGES &&
                !mbar_wait(bar_empty + 8 * slot, ((kb_cnt / FU_STAGES) - 1) & 1, err)) {
              ok = false;
              break;
            }
            mbar_expect_tx(bar_full + 8 * slot, UM_A_BYTES + b_bytes);
            tma_load_2d(smem_u32(sA + slot * UM_A_BYTES), tA, kb * UM_BK, arow,
                        bar_full + 8 * slot);
            tma_load_2d(smem_u32(sB + slot * FU_B_BYTES), tB, kb * UM_BK, brow,
                        bar_full + 8 * slot);
          }
        }
      }
      __syncwarp();
    } else if (warp == 1) {
      if (lane == 0) {  // MMA issuer
        const uint32_t idesc = idesc_bf16_f32(UM_BM, S.bn);
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++tile_cnt) {
          const uint32_t buf = tile_cnt & 1;
          if (tile_cnt >= 2 && !mbar_wait(bar_acce + 8 * buf, ((tile_cnt >> 1) - 1) & 1, err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t tacc = tmem + buf * FU_BN_MAX;
          for (int kb = 0; kb < nk; ++kb, ++kb_cnt) {
            const uint32_t slot = kb_cnt % FU_STAGES;
            if (!mbar_wait(bar_full + 8 * slot, (kb_cnt / FU_STAGES) & 1, err)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA + slot * UM_A_BYTES);
            const uint32_t b0 = smem_u32(sB + slot * FU_B_BYTES);
#pragma unroll
            for (int kk = 0; kk < UM_BK / 16; ++kk)
              mma_bf16(tacc, desc_k_sw128(a0 + kk * 32), desc_k_sw128(b0 + kk * 32), idesc,
                       (kb > 0 || kk > 0) ? 1u : 0u);
            mma_commit(bar_empty + 8 * slot);
          }
          if (ok) mma_commit(bar_accf + 8 * buf);
        }
        *consumed_slot = kb_cnt;
      }
      __syncwarp();
    } else {  // epilogue: warp w owns TMEM lanes 32 (w % 4) .., column half (w - 2) / 4
      const int ew = warp & 3;
      const int half = (warp - 2) >> 2;
      const int row = ew * 32 + lane;
      const OutMap& om = S.om;
      for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tile_cnt) {
        const uint32_t buf = tile_cnt & 1;
        const bool ok = mbar_wait(bar_accf + 8 * buf, (tile_cnt >> 1) & 1, err);
        tc_fence_after();
        if (!ok) break;
        const int mi = t % S.mt, rest = t / S.mt, ni = rest % S.nt, bz = rest / S.nt;
        const int m0 = mi * UM_BM, n0 = ni * S.bn;
        const int64_t m = int64_t(m0) + row;
        const bool row_ok = m < om.M;
        const int64_t roff = row_ok ? map2(m, om.r_s1, om.r_t1, om.r_t2) : 0;
        const int64_t boff = int64_t(bz) * om.batch_stride;
        const uint32_t tbase = tmem + (uint32_t(ew * 32) << 16) + buf * FU_BN_MAX;
#pragma unroll 1
        for (int c0 = 16 * half; c0 < S.bn; c0 += 32) {
          if (n0 + c0 >= om.N) break;  // uniform across the warp
          float v[16];
          tmem_ld16(tbase + uint32_t(c0), v);
          int64_t cq = int64_t(n0 + c0) / om.c_s1, cr = int64_t(n0 + c0) % om.c_s1;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int64_t n = int64_t(n0) + c0 + j;
            if (row_ok && n < om.N) {
              const int64_t off = boff + roff + cr * om.c_t1 + cq * om.c_t2;
              if (S.out_bf16)
                static_cast<__nv_bfloat16*>(om.base)[off] = __float2bfloat16_rn(v[j]);
              else
                static_cast<float*>(om.base)[off] = v[j];
            }
            if (++cr == om.c_s1) {
              cr = 0;
              ++cq;
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar_acce + 8 * buf);
      }
      if (s < 2) fence_proxy_async_global();  // this stage's stores, for the next TMA loads
    }
    if (s < 2) {
      __syncthreads();
      fu_grid_barrier(fa.bar, err);
      __syncthreads();
    }
  }
  __syncthreads();
  // Wind-down after an error: loads issued but never consumed must land
  // before the CTA (and its shared memory) goes away.  Bounded.
  if (threadIdx.x == 0 && *(volatile int*)err) {
    for (uint32_t k = *consumed_slot; k < kb_cnt; ++k)
      mbar_wait(bar_full + 8 * (k % FU_STAGES), (k / FU_STAGES) & 1, err, 1 << 16);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, FU_TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// Operand conversion kernels (FP64/FP32 -> BF16, K-major layouts)
// ---------------------------------------------------------------------------

// Phi2b[b + ldp*col] = Phi2[b, col], col = (be, k)  (zero padding b >= rx2)
TTG_BODY(k_cvt_phi2)(TTG_BLOCK, int64_t rx2, int64_t ncols, int64_t ldp, const double* __restrict__ P,
                           __nv_bfloat16* __restrict__ out) {
  pdl_begin();
  const int64_t total = ldp * ncols;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e % ldp, col = e / ldp;
    out[e] = __float2bfloat16_rn(b < rx2 ? float(P[b + rx2 * col]) : 0.f);
  }
}
TTG_KERNEL(k_cvt_phi2, 0);

// AT[(m + n*be) + ld1*(al + ra1*j)] = A[al, j, m, be]
TTG_BODY(k_cvt_AT)(TTG_BLOCK, int64_t ra1, int64_t n, int64_t ra2, int64_t ld1,
                         const double* __restrict__ A, __nv_bfloat16* __restrict__ out) {
  pdl_begin();
  const int64_t total = ld1 * ra1 * n;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t kk = e % ld1, row = e / ld1;
    float v = 0.f;
    if (kk < n * ra2) {
      const int64_t mm = kk % n, be = kk / n, al = row % ra1, j = row / ra1;
      v = float(A[al + ra1 * (j + n * (mm + n * be))]);
    }
    out[e] = __float2bfloat16_rn(v);
  }
}
TTG_KERNEL(k_cvt_AT, 0);

// Phi1T[(a + rx1*al) + ld2*i] = Phi1[i, a, al]
TTG_BODY(k_cvt_phi1)(TTG_BLOCK, int64_t ry1, int64_t rx1, int64_t ra1, int64_t ld2,
                           const double* __restrict__ P, __nv_bfloat16* __restrict__ out) {
  pdl_begin();
  const int64_t total = ld2 * ry1;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t kk = e % ld2, i = e / ld2;
    float v = 0.f;
    if (kk < rx1 * ra1) {
      const int64_t a = kk % rx1, al = kk / rx1;
      v = float(P[i + ry1 * (a + rx1 * al)]);
    }
    out[e] = __float2bfloat16_rn(v);
  }
}
TTG_KERNEL(k_cvt_phi1, 0);

// X[b + ldx*row] = v[b + rx2*row]  (row = m + n*a; zero padding)
TTG_BODY(k_cvt_x)(TTG_BLOCK, int64_t rx2, int64_t rows, int64_t ldx, const float* __restrict__ v,
                        __nv_bfloat16* __restrict__ out, const int* skip) {
  pdl_begin();
  if (skip && *skip) return;
  const int64_t total = ldx * rows;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = e % ldx, row = e / ldx;
    out[e] = __float2bfloat16_rn(b < rx2 ? v[b + rx2 * row] : 0.f);
  }
}
TTG_KERNEL(k_cvt_x, 0);

// Natural [i, j, k] (FP64) <-> reversed [k, j, i] (FP32) vector layouts.
TTG_BODY(k_nat_to_rev)(TTG_BLOCK, int64_t r1, int64_t n, int64_t r2, const double* __restrict__ x,
                             float* __restrict__ y, double scale) {
  pdl_begin();
  const int64_t total = r1 * n * r2;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t k = e % r2, j = (e / r2) % n, i = e / (r2 * n);
    y[e] = float(x[i + r1 * (j + n * k)] * scale);
  }
}
TTG_KERNEL(k_nat_to_rev, 0);

TTG_BODY(k_rev_to_nat_add)(TTG_BLOCK, int64_t r1, int64_t n, int64_t r2, const float* __restrict__ y,
                                 double* __restrict__ x, double scale) {
  pdl_begin();
  const int64_t total = r1 * n * r2;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e % r1, j = (e / r1) % n, k = e / (r1 * n);
    x[e] += scale * double(y[k + r2 * (j + n * i)]);
  }
}
TTG_KERNEL(k_rev_to_nat_add, 0);

int blocks_for(Context* c, int64_t n) {
  int64_t b = (n + 255) / 256;
  const int64_t cap = int64_t(c->num_sms) * 8;
  if (b > cap) b = cap;
  return int(b < 1 ? 1 : b);
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

void make_map(CUtensorMap* map, const void* ptr, int64_t K, int64_t rows, int64_t ld,
              int box_rows) {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!g_encode) fail(TTG_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  TTG_REQUIRE(ld % 8 == 0 && (reinterpret_cast<uintptr_t>(ptr) & 15) == 0,
              "TMA operand not 16-byte aligned");
  cuuint64_t gdim[2] = {cuuint64_t(K), cuuint64_t(rows)};
  cuuint64_t gstride[1] = {cuuint64_t(ld) * 2};
  cuuint32_t box[2] = {cuuint32_t(UM_BK), cuuint32_t(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), gdim,
                        gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(TTG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", int(r));
}

template <int BN, bool OB>
void launch_bn(Context* c, const CUtensorMap& ta, const CUtensorMap& tb, int64_t K,
               int64_t a_rows_pb, int64_t b_rows_pb, int64_t M, int64_t N, int64_t batch,
               const OutMap& om) {
  const size_t smem = umma_smem_bytes<BN>();
  ensure_smem_attr(reinterpret_cast<const void*>(k_umma_gemm<BN, OB>), c->device, int(smem));
  dim3 grid{unsigned((M + UM_BM - 1) / UM_BM), unsigned((N + BN - 1) / BN), unsigned(batch)};
  if (c->rec) {  // grouped batch: one record of the grouped GEMM
    UmmaPack p{};
    fill_pack(p, std::index_sequence_for<CUtensorMap, CUtensorMap, int, int, int, OutMap, int*,
                                         const int*>{},
              ta, tb, int(K), int(a_rows_pb), int(b_rows_pb), om, c->d_err + 1, c->skip);
    rec_group(c->rec, umma_info<BN, OB>(), grid, 128, smem, &p);
    rec_note_flop(c->rec, 2.0 * double(M) * double(N) * double(K) * double(batch));
    c->launches += 1;
    return;
  }
  launch(c, k_umma_gemm<BN, OB>, grid, 128, smem, ta, tb, int(K), int(a_rows_pb),
         int(b_rows_pb), om, c->d_err + 1, c->skip);
  TTG_CHECK_LAUNCH();
}

void umma_gemm(Context* c, const CUtensorMap& ta, const CUtensorMap& tb, int64_t K,
               int64_t a_rows_pb, int64_t b_rows_pb, int64_t M, int64_t N, int64_t batch,
               const OutMap& om, bool out_bf16, int bn) {
  TTG_REQUIRE(M < (1ll << 31) && N < (1ll << 31) && batch <= 65535, "umma gemm too large");
  if (out_bf16) {
    if (bn == 64) launch_bn<64, true>(c, ta, tb, K, a_rows_pb, b_rows_pb, M, N, batch, om);
    else if (bn == 128) launch_bn<128, true>(c, ta, tb, K, a_rows_pb, b_rows_pb, M, N, batch, om);
    else launch_bn<256, true>(c, ta, tb, K, a_rows_pb, b_rows_pb, M, N, batch, om);
  } else {
    if (bn == 64) launch_bn<64, false>(c, ta, tb, K, a_rows_pb, b_rows_pb, M, N, batch, om);
    else if (bn == 128) launch_bn<128, false>(c, ta, tb, K, a_rows_pb, b_rows_pb, M, N, batch, om);
    else launch_bn<256, false>(c, ta, tb, K, a_rows_pb, b_rows_pb, M, N, batch, om);
  }
}

// Tile width: the narrowest that keeps the grid within a few waves.  The
// local matvec's GEMMs are small (tens of CTAs at the widest tile), so
// narrower tiles mean more CTAs in flight, a shorter per-CTA epilogue and
// less shared memory per CTA (several CTAs per SM).
int pick_bn(Context* c, int64_t M, int64_t N, int64_t batch) {
  const int64_t mt = (M + UM_BM - 1) / UM_BM;
  for (int bn : {64, 128}) {
    if (N <= bn) return bn;
    if (mt * ((N + bn - 1) / bn) * batch <= 4 * int64_t(c->num_sms)) return bn;
  }
  return 256;
}

int64_t up8(int64_t v) { return (v + 7) / 8 * 8; }

// TTG_FUSED_MV=1 selects the single-launch persistent local matvec.  The
// three-launch form is the default: on the solve's local systems it is
// faster (22.8 us against 25.8 us per matvec on average in the d = 10,
// n = 64, rmax 128 anisotropic solve, each CTA of the three GEMMs draining one tile while the fused
// kernel's CTAs drain several in turn), while the fused form keeps T1/T2
// out of DRAM.
bool fused_enabled() {
  static const bool on = [] {
    const char* e = getenv("TTG_FUSED_MV");
    return e && e[0] == '1';
  }();
  return on;
}


}  // namespace

void MixedOp::prepare(Context* c, const MvDims& dd, const double* Phi1, const double* A,
                      const double* Phi2) {
  d = dd;
  TTG_REQUIRE(d.n == d.m, "mixed matvec needs square A cores");
  ldx = up8(d.rx2);
  ld1 = up8(d.n * d.ra2);
  ld2 = up8(d.rx1 * d.ra1);
  TTG_REQUIRE(d.n * d.rx1 < (1ll << 31) && d.rx1 * d.ry2 < (1ll << 31), "mixed matvec too large");
  phi2b.reset(c, ldx * d.ra2 * d.ry2);
  AT.reset(c, ld1 * d.ra1 * d.n);
  phi1T.reset(c, ld2 * d.ry1);
  X.reset(c, ldx * d.m * d.rx1);
  // Padding columns (b >= rx2) must read as zero: the Krylov kernels write
  // only the valid part of X.
  if (ldx != d.rx2) memset_async(c, X.p(), 0, sizeof(__nv_bfloat16) * X.size());
  T1.reset(c, ld1 * d.rx1 * d.ry2);
  T2.reset(c, ld2 * d.ry2 * d.n);
  launch(c, k_cvt_phi2, blocks_for(c, phi2b.size()), 256, 0, d.rx2, d.ra2 * d.ry2, ldx, Phi2,
         phi2b.p());
  launch(c, k_cvt_AT, blocks_for(c, AT.size()), 256, 0, d.ra1, d.n, d.ra2, ld1, A, AT.p());
  launch(c, k_cvt_phi1, blocks_for(c, phi1T.size()), 256, 0, d.ry1, d.rx1, d.ra1, ld2, Phi1,
         phi1T.p());
  TTG_CHECK_LAUNCH();
  make_map(&mapX, X.p(), d.rx2, d.m * d.rx1, ldx, UM_BM);
  make_map(&mapT1, T1.p(), d.n * d.ra2, d.rx1 * d.ry2, ld1, UM_BM);
  make_map(&mapT2, T2.p(), d.rx1 * d.ra1, d.ry2 * d.n, ld2, UM_BM);
  if (fused_enabled() && !c->rec) {  // a grouped batch takes the three-launch form
    prepare_fused(c);
    return;
  }
  bn1 = tuned_bn(c, 1);
  bn2 = tuned_bn(c, 2);
  bn3 = tuned_bn(c, 3);
  make_map(&mapP2, phi2b.p(), d.rx2, d.ra2 * d.ry2, ldx, bn1);
  make_map(&mapAT, AT.p(), d.n * d.ra2, d.ra1 * d.n, ld1, bn2);
  make_map(&mapP1, phi1T.p(), d.rx1 * d.ra1, d.ry1, ld2, bn3);
}

// ---------------------------------------------------------------------------
// Tile-width autotuner
//
// The first time a stage shape (M, N, K, batch) is met on a device, each
// admissible tile width is timed with CUDA events on the context stream
// (one warm-up and three timed launches, on the operands just converted and
// whatever the intermediates hold -- the values do not change the work) and
// the fastest is kept for the life of the process.  The width only decides
// which CTA computes which output columns; every output element is still
// the same K-ordered sequence of MMA steps.  TTG_AUTOTUNE=0 turns tuning off
// (the CTA-count heuristic pick_bn is used instead), e.g. for runs that must
// repeat the same launch configuration.
// ---------------------------------------------------------------------------

namespace {

struct TuneKey {
  int device, stage;
  int64_t M, N, K, batch;
  bool operator<(const TuneKey& o) const {
    if (device != o.device) return device < o.device;
    if (stage != o.stage) return stage < o.stage;
    if (M != o.M) return M < o.M;
    if (N != o.N) return N < o.N;
    if (K != o.K) return K < o.K;
    return batch < o.batch;
  }
};

std::mutex g_tune_mu;
std::map<TuneKey, int> g_tuned;

bool autotune_enabled() {
  static const bool on = [] {
    const char* e = getenv("TTG_AUTOTUNE");
    return !(e && e[0] == '0');
  }();
  return on;
}

}  // namespace

void MixedOp::run_stage(Context* c, int stage, int bn, const CUtensorMap& mapB, float* y) {
  const int64_t rows = d.m * d.rx1;
  if (stage == 1) {
    OutMap o1{T1.p(), rows, d.ra2 * d.ry2, d.m, 1, ld1, d.ra2, d.m, ld1 * d.rx1, 0};
    umma_gemm(c, mapX, mapB, d.rx2, 0, 0, rows, d.ra2 * d.ry2, 1, o1, true, bn);
  } else if (stage == 2) {
    OutMap o2{T2.p(), d.rx1, d.ra1 * d.n, d.rx1, 1, 0, d.ra1, d.rx1, ld2 * d.ry2, ld2};
    umma_gemm(c, mapT1, mapB, d.n * d.ra2, d.rx1, 0, d.rx1, d.ra1 * d.n, d.ry2, o2, true, bn);
  } else {
    const int64_t rows3 = d.ry2 * d.n;
    OutMap o3{y, rows3, d.ry1, rows3, 1, 0, d.ry1, rows3, 0, 0};
    umma_gemm(c, mapT2, mapB, d.rx1 * d.ra1, 0, 0, rows3, d.ry1, 1, o3, false, bn);
  }
}

int MixedOp::tuned_bn(Context* c, int stage) {
  int64_t M, N, K, batch = 1;
  if (stage == 1) {
    M = d.m * d.rx1; N = d.ra2 * d.ry2; K = d.rx2;
  } else if (stage == 2) {
    M = d.rx1; N = d.ra1 * d.n; K = d.n * d.ra2; batch = d.ry2;
  } else {
    M = d.ry2 * d.n; N = d.ry1; K = d.rx1 * d.ra1;
  }
  const int fallback = pick_bn(c, M, N, batch);
  if (!autotune_enabled() || c->skip) return fallback;
  const TuneKey key{c->device, stage, M, N, K, batch};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) return it->second;
  }
  if (c->rec) return fallback;  // recorded stream work cannot be timed
  DBuf<float> ysc;
  if (stage == 3) ysc.reset(c, d.ry2 * d.n * d.ry1);
  float best_ms = 1e30f;
  int best = fallback;
  cudaEvent_t e0, e1;
  TTG_CUDA(cudaEventCreate(&e0));
  TTG_CUDA(cudaEventCreate(&e1));
  for (int bn : {64, 128, 256}) {
    if (bn > 64 && bn / 2 >= N) break;  // wider tiles than N only waste columns
    CUtensorMap mb;
    if (stage == 1) make_map(&mb, phi2b.p(), d.rx2, N, ldx, bn);
    else if (stage == 2) make_map(&mb, AT.p(), K, N, ld1, bn);
    else make_map(&mb, phi1T.p(), K, N, ld2, bn);
    run_stage(c, stage, bn, mb, ysc.p());
    TTG_CUDA(cudaEventRecord(e0, c->stream));
    for (int rep = 0; rep < 3; ++rep) run_stage(c, stage, bn, mb, ysc.p());
    TTG_CUDA(cudaEventRecord(e1, c->stream));
    TTG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    TTG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best_ms) {
      best_ms = ms;
      best = bn;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tuned[key] = best;
  return best;
}

void MixedOp::apply(Context* c, const float* v, float* y) {
  MvTiming timing(c, 1);
  const int64_t rows = d.m * d.rx1;
  launch(c, k_cvt_x, blocks_for(c, ldx * rows), 256, 0, d.rx2, rows, ldx, v, X.p(), c->skip);
  TTG_CHECK_LAUNCH();
  stages(c, y);
}

void MixedOp::apply_converted(Context* c, float* y) {
  MvTiming timing(c, 1);
  stages(c, y);
}

void MixedOp::prepare_fused(Context* c) {
  // Tile width per stage: 128 columns when that still gives every SM a
  // tile, else 64 (more, shorter tiles).
  const int64_t M[3] = {d.m * d.rx1, d.rx1, d.ry2 * d.n};
  const int64_t N[3] = {d.ra2 * d.ry2, d.ra1 * d.n, d.ry1};
  const int64_t B[3] = {1, d.ry2, 1};
  int64_t most = 1;
  for (int s = 0; s < 3; ++s) {
    const int64_t mt = (M[s] + UM_BM - 1) / UM_BM;
    const int64_t t128 = mt * ((N[s] + 127) / 128) * B[s];
    fbn[s] = (N[s] > 64 && t128 >= c->num_sms) ? 128 : 64;
    most = std::max(most, mt * ((N[s] + fbn[s] - 1) / fbn[s]) * B[s]);
  }
  make_map(&fmapB[0], phi2b.p(), d.rx2, N[0], ldx, fbn[0]);
  make_map(&fmapB[1], AT.p(), d.n * d.ra2, N[1], ld1, fbn[1]);
  make_map(&fmapB[2], phi1T.p(), d.rx1 * d.ra1, N[2], ld2, fbn[2]);
  ensure_smem_attr(reinterpret_cast<const void*>(k_mv_fused), c->device,
                   int(fused_smem_bytes()));
  int occ = 0;
  TTG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mv_fused, FU_THREADS,
                                                         fused_smem_bytes()));
  TTG_REQUIRE(occ >= 1, "fused matvec: no resident CTA fits");
  fblocks = int(std::min<int64_t>(most, int64_t(c->num_sms) * occ));
  fbar.reset(c, 2);
  TTG_CUDA(cudaMemsetAsync(fbar.p(), 0, 2 * sizeof(unsigned), c->stream));
  TTG_REQUIRE(d.n * d.rx1 < (1ll << 31) && d.ry2 * d.n < (1ll << 31) && most < (1ll << 31),
              "fused matvec too large");
}

void MixedOp::stages_fused(Context* c, float* y) {
  const int64_t rows = d.m * d.rx1;
  FusedArgs fa{};
  const int64_t M[3] = {rows, d.rx1, d.ry2 * d.n};
  const int64_t N[3] = {d.ra2 * d.ry2, d.ra1 * d.n, d.ry1};
  const int64_t K[3] = {d.rx2, d.n * d.ra2, d.rx1 * d.ra1};
  const int64_t B[3] = {1, d.ry2, 1};
  fa.st[0].om = OutMap{T1.p(), rows, d.ra2 * d.ry2, d.m, 1, ld1, d.ra2, d.m, ld1 * d.rx1, 0};
  fa.st[1].om = OutMap{T2.p(), d.rx1, d.ra1 * d.n, d.rx1, 1, 0, d.ra1, d.rx1, ld2 * d.ry2, ld2};
  fa.st[2].om = OutMap{y, M[2], d.ry1, M[2], 1, 0, d.ry1, M[2], 0, 0};
  for (int s = 0; s < 3; ++s) {
    FusedStage& S = fa.st[s];
    S.K = int(K[s]);
    S.a_rows_pb = s == 1 ? int(d.rx1) : 0;
    S.b_rows_pb = 0;
    S.mt = int((M[s] + UM_BM - 1) / UM_BM);
    S.nt = int((N[s] + fbn[s] - 1) / fbn[s]);
    S.batch = int(B[s]);
    S.bn = fbn[s];
    S.out_bf16 = s < 2 ? 1 : 0;
  }
  fa.bar = fbar.p();
  fa.err = c->d_err + 1;
  fa.skip = c->skip;
  void* args[] = {(void*)&mapX, (void*)&fmapB[0], (void*)&mapT1, (void*)&fmapB[1],
                  (void*)&mapT2, (void*)&fmapB[2], (void*)&fa};
  TTG_CUDA(cudaLaunchCooperativeKernel((const void*)k_mv_fused, dim3(fblocks), dim3(FU_THREADS),
                                       args, fused_smem_bytes(), c->stream));
  c->launches += 1;
}

void MixedOp::stages(Context* c, float* y) {
  if (fblocks > 0) {
    stages_fused(c, y);  // T1, T2 and y in one launch
  } else {
    run_stage(c, 1, bn1, mapP2, y);  // T1[(m,a),(be,k)]
    run_stage(c, 2, bn2, mapAT, y);  // per k, T2_k[a,(al,j)]
    run_stage(c, 3, bn3, mapP1, y);  // y[(k,j), i] in the reversed vector layout
  }
  c->matvecs += 1;
  c->matvec_flops += int64_t(d.flops());
  c->mv_count[1] += 1;
  c->mv_flops[1] += d.flops();
  c->mv_bytes_lp += bytes_per_matvec();
}

namespace {
// out[kk + ldk * row] = bf16(src(row, kk)), zero for kk >= K, with
// src(row, kk) = src[row + ld * kk] (trans = 0) or src[kk + ld * row] (1).
TTG_BODY(k_cvt_kmajor)(TTG_BLOCK, int64_t rows, int64_t K, int64_t ldk, const double* __restrict__ src,
                             int64_t ld, int trans, __nv_bfloat16* __restrict__ out) {
  pdl_begin();
  const int64_t total = rows * ldk;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t kk = e % ldk, row = e / ldk;
    float v = 0.f;
    if (kk < K) v = float(trans ? src[kk + ld * row] : src[row + ld * kk]);
    out[e] = __float2bfloat16_rn(v);
  }
}
TTG_KERNEL(k_cvt_kmajor, 0);

// C[m + ldc n] = Cf[m + M n] (FP32 -> FP64)
TTG_BODY(k_f32_to_f64)(TTG_BLOCK, int64_t M, int64_t N, const float* __restrict__ Cf,
                             double* __restrict__ C, int64_t ldc) {
  pdl_begin();
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < M * N;
       e += int64_t(gridDim.x) * blockDim.x)
    C[(e % M) + ldc * (e / M)] = double(Cf[e]);
}
TTG_KERNEL(k_f32_to_f64, 0);
}  // namespace

void gemm_bf16(Context* c, bool tA, bool tB, int64_t M, int64_t N, int64_t K, const double* A,
               int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc) {
  TTG_REQUIRE(M >= 1 && N >= 1 && K >= 1 && M < (1ll << 31) && N < (1ll << 31),
              "bf16 gemm: sizes out of range");
  const int64_t ldk = up8(K);
  DBuf<__nv_bfloat16> Ab(c, ldk * M), Bb(c, ldk * N);
  DBuf<float> Cf(c, M * N);
  // A operand rows m: op(A)(m, kk); B operand rows n: op(B)(kk, n).
  launch(c, k_cvt_kmajor, blocks_for(c, ldk * M), 256, 0, M, K, ldk, A, lda, tA ? 1 : 0, Ab.p());
  launch(c, k_cvt_kmajor, blocks_for(c, ldk * N), 256, 0, N, K, ldk, B, ldb, tB ? 0 : 1, Bb.p());
  TTG_CHECK_LAUNCH();
  const int bn = pick_bn(c, M, N, 1);
  CUtensorMap mA, mB;
  make_map(&mA, Ab.p(), K, M, ldk, UM_BM);
  make_map(&mB, Bb.p(), K, N, ldk, bn);
  OutMap om{Cf.p(), M, N, M, 1, 0, N, M, 0, 0};
  umma_gemm(c, mA, mB, K, 0, 0, M, N, 1, om, false, bn);
  launch(c, k_f32_to_f64, blocks_for(c, M * N), 256, 0, M, N, Cf.p(), C, ldc);
  TTG_CHECK_LAUNCH();
}

void nat_to_rev(Context* c, int64_t r1, int64_t n, int64_t r2, const double* x, float* y,
                double scale) {
  launch(c, k_nat_to_rev, blocks_for(c, r1 * n * r2), 256, 0, r1, n, r2, x, y, scale);
  TTG_CHECK_LAUNCH();
}

void rev_to_nat_add(Context* c, int64_t r1, int64_t n, int64_t r2, const float* y, double* x,
                    double scale) {
  launch(c, k_rev_to_nat_add, blocks_for(c, r1 * n * r2), 256, 0, r1, n, r2, y, x, scale);
  TTG_CHECK_LAUNCH();
}

namespace {
// An mbarrier that expects one arrival which never comes: the bounded wait
// of the tcgen05 pipeline gives up after `limit` polls and raises *flag.
__global__ void k_selftest_mbar(int* flag, long long limit) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = umma::smem_u32(&bar);
  if (threadIdx.x == 0) {
    umma::mbar_init(b, 1);
    umma::fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) umma::mbar_wait(b, 0, flag, limit);
}
}  // namespace

void selftest_wait_mbarrier(Context* c, int* flag, long long limit) {
  k_selftest_mbar<<<1, 32, 0, c->stream>>>(flag, limit);
  TTG_CHECK_LAUNCH();
  sync(c);
}

}  // namespace ttg
