// BF16 tcgen05 local matvec (mixed-precision path).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>

#include "local_ops.h"

namespace ttg {

// One local operator (Phi1, A_k, Phi2) converted to BF16 K-major operands,
// with its scratch intermediates and TMA descriptors.  apply() maps a vector
// in the reversed layout v[k + rx2*(j + n*i)] (FP32) to y in the same layout.
struct MixedOp {
  MvDims d{};
  int64_t ldx = 0, ld1 = 0, ld2 = 0;
  int bn1 = 128, bn2 = 128, bn3 = 128;
  DBuf<__nv_bfloat16> phi2b, AT, phi1T, X, T1, T2;
  CUtensorMap mapX, mapP2, mapT1, mapAT, mapT2, mapP1;
  void prepare(Context* c, const MvDims& d, const double* Phi1, const double* A,
               const double* Phi2);
  void apply(Context* c, const float* v, float* y);
  // Same with X already holding the BF16 operand (written by the Arnoldi
  // kernels of the Krylov solver).
  void apply_converted(Context* c, float* y);
  // One GEMM stage (1, 2, 3) with tile width bn and B-operand map mapB;
  // stage 3 writes y.
  void run_stage(Context* c, int stage, int bn, const CUtensorMap& mapB, float* y);
  // Tile width of a stage: autotuned once per shape and device (mixed_ops.cu).
  int tuned_bn(Context* c, int stage);
  // Algorithmic DRAM bytes of one matvec: X (BF16), Phi2, A, Phi1 (BF16)
  // read once, y (FP32) written once.
  double bytes_per_matvec() const {
    return 2.0 * double(d.rx1) * d.m * d.rx2 +
           2.0 * (double(d.rx2) * d.ra2 * d.ry2 + double(d.ra1) * d.n * d.m * d.ra2 +
                  double(d.ry1) * d.rx1 * d.ra1) +
           4.0 * double(d.ry1) * d.n * d.ry2;
  }
  // The three GEMM stages from X to y, with the matvec counters: three GEMM
  // launches (default) or one fused persistent launch (TTG_FUSED_MV=1).
  void stages(Context* c, float* y);
  // Fused single-launch form: tile widths and B-operand maps per stage.
  int fbn[3] = {64, 64, 64};
  CUtensorMap fmapB[3];
  int fblocks = 0;
  DBuf<unsigned> fbar;
  void prepare_fused(Context* c);
  void stages_fused(Context* c, float* y);
};

// C (M x N, ld ldc, FP64) = op(A) op(B) on the BF16 tensor cores with FP32
// accumulation: FP64 operands converted to BF16 (K-major), one tcgen05
// GEMM, the FP32 result widened.  op(A) is M x K, op(B) K x N, column-major
// as gemm_f64.  The contractions of the mixed-precision rounding.
void gemm_bf16(Context* c, bool tA, bool tB, int64_t M, int64_t N, int64_t K, const double* A,
               int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc);

// Natural [i, j, k] FP64 <-> reversed [k, j, i] FP32 vector layouts.
void nat_to_rev(Context* c, int64_t r1, int64_t n, int64_t r2, const double* x, float* y,
                double scale);
// x[natural] += scale * y[reversed]
void rev_to_nat_add(Context* c, int64_t r1, int64_t n, int64_t r2, const float* y, double* x,
                    double scale);

}  // namespace ttg
