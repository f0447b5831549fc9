// Local operators of the AMEn inner loop.
#pragma once
#include "kernels.h"

namespace ttg {

// Sizes of one local matvec y = (Phi1 x A x Phi2) x  (amen_solve2.m:924-951).
//   Phi1 [ry1, rx1, ra1], A [ra1, n, m, ra2], Phi2 [rx2, ra2, ry2],
//   x [rx1, m, rx2] -> y [ry1, n, ry2].
struct MvDims {
  int64_t ry1, rx1, ra1, n, m, rx2, ra2, ry2;
  int64_t in_size() const { return rx1 * m * rx2; }
  int64_t out_size() const { return ry1 * n * ry2; }
  int64_t t1_size() const { return rx1 * m * ra2 * ry2; }
  int64_t t2_size() const { return rx1 * ra1 * n * ry2; }
  double flops() const {
    return 2.0 * (double(rx1) * m * ra2 * ry2 * rx2 + double(rx1) * ra1 * n * m * ra2 * ry2 +
                  double(ry1) * n * ry2 * rx1 * ra1);
  }
};

// FP64 local matvec; t1/t2 scratch of t1_size()/t2_size() doubles.
void local_matvec_f64(Context* c, const MvDims& d, const double* Phi1, const double* A,
                      const double* Phi2, const double* x, double* y, double* t1, double* t2);

// Same with scratch drawn from the context allocator.
void local_matvec_f64(Context* c, const MvDims& d, const double* Phi1, const double* A,
                      const double* Phi2, const double* x, double* y);

// compute_next_Phi (amen_solve2.m:834-920).  dir 0 = 'lr', 1 = 'rl'.
//   x [rx1, n, rx2], y [ry1, n, ry2], A [ra1, n, n, ra2] or nullptr.
//   'lr': Phi_prev [rx1, ry1, ra1] -> out [rx2, ry2, ra2]
//   'rl': Phi_prev [ry2, ra2, rx2] -> out [ry1, ra1, rx1]
// Returns the output element count.  Normalisation is done by the caller.
int64_t next_phi_f64(Context* c, int dir, int64_t rx1, int64_t n, int64_t rx2, int64_t ry1,
                     int64_t ry2, int64_t ra1, int64_t ra2, const double* Phi_prev,
                     const double* x, const double* A, const double* y, double* out);

// Dense local matrix B [(i,j,k),(a,m,b)] = sum Phi1[i,a,al] A[al,j,m,be] Phi2[b,be,k]
// (amen_solve2.m:472-480), N = rx1*n*rx2, column-major N x N.
void assemble_local_f64(Context* c, int64_t rx1, int64_t n, int64_t rx2, int64_t ra1,
                        int64_t ra2, const double* Phi1, const double* A, const double* Phi2,
                        double* B);

}  // namespace ttg
