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

// Images of rank-one terms under the local operator, for the candidate
// residuals of the truncation loop (amen_solve2.m:539-551): with the SVD
// sol = U diag(s) V^T, W[:, t] = s_k B (u_k v_k^T), k = k0 + t, t < cnt,
// where B = Phi1 x A x Phi2 (square local system, d.ry* = d.rx*).
// Because B is linear, rhs - B(U_r S_r V_r^T) = (rhs - B sol) + sum_{k>=r}
// W_k: every candidate residual follows from one contraction per rank-one
// term, 2 rx1 n ra2 (ra1 n + rx1 ra1 + rx2) flops each, instead of one full
// local matvec per candidate.  W: out_size() x cnt; scratch:
// rank1_scratch_size(d, cnt) doubles.  U: M x K (ldu), VT: K x rx2 (ldvt).
void rank1_images_f64(Context* c, const MvDims& d, const double* Phi1, const double* A,
                      const double* Phi2, const double* U, int64_t ldu, const double* VT,
                      int64_t ldvt, const double* s, int64_t k0, int64_t cnt, double* W,
                      double* scratch);
int64_t rank1_scratch_size(const MvDims& d, int64_t cnt);

// Running sums of candidate residuals: for b = 0..cnt-1,
//   R += W[:, cnt-1-b];  out[b] = ||R||      (R updated in place)
// deterministic two-kernel reduction.  part: cumulative_norms_part_size(c).
constexpr int CUMNORM_MAXC = 16;
void cumulative_norms_f64(Context* c, int64_t N, int64_t cnt, double* R, const double* W,
                          double* part, double* out);
int64_t cumulative_norms_part_size(Context* c);

}  // namespace ttg
