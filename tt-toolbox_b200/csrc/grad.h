// Gradients of TT functionals with respect to every core (FP64).
#pragma once
#include "internal.h"

namespace ttg {

// f(x) = <x, A x>; grad has x's flat core layout; *value (device) = f.
void grad_xAx(Context* c, const ttg_tt_s* x, const ttg_tt_s* A, double* grad, double* value);

// f(x) = <x, b>.
void grad_xb(Context* c, const ttg_tt_s* x, const ttg_tt_s* b, double* grad, double* value);

// f(x) = sum_s (X[idx_s] - y_s)^2 with idx column-major [S x d], 0-based.
void grad_sampled(Context* c, const ttg_tt_s* x, int64_t S, const int* idx, const double* y,
                  double* grad, double* value);

}  // namespace ttg
