#pragma once
#include <vector>

#include "internal.h"

namespace ttg {
// Truncation rank of my_chop2 (core/my_chop2.m:18-35).
int64_t my_chop2(const double* sv, int64_t n, double eps);
// TT rounding of round.m:20-108; returns a new handle on the same context.
ttg_tt_s* round_tt(ttg_tt_s* in, double eps, const std::vector<int64_t>& rmax, int precision,
                   ttg_round_stats* stats);
}  // namespace ttg
