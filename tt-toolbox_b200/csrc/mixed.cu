// Mixed-precision local solve (placeholder until the tensor-core path lands).
#include "mixed.h"

namespace ttg {

LocalSolveResult local_solve_mixed(Context*, const MvDims&, const double*, const double*,
                                   const double*, const double*, double, const double*, int64_t,
                                   int64_t, double*) {
  fail(TTG_ERR_UNSUPPORTED, "precision TTG_MIXED is not available in this build");
}

}  // namespace ttg
