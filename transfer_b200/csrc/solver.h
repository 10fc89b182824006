// Solver entry points shared between solver.cu and the C ABI layer.
#pragma once
#include "internal.h"

namespace transfer {
tr_status ensure_workspace(tr_ctx *c, int hist_cap);
// Solve A f = b (b: device vector of the context's FP64 layout, or NULL
// for the computed right-hand side); f: device output.
tr_status solve(tr_ctx *c, const tr_solve_opts *o, const double *b, double *f, tr_solve_report *rep);
}  // namespace transfer
