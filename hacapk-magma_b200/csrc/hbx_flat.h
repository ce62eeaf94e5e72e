// hbx_flat.h -- host BiCGSTAB loop of the flat drop-in solver.
#pragma once

namespace hbx {

// y = H x; returns 0 or an hbx_status.
typedef int (*FlatMatvec)(void *ctx, const double *x, double *y);

// HACApK_SOLVER.c:254-417 with host vectors; u is x0 in / solution out.
// Returns the number of steps; the first non-zero matvec status is stored
// in *status, or HBX_ERR_BREAKDOWN when alpha or zeta is not finite (the
// loop stops there and u keeps the last completed step).
int flat_bicgstab(int n, double *u, const double *b, double eps, int mstep, int verbose, FlatMatvec mv,
                  void *ctx, int *status);

}  // namespace hbx
