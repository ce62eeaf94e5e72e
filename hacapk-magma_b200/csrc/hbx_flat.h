// hbx_flat.h -- host BiCGSTAB loop of the flat drop-in solver.
#pragma once

namespace hbx {

// y = H x; returns 0 or an hbx_status.
typedef int (*FlatMatvec)(void *ctx, const double *x, double *y);

// HACApK_SOLVER.c:254-417 with host vectors; u is x0 in / solution out.
// Returns the number of steps; the first non-zero matvec status is stored
// in *status.
int flat_bicgstab(int n, double *u, const double *b, double eps, int mstep, int verbose, FlatMatvec mv,
                  void *ctx, int *status);

}  // namespace hbx
