// hbx_flat.cpp -- BiCGSTAB with host vectors and one H-matvec per product
// (the "flat" solver of HACApK_SOLVER.c:254-417): vector updates and the
// sequential dot products (c_hacapk_dotp_d, HACApK_SOLVER.c:7-14) on the
// host, in the reference's statement order; each product y = H x is a call
// of `mv`.  Host-only, so the loop can be checked without a GPU.
#include "hbx_flat.h"

#include "../../include/hacapk_b200.h"

#include <cmath>
#include <cstdio>
#include <vector>

namespace hbx {

int flat_bicgstab(int n, double *u, const double *b, double eps, int mstep, int verbose, FlatMatvec mv,
                  void *ctx, int *status) {
  std::vector<double> zr(n), zshdw(n), zp(n), zt(n), zkp(n), zakp(n), zkt(n), zakt(n);
  auto dot = [n](const double *x, const double *y) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
  };
  auto apply = [&](const double *x, double *y) {
    int rc = mv(ctx, x, y);
    if (rc != 0 && status && *status == 0) *status = rc;
  };
  double alpha = 0.0, beta = 0.0, zeta = 0.0, znorm, zden, znormold = 1.0;
  const double bnorm = std::sqrt(dot(b, b));
  for (int i = 0; i < n; ++i) zr[i] = b[i];
  apply(u, zshdw.data());
  for (int i = 0; i < n; ++i) zr[i] = zr[i] - zshdw[i];
  zshdw = zr;
  double zrnorm = std::sqrt(dot(zr.data(), zr.data()));
  int steps = 0;
  for (int step = 1; step <= mstep; ++step) {
    if (zrnorm / bnorm < eps) break;
    if (beta == 0.0) {
      zp = zr;
    } else {
      for (int i = 0; i < n; ++i) zp[i] = zp[i] + zeta * zakp[i];
      for (int i = 0; i < n; ++i) zp[i] = zp[i] * beta;
      for (int i = 0; i < n; ++i) zp[i] = zp[i] + zr[i];
    }
    zkp = zp;
    apply(zkp.data(), zakp.data());
    znorm = dot(zshdw.data(), zr.data());
    zden = dot(zshdw.data(), zakp.data());
    alpha = -znorm / zden;
    if (!std::isfinite(alpha)) {  // r^.Ap zero (HACApK_SOLVER.c:349 divides unchecked): stop, u kept
      if (status && *status == 0) *status = HBX_ERR_BREAKDOWN;
      break;
    }
    znormold = znorm;
    for (int i = 0; i < n; ++i) zt[i] = zr[i] + alpha * zakp[i];
    alpha = -alpha;
    zkt = zt;
    apply(zkt.data(), zakt.data());
    znorm = dot(zakt.data(), zt.data());
    zden = dot(zakt.data(), zakt.data());
    zeta = znorm / zden;
    if (!std::isfinite(zeta)) {  // At.At zero (HACApK_SOLVER.c:366): stop, u kept
      if (status && *status == 0) *status = HBX_ERR_BREAKDOWN;
      break;
    }
    for (int i = 0; i < n; ++i) u[i] = u[i] + alpha * zkp[i];
    for (int i = 0; i < n; ++i) u[i] = u[i] + zeta * zkt[i];
    zeta = -zeta;
    for (int i = 0; i < n; ++i) zr[i] = zt[i] + zeta * zakt[i];
    beta = dot(zshdw.data(), zr.data());
    zrnorm = std::sqrt(dot(zr.data(), zr.data()));
    beta = -alpha / zeta * beta / znormold;
    steps = step;
    if (verbose > 0) std::printf(" %d: log10(zrnorm/bnorm)=%.2e\n", step, std::log10(zrnorm / bnorm));
  }
  return steps;
}

}  // namespace hbx

extern "C" int hbx_test_flat_bicgstab(int n, double *u, const double *b, double eps, int mstep,
                                      hbx::FlatMatvec mv, void *ctx) {
  int st = 0;
  return hbx::flat_bicgstab(n, u, b, eps, mstep, 0, mv, ctx, &st);
}
