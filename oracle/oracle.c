/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference's
 * H-matvec and BiCGSTAB, used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the checker.  Nothing in the product
 * (hacapk-magma_b200/) links or calls this file.
 *
 *   orc_adot_lfmtx ........ HACApK_MAGMA.c:5-57 (zau += H zu, plain loops)
 *   orc_adot_lfmtx_blas ... HACApK_MAGMA.c:114-199 with the #define CPU
 *                           branch: one BLAS dgemv per leaf (:140-143,
 *                           :163-166, :184-187); dgemv is passed in by the
 *                           caller (OpenBLAS from scipy stands in for MKL)
 *   orc_adot_lfmtx_omp .... m_HACApK_solve.f90:203-253 (the "_hyp" form:
 *                           per-thread zaut accumulators, then summed),
 *                           OpenMP over leaves
 *   orc_adot_lfmtx_t ...... the transposed product zau += H^T zu: the same
 *                           loops with row/column roles and U/V swapped (the
 *                           reference has no transposed product; see
 *                           HACApK_BATCH_SORT.c:123, which only changes the
 *                           storage orientation of the same A*x)
 *   orc_bicgstab .......... HACApK_SOLVER.c:254-417 (c_hacapk_bicgstab_cax_
 *                           lfmtx_flat_), same statement order, with the
 *                           sequential dot c_hacapk_dotp_d (HACApK_SOLVER.c:7-14)
 *   orc_bicgstab_pipe ..... HACApK_SOLVER_PIPE.c:144-600 (pipelined BiCGSTAB,
 *                           version 1; _pipe2_ at :640 has the same arithmetic)
 *   orc_gcrm .............. m_HACApK_solve.f90:506-571 (HACApK_gcrm_lfmtx, GCR(m))
 *
 * The solvers take their product as a kind: the restated loops, the per-leaf
 * BLAS form, the OpenMP form, or an external zau += H zu function (the
 * reference's compiled c_hacapk_adot_body_lfmtx_, or a test's own product).
 *
 * Built with -ffp-contract=off.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <omp.h>

#include "../include/hacapk_b200.h"

typedef void (*dgemv_fn)(const char *trans, const int *m, const int *n, const double *alpha,
                         const double *a, const int *lda, const double *x, const int *incx,
                         const double *beta, double *y, const int *incy);

static const stc_HACApK_leafmtx *leaf_at(const stc_HACApK_leafmtxp *st, int ip) {
  return (const stc_HACApK_leafmtx *)((const char *)st->st_lf + (size_t)st->st_lf_stride * ip);
}

static const double *a2_of(const stc_HACApK_leafmtx *s) {
  return (const double *)((const char *)s->a1 + s->a1size);
}

/* HACApK_MAGMA.c:5-57 */
void orc_adot_lfmtx(double *zau, const stc_HACApK_leafmtxp *st, const double *zu, double *zbu) {
  const int nlf = st->nlf;
  for (int ip = 0; ip < nlf; ip++) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    const int ndl = s->ndl, ndt = s->ndt, nstrtl = s->nstrtl, nstrtt = s->nstrtt;
    if (s->ltmtx == 1) {
      const double *a2 = a2_of(s);
      const int kt = s->kt;
      for (int il = 0; il < kt; il++) {
        zbu[il] = 0.0;
        for (int it = 0; it < ndt; it++) zbu[il] += s->a1[it + il * ndt] * zu[it + nstrtt - 1];
      }
      for (int il = 0; il < kt; il++)
        for (int it = 0; it < ndl; it++) zau[it + nstrtl - 1] += a2[it + il * ndl] * zbu[il];
    } else if (s->ltmtx == 2) {
      for (int il = 0; il < ndl; il++)
        for (int it = 0; it < ndt; it++)
          zau[il + nstrtl - 1] += s->a1[it + il * ndt] * zu[it + nstrtt - 1];
    }
  }
}

/* HACApK_MAGMA.c:114-199, CPU branch (per-leaf dgemv). */
void orc_adot_lfmtx_blas(double *zau, const stc_HACApK_leafmtxp *st, const double *zu, double *zbu,
                         void *dgemv_ptr) {
  dgemv_fn dgemv = (dgemv_fn)dgemv_ptr;
  const int ione = 1;
  const double one = 1.0, zero = 0.0;
  for (int ip = 0; ip < st->nlf; ip++) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    int ndl = s->ndl, ndt = s->ndt, kt = s->kt;
    if (s->ltmtx == 1) {
      if (kt == 0) continue;
      dgemv("T", &ndt, &kt, &one, s->a1, &ndt, &zu[s->nstrtt - 1], &ione, &zero, zbu, &ione);
      dgemv("N", &ndl, &kt, &one, a2_of(s), &ndl, zbu, &ione, &one, &zau[s->nstrtl - 1], &ione);
    } else if (s->ltmtx == 2) {
      dgemv("T", &ndt, &ndl, &one, s->a1, &ndt, &zu[s->nstrtt - 1], &ione, &one,
            &zau[s->nstrtl - 1], &ione);
    }
  }
}

/* m_HACApK_solve.f90:203-253 with OpenMP threads over the leaf list: each
 * thread accumulates a private zaut, then the copies are added in thread
 * order (deterministic for a fixed thread count). */
void orc_adot_lfmtx_omp(double *zau, const stc_HACApK_leafmtxp *st, const double *zu, int nthreads) {
  const int nd = st->nd;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  double *zaut = (double *)calloc((size_t)nd * nthreads, sizeof(double));
  double *zbut = (double *)calloc((size_t)(st->ktmax > 0 ? st->ktmax : 1) * nthreads, sizeof(double));
#pragma omp parallel num_threads(nthreads)
  {
    const int th = omp_get_thread_num();
    double *za = zaut + (size_t)nd * th;
    double *zb = zbut + (size_t)(st->ktmax > 0 ? st->ktmax : 1) * th;
#pragma omp for schedule(dynamic, 16)
    for (int ip = 0; ip < st->nlf; ip++) {
      const stc_HACApK_leafmtx *s = leaf_at(st, ip);
      const int ndl = s->ndl, ndt = s->ndt, nl0 = s->nstrtl - 1, nt0 = s->nstrtt - 1;
      if (s->ltmtx == 1) {
        const double *a2 = a2_of(s);
        for (int il = 0; il < s->kt; il++) {
          double acc = 0.0;
          const double *v = s->a1 + (size_t)il * ndt;
          for (int it = 0; it < ndt; it++) acc += v[it] * zu[nt0 + it];
          zb[il] = acc;
        }
        for (int il = 0; il < s->kt; il++) {
          const double *u = a2 + (size_t)il * ndl;
          for (int it = 0; it < ndl; it++) za[nl0 + it] += u[it] * zb[il];
        }
      } else if (s->ltmtx == 2) {
        for (int il = 0; il < ndl; il++) {
          const double *a = s->a1 + (size_t)il * ndt;
          double acc = 0.0;
          for (int it = 0; it < ndt; it++) acc += a[it] * zu[nt0 + it];
          za[nl0 + il] += acc;
        }
      }
    }
  }
  for (int t = 0; t < nthreads; t++)
    for (int i = 0; i < nd; i++) zau[i] += zaut[(size_t)nd * t + i];
  free(zaut);
  free(zbut);
}

/* zau += H^T zu (row/column roles and U/V swapped). */
void orc_adot_lfmtx_t(double *zau, const stc_HACApK_leafmtxp *st, const double *zu, double *zbu) {
  for (int ip = 0; ip < st->nlf; ip++) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    const int ndl = s->ndl, ndt = s->ndt, nstrtl = s->nstrtl, nstrtt = s->nstrtt;
    if (s->ltmtx == 1) {
      const double *a2 = a2_of(s);
      for (int il = 0; il < s->kt; il++) {
        zbu[il] = 0.0;
        for (int it = 0; it < ndl; it++) zbu[il] += a2[it + il * ndl] * zu[it + nstrtl - 1];
      }
      for (int il = 0; il < s->kt; il++)
        for (int it = 0; it < ndt; it++) zau[it + nstrtt - 1] += s->a1[it + il * ndt] * zbu[il];
    } else if (s->ltmtx == 2) {
      for (int il = 0; il < ndl; il++)
        for (int it = 0; it < ndt; it++)
          zau[it + nstrtt - 1] += s->a1[it + il * ndt] * zu[il + nstrtl - 1];
    }
  }
}

/* HACApK_SOLVER.c:7-14 */
static double dotp_d(int nd, const double *b, const double *a) {
  double norm = 0.0;
  for (int ii = 0; ii < nd; ii++) norm += b[ii] * a[ii];
  return norm;
}
static void daxpy(int n, double a, const double *x, double *y) {
  for (int i = 0; i < n; i++) y[i] = y[i] + a * x[i];
}

enum { ORC_MV_REF = 0, ORC_MV_BLAS = 1, ORC_MV_OMP = 2, ORC_MV_EXTERNAL = 3 };

typedef void (*ext_matvec_fn)(double *zau, const stc_HACApK_leafmtxp *st, const double *zu, double *zbu);

typedef struct orc_mv {
  int kind;
  void *fn;          /* dgemv (BLAS) or an external zau += H zu function */
  const void *ext_st;/* container handed to the external function (its own layout) */
  int nthreads;
  double seconds;    /* accumulated matvec wall time */
  int count;
} orc_mv;

static double wall(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static void mv_apply(orc_mv *mv, double *zau, const stc_HACApK_leafmtxp *st, const double *zu, double *zbu) {
  double t0 = wall();
  switch (mv->kind) {
    case ORC_MV_BLAS: orc_adot_lfmtx_blas(zau, st, zu, zbu, mv->fn); break;
    case ORC_MV_OMP: orc_adot_lfmtx_omp(zau, st, zu, mv->nthreads); break;
    case ORC_MV_EXTERNAL: ((ext_matvec_fn)mv->fn)(zau, (const stc_HACApK_leafmtxp *)mv->ext_st, zu, zbu); break;
    default: orc_adot_lfmtx(zau, st, zu, zbu); break;
  }
  mv->seconds += wall() - t0;
  mv->count++;
}

/* HACApK_SOLVER.c:254-417.  u: x0 in / solution out.  For mv_kind ==
 * ORC_MV_EXTERNAL the matvec mv_fn is called with ext_st as its container.  hist[0..nstp] receives
 * ||r||/||b|| (hist may be NULL).  Returns the number of steps (nstp). */
int orc_bicgstab(const stc_HACApK_leafmtxp *st, int nd, double *u, const double *b, double eps,
                 int mstep, int mv_kind, void *mv_fn, const void *ext_st, int nthreads,
                 double *hist, double *matvec_seconds) {
  orc_mv mv = {mv_kind, mv_fn, ext_st, nthreads, 0.0, 0};
  const size_t n = (size_t)nd;
  double *zt = calloc(n, 8), *zr = calloc(n, 8), *zp = calloc(n, 8), *zkp = calloc(n, 8);
  double *zakp = calloc(n, 8), *zkt = calloc(n, 8), *zakt = calloc(n, 8), *zshdw = calloc(n, 8);
  double *wws = calloc(n > 0 ? n : 1, 8);
  double alpha = 0.0, beta = 0.0, zeta = 0.0, zz, zden, znorm, znormold = 1.0, bnorm, zrnorm;
  int nstp = 0;
  zz = dotp_d(nd, b, b);
  bnorm = sqrt(zz);
  memcpy(zr, b, n * 8);
  memset(zshdw, 0, n * 8);
  mv_apply(&mv, zshdw, st, u, wws);
  daxpy(nd, -1.0, zshdw, zr);
  memcpy(zshdw, zr, n * 8);
  zrnorm = dotp_d(nd, zr, zr);
  zrnorm = sqrt(zrnorm);
  if (hist) hist[0] = zrnorm / bnorm;
  for (int step = 1; step <= mstep; step++) {
    if (zrnorm / bnorm < eps) break;
    if (beta == 0.0) {
      memcpy(zp, zr, n * 8);
    } else {
      daxpy(nd, zeta, zakp, zp);
      for (int i = 0; i < nd; i++) zp[i] = zp[i] * beta;
      daxpy(nd, 1.0, zr, zp);
    }
    memcpy(zkp, zp, n * 8);
    memset(zakp, 0, n * 8);
    mv_apply(&mv, zakp, st, zkp, wws);
    znorm = dotp_d(nd, zshdw, zr);
    zden = dotp_d(nd, zshdw, zakp);
    alpha = -znorm / zden;
    znormold = znorm;
    memcpy(zt, zr, n * 8);
    daxpy(nd, alpha, zakp, zt);
    alpha = -alpha;
    memcpy(zkt, zt, n * 8);
    memset(zakt, 0, n * 8);
    mv_apply(&mv, zakt, st, zkt, wws);
    znorm = dotp_d(nd, zakt, zt);
    zden = dotp_d(nd, zakt, zakt);
    zeta = znorm / zden;
    daxpy(nd, alpha, zkp, u);
    daxpy(nd, zeta, zkt, u);
    zeta = -zeta;
    memcpy(zr, zt, n * 8);
    daxpy(nd, zeta, zakt, zr);
    beta = dotp_d(nd, zshdw, zr);
    zrnorm = dotp_d(nd, zr, zr);
    beta = -alpha / zeta * beta / znormold;
    zrnorm = sqrt(zrnorm);
    nstp = step;
    if (hist) hist[step] = zrnorm / bnorm;
  }
  if (matvec_seconds) *matvec_seconds = mv.seconds;
  free(zt); free(zr); free(zp); free(zkp); free(zakp); free(zkt); free(zakt); free(zshdw); free(wws);
  return nstp;
}

/* Pipelined BiCGSTAB, c_hacapk_bicgstab_cax_lfmtx_pipe_ (HACApK_SOLVER_PIPE.c:144-600;
 * the second version, _pipe2_ at :640-1148, runs the same arithmetic with its
 * host gathers moved beside the dot products).  The auxiliary products
 * s = A p and z = A s are carried by recurrences, so a step takes two products
 * (v = A z, t = A w).  Statement order and the daxpy / dlascl roundings are
 * the reference's (y = y + a x; x = c x); the dots are the sequential
 * HACApK_dotp_d (the reference calls magma_ddot).  The iterate accumulates in
 * u (x0 in / solution out): the reference adds the corrections to zx, a
 * device vector it never initialises, and copies back the unchanged u
 * (:592), so its own output is the initial guess.  hist[0..nstp] receives
 * ||r||/||b||.  Returns nstp. */
int orc_bicgstab_pipe(const stc_HACApK_leafmtxp *st, int nd, double *u, const double *b, double eps, int mstep,
                      int mv_kind, void *mv_fn, const void *ext_st, int nthreads, double *hist,
                      double *matvec_seconds) {
  orc_mv mv = {mv_kind, mv_fn, ext_st, nthreads, 0.0, 0};
  const size_t n = (size_t)nd;
  double *zr = calloc(n, 8), *zr0 = calloc(n, 8), *zw = calloc(n, 8), *zt = calloc(n, 8), *zv = calloc(n, 8);
  double *zp = calloc(n, 8), *zs = calloc(n, 8), *zz = calloc(n, 8), *zq = calloc(n, 8), *zy = calloc(n, 8);
  double *wws = calloc(n > 0 ? n : 1, 8);
  double alpha, beta = 0.0, zeta = 0.0, zden, znorm, znormold, zrnorm, zwnorm, zsnorm, zznorm;
  int nstp = 0;
  const double bnorm = sqrt(dotp_d(nd, b, b));
  memset(zv, 0, n * 8);
  mv_apply(&mv, zv, st, u, wws);
  memcpy(zr, b, n * 8);
  daxpy(nd, -1.0, zv, zr);
  memcpy(zr0, zr, n * 8);
  memset(zw, 0, n * 8);
  mv_apply(&mv, zw, st, zr, wws);
  memset(zt, 0, n * 8);
  mv_apply(&mv, zt, st, zw, wws);
  znorm = dotp_d(nd, zr, zr);
  zrnorm = dotp_d(nd, zw, zr);
  alpha = znorm / zrnorm;
  zrnorm = sqrt(znorm);
  if (hist) hist[0] = zrnorm / bnorm;
  for (int step = 1; step <= mstep; step++) {
    if (zrnorm / bnorm < eps) break;
    if (step > 1) {
      daxpy(nd, -zeta, zs, zp);
      for (int i = 0; i < nd; i++) zp[i] = zp[i] * beta;
      daxpy(nd, 1.0, zr, zp);
      daxpy(nd, -zeta, zz, zs);
      for (int i = 0; i < nd; i++) zs[i] = zs[i] * beta;
      daxpy(nd, 1.0, zw, zs);
      daxpy(nd, -zeta, zv, zz);
      for (int i = 0; i < nd; i++) zz[i] = zz[i] * beta;
      daxpy(nd, 1.0, zt, zz);
    } else {
      memcpy(zp, zr, n * 8);
      memcpy(zs, zw, n * 8);
      memcpy(zz, zt, n * 8);
    }
    memcpy(zq, zr, n * 8);
    daxpy(nd, -alpha, zs, zq);
    memcpy(zy, zw, n * 8);
    daxpy(nd, -alpha, zz, zy);
    zrnorm = dotp_d(nd, zy, zq);
    zden = dotp_d(nd, zy, zy);
    zeta = zrnorm / zden;
    memset(zv, 0, n * 8);
    mv_apply(&mv, zv, st, zz, wws);
    daxpy(nd, alpha, zp, u);
    daxpy(nd, zeta, zq, u);
    memcpy(zr, zq, n * 8);
    daxpy(nd, -zeta, zy, zr);
    memcpy(zw, zt, n * 8);
    daxpy(nd, -alpha, zv, zw);
    for (int i = 0; i < nd; i++) zw[i] = zw[i] * -zeta;
    daxpy(nd, 1.0, zy, zw);
    znormold = znorm;
    znorm = dotp_d(nd, zr, zr0);
    zwnorm = dotp_d(nd, zw, zr0);
    zsnorm = dotp_d(nd, zs, zr0);
    zznorm = dotp_d(nd, zz, zr0);
    zrnorm = dotp_d(nd, zr, zr);
    beta = (alpha / zeta) * (znorm / znormold);
    alpha = znorm / (zwnorm + beta * zsnorm - beta * zeta * zznorm);
    zrnorm = sqrt(zrnorm);
    nstp = step;
    if (hist) hist[step] = zrnorm / bnorm;
    memset(zt, 0, n * 8);
    mv_apply(&mv, zt, st, zw, wws);
  }
  if (matvec_seconds) *matvec_seconds = mv.seconds;
  free(zr); free(zr0); free(zw); free(zt); free(zv); free(zp); free(zs); free(zz); free(zq); free(zy); free(wws);
  return nstp;
}

/* HACApK_gcrm_lfmtx (m_HACApK_solve.f90:506-571): GCR(m) restarted every
 * mreset steps (param(87)), the product zau = H zu (the Fortran's
 * HACApK_adot_lfmtx_hyp; any of the oracle's products), the sequential dot
 * HACApK_dotp_d.  The statement order is the Fortran's, including the
 * restart: when step `in` fills the last slot, the next direction is written
 * into slot 1 and then orthogonalized against every slot, slot 1 (the new
 * vector itself, with the old slot's |A p|^2) included.  u: x0 in / solution
 * out; hist[0..nstp] receives ||r||/||b||.  Returns nstp. */
int orc_gcrm(const stc_HACApK_leafmtxp *st, int nd, double *u, const double *b, double eps, int mstep, int mreset,
             int mv_kind, void *mv_fn, const void *ext_st, int nthreads, double *hist, double *matvec_seconds) {
  orc_mv mv = {mv_kind, mv_fn, ext_st, nthreads, 0.0, 0};
  const size_t n = (size_t)nd;
  if (mreset < 1) mreset = 1;
  double *zr = calloc(n, 8), *zar = calloc(n, 8), *capap = calloc((size_t)mreset, 8);
  double *zp = calloc(n * (size_t)mreset, 8), *zap = calloc(n * (size_t)mreset, 8);
  double *wws = calloc(n > 0 ? n : 1, 8);
  int in = 0, nstp = 0;
  const double bnorm = sqrt(dotp_d(nd, b, b));
  memset(zar, 0, n * 8);
  mv_apply(&mv, zar, st, u, wws);
  for (int i = 0; i < nd; i++) zr[i] = b[i] - zar[i];
  memcpy(zp, zr, n * 8);
  double zrnorm2 = dotp_d(nd, zr, zr), zrnorm = sqrt(zrnorm2);
  if (hist) hist[0] = zrnorm / bnorm;
  if (!(zrnorm / bnorm < eps)) {
    memset(zap, 0, n * 8);
    mv_apply(&mv, zap, st, zp, wws);
    for (in = 1; in <= mstep; in++) {
      const int ik = (in - 1) % mreset + 1;
      const double *zq = zap + n * (size_t)(ik - 1);
      const double znom = dotp_d(nd, zq, zr);
      capap[ik - 1] = dotp_d(nd, zq, zq);
      const double alpha = znom / capap[ik - 1];
      const double *pk = zp + n * (size_t)(ik - 1);
      for (int i = 0; i < nd; i++) u[i] = u[i] + alpha * pk[i];
      for (int i = 0; i < nd; i++) zr[i] = zr[i] - alpha * zq[i];
      zrnorm2 = dotp_d(nd, zr, zr);
      zrnorm = sqrt(zrnorm2);
      if (hist) hist[in] = zrnorm / bnorm;
      nstp = in;
      if (zrnorm / bnorm < eps || in == mstep) break;
      memset(zar, 0, n * 8);
      mv_apply(&mv, zar, st, zr, wws);
      const int ikn = in % mreset + 1;
      double *pn = zp + n * (size_t)(ikn - 1), *apn = zap + n * (size_t)(ikn - 1);
      memcpy(pn, zr, n * 8);
      memcpy(apn, zar, n * 8);
      for (int il = 1; il <= ik; il++) {
        const double *ql = zap + n * (size_t)(il - 1), *pl = zp + n * (size_t)(il - 1);
        const double beta = -dotp_d(nd, ql, zar) / capap[il - 1];
        for (int i = 0; i < nd; i++) pn[i] = pn[i] + beta * pl[i];
        for (int i = 0; i < nd; i++) apn[i] = apn[i] + beta * ql[i];
      }
    }
  }
  if (matvec_seconds) *matvec_seconds = mv.seconds;
  free(zr); free(zar); free(capap); free(zp); free(zap); free(wws);
  return nstp;
}
