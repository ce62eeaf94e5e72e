// hbx_build.cpp -- host construction of HACApK leaf lists (input side of the
// H-matvec path).  CPU restatement of the reference's construction:
//
//   face_integral ............ m_ppohBEM_user_func.f90:49-99
//   matrix entry / centroids . m_ppohBEM_matrix_element_ij.f90:49-76,
//                              m_ppohBEM_bembb2hacapk.f90:101-106
//   cluster tree ............. m_HACApK_base.f90:1385-1445 (generate_cbitree)
//   bounding boxes ........... m_HACApK_base.f90:1344-1382 (bndbox)
//   block partition .......... m_HACApK_base.f90:1172-1206, 1236-1282
//   leaf sort ................ m_HACApK_base.f90:451-461, 1285-1320
//   ACA+ ..................... m_HACApK_base.f90:783-975 with calc_vec :677-698
//                              and HACApK_lib.f90:31-81 (unrm, maxabs, minabs)
//   fill ..................... m_HACApK_base.f90:978-1051
//   statistics ............... m_HACApK_base.f90:1108-1169, 538-561
//
// Leaves are independent, so the fill runs OpenMP-parallel over leaves; the
// per-leaf arithmetic follows the Fortran statement order.  The file is built
// with -ffp-contract=off so the result does not depend on FMA contraction.
#include "../../include/hacapk_b200_build.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include <omp.h>

namespace {

// ---------------------------------------------------------------- kernel
// m_ppohBEM_user_func.f90:42-43: the literals carry no d0 suffix, so they are
// rounded to single precision before being stored in the real(8) parameters.
const double kPiF = (double)3.141592653589793f;
const double kEps0 = (double)8.854187818f * 1e-12;

inline void cross3(const double u[3], const double v[3], double w[3]) {
  w[0] = u[1] * v[2] - u[2] * v[1];
  w[1] = u[2] * v[0] - u[0] * v[2];
  w[2] = u[0] * v[1] - u[1] * v[0];
}

// face_integral(xs,ys,zs,x,y,z): analytic integral of 1/r over the flat
// triangle (xs,ys,zs) seen from (x,y,z); returns the unscaled |sum|.
double face_integral_raw(const double xs[3], const double ys[3], const double zs[3],
                         double x, double y, double z) {
  double r[3];
  for (int a = 0; a < 3; ++a) {
    double dx = xs[a] - x, dy = ys[a] - y, dz = zs[a] - z;
    r[a] = std::sqrt(dx * dx + dy * dy + dz * dz);
  }
  double u[3], v[3], w[3];
  u[0] = xs[1] - xs[0]; v[0] = xs[2] - xs[1];
  u[1] = ys[1] - ys[0]; v[1] = ys[2] - ys[1];
  u[2] = zs[1] - zs[0]; v[2] = zs[2] - zs[1];
  cross3(u, v, w);
  double wn = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  w[0] = w[0] / wn; w[1] = w[1] / wn; w[2] = w[2] / wn;
  u[0] = x - xs[0]; u[1] = y - ys[0]; u[2] = z - zs[0];
  double zp = u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
  double ox = x - zp * w[0], oy = y - zp * w[1], oz = z - zp * w[2];
  double zpabs = std::fabs(zp);
  double sum = 0.0;
  for (int i = 0; i < 3; ++i) {
    int j = (i + 1) % 3;
    u[0] = xs[j] - ox; u[1] = ys[j] - oy; u[2] = zs[j] - oz;
    double xj = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    u[0] = u[0] / xj; u[1] = u[1] / xj; u[2] = u[2] / xj;
    cross3(w, u, v);
    double xi = (xs[i] - ox) * u[0] + (ys[i] - oy) * u[1] + (zs[i] - oz) * u[2];
    double yi = (xs[i] - ox) * v[0] + (ys[i] - oy) * v[1] + (zs[i] - oz) * v[2];
    double dx = xj - xi, dy = -yi;
    double t = std::sqrt(dx * dx + dy * dy);
    double l = dx / t, m = dy / t;
    double d = l * yi - m * xi;
    double ti = l * xi + m * yi, tj = l * xj;
    double theta = std::atan2(yi, xi);
    double omega = theta - std::atan2(r[i] * d, zpabs * ti) + std::atan2(r[j] * d, zpabs * tj);
    double q = std::log((r[j] + tj) / (r[i] + ti));
    double g = d * q - zpabs * omega;
    sum = sum + g;
  }
  return std::fabs(sum);
}

// ---------------------------------------------------------------- helpers
// HACApK_lib.f90:31-46, scaled 2-norm that skips |a| < 1e-30.
double unrm(int nd, const double *za) {
  double zscl = 0.0, zzz = 1.0;
  for (int il = 0; il < nd; ++il) {
    double zza = std::fabs(za[il]);
    if (zza < 1.0e-30) continue;
    if (zscl < zza) {
      double t = zscl / zza;
      zzz = 1.0 + zzz * t * t;
      zscl = zza;
    } else {
      double t = zza / zscl;
      zzz = zzz + t * t;
    }
  }
  return zscl * std::sqrt(zzz);
}
// HACApK_lib.f90:48-57 (1-based index returned).
void maxabsvalloc(const double *za, double &zz, int &il, int nd) {
  il = 1; zz = std::fabs(za[0]);
  for (int it = 2; it <= nd; ++it)
    if (std::fabs(za[it - 1]) > zz) { il = it; zz = std::fabs(za[it - 1]); }
}
// HACApK_lib.f90:72-81.
void minabsvalloc(const double *za, double &zz, int &il, int nd) {
  il = 1; zz = std::fabs(za[0]);
  for (int it = 2; it <= nd; ++it)
    if (std::fabs(za[it - 1]) < zz) { il = it; zz = std::fabs(za[it - 1]); }
}
// HACApK_lib.f90:156-162.
int med3(int nl, int nr, int nlr2) {
  if (nl < nr) {
    if (nr < nlr2) return nr;
    else if (nlr2 < nl) return nl;
    else return nlr2;
  } else {
    if (nlr2 < nr) return nr;
    else if (nl < nlr2) return nl;
    else return nlr2;
  }
}

struct Cluster {
  int nstrt, nsize, ndpth, nnson, nmbr;
  int son[2];
  double bmin[3], bmax[3], zwdth;
};

struct Leaf {
  int ltmtx, kt, nstrtl, ndl, nstrtt, ndt;
};

}  // namespace

struct hbx_hbuild {
  int nofc = 0, nond = 0;
  int kernel = HBX_KERNEL_LAPLACE;
  std::vector<double> fx, fy, fz;        // face vertices, 3 per face
  std::vector<double> zgmid;             // nofc x 3, column-major
  std::vector<int> lod;                  // 1-based face ids
  std::vector<Cluster> clt;
  std::vector<Leaf> leaves;
  std::vector<stc_HACApK_leafmtx> st_lf;
  std::vector<double *> storage;         // per-leaf a1|a2 blocks
  stc_HACApK_leafmtxp st{};
  hbx_build_stats stats{};

  // entry(i,j), 1-based face ids: collocation at centroid of face i,
  // integration over face j (m_ppohBEM_matrix_element_ij.f90:60-74).
  double entry(int i, int j) const {
    const double x = zgmid[(size_t)(i - 1)];
    const double y = zgmid[(size_t)nofc + (i - 1)];
    const double z = zgmid[2 * (size_t)nofc + (i - 1)];
    const double *xs = &fx[3 * (size_t)(j - 1)];
    const double *ys = &fy[3 * (size_t)(j - 1)];
    const double *zs = &fz[3 * (size_t)(j - 1)];
    double s = face_integral_raw(xs, ys, zs, x, y, z);
    if (kernel == HBX_KERNEL_PPOHBEM) return s / (4.0 * kPiF * kEps0);
    return s / (4.0 * M_PI);
  }
  ~hbx_hbuild() {
    for (double *p : storage) std::free(p);
  }
};

namespace {

// m_HACApK_base.f90:1385-1445.  `lod` points at the first face id of this
// cluster's slice; clusters are numbered in creation (pre-)order.
int gen_cbitree(hbx_hbuild &B, int minsz, int *lod, int &ndpth, int nsrt, int nd) {
  ndpth = ndpth + 1;
  const int nofc = B.nofc;
  const double *zg = B.zgmid.data();
  Cluster c{};
  c.nstrt = nsrt; c.nsize = nd; c.ndpth = ndpth;
  c.son[0] = c.son[1] = -1;
  if (nd <= minsz) {
    c.nnson = 0;
    c.nmbr = (int)B.clt.size() + 1;
    B.clt.push_back(c);
    return (int)B.clt.size() - 1;
  }
  double zlmin[3], zlmax[3];
  for (int id = 0; id < 3; ++id) {
    zlmin[id] = zg[(size_t)id * nofc + (lod[0] - 1)];
    zlmax[id] = zlmin[id];
    for (int il = 2; il <= nd; ++il) {
      double zgv = zg[(size_t)id * nofc + (lod[il - 1] - 1)];
      if (zgv < zlmin[id]) zlmin[id] = zgv;
      else if (zlmax[id] < zgv) zlmax[id] = zgv;
    }
  }
  double zdiff = zlmax[0] - zlmin[0];
  int ncut = 0;
  for (int id = 0; id < 3; ++id) {
    double zidiff = zlmax[id] - zlmin[id];
    if (zidiff > zdiff) { zdiff = zidiff; ncut = id; }
  }
  const double zlmid = (zlmax[ncut] + zlmin[ncut]) / 2;
  auto zv = [&](int pos1) { return zg[(size_t)ncut * nofc + (lod[pos1 - 1] - 1)]; };
  int nl = 1, nr = nd;
  while (nl < nr) {
    while (nl < nd && zv(nl) <= zlmid) nl = nl + 1;
    while (nr >= 1 && zv(nr) > zlmid) nr = nr - 1;
    if (nl < nr) std::swap(lod[nl - 1], lod[nr - 1]);
  }
  c.nnson = 2;
  c.nmbr = (int)B.clt.size() + 1;
  B.clt.push_back(c);
  const int me = (int)B.clt.size() - 1;
  int s0 = gen_cbitree(B, minsz, lod, ndpth, nsrt, nl - 1);
  ndpth = ndpth - 1;
  int s1 = gen_cbitree(B, minsz, lod + (nl - 1), ndpth, nsrt + nl - 1, nd - nl + 1);
  ndpth = ndpth - 1;
  B.clt[me].son[0] = s0;
  B.clt[me].son[1] = s1;
  return me;
}

// m_HACApK_base.f90:1344-1382 (post-order).
void bndbox(hbx_hbuild &B, int ic) {
  Cluster &c0 = B.clt[ic];
  for (int s = 0; s < c0.nnson; ++s) bndbox(B, c0.son[s]);
  Cluster &c = B.clt[ic];
  const int nofc = B.nofc;
  const double *zg = B.zgmid.data();
  const int *lod = B.lod.data() + (c.nstrt - 1);
  if (c.nnson == 0) {
    for (int id = 0; id < 3; ++id) {
      c.bmin[id] = (c.nsize > 0) ? zg[(size_t)id * nofc + (lod[0] - 1)] : 0.0;
      c.bmax[id] = c.bmin[id];
    }
    for (int id = 0; id < 3; ++id)
      for (int il = 2; il <= c.nsize; ++il) {
        double v = zg[(size_t)id * nofc + (lod[il - 1] - 1)];
        if (v < c.bmin[id]) c.bmin[id] = v;
        if (c.bmax[id] < v) c.bmax[id] = v;
      }
  } else {
    const Cluster &a = B.clt[c.son[0]];
    for (int id = 0; id < 3; ++id) { c.bmin[id] = a.bmin[id]; c.bmax[id] = a.bmax[id]; }
    for (int s = 1; s < c.nnson; ++s) {
      const Cluster &b = B.clt[c.son[s]];
      for (int id = 0; id < 3; ++id) {
        if (b.bmin[id] < c.bmin[id]) c.bmin[id] = b.bmin[id];
        if (c.bmax[id] < b.bmax[id]) c.bmax[id] = b.bmax[id];
      }
    }
  }
  double zw = (c.bmax[0] - c.bmin[0]) * (c.bmax[0] - c.bmin[0]);
  for (int id = 1; id < 3; ++id) zw = zw + (c.bmax[id] - c.bmin[id]) * (c.bmax[id] - c.bmin[id]);
  c.zwdth = std::sqrt(zw);
}

// m_HACApK_base.f90:1236-1282 (and the counting twin :1172-1206).
void gen_leaves(hbx_hbuild &B, int il_c, int it_c, int nleaf, int nlmax, double zeta,
                int &n_hnode) {
  const Cluster &l = B.clt[il_c];
  const Cluster &t = B.clt[it_c];
  const int ndl = l.nsize, ndt = t.nsize;
  double zs = 0.0;
  for (int id = 0; id < 3; ++id) {
    if (l.bmax[id] < t.bmin[id]) zs = zs + (t.bmin[id] - l.bmax[id]) * (t.bmin[id] - l.bmax[id]);
    else if (t.bmax[id] < l.bmin[id]) zs = zs + (l.bmin[id] - t.bmax[id]) * (l.bmin[id] - t.bmax[id]);
  }
  const double zdistlt = std::sqrt(zs);
  if ((l.zwdth <= zeta * zdistlt || t.zwdth <= zeta * zdistlt) &&
      (ndl >= nleaf && ndt >= nleaf && ndl <= nlmax && ndt <= nlmax)) {
    B.leaves.push_back(Leaf{1, 0, l.nstrt, ndl, t.nstrt, ndt});
  } else if (l.nnson == 0 || t.nnson == 0 || ndl <= nleaf || ndt <= nleaf) {
    B.leaves.push_back(Leaf{2, 0, l.nstrt, ndl, t.nstrt, ndt});
  } else {
    n_hnode++;
    const int ls0 = l.son[0], ls1 = l.son[1], ts0 = t.son[0], ts1 = t.son[1];
    const int lsons[2] = {ls0, ls1}, tsons[2] = {ts0, ts1};
    for (int a = 0; a < l.nnson; ++a)
      for (int b = 0; b < t.nnson; ++b) gen_leaves(B, lsons[a], tsons[b], nleaf, nlmax, zeta, n_hnode);
  }
}

// m_HACApK_base.f90:1285-1320 (1-based bounds, Hoare partition, med3 pivot).
template <class Key>
void qsort_leaves(std::vector<Leaf> &v, int s, int e, Key key) {
  if (s >= e) return;
  int nl = s, nr = e, nlr2 = nl + (nr - nl) / 2;
  int nmid = med3(key(v[nl - 1]), key(v[nr - 1]), key(v[nlr2 - 1]));
  for (;;) {
    while (key(v[nl - 1]) < nmid) nl = nl + 1;
    while (key(v[nr - 1]) > nmid) nr = nr - 1;
    if (nl >= nr) break;
    std::swap(v[nl - 1], v[nr - 1]);
    nl = nl + 1; nr = nr - 1;
  }
  qsort_leaves(v, s, nl - 1, key);
  qsort_leaves(v, nr + 1, e, key);
}

// calc_vec (m_HACApK_base.f90:677-698).  Column mode (fixed column `ip`,
// varying rows, mask over rows) or row mode (fixed row, varying columns).
// U holds columns of length ndl, V columns of length ndt (capacity-strided).
struct AcaCtx {
  const hbx_hbuild *B;
  int ndl, ndt, nstrtl, nstrtt;
  std::vector<double> U, V;  // zaa(ndl,cap), zab(ndt,cap)
  int cap = 0;
  std::vector<double> tmp;
  void ensure(int ncols) {
    if (ncols <= cap) return;
    int nc = std::max(ncols, std::max(8, cap * 2));
    U.resize((size_t)ndl * nc, 0.0);
    V.resize((size_t)ndt * nc, 0.0);
    cap = nc;
  }
  double *ucol(int k1) { return &U[(size_t)ndl * (k1 - 1)]; }  // 1-based column
  double *vcol(int k1) { return &V[(size_t)ndt * (k1 - 1)]; }
  // column j of the residual after k terms -> vec (length ndl)
  void calc_col(int k, int jcol, double *vec, const std::vector<int> &rmsk) {
    const int *lod = B->lod.data();
    const int itt = jcol + nstrtt - 1;
    for (int ii = 1; ii <= ndl; ++ii)
      if (rmsk[ii - 1] == 0) vec[ii - 1] = B->entry(lod[ii + nstrtl - 2], lod[itt - 1]);
    if (k == 0) return;
    tmp.assign(ndl, 0.0);
    for (int it = 1; it <= k; ++it) {
      const double zz = V[(size_t)ndt * (it - 1) + (jcol - 1)];
      const double *uc = &U[(size_t)ndl * (it - 1)];
      for (int ii = 0; ii < ndl; ++ii) tmp[ii] = tmp[ii] + uc[ii] * zz;
    }
    for (int ii = 0; ii < ndl; ++ii) vec[ii] = vec[ii] - tmp[ii];
    for (int ii = 0; ii < ndl; ++ii) if (rmsk[ii] == 1) vec[ii] = 0.0;
  }
  // row i of the residual after k terms -> vec (length ndt)
  void calc_row(int k, int irow, double *vec, const std::vector<int> &cmsk) {
    const int *lod = B->lod.data();
    const int ill = irow + nstrtl - 1;
    for (int ii = 1; ii <= ndt; ++ii)
      if (cmsk[ii - 1] == 0) vec[ii - 1] = B->entry(lod[ill - 1], lod[ii + nstrtt - 2]);
    if (k == 0) return;
    tmp.assign(ndt, 0.0);
    for (int it = 1; it <= k; ++it) {
      const double zz = U[(size_t)ndl * (it - 1) + (irow - 1)];
      const double *vc = &V[(size_t)ndt * (it - 1)];
      for (int ii = 0; ii < ndt; ++ii) tmp[ii] = tmp[ii] + vc[ii] * zz;
    }
    for (int ii = 0; ii < ndt; ++ii) vec[ii] = vec[ii] - tmp[ii];
    for (int ii = 0; ii < ndt; ++ii) if (cmsk[ii] == 1) vec[ii] = 0.0;
  }
};

// HACApK_acaplus (m_HACApK_base.f90:783-975), param(61)=1 (MREM norm).
// Returns kt; the factors are columns 1..kt of ctx.U (zaa) and ctx.V (zab).
int acaplus(AcaCtx &C, const hbx_build_params &P, double eps, double pACA_EPS) {
  const int ndl = C.ndl, ndt = C.ndt;
  const double za_ACA_EPS = (double)1.0e-30f;
  const double ACA_EPS = pACA_EPS;
  const int kmax = P.kmax, kmin = P.kmin;
  int ntries = std::max(ndl, ndt) + 1, ntries_row = 6, ntries_col = 6;
  std::vector<int> lrow_msk(ndl, 0), lcol_msk(ndt, 0);
  int k = 0;
  C.ensure(1);
  int j_ref = 1;
  std::vector<double> pa_ref(ndl, 0.0), pb_ref(ndt, 0.0);
  C.calc_col(k, j_ref, pa_ref.data(), lrow_msk);
  double colnorm = unrm(ndl, pa_ref.data());
  double rownorm;
  int i_ref;
  minabsvalloc(pa_ref.data(), rownorm, i_ref, ndl);
  C.calc_row(k, i_ref, pb_ref.data(), lcol_msk);
  rownorm = unrm(ndt, pb_ref.data());
  double apxnorm = 0.0;
  int lstop_aca = 0;
  double col_maxval = 0.0, row_maxval = 0.0;
  int i = 0, j = 0;
  while ((k < kmax) && (ntries_row > 0 || ntries_col > 0) && (ntries > 0)) {
    ntries = ntries - 1;
    C.ensure(k + 1);
    double *pcol = C.ucol(k + 1);
    double *prow = C.vcol(k + 1);
    col_maxval = 0.0; maxabsvalloc(pa_ref.data(), col_maxval, i, ndl);
    row_maxval = 0.0; maxabsvalloc(pb_ref.data(), row_maxval, j, ndt);
    if (row_maxval > col_maxval) {
      if (j != j_ref) C.calc_col(k, j, pcol, lrow_msk);
      else std::copy(pa_ref.begin(), pa_ref.end(), pcol);
      maxabsvalloc(pcol, col_maxval, i, ndl);
      if (col_maxval < ACA_EPS && k >= kmin) {
        lstop_aca = 1;
      } else {
        C.calc_row(k, i, prow, lcol_msk);
        double zinvmax;
        if (std::fabs(pcol[i - 1]) > (double)1.0e-20f) zinvmax = 1.0 / pcol[i - 1];
        else { k = std::max(k - 1, 0); break; }
        for (int a = 0; a < ndl; ++a) pcol[a] = pcol[a] * zinvmax;
      }
    } else {
      if (i != i_ref) C.calc_row(k, i, prow, lcol_msk);
      else std::copy(pb_ref.begin(), pb_ref.end(), prow);
      maxabsvalloc(prow, row_maxval, j, ndt);
      if (row_maxval < ACA_EPS && k >= kmin) {
        lstop_aca = 1;
      } else {
        C.calc_col(k, j, pcol, lrow_msk);
        double zinvmax;
        if (std::fabs(prow[j - 1]) > (double)1.0e-20f) zinvmax = 1.0 / prow[j - 1];
        else { k = std::max(k - 1, 0); break; }
        for (int a = 0; a < ndt; ++a) prow[a] = prow[a] * zinvmax;
      }
    }
    lrow_msk[i - 1] = 1; lcol_msk[j - 1] = 1;

    if (i != i_ref) {
      double zinvmax = -pcol[i_ref - 1];
      for (int a = 0; a < ndt; ++a) pb_ref[a] = pb_ref[a] + prow[a] * zinvmax;
      rownorm = unrm(ndt, pb_ref.data());
    }
    if (i == i_ref || rownorm < ACA_EPS) {
      if (i == i_ref) ntries_row = ntries_row + 1;
      if (ntries_row > 0) {
        rownorm = 0.0; i = i_ref;
        while (i != ((i_ref + ndl - 2) % ndl) + 1 && rownorm < za_ACA_EPS && ntries_row > 0) {
          if (lrow_msk[i - 1] == 0) {
            C.calc_row(k + 1, i, pb_ref.data(), lcol_msk);
            rownorm = unrm(ndt, pb_ref.data());
            if (rownorm < ACA_EPS) lrow_msk[i - 1] = 1;
            ntries_row = ntries_row - 1;
          } else {
            rownorm = 0.0;
          }
          i = (i % ndl) + 1;
        }
        i_ref = ((i + ndl - 2) % ndl) + 1;
      }
    }

    if (j != j_ref) {
      double zinvmax = -prow[j_ref - 1];
      for (int a = 0; a < ndl; ++a) pa_ref[a] = pa_ref[a] + pcol[a] * zinvmax;
      colnorm = unrm(ndl, pa_ref.data());
    }
    if (j == j_ref || colnorm < ACA_EPS) {
      if (j == j_ref) ntries_col = ntries_col + 1;
      if (ntries_col > 0) {
        colnorm = 0.0; j = j_ref;
        while (j != ((j_ref + ndt - 2) % ndt) + 1 && colnorm < za_ACA_EPS && ntries_col > 0) {
          if (lcol_msk[j - 1] == 0) {
            C.calc_col(k + 1, j, pa_ref.data(), lrow_msk);
            colnorm = unrm(ndl, pa_ref.data());
            if (colnorm < ACA_EPS) lcol_msk[j - 1] = 1;
            ntries_col = ntries_col - 1;
          } else {
            colnorm = 0.0;
          }
          j = (j % ndt) + 1;
        }
        j_ref = ((j + ndt - 2) % ndt) + 1;
      }
    }

    if (colnorm < ACA_EPS && rownorm < ACA_EPS && k >= kmin) {
      lstop_aca = 1; k = k + 1;
    }
    if (lstop_aca == 0) {
      double blknorm = unrm(ndl, pcol) * unrm(ndt, prow);
      if (k == 0) {
        apxnorm = blknorm;
      } else if (blknorm < apxnorm * eps && rownorm < apxnorm * eps &&
                 colnorm < apxnorm * eps && k >= kmin) {
        lstop_aca = 1;
      }
    }
    if (lstop_aca == 1 && k >= kmin) break;
    k = k + 1;
  }
  return k;
}


// HACApK_lib.f90:59-70: masked max-abs locator (index 0 when all masked).
void maxabsvallocm(const double *za, double &zz, int &il, int nd, const std::vector<int> &lmask) {
  il = 0; zz = 0.0;
  for (int it = 1; it <= nd; ++it) {
    if (lmask[it - 1] == 1) continue;
    if (std::fabs(za[it - 1]) > zz) { il = it; zz = std::fabs(za[it - 1]); }
  }
}

// HACApK_aca (m_HACApK_base.f90:701-780), param(61)=1.  Returns kt.
int aca(AcaCtx &C, const hbx_build_params &P, double eps, double pACA_EPS) {
  const int ndl = C.ndl, ndt = C.ndt;
  const int krank = std::min(ndl, ndt);
  const double ACA_EPS = pACA_EPS;
  double znrm = 0.0;
  std::vector<int> lrow_msk(ndl, 0), lcol_msk(ndt, 0);
  int k = 1;
  int lstop_aca = 0;
  const int kstop = std::min(P.kmax, krank);
  int ist = (C.nstrtl > C.nstrtt) ? 1 : ndl;
  double zeps = 0.0;
  for (;;) {
    C.ensure(k);
    double *pcol = C.ucol(k);
    double *prow = C.vcol(k);
    C.calc_row(k - 1, ist, prow, lcol_msk);
    double row_maxval; int jst;
    maxabsvallocm(prow, row_maxval, jst, ndt, lcol_msk);
    if (jst == 0) break;  // every column masked or zero (the reference would index prow(0))
    double zdltinv = 1.0 / prow[jst - 1];
    for (int a = 0; a < ndt; ++a) prow[a] = prow[a] * zdltinv;
    C.calc_col(k - 1, jst, pcol, lrow_msk);
    lrow_msk[ist - 1] = 1;
    double col_maxval; int istn;
    maxabsvallocm(pcol, col_maxval, istn, ndl, lrow_msk);
    lcol_msk[jst - 1] = 1;
    ist = istn;
    if (std::fabs(row_maxval) < ACA_EPS && std::fabs(col_maxval) < ACA_EPS && k >= P.kmin) break;
    zeps = unrm(ndl, pcol) * unrm(ndt, prow);
    if (k == 1) znrm = zeps;
    zeps = zeps / znrm;
    if (zeps < eps || k == kstop) lstop_aca = 1;
    if (lstop_aca == 1 && k >= P.kmin) break;
    if (ist == 0) break;  // every row masked
    k = k + 1;
  }
  return k;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

void hbx_build_default_params(hbx_build_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->leaf_size = 15;
  p->eta = 2.0;
  p->aca_eps = 1.0e-6;
  p->aca_abs_factor = (double)1.0e-3f;  // param(72)=1.0e-3 (single literal)
  p->kmax = 1000;
  p->kmin = 1;
  p->kernel = HBX_KERNEL_LAPLACE;
  p->nthreads = 0;
  p->fill = 1;
  p->aca_method = 2;
}

int hbx_mesh_icosphere(int level, double *xyz, int *faces) {
  if (level < 0 || level > 10 || !xyz || !faces) return HBX_ERR_INVALID;
  const double t = (1.0 + std::sqrt(5.0)) / 2.0;
  std::vector<double> V = {-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0,
                           0, -1, t, 0, 1, t, 0, -1, -t, 0, 1, -t,
                           t, 0, -1, t, 0, 1, -t, 0, -1, -t, 0, 1};
  for (int v = 0; v < 12; ++v) {
    double n = std::sqrt(V[3 * v] * V[3 * v] + V[3 * v + 1] * V[3 * v + 1] + V[3 * v + 2] * V[3 * v + 2]);
    for (int a = 0; a < 3; ++a) V[3 * v + a] /= n;
  }
  std::vector<int> F = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11,
                        1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
                        3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9,
                        4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
  for (int lv = 0; lv < level; ++lv) {
    std::map<std::pair<int, int>, int> mid;
    auto midpoint = [&](int a, int b) {
      std::pair<int, int> key(std::min(a, b), std::max(a, b));
      auto it = mid.find(key);
      if (it != mid.end()) return it->second;
      double p[3];
      for (int c = 0; c < 3; ++c) p[c] = 0.5 * (V[3 * a + c] + V[3 * b + c]);
      double n = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      int id = (int)(V.size() / 3);
      for (int c = 0; c < 3; ++c) V.push_back(p[c] / n);
      mid[key] = id;
      return id;
    };
    std::vector<int> NF;
    NF.reserve(F.size() * 4);
    for (size_t f = 0; f < F.size(); f += 3) {
      int a = F[f], b = F[f + 1], c = F[f + 2];
      int ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
      int tri[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
      NF.insert(NF.end(), tri, tri + 12);
    }
    F.swap(NF);
  }
  std::memcpy(xyz, V.data(), V.size() * sizeof(double));
  std::memcpy(faces, F.data(), F.size() * sizeof(int));
  return HBX_OK;
}

int hbx_build(const double *xyz, int nond, const int *face2node, int nofc,
              const hbx_build_params *params, hbx_hbuild **out) {
  if (!xyz || !face2node || nond <= 0 || nofc <= 0 || !out) return HBX_ERR_INVALID;
  hbx_build_params P;
  if (params) P = *params; else hbx_build_default_params(&P);
  if (P.leaf_size < 2) P.leaf_size = 3;  // HACApK_chk_st_ctl (m_HACApK_base.f90:394-398)
  hbx_hbuild *B = new (std::nothrow) hbx_hbuild();
  if (!B) return HBX_ERR_NOMEM;
  B->nofc = nofc; B->nond = nond; B->kernel = P.kernel;
  B->fx.resize(3 * (size_t)nofc); B->fy.resize(3 * (size_t)nofc); B->fz.resize(3 * (size_t)nofc);
  B->zgmid.resize(3 * (size_t)nofc);
  for (int f = 0; f < nofc; ++f) {
    for (int a = 0; a < 3; ++a) {
      int n = face2node[3 * (size_t)f + a];
      if (n < 0 || n >= nond) { delete B; return HBX_ERR_INVALID; }
      B->fx[3 * (size_t)f + a] = xyz[3 * (size_t)n];
      B->fy[3 * (size_t)f + a] = xyz[3 * (size_t)n + 1];
      B->fz[3 * (size_t)f + a] = xyz[3 * (size_t)n + 2];
    }
    const double *x = &B->fx[3 * (size_t)f], *y = &B->fy[3 * (size_t)f], *z = &B->fz[3 * (size_t)f];
    B->zgmid[f] = (x[0] + x[1] + x[2]) / 3.0;
    B->zgmid[(size_t)nofc + f] = (y[0] + y[1] + y[2]) / 3.0;
    B->zgmid[2 * (size_t)nofc + f] = (z[0] + z[1] + z[2]) / 3.0;
  }
  const double t0 = now_s();
  B->lod.resize(nofc);
  for (int i = 0; i < nofc; ++i) B->lod[i] = i + 1;
  B->clt.reserve(4 * (size_t)nofc / std::max(1, P.leaf_size) + 16);
  int ndpth = 0;
  int root = gen_cbitree(*B, P.leaf_size, B->lod.data(), ndpth, 1, nofc);
  bndbox(*B, root);
  const int nleaf = P.leaf_size + 1;
  const int nlmax = nofc;  // param(22)=1.0 -> 1.0*nofc
  int n_hnode = 0;
  gen_leaves(*B, root, root, nleaf, nlmax, P.eta, n_hnode);
  const int nlf = (int)B->leaves.size();
  auto keyl = [](const Leaf &a) { return a.nstrtl; };
  auto keyt = [](const Leaf &a) { return a.nstrtt; };
  qsort_leaves(B->leaves, 1, nlf, keyl);
  {
    int ilp = 1, ips = 1;
    for (int ip = 1; ip <= nlf; ++ip) {
      int il = B->leaves[ip - 1].nstrtl;
      if (il > ilp) {
        qsort_leaves(B->leaves, ips, ip - 1, keyt);
        ilp = il; ips = ip;
      }
    }
  }
  B->stats.nd = nofc;
  B->stats.nclst = (int)B->clt.size();
  B->stats.n_hnode = n_hnode;
  long long ncpc = 0;
  int nrk = 0, nde = 0;
  for (const Leaf &L : B->leaves) {
    if (L.ltmtx == 1) { nrk++; ncpc += (long long)(L.ndl + L.ndt) * 7; }
    else { nde++; ncpc += (long long)L.ndl * L.ndt; }
  }
  B->stats.n_lowrank = nrk; B->stats.n_dense = nde; B->stats.ncpc7 = ncpc;
  const double t1 = now_s();
  B->stats.seconds_tree = t1 - t0;

  // ---- fill (m_HACApK_base.f90:978-1051), parallel over leaves
  B->storage.assign(nlf, nullptr);
  int fail = 0;
  if (P.fill) {
    const double eps = P.aca_eps;
    const double pACA = P.aca_abs_factor * eps;
    std::vector<int> order(nlf);
    for (int i = 0; i < nlf; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
      const Leaf &x = B->leaves[a], &y = B->leaves[b];
      long long cx = (long long)x.ndl * x.ndt, cy = (long long)y.ndl * y.ndt;
      return cx != cy ? cx > cy : a < b;
    });
    if (P.nthreads > 0) omp_set_num_threads(P.nthreads);
#pragma omp parallel
    {
      AcaCtx C;
      C.B = B;
#pragma omp for schedule(dynamic, 1)
      for (int oi = 0; oi < nlf; ++oi) {
        const int ip = order[oi];
        Leaf &L = B->leaves[ip];
        if (L.ltmtx == 1) {
          C.ndl = L.ndl; C.ndt = L.ndt; C.nstrtl = L.nstrtl; C.nstrtt = L.nstrtt;
          C.U.assign((size_t)L.ndl * 8, 0.0);
          C.V.assign((size_t)L.ndt * 8, 0.0);
          C.cap = 8;
          int kt = (P.aca_method == 1) ? aca(C, P, eps, pACA) : acaplus(C, P, eps, pACA);
          L.kt = kt;
          size_t n1 = (size_t)L.ndt * kt, n2 = (size_t)L.ndl * kt;
          double *mem = (double *)std::malloc(std::max<size_t>(1, n1 + n2) * sizeof(double));
          if (!mem) { fail = 1; continue; }
          for (int c = 0; c < kt; ++c) {
            std::memcpy(mem + (size_t)c * L.ndt, &C.V[(size_t)c * L.ndt], L.ndt * sizeof(double));
            std::memcpy(mem + n1 + (size_t)c * L.ndl, &C.U[(size_t)c * L.ndl], L.ndl * sizeof(double));
          }
          B->storage[ip] = mem;
        } else {
          size_t n = (size_t)L.ndl * L.ndt;
          double *mem = (double *)std::malloc(std::max<size_t>(1, n) * sizeof(double));
          if (!mem) { fail = 1; continue; }
          const int *lod = B->lod.data();
          for (int il = 1; il <= L.ndl; ++il) {
            const int ill = il + L.nstrtl - 1;
            for (int it = 1; it <= L.ndt; ++it) {
              const int itt = it + L.nstrtt - 1;
              mem[(size_t)(it - 1) + (size_t)(il - 1) * L.ndt] = B->entry(lod[ill - 1], lod[itt - 1]);
            }
          }
          B->storage[ip] = mem;
        }
      }
    }
  }
  if (fail) { delete B; return HBX_ERR_NOMEM; }
  B->stats.seconds_fill = now_s() - t1;

  // ---- leaf list in the reference layout + HACApK_chk_leafmtx statistics
  B->st_lf.resize(nlf);
  long long mem8 = 0;
  int ktmax = 0;
  for (int ip = 0; ip < nlf; ++ip) {
    const Leaf &L = B->leaves[ip];
    stc_HACApK_leafmtx &s = B->st_lf[ip];
    s.ltmtx = L.ltmtx; s.kt = L.kt;
    s.nstrtl = L.nstrtl; s.ndl = L.ndl; s.nstrtt = L.nstrtt; s.ndt = L.ndt;
    s.a1 = B->storage[ip];
    if (L.ltmtx == 1) {
      s.a1size = (long long)L.ndt * L.kt * (long long)sizeof(double);
      s.a2 = s.a1 ? s.a1 + (size_t)L.ndt * L.kt : nullptr;
      mem8 += (long long)(L.ndt + L.ndl) * L.kt;
      ktmax = std::max(ktmax, L.kt);
    } else {
      s.a1size = (long long)L.ndt * L.ndl * (long long)sizeof(double);
      s.a2 = nullptr;
      mem8 += (long long)L.ndl * L.ndt;
    }
  }
  B->stats.ktmax = ktmax;
  B->stats.mem_words = mem8;
  B->stats.memh_words = mem8 + nrk + nde;
  std::memset(&B->st, 0, sizeof(B->st));
  B->st.nd = nofc;
  B->st.nlf = nlf;
  B->st.nlfkt = nrk;
  B->st.ktmax = ktmax;
  B->st.st_lf_stride = (int)sizeof(stc_HACApK_leafmtx);
  B->st.st_lf = B->st_lf.data();
  *out = B;
  return HBX_OK;
}

void hbx_build_free(hbx_hbuild *b) { delete b; }

stc_HACApK_leafmtxp *hbx_build_leafmtxp(hbx_hbuild *b) { return b ? &b->st : nullptr; }

const int *hbx_build_lod(const hbx_hbuild *b) { return b ? b->lod.data() : nullptr; }

const double *hbx_build_centroids(const hbx_hbuild *b) { return b ? b->zgmid.data() : nullptr; }

int hbx_build_get_stats(const hbx_hbuild *b, hbx_build_stats *s) {
  if (!b || !s) return HBX_ERR_INVALID;
  *s = b->stats;
  return HBX_OK;
}

double hbx_build_entry(const hbx_hbuild *b, int i, int j) {
  if (!b || i < 1 || j < 1 || i > b->nofc || j > b->nofc) return NAN;
  return b->entry(i, j);
}

int hbx_build_dense_block(const hbx_hbuild *b, int r0, int nr, int c0, int nc, double *out) {
  if (!b || !out || r0 < 0 || c0 < 0 || nr < 0 || nc < 0 || r0 + nr > b->nofc || c0 + nc > b->nofc)
    return HBX_ERR_INVALID;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nc; ++c)
    for (int r = 0; r < nr; ++r)
      out[(size_t)r + (size_t)c * nr] = b->entry(b->lod[r0 + r], b->lod[c0 + c]);
  return HBX_OK;
}

}  // extern "C"
