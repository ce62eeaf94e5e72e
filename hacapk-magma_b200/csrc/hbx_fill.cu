// hbx_fill.cu -- the leaf fill on the GPU (HACApK_fill_leafmtx,
// m_HACApK_base.f90:978-1051): dense leaves receive their matrix entries,
// admissible leaves the ACA+ factors of HACApK_acaplus (:783-975), with the
// ppohBEM collocation kernel (m_ppohBEM_user_func.f90:49-99) evaluated on the
// device wherever the algorithm asks for an entry.
//
//   k_fill_dense  one CTA per dense leaf (grid-stride), one thread per entry.
//   k_fill_aca    one warp per admissible leaf: the rank loop is the
//                 reference's, scalar decisions are taken by every lane on the
//                 same broadcast values, and each vector step (a residual row
//                 or column, a scaling, an update of the reference row or
//                 column) is spread over the lanes.  Pivot searches are warp
//                 reductions that keep the reference's first-index tie rule;
//                 the scaled 2-norms (HACApK_lib.f90:31-46) are warp
//                 reductions too, equal to the reference's up to rounding.
//
// The file is compiled without FMA contraction (-fmad=false), like the host
// restatement, so every entry and every update is rounded as the reference
// writes it; only the device's atan2 and log may differ from the host C
// library's in the last bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/hacapk_b200.h"

namespace hbx {
namespace {

struct FillGeom {
  const double *fv;   // [nofc][9]: the face's vertex x0 x1 x2 y0 y1 y2 z0 z1 z2
  const double *zg;   // [3][nofc]: centroids (column-major zgmid)
  const int *lod;     // [nofc]: 1-based face id of each cluster-order position
  int nofc;
  int kernel;         // HBX_FILL_KERNEL_*
};

__device__ __forceinline__ void cross3(const double u[3], const double v[3], double w[3]) {
  w[0] = u[1] * v[2] - u[2] * v[1];
  w[1] = u[2] * v[0] - u[0] * v[2];
  w[2] = u[0] * v[1] - u[1] * v[0];
}

// face_integral of m_ppohBEM_user_func.f90:49-99: the analytic integral of
// 1/r over the flat triangle (xs, ys, zs) seen from (x, y, z); |sum|.
__device__ double face_integral_raw(const double *xs, const double *ys, const double *zs, double x, double y,
                                    double z) {
  double r[3];
  for (int a = 0; a < 3; ++a) {
    const double dx = xs[a] - x, dy = ys[a] - y, dz = zs[a] - z;
    r[a] = sqrt(dx * dx + dy * dy + dz * dz);
  }
  double u[3], v[3], w[3];
  u[0] = xs[1] - xs[0];
  v[0] = xs[2] - xs[1];
  u[1] = ys[1] - ys[0];
  v[1] = ys[2] - ys[1];
  u[2] = zs[1] - zs[0];
  v[2] = zs[2] - zs[1];
  cross3(u, v, w);
  const double wn = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  w[0] = w[0] / wn;
  w[1] = w[1] / wn;
  w[2] = w[2] / wn;
  u[0] = x - xs[0];
  u[1] = y - ys[0];
  u[2] = z - zs[0];
  const double zp = u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
  const double ox = x - zp * w[0], oy = y - zp * w[1], oz = z - zp * w[2];
  const double zpabs = fabs(zp);
  double sum = 0.0;
  for (int i = 0; i < 3; ++i) {
    const int j = (i + 1) % 3;
    u[0] = xs[j] - ox;
    u[1] = ys[j] - oy;
    u[2] = zs[j] - oz;
    const double xj = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    u[0] = u[0] / xj;
    u[1] = u[1] / xj;
    u[2] = u[2] / xj;
    cross3(w, u, v);
    const double xi = (xs[i] - ox) * u[0] + (ys[i] - oy) * u[1] + (zs[i] - oz) * u[2];
    const double yi = (xs[i] - ox) * v[0] + (ys[i] - oy) * v[1] + (zs[i] - oz) * v[2];
    const double dx = xj - xi, dy = -yi;
    const double t = sqrt(dx * dx + dy * dy);
    const double l = dx / t, m = dy / t;
    const double d = l * yi - m * xi;
    const double ti = l * xi + m * yi, tj = l * xj;
    const double theta = atan2(yi, xi);
    const double omega = theta - atan2(r[i] * d, zpabs * ti) + atan2(r[j] * d, zpabs * tj);
    const double q = log((r[j] + tj) / (r[i] + ti));
    const double g = d * q - zpabs * omega;
    sum = sum + g;
  }
  return fabs(sum);
}

// HACApK_entry_ij for 1-based face ids: collocation at the centroid of face
// i, integration over face j (m_ppohBEM_matrix_element_ij.f90:60-74).  The
// ppohBEM scale keeps the reference's single-precision literals PI and
// EPSILON_0 (m_ppohBEM_user_func.f90:42-43).
__device__ double entry(const FillGeom &g, int i, int j) {
  const double x = g.zg[i - 1], y = g.zg[(size_t)g.nofc + (i - 1)], z = g.zg[2 * (size_t)g.nofc + (i - 1)];
  const double *f = g.fv + 9 * (size_t)(j - 1);
  const double s = face_integral_raw(f, f + 3, f + 6, x, y, z);
  if (g.kernel == HBX_FILL_KERNEL_PPOHBEM) {
    const double pif = (double)3.141592653589793f, eps0 = (double)8.854187818f * 1e-12;
    return s / (4.0 * pif * eps0);
  }
  return s / (4.0 * 3.141592653589793);
}

struct DenseJob {
  int nstrtl, ndl, nstrtt, ndt;
  long long off;  // first word of the leaf in the output
};

// mem[(it-1) + (il-1) ndt] = entry(lod(il + nstrtl - 1), lod(it + nstrtt - 1))
__global__ void k_fill_dense(FillGeom g, const DenseJob *jobs, int njobs, double *out) {
  for (int q = blockIdx.x; q < njobs; q += gridDim.x) {
    const DenseJob J = jobs[q];
    const long long n = (long long)J.ndl * J.ndt;
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
      const int il = (int)(e / J.ndt), it = (int)(e % J.ndt);
      out[J.off + e] = entry(g, g.lod[il + J.nstrtl - 1], g.lod[it + J.nstrtt - 1]);
    }
  }
}


// A team of NT threads works on one leaf: NT = 32 is one warp, NT > 32 one
// CTA (the largest leaves, whose row and column steps have tens of thousands
// of entries).  Every member runs the same scalar control flow on the same
// values; `sd` / `si` are the team's shared scratch for cross-warp
// reductions (NT > 32 only).
template <int NT>
struct Team {
  int r;  // rank in the team
  double *sd;
  int *si;
  __device__ void sync() const {
    if (NT == 32) __syncwarp();
    else __syncthreads();
  }
  __device__ double max(double v) const {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (NT == 32) return v;
    sync();
    if ((r & 31) == 0) sd[r >> 5] = v;
    sync();
    double m = sd[0];
    for (int k = 1; k < NT / 32; ++k) m = fmax(m, sd[k]);
    return m;
  }
  __device__ double sum(double v) const {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (NT == 32) return v;
    sync();
    if ((r & 31) == 0) sd[r >> 5] = v;
    sync();
    double m = sd[0];
    for (int k = 1; k < NT / 32; ++k) m += sd[k];
    return m;
  }
};

// First 1-based index of the largest (kMax) or smallest |za| and the value
// (HACApK_lib.f90:48-57, :72-81): member-local scans in index order, then
// reductions in which equal values keep the smaller index.
template <bool kMax, int NT>
__device__ void team_absloc(const Team<NT> &T, const double *za, int nd, double &zz, int &il) {
  constexpr int kNone = 0x7fffffff;
  double best = 0.0;
  int bi = kNone;
  for (int it = T.r; it < nd; it += NT) {
    const double a = fabs(za[it]);
    if (bi == kNone || (kMax ? a > best : a < best)) {
      best = a;
      bi = it;
    }
  }
  auto better = [](double ob, int oi, double b, int i) {
    return oi != kNone && (i == kNone || (kMax ? ob > b : ob < b) || (ob == b && oi < i));
  };
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (better(ob, oi, best, bi)) {
      best = ob;
      bi = oi;
    }
  }
  // lane 0's result for the warp (a NaN makes the pairwise choice one-sided;
  // the lanes must still agree)
  best = __shfl_sync(0xffffffffu, best, 0);
  bi = __shfl_sync(0xffffffffu, bi, 0);
  if (NT > 32) {
    T.sync();
    if ((T.r & 31) == 0) {
      T.sd[T.r >> 5] = best;
      T.si[T.r >> 5] = bi;
    }
    T.sync();
    best = T.sd[0];
    bi = T.si[0];
    for (int k = 1; k < NT / 32; ++k)
      if (better(T.sd[k], T.si[k], best, bi)) {
        best = T.sd[k];
        bi = T.si[k];
      }
  }
  zz = best;
  il = bi + 1;
}

// The 2-norm of HACApK_lib.f90:31-46 (entries below 1e-30 in magnitude
// skipped, scaled by the largest one so that squares cannot overflow),
// reduced over the team: the same value as the reference's sequential
// scaled sum up to rounding in the last bits.
template <int NT>
__device__ double team_unrm(const Team<NT> &T, int nd, const double *za) {
  double zscl = 0.0;
  for (int il = T.r; il < nd; il += NT) {
    const double a = fabs(za[il]);
    if (a >= 1.0e-30 && a > zscl) zscl = a;
  }
  zscl = T.max(zscl);
  if (zscl == 0.0) return 0.0;
  const double inv = 1.0 / zscl;
  double s = 0.0;
  for (int il = T.r; il < nd; il += NT) {
    const double a = fabs(za[il]);
    if (a >= 1.0e-30) {
      const double t = a * inv;
      s = s + t * t;
    }
  }
  return zscl * sqrt(T.sum(s));
}

// One team's view of one leaf.
template <int NT>
struct LeafAca {
  FillGeom g;
  Team<NT> T;
  int ndl, ndt, nstrtl, nstrtt, cap;
  double *U, *V;  // column-major, capacity cap
  int *rmsk, *cmsk;

  __device__ double *ucol(int k1) const { return U + (size_t)ndl * (k1 - 1); }
  __device__ double *vcol(int k1) const { return V + (size_t)ndt * (k1 - 1); }

  // column jcol of the residual after k terms (calc_vec, m_HACApK_base.f90:677-698)
  __device__ void calc_col(int k, int jcol, double *vec) const {
    const int fcol = g.lod[jcol + nstrtt - 2];
    for (int ii = T.r; ii < ndl; ii += NT) {
      double v = vec[ii];
      if (rmsk[ii] == 0) v = entry(g, g.lod[ii + nstrtl - 1], fcol);
      if (k > 0) {
        double tmp = 0.0;
        for (int it = 1; it <= k; ++it) tmp = tmp + U[(size_t)ndl * (it - 1) + ii] * V[(size_t)ndt * (it - 1) + (jcol - 1)];
        v = v - tmp;
        if (rmsk[ii] == 1) v = 0.0;
      }
      vec[ii] = v;
    }
    T.sync();
  }
  // row irow of the residual after k terms
  __device__ void calc_row(int k, int irow, double *vec) const {
    const int frow = g.lod[irow + nstrtl - 2];
    for (int ii = T.r; ii < ndt; ii += NT) {
      double v = vec[ii];
      if (cmsk[ii] == 0) v = entry(g, frow, g.lod[ii + nstrtt - 1]);
      if (k > 0) {
        double tmp = 0.0;
        for (int it = 1; it <= k; ++it) tmp = tmp + V[(size_t)ndt * (it - 1) + ii] * U[(size_t)ndl * (it - 1) + (irow - 1)];
        v = v - tmp;
        if (cmsk[ii] == 1) v = 0.0;
      }
      vec[ii] = v;
    }
    T.sync();
  }
  __device__ void set_mask(int *m, int idx1) const {
    if (T.r == 0) m[idx1 - 1] = 1;
    T.sync();
  }
  __device__ void copy(double *dst, const double *src, int n) const {
    for (int a = T.r; a < n; a += NT) dst[a] = src[a];
    T.sync();
  }
  __device__ void scale(double *x, int n, double s) const {
    for (int a = T.r; a < n; a += NT) x[a] = x[a] * s;
    T.sync();
  }
  __device__ void axpy(double *y, const double *x, int n, double s) const {  // y = y + x s
    for (int a = T.r; a < n; a += NT) y[a] = y[a] + x[a] * s;
    T.sync();
  }
};

struct AcaJob {
  int nstrtl, ndl, nstrtt, ndt;
  int cap;            // columns of U and V in the workspace
  int kt;             // out: the rank; -1 when it would exceed cap
  long long woff;     // first double of the leaf's workspace: U (ndl cap), V (ndt cap), pa_ref (ndl), pb_ref (ndt)
  long long moff;     // first int of its masks: row (ndl), column (ndt)
};

struct AcaParams {
  double eps, aca_eps;  // relative tolerance, ACA_EPS = aca_abs_factor * eps
  int kmax, kmin;
};

// HACApK_acaplus (m_HACApK_base.f90:783-975) with param(61) = 1 for one leaf;
// returns kt, or -1 when the rank would exceed the workspace's columns.
template <int NT>
__device__ int aca_plus(const LeafAca<NT> &C, const AcaParams &P, double *pa_ref, double *pb_ref) {
  const Team<NT> &T = C.T;
  const int ndl = C.ndl, ndt = C.ndt;
  const double za_ACA_EPS = (double)1.0e-30f;
  const double ACA_EPS = P.aca_eps, eps = P.eps;
  const int kmax = P.kmax, kmin = P.kmin;
  int ntries = max(ndl, ndt) + 1, ntries_row = 6, ntries_col = 6;
  for (int a = T.r; a < ndl; a += NT) {
    C.rmsk[a] = 0;
    pa_ref[a] = 0.0;
  }
  for (int a = T.r; a < ndt; a += NT) {
    C.cmsk[a] = 0;
    pb_ref[a] = 0.0;
  }
  T.sync();
  int k = 0;
  if (C.cap < 1) return -1;
  int j_ref = 1;
  C.calc_col(k, j_ref, pa_ref);
  double colnorm = team_unrm(T, ndl, pa_ref);
  double rownorm;
  int i_ref;
  team_absloc<false>(T, pa_ref, ndl, rownorm, i_ref);
  C.calc_row(k, i_ref, pb_ref);
  rownorm = team_unrm(T, ndt, pb_ref);
  double apxnorm = 0.0;
  int lstop_aca = 0;
  double col_maxval = 0.0, row_maxval = 0.0;
  int i = 0, j = 0;
  while ((k < kmax) && (ntries_row > 0 || ntries_col > 0) && (ntries > 0)) {
    ntries = ntries - 1;
    if (k + 1 > C.cap) return -1;
    double *pcol = C.ucol(k + 1);
    double *prow = C.vcol(k + 1);
    team_absloc<true>(T, pa_ref, ndl, col_maxval, i);
    team_absloc<true>(T, pb_ref, ndt, row_maxval, j);
    if (row_maxval > col_maxval) {
      if (j != j_ref) C.calc_col(k, j, pcol);
      else C.copy(pcol, pa_ref, ndl);
      team_absloc<true>(T, pcol, ndl, col_maxval, i);
      if (col_maxval < ACA_EPS && k >= kmin) {
        lstop_aca = 1;
      } else {
        C.calc_row(k, i, prow);
        const double piv = pcol[i - 1];
        if (!(fabs(piv) > (double)1.0e-20f)) {
          k = max(k - 1, 0);
          break;
        }
        T.sync();  // every member has read the pivot before the column is scaled
        C.scale(pcol, ndl, 1.0 / piv);
      }
    } else {
      if (i != i_ref) C.calc_row(k, i, prow);
      else C.copy(prow, pb_ref, ndt);
      team_absloc<true>(T, prow, ndt, row_maxval, j);
      if (row_maxval < ACA_EPS && k >= kmin) {
        lstop_aca = 1;
      } else {
        C.calc_col(k, j, pcol);
        const double piv = prow[j - 1];
        if (!(fabs(piv) > (double)1.0e-20f)) {
          k = max(k - 1, 0);
          break;
        }
        T.sync();
        C.scale(prow, ndt, 1.0 / piv);
      }
    }
    C.set_mask(C.rmsk, i);
    C.set_mask(C.cmsk, j);

    if (i != i_ref) {
      C.axpy(pb_ref, prow, ndt, -pcol[i_ref - 1]);
      rownorm = team_unrm(T, ndt, pb_ref);
    }
    if (i == i_ref || rownorm < ACA_EPS) {
      if (i == i_ref) ntries_row = ntries_row + 1;
      if (ntries_row > 0) {
        rownorm = 0.0;
        i = i_ref;
        while (i != ((i_ref + ndl - 2) % ndl) + 1 && rownorm < za_ACA_EPS && ntries_row > 0) {
          if (C.rmsk[i - 1] == 0) {
            if (k + 1 > C.cap) return -1;
            C.calc_row(k + 1, i, pb_ref);
            rownorm = team_unrm(T, ndt, pb_ref);
            if (rownorm < ACA_EPS) C.set_mask(C.rmsk, i);
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
      C.axpy(pa_ref, pcol, ndl, -prow[j_ref - 1]);
      colnorm = team_unrm(T, ndl, pa_ref);
    }
    if (j == j_ref || colnorm < ACA_EPS) {
      if (j == j_ref) ntries_col = ntries_col + 1;
      if (ntries_col > 0) {
        colnorm = 0.0;
        j = j_ref;
        while (j != ((j_ref + ndt - 2) % ndt) + 1 && colnorm < za_ACA_EPS && ntries_col > 0) {
          if (C.cmsk[j - 1] == 0) {
            if (k + 1 > C.cap) return -1;
            C.calc_col(k + 1, j, pa_ref);
            colnorm = team_unrm(T, ndl, pa_ref);
            if (colnorm < ACA_EPS) C.set_mask(C.cmsk, j);
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
      lstop_aca = 1;
      k = k + 1;
    }
    if (lstop_aca == 0) {
      const double blknorm = team_unrm(T, ndl, pcol) * team_unrm(T, ndt, prow);
      if (k == 0) {
        apxnorm = blknorm;
      } else if (blknorm < apxnorm * eps && rownorm < apxnorm * eps && colnorm < apxnorm * eps && k >= kmin) {
        lstop_aca = 1;
      }
    }
    if (lstop_aca == 1 && k >= kmin) break;
    k = k + 1;
  }
  return k;
}

// One team per leaf: NT = 32 runs eight warps per CTA, each its own leaf;
// NT > 32 one CTA per leaf.
template <int NT>
__global__ void __launch_bounds__(NT == 32 ? 256 : NT) k_fill_aca(FillGeom g, AcaJob *jobs, int njobs, AcaParams P,
                                                                 double *work, int *masks) {
  __shared__ double sd[NT == 32 ? 1 : NT / 32];
  __shared__ int si[NT == 32 ? 1 : NT / 32];
  const int teams_per_cta = NT == 32 ? (int)(blockDim.x >> 5) : 1;
  const int team = NT == 32 ? (int)(threadIdx.x >> 5) : 0;
  const Team<NT> T{(int)(NT == 32 ? (threadIdx.x & 31) : threadIdx.x), sd, si};
  for (int q = blockIdx.x * teams_per_cta + team; q < njobs; q += gridDim.x * teams_per_cta) {
    AcaJob &J = jobs[q];
    double *w = work + J.woff;
    const LeafAca<NT> C{g, T, J.ndl, J.ndt, J.nstrtl, J.nstrtt, J.cap, w, w + (size_t)J.ndl * J.cap,
                        masks + J.moff, masks + J.moff + J.ndl};
    double *pa_ref = w + (size_t)(J.ndl + J.ndt) * J.cap;
    double *pb_ref = pa_ref + J.ndl;
    const int kt = aca_plus<NT>(C, P, pa_ref, pb_ref);
    if (T.r == 0) J.kt = kt;
    T.sync();
  }
}

// The factors of job q, columns 1..kt, from its workspace into the packed
// output: V (ndt x kt) then U (ndl x kt), both column-major (a1 and a2 of
// the reference leaf, m_HACApK_base.f90:1021-1028).
struct PackJob {
  long long woff, out;
  int ndl, ndt, cap, kt;
};
__global__ void k_pack_aca(const PackJob *jobs, int njobs, const double *work, double *out) {
  for (int q = blockIdx.x; q < njobs; q += gridDim.x) {
    const PackJob J = jobs[q];
    const double *U = work + J.woff, *V = U + (size_t)J.ndl * J.cap;
    const long long nv = (long long)J.ndt * J.kt, nu = (long long)J.ndl * J.kt;
    for (long long e = threadIdx.x; e < nv; e += blockDim.x) out[J.out + e] = V[e];
    for (long long e = threadIdx.x; e < nu; e += blockDim.x) out[J.out + nv + e] = U[e];
  }
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace hbx

struct hbx_fill {
  double *storage = nullptr;  // host memory of every leaf's a1 (and a2)
  size_t words = 0;
};

namespace {

thread_local std::string g_fill_error;

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

extern "C" {

void hbx_fill_free(hbx_fill *f);

int hbx_fill_leaves(const double *xyz, int nond, const int *face2node, int nofc, const int *lod,
                    const hbx_fill_params *params, stc_HACApK_leafmtxp *st, hbx_fill **out, hbx_fill_stats *stats) {
  using namespace hbx;
  if (out) *out = nullptr;
  if (!xyz || !face2node || !lod || !params || !st || !out || nond <= 0 || nofc <= 0 || st->nlf < 0 ||
      (st->nlf > 0 && !st->st_lf) || st->st_lf_stride < (int)sizeof(stc_HACApK_leafmtx))
    return HBX_ERR_INVALID;
  if (params->kernel != HBX_FILL_KERNEL_PPOHBEM && params->kernel != HBX_FILL_KERNEL_LAPLACE) return HBX_ERR_INVALID;
  if (!(params->aca_eps > 0.0) || params->kmax < 1 || params->kmin < 0) return HBX_ERR_INVALID;
  const double t0 = now_s();
  const int nlf = st->nlf;
  auto leaf = [&](int ip) -> stc_HACApK_leafmtx & {
    return *reinterpret_cast<stc_HACApK_leafmtx *>(reinterpret_cast<char *>(st->st_lf) + (size_t)ip * st->st_lf_stride);
  };
  // geometry: face vertices and centroids as hbx_build forms them
  std::vector<double> fv(9 * (size_t)nofc), zg(3 * (size_t)nofc);
  for (int f = 0; f < nofc; ++f) {
    double *o = &fv[9 * (size_t)f];
    for (int a = 0; a < 3; ++a) {
      const int n = face2node[3 * (size_t)f + a];
      if (n < 0 || n >= nond) return HBX_ERR_INVALID;
      o[a] = xyz[3 * (size_t)n];
      o[3 + a] = xyz[3 * (size_t)n + 1];
      o[6 + a] = xyz[3 * (size_t)n + 2];
    }
    zg[f] = (o[0] + o[1] + o[2]) / 3.0;
    zg[(size_t)nofc + f] = (o[3] + o[4] + o[5]) / 3.0;
    zg[2 * (size_t)nofc + f] = (o[6] + o[7] + o[8]) / 3.0;
  }
  for (int i = 0; i < nofc; ++i)
    if (lod[i] < 1 || lod[i] > nofc) return HBX_ERR_INVALID;
  std::vector<DenseJob> dense;
  std::vector<int> dense_ip, aca_ip;
  long long dense_words = 0;
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx &L = leaf(ip);
    if (L.ndl <= 0 || L.ndt <= 0 || L.nstrtl < 1 || L.nstrtt < 1 || L.nstrtl - 1 + L.ndl > nofc ||
        L.nstrtt - 1 + L.ndt > nofc || (L.ltmtx != 1 && L.ltmtx != 2))
      return HBX_ERR_INVALID;
    if (L.ltmtx == 2) {
      dense.push_back(DenseJob{L.nstrtl, L.ndl, L.nstrtt, L.ndt, dense_words});
      dense_ip.push_back(ip);
      dense_words += (long long)L.ndl * L.ndt;
    } else {
      aca_ip.push_back(ip);
    }
  }
  cudaError_t e;
  DevBuf d_fv, d_zg, d_lod;
  if ((e = cudaMalloc(&d_fv.p, fv.size() * 8)) != cudaSuccess || (e = cudaMalloc(&d_zg.p, zg.size() * 8)) != cudaSuccess ||
      (e = cudaMalloc(&d_lod.p, (size_t)nofc * 4)) != cudaSuccess)
    return e == cudaErrorMemoryAllocation ? HBX_ERR_NOMEM : HBX_ERR_CUDA;
  cudaMemcpy(d_fv.p, fv.data(), fv.size() * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(d_zg.p, zg.data(), zg.size() * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(d_lod.p, lod, (size_t)nofc * 4, cudaMemcpyHostToDevice);
  const FillGeom g{static_cast<const double *>(d_fv.p), static_cast<const double *>(d_zg.p),
                   static_cast<const int *>(d_lod.p), nofc, params->kernel};
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);

  // largest leaves first, so that the warps that take them start at once
  std::stable_sort(aca_ip.begin(), aca_ip.end(), [&](int a, int b) {
    const stc_HACApK_leafmtx &x = leaf(a), &y = leaf(b);
    return (long long)x.ndl * x.ndt > (long long)y.ndl * y.ndt;
  });
  // ---- ACA+ in batches of leaves whose workspaces fit the budget; a leaf
  // whose rank outgrows its columns is run again with twice as many.  The
  // packed factors of every batch stay on the device until the end.
  const AcaParams P{params->aca_eps, params->aca_abs_factor * params->aca_eps, params->kmax, params->kmin};
  const size_t budget = (params->workspace_mb > 0 ? (size_t)params->workspace_mb : 4096) << 20;
  const bool verbose = std::getenv("HBX_FILL_VERBOSE") != nullptr;
  std::vector<int> kt_of(aca_ip.size(), 0);
  std::vector<int> out_buf(aca_ip.size(), -1);        // device output buffer of each ACA leaf
  std::vector<long long> out_off(aca_ip.size(), 0);   // its first word there
  std::vector<DevBuf> outs;                           // packed factors, one buffer per batch
  outs.reserve(64);
  std::vector<long long> out_words;
  std::vector<size_t> todo(aca_ip.size());
  for (size_t q = 0; q < todo.size(); ++q) todo[q] = q;
  const int first_cap = params->first_cap > 0 ? params->first_cap : 64;
  long long retried = 0;
  double t_aca = 0.0;
  // leaves with more rows plus columns than this get a CTA, the rest a warp
  constexpr int kBigLeaf = 4096, kBigTeam = 512;
  DevBuf d_work, d_mask, d_jobs;
  size_t work_cap = 0, mask_cap = 0, jobs_cap = 0;
  auto ensure = [&](DevBuf &b, size_t &cap, size_t bytes) -> cudaError_t {
    if (bytes <= cap) return cudaSuccess;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    cap = 0;
    cudaError_t r = cudaMalloc(&b.p, bytes);
    if (r == cudaSuccess) cap = bytes;
    return r;
  };
  for (int round = 0; !todo.empty(); ++round) {
    if (round > 24) return HBX_ERR_INVALID;  // cannot happen: the capacity doubles up to every leaf's full rank
    std::vector<size_t> again;
    size_t pos = 0;
    while (pos < todo.size()) {
      std::vector<AcaJob> jobs;
      std::vector<size_t> which;
      long long wd = 0, wm = 0;
      bool big = false;
      while (pos < todo.size()) {
        const stc_HACApK_leafmtx &L = leaf(aca_ip[todo[pos]]);
        const bool b = L.ndl + L.ndt >= kBigLeaf;
        if (!jobs.empty() && b != big) break;
        // the rank never exceeds min(ndl, ndt) (one row and one column are
        // retired per step) nor kmax, and a step may look one column ahead
        const int full = std::min(std::min(L.ndl, L.ndt), params->kmax) + 2;
        const long long c = (long long)first_cap << std::min(round, 20);
        const int cap = (int)std::min<long long>(c, full);
        const long long need = (long long)(L.ndl + L.ndt) * (cap + 1);
        if (!jobs.empty() && (size_t)(wd + need) * 8 + (size_t)(wm + L.ndl + L.ndt) * 4 > budget) break;
        big = b;
        jobs.push_back(AcaJob{L.nstrtl, L.ndl, L.nstrtt, L.ndt, cap, 0, wd, wm});
        which.push_back(todo[pos]);
        wd += need;
        wm += L.ndl + L.ndt;
        ++pos;
      }
      const double tb = now_s();
      if ((e = ensure(d_jobs, jobs_cap, jobs.size() * sizeof(AcaJob))) != cudaSuccess ||
          (e = ensure(d_work, work_cap, (size_t)wd * 8)) != cudaSuccess ||
          (e = ensure(d_mask, mask_cap, (size_t)wm * 4)) != cudaSuccess)
        return e == cudaErrorMemoryAllocation ? HBX_ERR_NOMEM : HBX_ERR_CUDA;
      cudaMemcpy(d_jobs.p, jobs.data(), jobs.size() * sizeof(AcaJob), cudaMemcpyHostToDevice);
      if (big) {
        const int nblk = (int)std::min<size_t>(jobs.size(), (size_t)nsm * 4);
        k_fill_aca<kBigTeam><<<nblk, kBigTeam>>>(g, static_cast<AcaJob *>(d_jobs.p), (int)jobs.size(), P,
                                                 static_cast<double *>(d_work.p), static_cast<int *>(d_mask.p));
      } else {
        const int wpb = 8;
        const int nblk = (int)std::min<size_t>((jobs.size() + wpb - 1) / wpb, (size_t)nsm * 16);
        k_fill_aca<32><<<nblk, 32 * wpb>>>(g, static_cast<AcaJob *>(d_jobs.p), (int)jobs.size(), P,
                                           static_cast<double *>(d_work.p), static_cast<int *>(d_mask.p));
      }
      if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess) {
        g_fill_error = cudaGetErrorString(e);
        return HBX_ERR_CUDA;
      }
      cudaMemcpy(jobs.data(), d_jobs.p, jobs.size() * sizeof(AcaJob), cudaMemcpyDeviceToHost);
      const double tk = now_s();
      // pack the finished leaves' factors into this batch's output buffer
      std::vector<PackJob> pk;
      long long ow = 0;
      const int ob = (int)outs.size();
      for (size_t q = 0; q < jobs.size(); ++q) {
        if (jobs[q].kt < 0) {
          again.push_back(which[q]);
          continue;
        }
        pk.push_back(PackJob{jobs[q].woff, ow, jobs[q].ndl, jobs[q].ndt, jobs[q].cap, jobs[q].kt});
        kt_of[which[q]] = jobs[q].kt;
        out_buf[which[q]] = ob;
        out_off[which[q]] = ow;
        ow += (long long)(jobs[q].ndl + jobs[q].ndt) * jobs[q].kt;
      }
      if (!pk.empty()) {
        outs.emplace_back();
        out_words.push_back(ow);
        DevBuf d_pk;
        if ((e = cudaMalloc(&d_pk.p, pk.size() * sizeof(PackJob))) != cudaSuccess ||
            (e = cudaMalloc(&outs.back().p, std::max<long long>(1, ow) * 8)) != cudaSuccess)
          return e == cudaErrorMemoryAllocation ? HBX_ERR_NOMEM : HBX_ERR_CUDA;
        cudaMemcpy(d_pk.p, pk.data(), pk.size() * sizeof(PackJob), cudaMemcpyHostToDevice);
        k_pack_aca<<<(int)std::min<size_t>(pk.size(), (size_t)nsm * 8), 256>>>(
            static_cast<PackJob *>(d_pk.p), (int)pk.size(), static_cast<double *>(d_work.p),
            static_cast<double *>(outs.back().p));
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) return HBX_ERR_CUDA;
      }
      t_aca += tk - tb;
      if (verbose)
        std::fprintf(stderr, "hbx_fill: round %d batch of %zu %s leaves, workspace %.2f GB, ACA+ %.3f s, pack %.3f s\n",
                     round, jobs.size(), big ? "large" : "small", wd * 8e-9, tk - tb, now_s() - tk);
    }
    retried += round == 0 ? (long long)again.size() : 0;
    todo.swap(again);
  }
  const double t1 = now_s();

  // ---- dense leaves, on the device
  DevBuf d_dense;
  if (!dense.empty()) {
    DevBuf d_jobs;
    if ((e = cudaMalloc(&d_jobs.p, dense.size() * sizeof(DenseJob))) != cudaSuccess ||
        (e = cudaMalloc(&d_dense.p, std::max<long long>(1, dense_words) * 8)) != cudaSuccess)
      return e == cudaErrorMemoryAllocation ? HBX_ERR_NOMEM : HBX_ERR_CUDA;
    cudaMemcpy(d_jobs.p, dense.data(), dense.size() * sizeof(DenseJob), cudaMemcpyHostToDevice);
    k_fill_dense<<<(int)std::min<size_t>(dense.size(), (size_t)nsm * 16), 256>>>(
        g, static_cast<DenseJob *>(d_jobs.p), (int)dense.size(), static_cast<double *>(d_dense.p));
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess) return HBX_ERR_CUDA;
  }
  const double t2 = now_s();

  // ---- leaf storage in the reference layout: the dense entries, then every
  // batch's packed factors, each copied from the device once
  size_t words = (size_t)dense_words;
  for (long long w : out_words) words += (size_t)w;
  hbx_fill *F = new (std::nothrow) hbx_fill();
  if (!F) return HBX_ERR_NOMEM;
  F->words = words;
  F->storage = static_cast<double *>(std::malloc(std::max<size_t>(1, words) * 8));
  if (!F->storage) {
    delete F;
    return HBX_ERR_NOMEM;
  }
  std::vector<size_t> base(outs.size());
  {
    size_t o = (size_t)dense_words;
    for (size_t k = 0; k < outs.size(); ++k) {
      base[k] = o;
      o += (size_t)out_words[k];
    }
  }
  // first touch of the destination pages by every host core (a pageable
  // copy into untouched memory runs at a tenth of the speed)
  const double t3 = now_s();
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)words; i += 512) F->storage[i] = 0.0;
  const double t4 = now_s();
  if (dense_words > 0) e = cudaMemcpy(F->storage, d_dense.p, (size_t)dense_words * 8, cudaMemcpyDeviceToHost);
  for (size_t k = 0; k < outs.size() && e == cudaSuccess; ++k)
    if (out_words[k] > 0) e = cudaMemcpy(F->storage + base[k], outs[k].p, (size_t)out_words[k] * 8, cudaMemcpyDeviceToHost);
  if (verbose) std::fprintf(stderr, "hbx_fill: first touch %.3f s, copies %.3f s\n", t4 - t3, now_s() - t4);
  if (e != cudaSuccess) {
    hbx_fill_free(F);
    return HBX_ERR_CUDA;
  }
  int ktmax = 0, nlfkt = 0;
  for (size_t q = 0; q < dense.size(); ++q) {
    stc_HACApK_leafmtx &L = leaf(dense_ip[q]);
    L.kt = 0;
    L.a1 = F->storage + dense[q].off;
    L.a2 = nullptr;
    L.a1size = (long long)L.ndl * L.ndt * 8;
  }
  for (size_t q = 0; q < aca_ip.size(); ++q) {
    stc_HACApK_leafmtx &L = leaf(aca_ip[q]);
    const int kt = kt_of[q];
    double *p = F->storage + base[out_buf[q]] + out_off[q];
    L.kt = kt;
    L.a1 = p;
    L.a1size = (long long)L.ndt * kt * 8;
    L.a2 = p + (size_t)L.ndt * kt;
    ktmax = std::max(ktmax, kt);
    ++nlfkt;
  }
  st->ktmax = ktmax;
  st->nlfkt = nlfkt;
  if (verbose)
    std::fprintf(stderr, "hbx_fill: ACA+ %.3f s (kernels), all batches %.3f s, dense %.3f s, to the host %.3f s\n",
                 t_aca, t1 - t0, t2 - t1, now_s() - t2);
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->n_lowrank = nlfkt;
    stats->n_dense = (int)dense.size();
    stats->ktmax = ktmax;
    stats->words = (long long)words;
    stats->retried = retried;
    stats->seconds = now_s() - t0;
  }
  *out = F;
  return HBX_OK;
}

void hbx_fill_free(hbx_fill *f) {
  if (!f) return;
  std::free(f->storage);
  delete f;
}

}  // extern "C"
