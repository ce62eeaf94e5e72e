/*
 * hacapk_b200_build.h -- host-side construction of HACApK leaf lists.
 *
 * This is the input side of the H-matvec path: surface meshes, the
 * ppohBEM collocation kernel, HACApK's cluster tree, block partition and
 * ACA+ fill, producing a stc_HACApK_leafmtxp in exactly the layout the
 * reference's C layer reads.  It is a CPU restatement of
 * m_HACApK_base.f90 / m_ppohBEM_user_func.f90 (OpenMP over leaves), not a
 * GPU deliverable; libhacapk_build.so has no CUDA dependency.
 */
#ifndef HACAPK_B200_BUILD_H
#define HACAPK_B200_BUILD_H

#include "hacapk_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Kernel selector for the BEM matrix entry. */
enum {
  /* face_integral of m_ppohBEM_user_func.f90:49-99 as written: the
   * single-precision literals PI and EPSILON_0 (:42-43) and the
   * 1/(4*PI*EPSILON_0) scale (:98). */
  HBX_KERNEL_PPOHBEM = 0,
  /* The same analytic flat-triangle integral of 1/r with the scale
   * 1/(4*pi) in double precision (Laplace single layer). */
  HBX_KERNEL_LAPLACE = 1
};

typedef struct hbx_build_params {
  int leaf_size;        /* param(21): cluster leaf size (reference default 15) */
  double eta;           /* param(51): admissibility parameter (2.0)            */
  double aca_eps;       /* param(71): ACA+ relative tolerance                  */
  double aca_abs_factor;/* param(72): ACA_EPS = aca_abs_factor * aca_eps       */
  int kmax;             /* param(63): rank limit (1000)                        */
  int kmin;             /* param(64): minimum rank (1)                         */
  int kernel;           /* HBX_KERNEL_*                                         */
  int nthreads;         /* OpenMP threads for the fill; 0 = runtime default    */
  int fill;             /* 0: block structure only (no ACA+/dense fill)        */
  int aca_method;       /* param(60): 1 = ACA, 2 = ACA+ (reference default 2)  */
  int reserved[6];
} hbx_build_params;

/* Fills `p` with the reference defaults of HACApK_init (m_HACApK_base.f90:294-313). */
void hbx_build_default_params(hbx_build_params *p);

typedef struct hbx_build_stats {
  int nd;
  int nclst;            /* clusters created (m_HACApK_base.f90:433)           */
  int n_lowrank;        /* lnmtx(1) */
  int n_dense;          /* lnmtx(2) */
  int n_hnode;          /* lnmtx(3): non-leaf block nodes                      */
  int ktmax;
  long long mem_words;  /* sum (ndl+ndt)*kt + sum ndl*ndt (HACApK_chk_leafmtx) */
  long long memh_words; /* mem_words + nlf (the reference's "H matrix memory") */
  long long ncpc7;      /* the same with kt := param(62)=7 (HACApK_setcutrow)  */
  double seconds_tree;
  double seconds_fill;
  int reserved[8];
} hbx_build_stats;

typedef struct hbx_hbuild hbx_hbuild;

/* Unit icosphere by repeated 4-way subdivision of the icosahedron with
 * midpoints projected to the sphere: 10*4^L+2 vertices, 20*4^L faces.
 * xyz: 3*nv doubles (x,y,z per vertex); faces: 3*nf 0-based vertex ids. */
int hbx_mesh_icosphere(int level, double *xyz, int *faces);

/* Builds the H-matrix of the collocation matrix of `kernel` on the mesh:
 * row i = centroid of face i, column j = integral over face j.
 * face2node is 0-based (the .pbf/.pbs convention). */
int hbx_build(const double *xyz, int nond, const int *face2node, int nofc,
              const hbx_build_params *params, hbx_hbuild **out);
void hbx_build_free(hbx_hbuild *b);

/* Leaf list in the reference layout (stride sizeof(stc_HACApK_leafmtx)). */
stc_HACApK_leafmtxp *hbx_build_leafmtxp(hbx_hbuild *b);
/* lod(1:nd): 1-based face id of cluster-order position i. */
const int *hbx_build_lod(const hbx_hbuild *b);
int hbx_build_get_stats(const hbx_hbuild *b, hbx_build_stats *s);
/* Face centroids zgmid(nofc,3) (column-major, as m_ppohBEM_bembb2hacapk.f90:102-106). */
const double *hbx_build_centroids(const hbx_hbuild *b);

/* Matrix entry for 1-based face ids (HACApK_entry_ij). */
double hbx_build_entry(const hbx_hbuild *b, int i, int j);
/* Dense block of the matrix in cluster order: out[(r-r0) + (c-c0)*nr] for
 * cluster-order rows r0..r0+nr-1, columns c0..c0+nc-1 (0-based). */
int hbx_build_dense_block(const hbx_hbuild *b, int r0, int nr, int c0, int nc, double *out);

#ifdef __cplusplus
}
#endif
#endif /* HACAPK_B200_BUILD_H */
