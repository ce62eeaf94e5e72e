// hbx_engine.h -- engine state behind the opaque hbx_hmat handle, and the
// kernel launchers shared by the hbx_* API and the HACApK drop-in symbols.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "hbx_plan.h"

namespace hbx {

// Partial-sum slots of the BiCGSTAB reductions (per CTA, compensated pairs).
enum : int {
  kSlotRhoR = 0,   // rh . r
  kSlotRR = 1,     // r . r
  kSlotRhAp = 2,   // rh . Ap
  kSlotAtT = 3,    // At . t
  kSlotAtAt = 4,   // At . At
  kSlotBB = 5,     // b . b
  kSlotAux = 6,    // scratch (true residual)
  kSlots = 8
};

// Solver scalars carried from one iteration launch to the next.
struct BicgState {
  double alpha, zeta, rho, beta;
  double relres, bnorm;
  int iter, done, status, breakdown;
};

struct MatvecArgs {
  const uint8_t *stream;
  const RunRec *recs;
  const CtaInfo *ctas;
  const RunLite *lite;
  const double *x;
  const double *yin;
  double *y;
  double *zbu;
  const float *x32;  // FP32 engines: x rounded to float (gathered instead of x)
  float *zbu32;      // FP32 engines: zbu rounded to float (gathered by the U runs)
  uint64_t zbu_len;
  double alpha, beta;
  unsigned *gbar;
  int *err;
  unsigned long long timeout_ns;
  unsigned long long *prof;  // optional: per-CTA %globaltimer stamps [num_ctas][16], slots 0-5
  uint32_t keep_frac;        // fraction (of 2^16) of each CTA's stream kept in L2 between passes; 0: no hints
  uint32_t stall;            // test hook: the launch's grid barrier waits for one instance more than can
                             // complete, so its bounded waits expire (hbx_debug_stall_next_barrier)
  const int *skip;           // optional: the launch does nothing while *skip is set (a solver's done flag)
  // optional (block-diagonal engines): chunk g of CTA c covers instances
  // [lo, hi] = chunk_inst[chunk_base[c] + g] (lo | hi << 16); a chunk none of
  // whose instances is active (inst_pre: prefix counts of active instances,
  // count + 1 entries) is not copied, and the rows of inactive instances
  // come out undefined
  const uint32_t *chunk_inst, *chunk_base;
  const int *inst_pre;
};

struct BicgArgs {
  const uint8_t *stream;
  const RunRec *recs;
  const CtaInfo *ctas;
  const RunLite *lite;
  const Atom *atoms;
  double *zbu;      // [2][zbu_len]: one copy per H-matvec of a step
  uint64_t zbu_len;
  unsigned *gbar;
  int *err;
  unsigned long long timeout_ns;
  const double *b;
  double *u, *r, *rh, *p, *ap, *t, *at;
  float *p32, *t32, *zbu32;  // FP32 engines: float copies of the matvec inputs (zbu32: [2][zbu_len])
  double *part;   // [num_ctas][kSlots][2]
  BicgState *state;
  double *hist;   // relres per iteration (max_iter + 1 entries)
  unsigned long long *prof;  // optional: per-CTA %globaltimer stamps [num_ctas][16], slots 8-15
  double tol;
  int max_iter;
  uint32_t keep_frac;  // as MatvecArgs::keep_frac
};

// Multi-RHS product on the tensor cores (hbx_mrhs.cu): Y = alpha*H*X +
// beta*Yin for kNrhs right-hand sides, rows of kNrhs values (RHS-contiguous).
constexpr int kNrhs = 64;
struct MatmatArgs {
  const uint8_t *stream;  // packed with pair_panels (FP32)
  const RunRec *recs;
  const CtaInfo *ctas;
  const RunLite *lite;
  const float *x;     // [nd][kNrhs]
  const double *yin;  // [nd][kNrhs], read when beta != 0
  double *y;          // [nd][kNrhs]
  float *zbu;         // [zbu_len][kNrhs]
  double alpha, beta;
  unsigned *gbar;
  int *err;
  unsigned long long timeout_ns;
};
size_t matmat_smem_bytes();
cudaError_t configure_matmat();
cudaError_t launch_matmat(const MatmatArgs &a, int num_ctas, cudaStream_t s);

// Multi-RHS BiCGSTAB (hbx_mrhs_solve.cu): scalars of one right-hand side.
struct MrScal {
  double alpha, zeta, rho, beta, rr, rtol;
  int active, iters, status, pad;
};
// One step for every right-hand side still running (10 launches, two of
// them the product through `matmat`).
struct MrStep {
  int nd, max_iter;
  MrScal *sc;
  int *any_active;
  double *r, *rh, *p, *ap, *t, *at, *x, *part;
  float *f32;  // the product's input (p, then t, rounded to float)
  cudaError_t (*matmat)(void *ctx, const float *x, double *y, cudaStream_t s);
  void *ctx;
};
int mr_row_blocks(int nd);
cudaError_t mr_launch_dots(int nq, int nd, const double *x0, const double *y0, const double *x1, const double *y1,
                           double *part, cudaStream_t s);
cudaError_t mr_launch_setup(int nd, const double *R, double *r, double *rh, double *p, double *ap, double *x,
                            cudaStream_t s);
cudaError_t mr_launch_init(int nd, const double *part, const double *thresh, const int *mask, MrScal *sc,
                           int *any_active, cudaStream_t s);
cudaError_t mr_launch_step(const MrStep &a, cudaStream_t s);
cudaError_t mr_launch_colsum(int nd, const double *part, double *out, cudaStream_t s);
cudaError_t mr_launch_transpose(int rows, int cols, const double *in, double *out, cudaStream_t s);
cudaError_t mr_launch_resid(int nd, const double *B, const double *HU, double *R, cudaStream_t s);
cudaError_t mr_launch_add(int nd, const int *mask, const double *D, double *U, cudaStream_t s);

// Batched BiCGSTAB over the instances of a block-diagonal engine
// (hbx_batch.cu); one MrScal per instance, rtol = the relative tolerance.
struct BtStep {
  size_t n;
  int count, max_iter;
  int *pre;  // optional: prefix counts of active instances, refreshed before each product
  const int *off, *rinst;  // instance row offsets [count + 1], instance of every row
  MrScal *sc;
  int *any_active;
  double *r, *rh, *p, *ap, *t, *at, *u, *dots, *bnorm;
  cudaError_t (*matvec)(void *ctx, const double *x, double *y, cudaStream_t s);
  void *ctx;
};
cudaError_t bt_launch_dots(int nq, int count, const int *off, const double *x0, const double *y0, const double *x1,
                           const double *y1, double *out, cudaStream_t s);
cudaError_t bt_launch_setup(size_t n, const double *r, double *rh, double *p, double *ap, cudaStream_t s);
cudaError_t bt_launch_init(int count, const double *dots, double tol, const double *rtol, int max_iter, MrScal *sc,
                           double *bnorm, int *any_active, cudaStream_t s);
cudaError_t bt_launch_mask(size_t n, const int *rinst, const int *flag, double *r, cudaStream_t s);
cudaError_t bt_launch_step(const BtStep &a, cudaStream_t s);
cudaError_t bt_launch_prefix(int count, const MrScal *sc, int *pre, cudaStream_t s);

// Dot products of up to kMaxDots vector pairs per launch (hbx_gcr.cu;
// compensated per-block partials part[blocks][kMaxDots][2], summed in block
// order into out[k]); the GCR restart length is at most kMaxDots.
constexpr int kMaxDots = 64;
int gcr_dot_blocks(size_t n);
cudaError_t gcr_launch_dots(int k, const double *const *x, const double *const *y, size_t n, double *part,
                            double *out, cudaStream_t s);

// GCR(m) (hbx_gcr.cu; m_HACApK_solve.f90:506-571), state on the device.
struct GcrState {
  double bnorm, relres, tol, alpha;
  double capap[kMaxDots], beta[kMaxDots];
  int step, max_iter, done, status;
  unsigned ticket;  // last-block counter of the fused reductions
  int pad;
};
struct GcrVecs {
  const double *b;
  double *u, *r, *ar;  // ar: A r of the current step
  double *p, *ap;      // m slots of nd each
};
cudaError_t gcr_launch_init(const GcrVecs &v, size_t n, GcrState *st, double *part, double tol, int max_iter,
                            cudaStream_t s);
cudaError_t gcr_launch_alpha0(const GcrVecs &v, size_t n, GcrState *st, double *part, cudaStream_t s);
cudaError_t gcr_launch_update(const GcrVecs &v, size_t n, int ik, GcrState *st, double *part, cudaStream_t s);
cudaError_t gcr_launch_orth(const GcrVecs &v, size_t n, int ik, int ikn, GcrState *st, double *part,
                            cudaStream_t s);

// Pipelined BiCGSTAB (hbx_pipe.cu; HACApK_SOLVER_PIPE.c:144-600).  The state
// lives on the device so that a batch of steps runs as one captured graph.
struct PipeState {
  double alpha, beta, zeta, znorm, bnorm, relres, tol;
  int step, max_iter, done, status;
  unsigned ticket;  // last-block counter of the fused reductions
  int pad;
};
struct PipeVecs {
  const double *b;
  double *u, *r, *r0, *w, *t, *v, *p, *s, *z, *q, *y;
};
constexpr int kPipeVecs = 10;  // r, r0, w, t, v, p, s, z, q, y
cudaError_t pipe_launch_init(const PipeVecs &v, size_t n, PipeState *st, double *part, double *hist, double tol,
                             int max_iter, cudaStream_t s);
cudaError_t pipe_launch_a(const PipeVecs &v, size_t n, PipeState *st, double *part, cudaStream_t s);
cudaError_t pipe_launch_b(const PipeVecs &v, size_t n, PipeState *st, double *part, double *hist, cudaStream_t s);

// Static scratch of hbx_matvec_noalloc (hbx_kernels.cu): 256 bytes of
// barrier words, then room for kNoallocZbuMax zbu doubles.
constexpr size_t kNoallocScratchBytes = size_t(1) << 20;
constexpr size_t kNoallocCtlBytes = 256;
constexpr uint64_t kNoallocZbuMax = (kNoallocScratchBytes - kNoallocCtlBytes) / sizeof(double);
cudaError_t noalloc_scratch_address(void **ptr);

// Kernel launchers (hbx_kernels.cu).
size_t kernel_smem_bytes();
cudaError_t configure_kernels();
cudaError_t configure_step_kernels();     // the step kernels' translation unit
cudaError_t configure_step_kernels_lp();  // the FP32 / BF16 step kernels' unit
cudaError_t launch_bicg_iter_lp(const BicgArgs &a, int num_ctas, cudaStream_t s, int precision);
cudaError_t launch_matvec(const MatvecArgs &a, int num_ctas, cudaStream_t s, int precision);
cudaError_t launch_bicg_setup(const BicgArgs &a, int num_ctas, cudaStream_t s);
cudaError_t launch_bicg_iter(const BicgArgs &a, int num_ctas, cudaStream_t s, int precision);
// part[.][slot] = sum over own rows of x.y; then out[0] = the total (one block).
cudaError_t launch_axpy(double alpha, const double *x, double *y, size_t n, cudaStream_t s);
cudaError_t launch_to_float(const double *x, float *y, size_t n, cudaStream_t s);
cudaError_t launch_dot(const BicgArgs &a, const double *x, const double *y, int slot, double *out,
                       int num_ctas, cudaStream_t s);

}  // namespace hbx

struct hbx_hmat {
  int device = 0;
  int num_ctas = 0;
  int transposed = 0;  // the packed stream holds H^T
  int nrhs = 1;        // right-hand sides per product (kNrhs: multi-RHS engine, hbx_matmat only)
  float *d_zbum = nullptr;  // multi-RHS engine: zbu for all right-hand sides [zbu_len][kNrhs]
  // multi-RHS solver workspace (hbx_bicgstab_multi)
  double *d_mrv = nullptr;      // r, rh, p, ap, t, at, x, R, and two kNrhs x nd scratch arrays
  float *d_mr32 = nullptr;      // nd x kNrhs
  double *d_mrpart = nullptr;   // [row blocks][2][kNrhs]
  hbx::MrScal *d_mrsc = nullptr;
  int *d_mrint = nullptr;       // any_active, mask[kNrhs]
  double *d_mrdbl = nullptr;    // thresholds[kNrhs], norms[kNrhs]
  void *h_mrpin = nullptr;      // pinned: MrScal[kNrhs], norms, thresholds, ints
  // block-diagonal batch of independent instances (hbx_create_batch)
  std::vector<int> inst_off;    // row offsets, count + 1 entries (empty: one instance)
  int *d_inst_off = nullptr;    // the same on the device
  int *d_rinst = nullptr;       // instance of every row
  // per-instance stream skipping (hbx_create_batch; MatvecArgs::chunk_inst):
  // the chunk table, each CTA's first entry, prefix counts of active
  // instances, and whether products skip inactive instances right now
  uint32_t *d_chunk_inst = nullptr, *d_chunk_base = nullptr;
  int *d_inst_pre = nullptr;
  int skip_inactive = 0;
  int merge_keep = -1;  // the planner's merged D+U setting in use
  int l2_keep_mb = 0;   // the L2 budget of the stream in use (MB; 0: no hints)
  void *d_rflag = nullptr;  // refined batch: per-instance flags and inner tolerances
  double *d_btv = nullptr;      // r, rh, p, ap, t, at (6 nd)
  hbx::MrScal *d_btsc = nullptr;
  double *d_btdbl = nullptr;    // dots [count][2], bnorm [count], true norms [count]
  int *d_btany = nullptr;
  hbx::Plan plan;
  uint8_t *d_stream = nullptr;
  hbx::RunRec *d_recs = nullptr;
  long long num_runs = 0;
  hbx::CtaInfo *d_ctas = nullptr;
  hbx::RunLite *d_lite = nullptr;
  hbx::Atom *d_atoms = nullptr;
  double *d_zbu = nullptr;
  unsigned *d_gbar = nullptr;
  int *d_err = nullptr;
  unsigned long long timeout_ns = 2000000000ull;
  uint32_t keep_frac = 0;  // fraction (of 2^16) of every CTA's stream kept in L2 between passes
  uint32_t stall_next = 0; // test hook: the next k_matvec launch's grid barrier cannot complete
  unsigned long long *d_prof = nullptr;  // phase stamps of the last matvec (HBX_PROFILE=1)
  double setup_seconds = 0.0;
  cudaStream_t stream = nullptr;  // used by the host-vector calls
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr, ev4 = nullptr;
  // host-vector staging
  double *d_x = nullptr, *d_y = nullptr;
  double *h_pin = nullptr;        // pinned staging, 2*nd doubles
  // solver workspace
  double *d_work = nullptr;       // r, rh, p, ap, t, at, b, u  (8*nd)
  double *d_part = nullptr;
  double *d_dot = nullptr;
  hbx::BicgState *d_state = nullptr;
  hbx::BicgState *h_state = nullptr;  // pinned
  double *d_hist = nullptr;
  double *d_refine = nullptr;     // mixed-precision solve: outer residual and correction (2*nd)
  float *d_f32 = nullptr;         // FP32 engines: x, p, t (3*nd) and zbu (zbu_len) rounded to float
  int hist_cap = 0;
  // GCR(m): r, A r, p[m], Ap[m] (nd each); device state and its pinned copy;
  // per-block partials; the captured restart cycle(s)
  double *d_gcr = nullptr;
  int gcr_m = 0;
  hbx::GcrState *d_gcrs = nullptr, *h_gcrs = nullptr;
  double *d_gcrpart = nullptr;
  cudaGraphExec_t ggraph = nullptr;
  int ggraph_m = 0, ggraph_cycles = 0;
  const void *ggraph_key = nullptr;
  // pipelined BiCGSTAB: vectors (kPipeVecs*nd), device state, pinned copy,
  // per-block partials, relres history, captured step batch
  double *d_pipe = nullptr;
  hbx::PipeState *d_pstate = nullptr, *h_pstate = nullptr;
  double *d_ppart = nullptr, *d_phist = nullptr;
  int phist_cap = 0;
  cudaGraphExec_t pgraph = nullptr;
  int pgraph_batch = 0;
  const void *pgraph_key = nullptr;
  // captured iteration batch
  cudaGraphExec_t graph = nullptr;
  int graph_batch = 0;
  const void *graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
};
