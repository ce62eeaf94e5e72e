/*
 * hacapk_b200.h -- C ABI of the B200-native H-matrix matvec / BiCGSTAB engine.
 *
 * Two layers live behind this header:
 *
 *  1. The HACApK drop-in symbols.  They keep the names, argument lists and
 *     by-reference (Fortran) calling convention of the HACApK-MAGMA C layer so
 *     that the Fortran driver (m_HACApK_solve.f90 / m_HACApK_use.f90) links
 *     against libhacapk_b200.so instead of the MAGMA batched-GEMV objects.
 *     Each declaration cites the reference function it replaces.
 *
 *  2. The hbx_* API: status-returning, stream-aware calls on an opaque
 *     engine handle.  The drop-in symbols are thin wrappers around it.
 *
 * All vectors are in HACApK's cluster (permuted) order and all leaf offsets
 * (nstrtl, nstrtt) are 1-based, exactly as in the reference leaf list.
 * No torch or CUDA types appear in any signature; streams are passed as
 * `void *` holding a cudaStream_t (NULL = the legacy default stream).
 */
#ifndef HACAPK_B200_H
#define HACAPK_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define HBX_ABI_VERSION 1

/* ------------------------------------------------------------------------ */
/* Leaf-matrix layout (mirrors HACApK_MAGMA.h:12-121, HAVE_MAGMA_BATCH build) */
/* ------------------------------------------------------------------------ */

/* One leaf of the H-matrix (HACApK_MAGMA.h:12-20, m_HACApK_base.f90:54-61).
 *  ltmtx = 1: low-rank, A ~= U V^T with V = a1 (ndt x kt, column-major) and
 *             U = a2 (ndl x kt, column-major) found at (char*)a1 + a1size.
 *  ltmtx = 2: dense, a1 is ndt x ndl column-major, A(il,it) = a1[it + il*ndt].
 * Only a1 (the first word of the Fortran pointer descriptor) and a1size are
 * read; `a2` is never dereferenced, matching HACApK_MAGMA.c:27. */
typedef struct stc_HACApK_leafmtx {
  int ltmtx;
  int kt;
  int nstrtl, ndl;
  int nstrtt, ndt;
  long long int a1size;
  double *a1;
  double *a2;
} stc_HACApK_leafmtx;

/* Container (HACApK_MAGMA.h:28-106, m_HACApK_base.f90:64-235).  The GPU/batch
 * fields are kept only so that `st_lf` sits at the offset a MAGMA build of the
 * Fortran type expects; this engine keeps its own state in a side table keyed
 * by the container address and never writes these fields.  The leaves are
 * found at (char*)st_lf + ip*st_lf_stride. */
typedef struct stc_HACApK_leafmtxp {
  int nd;
  int nlf;
  int nlfkt;
  int ktmax;
  int st_lf_stride;
  /* HAVE_MAGMA | HAVE_MAGMA_BATCH block */
  int m, n, gn, max_block;
  double gflops;
  void *mtx1_gpu, *mtx2_gpu, *zu_gpu, *zau_gpu, *zau_pin, *zbu_gpu;
  int num_batch, total_size_y, transA;
  void *d_A_array, *d_X_array, *d_Y_array;
  void *d_M, *d_N, *d_lda, *d_inc;
  void *batch_order;
  void *h_A_array, *h_X_array, *h_Y_array;
  void *h_type, *h_I, *h_J, *h_M, *h_N, *h_lda, *max_M, *max_N, *batch_size;
  int num_streamed, num_streamed_t;
  void *h_A_array_streamed, *h_X_array_streamed, *h_Y_array_streamed;
  void *h_M_streamed, *h_N_streamed, *h_lda_streamed;
  void *d_A_mgpu, *d_X_mgpu, *d_Y_mgpu, *d_M_mgpu, *d_N_mgpu, *d_lda_mgpu, *d_inc_mgpu;
  void *zu_mgpu, *zau_mgpu, *zbu_mgpu;
  void *h_A_mgpu, *h_X_mgpu, *h_Y_mgpu, *h_type_mgpu, *h_I_mgpu, *h_J_mgpu;
  void *h_M_mgpu, *h_N_mgpu, *h_lda_mgpu, *max_M_mgpu, *max_N_mgpu;
  void *nlf_mgpu, *num_batch_mgpu, *total_size_y_mgpu;
  int *iwork;
  int mpi_rank;
  /* end of HAVE_MAGMA block */
  stc_HACApK_leafmtx *st_lf;
} stc_HACApK_leafmtxp;

/* Control block (HACApK_MAGMA.h:108-121).  `param` is HACApK's param(1:100)
 * array; lpmd/lod/lsp/lnp/lthr are found at byte offsets from `param`.
 * C indices used here: param[0] verbosity, param[82] max steps,
 * param[90] BiCGSTAB tolerance, lpmd[1] nrank, lpmd[2] rank. */
typedef struct stc_HACApK_lcontrol {
  int lf_umpi;
  int lpmd_offset;
  int lod_offset;
  int lsp_offset;
  int lnp_offset;
  int lthr_offset;
  double *param;
} stc_HACApK_lcontrol;

/* ------------------------------------------------------------------------ */
/* hbx_* API                                                                */
/* ------------------------------------------------------------------------ */

typedef enum hbx_status {
  HBX_OK = 0,
  HBX_ERR_INVALID = 1,       /* bad argument or malformed leaf list        */
  HBX_ERR_NOMEM = 2,         /* host or device allocation failed           */
  HBX_ERR_CUDA = 3,          /* CUDA runtime error                         */
  HBX_ERR_TIMEOUT = 4,       /* a bounded device wait expired              */
  HBX_ERR_BREAKDOWN = 5,     /* BiCGSTAB breakdown (zero/non-finite scalar)*/
  HBX_ERR_NOT_CONVERGED = 6, /* iteration limit reached before tolerance   */
  HBX_ERR_NONFINITE = 7,     /* NaN or Inf in an input vector              */
  HBX_ERR_UNSUPPORTED = 8    /* e.g. more than one MPI rank                */
} hbx_status;

/* Storage precision of the packed factors.  HBX_FP32 rounds every factor
 * to float once, at hbx_create, and multiplies in float (four columns per
 * 16-byte load), adding each run's products to double row sums; vectors,
 * dot products and solver scalars stay double.  HBX_BF16 rounds every
 * factor to bfloat16 (8 significant bits, nearest, ties to even) and
 * multiplies the widened factors by float vectors in float, eight columns
 * per 16-byte load: a quarter of the FP64 bytes.  bfloat16 has float's
 * exponent range, so no per-leaf scale is needed to keep the factors in
 * range.  No counterpart in the reference, which is FP64 throughout. */
enum { HBX_FP64 = 0, HBX_FP32 = 1, HBX_BF16 = 2 };

typedef struct hbx_hmat hbx_hmat;

typedef struct hbx_options {
  int precision;   /* HBX_FP64, HBX_FP32 or HBX_BF16 (factor storage)     */
  int num_ctas;    /* persistent CTAs; 0 = one per SM                     */
  int transpose;   /* 1: the engine holds H^T (adjoint products and solves;
                      no counterpart in the reference)                    */
  int nrhs;        /* 0 or 1: single-vector engine (hbx_matvec, solves);
                      HBX_NRHS: multi-RHS engine for hbx_matmat (needs
                      precision = HBX_FP32; no counterpart in the reference) */
  int block_cost;  /* balancing cost model of the CTA schedule: the fixed   */
  int run_cost;    /* cost of a block end and of a run, in bytes (0 = the
                      defaults 8192 and 4096; hbx_autotune picks them)      */
  int merge;       /* single-vector engines: an atom's dense and low-rank
                      columns in one run ("merged D+U") for every atom with
                      low-rank rows except each CTA's first k, which stay
                      split; merge = k + 1, -1 for no merged runs, 0 for the
                      default k = 4 (HBX_MERGE_KEEP overrides the default) */
  int l2_keep_mb;  /* megabytes of the factor stream kept in L2 from one
                      product to the next (the head of every CTA's stream is
                      read with evict_last); 0 = the default 24
                      (HBX_L2_KEEP_MB overrides it), -1 = no cache hints   */
  int reserved[8];
} hbx_options;

/* Right-hand sides of one hbx_matmat call on a multi-RHS engine. */
#define HBX_NRHS 64

typedef struct hbx_info {
  int nd, nlf, nlfkt, ktmax;
  int num_ctas, num_atoms, num_runs, precision;
  long long stream_bytes;  /* packed factor bytes streamed per matvec        */
  long long alg_bytes;     /* algorithmic bytes per single-RHS matvec with
                              FP64 factors (B_H), whatever the storage       */
  long long alg_flops;     /* 2*(sum dense ndl*ndt + sum kt*(ndl+ndt))       */
  long long zbu_len;       /* sum of kt over low-rank leaves                  */
  long long dense_words, lowrank_words;
  double setup_seconds;
  int transposed;          /* 1 when the engine holds H^T                    */
  int nrhs;                /* right-hand sides per product (1 or HBX_NRHS)   */
  int instances;           /* independent H-matrices (hbx_create_batch)     */
  int block_cost, run_cost; /* the CTA schedule's cost model in use          */
  int merge_keep;           /* atoms kept split per CTA (-1: no merged runs)  */
  int l2_keep_mb;           /* L2 budget of the stream in MB (0: no hints)    */
  int reserved[1];
} hbx_info;

typedef struct hbx_solve_opts {
  double tol;          /* stop when ||r||/||b|| < tol (checked before each step) */
  int max_iter;        /* iteration limit (param[82] in the drop-in)             */
  int verbose;         /* >0: print the residual history like the reference     */
  int batch;           /* iterations per graph replay between host checks (0=8) */
  int restart;         /* hbx_gcr: restart length m, param(87) (0 = 8; at most 64) */
  double inner_tol;    /* mixed-precision solve: relative residual reduction asked
                          of each inner solve at most (0 = 1e-6)                 */
  int reserved[8];
} hbx_solve_opts;

typedef struct hbx_solve_info {
  int iterations;      /* completed BiCGSTAB steps (nstp)                     */
  int status;          /* hbx_status of the solve                             */
  double bnorm;        /* ||b||_2                                             */
  double relres;       /* recursive residual ||r||/||b|| at exit              */
  double true_relres;  /* ||b - H u|| / ||b|| recomputed after the solve      */
  double seconds;      /* device time from r0 = b - H u0 to the last step     */
  double iter_kernel_seconds; /* device time of the iteration launches only   */
  int iter_launches;   /* iteration-kernel launches (includes the final
                          launches that only observe convergence)             */
  int launches;        /* all kernel launches of the solve                    */
  int outer;           /* mixed-precision solve: refinement steps (FP64 residuals) */
  int reserved[5];
} hbx_solve_info;

/* Packs the leaf list into the engine's per-CTA streaming layout and uploads
 * it to the current device.  Replaces the setup half of
 * c_hacapk_adot_body_lfcpy_batch_sorted_ (HACApK_BATCH_SORT.c:86-858). */
int hbx_create(const stc_HACApK_leafmtxp *st, int nd, const hbx_options *opt,
               hbx_hmat **out);
/* One engine over `count` independent H-matrices (no counterpart in the
 * reference, which holds one body): their leaves form one block-diagonal
 * H, instance k owning rows and columns [off_k, off_k + nd[k]) with
 * off_k = nd[0] + ... + nd[k-1], so hbx_matvec multiplies every body in one
 * persistent launch and hbx_bicgstab_batch solves them all at once.  Vectors
 * are the instances' vectors (each in its own cluster order) one after the
 * other.  Same options as hbx_create except nrhs. */
int hbx_create_batch(const stc_HACApK_leafmtxp *const *st, const int *nd, int count, const hbx_options *opt,
                     hbx_hmat **out);

/* Autotuner of the schedule and layout (no counterpart in the reference,
 * whose size-class batches are fixed by HACApK_BATCH_SORT.c): builds engines
 * for a grid of CTA schedules -- the planner's block and run costs, and the
 * number of CTAs -- then, for single-vector engines and around the best
 * schedule, for the merged D+U layout (`merge`) and then for the L2 budget of
 * the stream (`l2_keep_mb`), with `base`'s precision, orientation and nrhs;
 * times the product of each on the current device (hbx_matvec, or
 * hbx_matmat for a multi-RHS base; 3 untimed and `reps` timed launches, CUDA
 * events) and returns in `best` the options of the fastest, in `best_us` its
 * time and in `default_us` the time of the defaults (both nullable).  Takes
 * one engine build per candidate (10 for multi-RHS engines, 17 otherwise). */
int hbx_autotune(const stc_HACApK_leafmtxp *st, int nd, const hbx_options *base, int reps, hbx_options *best,
                 double *best_us, double *default_us);

/* Frees device and host state (HACApK_BATCH.c:812-859). */
int hbx_destroy(hbx_hmat *h);
int hbx_get_info(const hbx_hmat *h, hbx_info *info);

/* y = alpha * H x + beta * yin on device pointers; yin may equal y; beta == 0
 * ignores yin.  One persistent kernel launch on `stream`.  Replaces
 * c_hacapk_adot_body_lfmtx_batch_queue with on_gpu=1 (HACApK_BATCH.c:47-255). */
int hbx_matvec(hbx_hmat *h, double alpha, const double *x, double beta,
               const double *yin, double *y, void *stream);

/* Allocation-free variant of hbx_matvec (no counterpart in the reference).
 * For callers that cannot call cudaMalloc once they are running: a host code
 * that reserves the GPU's memory for its own pool at start-up, where a later
 * cudaMalloc fails for lack of room, and a time-stepping loop that must not
 * stall, where cudaFree would synchronize the whole device.  Same kernel and
 * same result as hbx_matvec, but the per-call scratch (the V^T x segments and
 * the grid-barrier words) comes from one fixed 1 MiB device array compiled
 * into the library, reserved when the library's kernels load and held by
 * every GPU that loads them until the process exits.  Limit: matrices whose
 * low-rank ranks sum to more than 131040 are rejected with HBX_ERR_INVALID.
 * The call allocates nothing: it clears the barrier words and launches on
 * `stream`.  The array's address is looked up on a device's first call and
 * kept: make that first call before any stream capture, and do not use the
 * call again in a process after cudaDeviceReset (or another teardown of the
 * device's context), which leaves the kept address stale.  All calls share the array, so
 * calls that overlap on the GPU (other streams, other engines) race:
 * serialize them.  Device-side wait failures latch in the engine's error
 * word (hbx_sync). */
int hbx_matvec_noalloc(hbx_hmat *h, double alpha, const double *x, double beta,
                       const double *yin, double *y, void *stream);

/* Y = alpha * H X + beta * Yin for HBX_NRHS right-hand sides at once, on an
 * engine created with hbx_options.nrhs = HBX_NRHS (no counterpart in the
 * reference, whose batched GEMV takes one vector).  X is nd x HBX_NRHS floats,
 * Yin and Y nd x HBX_NRHS doubles, all row-major (the HBX_NRHS values of a row
 * adjacent) on the device; beta == 0 ignores Yin.  The products run on the
 * tensor cores (TF32 inputs: factors and X rounded to 10-bit mantissas, FP32
 * accumulation): a relative error of order 1e-3 per entry, meant as the inner
 * product of an iterative refinement.  One persistent launch on `stream`. */
int hbx_matmat(hbx_hmat *h, double alpha, const float *X, double beta, const double *Yin, double *Y,
               void *stream);

/* BiCGSTAB of every instance of a batch engine at once (no counterpart in the
 * reference): each instance runs the algorithm of HACApK_SOLVER.c:602-732
 * with its own scalars and stops on its own when ||r||/||b|| of its rows is
 * below opts->tol (checked before every step, as HACApK_SOLVER.c:631) or
 * after opts->max_iter steps (a convergence mask: its rows of the products
 * are zero from then on).  Both products of a step are one block-diagonal
 * launch each.  b, u: device vectors of the engine's size (u: x0 in, solutions
 * out); info (nullable) receives one entry per instance, true_relres being
 * recomputed as ||b - H u||/||b|| after the solve.  On a plain engine this is
 * BiCGSTAB with plain (not compensated) dot products.  Returns HBX_OK when
 * every instance converged. */
int hbx_bicgstab_batch(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info,
                       void *stream);
/* The same with host vectors (copies inside). */
int hbx_bicgstab_batch_host(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts,
                            hbx_solve_info *info);
/* Mixed-precision batched solve (the uneven-batch form with FP32 or BF16
 * factors): h an FP64 batch engine, hl a batch engine over the same
 * instances with precision HBX_FP32 or HBX_BF16.  Each outer step computes
 * every instance's FP64 residual on h; instances still above opts->tol get
 * a correction from the batched BiCGSTAB on hl, each to its own inner
 * tolerance max(opts->inner_tol (1e-6 when 0), tol / (2 relres)); the others
 * are masked out (their chunks are not streamed).  info: one entry per
 * instance (iterations = its inner steps, outer = refinement steps,
 * true_relres = its last FP64 residual). */
int hbx_bicgstab_batch_refined(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u, const hbx_solve_opts *opts,
                               hbx_solve_info *info, void *stream);
int hbx_bicgstab_batch_refined_host(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u,
                                    const hbx_solve_opts *opts, hbx_solve_info *info);

/* BiCGSTAB for HBX_NRHS right-hand sides at once (no counterpart in the
 * reference): FP64 iterative refinement around the algorithm of
 * c_hacapk_bicgstab_cax_lfmtx_gpu_ (HACApK_SOLVER.c:602-732) run for every
 * right-hand side with its own scalars and its own stop test (a convergence
 * mask) on `hm`, a multi-RHS engine (hbx_options.nrhs = HBX_NRHS) of the same
 * leaf list, so both products of a step go through one tensor-core launch.
 * Each refinement step forms R = B - H U with the FP64 engine `h` (one
 * product per unconverged right-hand side), solves H D = R on `hm` until each
 * residual falls by max(opts->inner_tol (0 = 1e-3), tol*||b||/||r||/2) and
 * adds D to U; a right-hand side stops once its FP64 residual
 * ||b - H u||/||b|| is below opts->tol, or after opts->max_iter inner steps.
 * B and U are nd x HBX_NRHS doubles, row-major, on the device (U: x0 in,
 * solutions out); info (nullable) receives HBX_NRHS entries, one per
 * right-hand side (iterations = its inner steps, outer = refinement steps,
 * true_relres = its final FP64 residual).  Returns HBX_OK when every
 * right-hand side converged. */
int hbx_bicgstab_multi(hbx_hmat *h, hbx_hmat *hm, const double *B, double *U, const hbx_solve_opts *opts,
                       hbx_solve_info *info, void *stream);
/* The same with host arrays (copies inside, on an internal stream). */
int hbx_bicgstab_multi_host(hbx_hmat *h, hbx_hmat *hm, const double *B, double *U, const hbx_solve_opts *opts,
                            hbx_solve_info *info);

/* GCR(m) on device vectors (HACApK_gcrm_lfmtx, m_HACApK_solve.f90:506-571,
 * which the reference runs on the host only): restarted every opts->restart
 * steps (param(87)), the stop test ||r||/||b|| < opts->tol after each step,
 * at most opts->max_iter steps (param(83)).  Each step is one H-matvec
 * launch and a few vector launches; dot products are compensated and summed
 * in a fixed order.  u: x0 in, solution out; info->iterations = nstp. */
int hbx_gcr(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info,
            void *stream);
/* The same with host vectors (copies inside). */
int hbx_gcr_host(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info);

/* Pipelined BiCGSTAB on device vectors (c_hacapk_bicgstab_cax_lfmtx_pipe_,
 * HACApK_SOLVER_PIPE.c:144-600; _pipe2_, :640, is the same arithmetic): the
 * products of p and s are carried by recurrences, so a step is two H-matvecs
 * and two fused reduction kernels; batches of opts->batch steps (8 by
 * default) run as one CUDA graph.  Stop test ||r||/||b|| < opts->tol before
 * each step, at most opts->max_iter steps.  u: x0 in, solution out (the
 * reference accumulates the iterate in an uninitialised vector and returns
 * u unchanged, HACApK_SOLVER_PIPE.c:592).  HBX_ERR_BREAKDOWN when a
 * denominator of the recurrences is zero or not finite. */
int hbx_bicgstab_pipe(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts, hbx_solve_info *info,
                      void *stream);
/* The same with host vectors (copies inside). */
int hbx_bicgstab_pipe_host(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts,
                           hbx_solve_info *info);

/* Mixed-precision BiCGSTAB (no counterpart in the reference): FP64
 * iterative refinement around BiCGSTAB on `hl`, an engine created on the same
 * leaf list with hbx_options.precision = HBX_FP32.  Each refinement step
 * forms the residual r = b - H u with the FP64 engine `h`, solves H d = r on
 * `hl` until its residual falls by max(opts->inner_tol, tol*||b||/||r||/2)
 * and adds d to u, until ||b - H u|| / ||b|| < opts->tol (FP64, measured) or
 * opts->max_iter inner steps in all.  info->iterations counts the inner
 * steps, info->outer the refinement steps, info->true_relres is the final
 * FP64 residual.  u: x0 in, solution out (device pointers, on `stream`). */
int hbx_bicgstab_refined(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u, const hbx_solve_opts *opts,
                         hbx_solve_info *info, void *stream);
/* The same with host vectors (copies inside). */
int hbx_bicgstab_refined_host(hbx_hmat *h, hbx_hmat *hl, const double *b, double *u, const hbx_solve_opts *opts,
                              hbx_solve_info *info);

/* Adjoint sensitivity of J(g) = 0.5 ||sigma - sigma_t||^2 where H sigma = g
 * (no counterpart in the reference): solves H sigma = g with `h`, then
 * H^T lambda = sigma - sigma_t with `ht` (an engine created with
 * hbx_options.transpose = 1 on the same leaf list), and returns
 * grad = dJ/dg = lambda.  Host vectors of nd doubles; sigma and grad are
 * written (their contents on entry are ignored: both solves start from 0).
 * `fwd` / `adj` (optional) receive the two solves' statistics. */
int hbx_gradient_host(hbx_hmat *h, hbx_hmat *ht, const double *g, const double *sigma_t, double *sigma,
                      double *grad, double *J, const hbx_solve_opts *opts, hbx_solve_info *fwd,
                      hbx_solve_info *adj);

/* Waits for `stream` and returns the device error latched by earlier async
 * calls on this engine (HBX_ERR_TIMEOUT when a bounded device wait expired),
 * clearing it. */
int hbx_sync(hbx_hmat *h, void *stream);

/* Host vectors: zau = (accumulate ? zau : 0) + H zu, with the H2D/D2H copies
 * inside the call (HACApK_BATCH.c:257-271 semantics when accumulate=1).
 * kernel_seconds / copy_seconds (nullable) are incremented. */
int hbx_matvec_host(hbx_hmat *h, const double *zu, double *zau, int accumulate,
                    double *kernel_seconds, double *copy_seconds);

/* BiCGSTAB on device vectors (u holds x0 on entry, the solution on exit).
 * Algorithm of c_hacapk_bicgstab_cax_lfmtx_gpu_ (HACApK_SOLVER.c:421-807). */
int hbx_bicgstab(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts,
                 hbx_solve_info *info, void *stream);
/* Same with host vectors; copies are inside the call. */
int hbx_bicgstab_host(hbx_hmat *h, const double *b, double *u, const hbx_solve_opts *opts,
                      hbx_solve_info *info);

/* Diagnostics: per-CTA %globaltimer stamps of the phases of the last matvec
 * (only when the engine was created with HBX_PROFILE=1 in the environment);
 * copies up to cap values into out, returns how many. */
int hbx_debug_phase_stamps(hbx_hmat *h, unsigned long long *out, int cap);

/* ------------------------------------------------------------------------ */
/* Leaf fill on the GPU                                                     */
/* ------------------------------------------------------------------------ */

/* Collocation kernel of the fill: HBX_FILL_KERNEL_PPOHBEM is face_integral of
 * m_ppohBEM_user_func.f90:49-99 as written (single-precision literals PI and
 * EPSILON_0 of :42-43, scale 1/(4 PI EPSILON_0)); HBX_FILL_KERNEL_LAPLACE the
 * same analytic flat-triangle integral of 1/r scaled by 1/(4 pi) in double. */
enum { HBX_FILL_KERNEL_PPOHBEM = 0, HBX_FILL_KERNEL_LAPLACE = 1 };

typedef struct hbx_fill_params {
  int kernel;            /* HBX_FILL_KERNEL_*                                    */
  double aca_eps;        /* param(71): ACA+ relative tolerance                   */
  double aca_abs_factor; /* param(72): ACA_EPS = aca_abs_factor * aca_eps        */
  int kmax;              /* param(63): rank limit                                */
  int kmin;              /* param(64): minimum rank                              */
  int workspace_mb;      /* device workspace of one batch of leaves (0 = 4096)   */
  int first_cap;         /* rank columns tried first per leaf (0 = 64); a leaf
                            that needs more is run again with twice as many     */
  int reserved[8];
} hbx_fill_params;

typedef struct hbx_fill_stats {
  int n_lowrank, n_dense, ktmax;
  long long words;       /* factor and entry words stored                       */
  long long retried;     /* leaves run again with more rank columns            */
  double seconds;
  int reserved[6];
} hbx_fill_stats;

typedef struct hbx_fill hbx_fill;

/* Fills the leaves of `st` on the current device, replacing
 * HACApK_fill_leafmtx (m_HACApK_base.f90:978-1051): every dense leaf
 * (ltmtx 2) receives its entries, every admissible leaf (ltmtx 1) the
 * factors of HACApK_acaplus (:783-975, param(61) = 1) and its rank kt, with
 * the collocation kernel evaluated on the GPU (collocation at the centroid of
 * face lod(i), integration over face lod(j); xyz: 3 nond doubles, face2node:
 * 3 nofc 0-based vertex ids, lod: nofc 1-based face ids in cluster order).
 * On entry the leaves carry ltmtx, nstrtl, ndl, nstrtt, ndt (the block
 * partition, e.g. from hbx_build with fill = 0); on return kt, a1size, a1 and
 * a2 are set as the reference lays them out, st->ktmax and st->nlfkt too,
 * and the factor storage belongs to *out until hbx_fill_free. */
int hbx_fill_leaves(const double *xyz, int nond, const int *face2node, int nofc, const int *lod,
                    const hbx_fill_params *params, stc_HACApK_leafmtxp *st, hbx_fill **out,
                    hbx_fill_stats *stats);
void hbx_fill_free(hbx_fill *f);

/* Test hooks of the failure paths (no counterpart in the reference).
 * hbx_debug_stall_next_barrier: the engine's next hbx_matvec launch waits on
 * a grid-barrier instance that cannot complete, so its bounded device waits
 * expire after the engine's timeout (HBX_TIMEOUT_MS at create, 2 s by
 * default) and the launch ends; hbx_sync then reports HBX_ERR_TIMEOUT and
 * resets the barrier words, and the engine works again.
 * hbx_debug_fail_alloc(n): the n-th device allocation made by this library
 * from now on (n = 0: the next one) fails as cudaMalloc does on a full
 * device; n < 0 turns the hook off. */
int hbx_debug_stall_next_barrier(hbx_hmat *h);
int hbx_debug_fail_alloc(int n);

const char *hbx_status_string(int status);
/* Message of the last failing hbx_* call on this host thread. */
const char *hbx_last_error(void);

/* ------------------------------------------------------------------------ */
/* HACApK drop-in entry points (Fortran calling convention)                 */
/* ------------------------------------------------------------------------ */

/* HACApK_MAGMA.c:69-75 -- device initialisation / release. */
void magma_init_(void);
void magma_finalize_(void);

/* HACApK_BATCH_SORT.c:86 -- pack and upload the leaf list. */
void c_hacapk_adot_body_lfcpy_batch_sorted_(int *nd, stc_HACApK_leafmtxp *st_leafmtxp);
/* HACApK_BATCH.c:257 -- zau += H zu with host vectors; zbu is unused
 * (host workspace in the reference); the three timers are incremented. */
void c_hacapk_adot_body_lfmtx_batch_(double *zau, stc_HACApK_leafmtxp *st_leafmtxp,
                                     double *zu, double *zbu, double *time_batch,
                                     double *time_set, double *time_copy);
/* HACApK_BATCH.c:812 -- release device state. */
void c_hacapk_adot_body_lfdel_batch_(stc_HACApK_leafmtxp *st_leafmtxp);

/* HACApK_MAGMA.c:231 / :79 / :369 -- the per-leaf GPU variants; mapped onto
 * the same engine (zau += H zu). */
void c_hacapk_adot_body_lfcpy_gpu_(int *nd, stc_HACApK_leafmtxp *st_leafmtxp);
void c_hacapk_adot_body_lfmtx_gpu_(double *zau, stc_HACApK_leafmtxp *st_leafmtxp,
                                   double *zu, double *zbu);
void c_hacapk_adot_body_lfdel_gpu_(stc_HACApK_leafmtxp *st_leafmtxp);

/* HACApK_SOLVER.c:421 -- BiCGSTAB with all vectors on the GPU.
 * HACApK_SOLVER.c:254 -- "flat" BiCGSTAB: host vectors, GPU matvec per step.
 * u: x0 in / solution out; b: rhs; param: HACApK param(1:100); *nstp: steps.
 * *lrtrn is set to the hbx_status (0 on success); the reference never set it. */
void c_hacapk_bicgstab_cax_lfmtx_gpu_(stc_HACApK_leafmtxp *st_leafmtxp,
                                      stc_HACApK_lcontrol *st_ctl, double *u, double *b,
                                      double *param, int *nd, int *nstp, int *lrtrn);
void c_hacapk_bicgstab_cax_lfmtx_flat_(stc_HACApK_leafmtxp *st_leafmtxp,
                                       stc_HACApK_lcontrol *st_ctl, double *u, double *b,
                                       double *param, int *nd, int *nstp, int *lrtrn);
/* HACApK_SOLVER_PIPE.c:144 and :640 -- the two pipelined BiCGSTAB versions,
 * both on hbx_bicgstab_pipe_host (same arguments as above). */
void c_hacapk_bicgstab_cax_lfmtx_pipe_(stc_HACApK_leafmtxp *st_leafmtxp,
                                       stc_HACApK_lcontrol *st_ctl, double *u, double *b,
                                       double *param, int *nd, int *nstp, int *lrtrn);
void c_hacapk_bicgstab_cax_lfmtx_pipe2_(stc_HACApK_leafmtxp *st_leafmtxp,
                                        stc_HACApK_lcontrol *st_ctl, double *u, double *b,
                                        double *param, int *nd, int *nstp, int *lrtrn);
/* HACApK_SOLVER.c:815 / :1405 / :2137 -- the multi-GPU-per-process BiCGSTAB
 * versions (the reference's default build calls _mgpu1_ from HACApK_solve_cax,
 * m_HACApK_use.f90:349).  The same recurrence as _gpu_; here each process
 * drives one GPU holding the whole H, so all three run hbx_bicgstab_host on
 * it (same arguments as above; H is copied in and released after the solve
 * unless lfcpy already made an engine for st_leafmtxp). */
void c_hacapk_bicgstab_cax_lfmtx_mgpu1_(stc_HACApK_leafmtxp *st_leafmtxp,
                                        stc_HACApK_lcontrol *st_ctl, double *u, double *b,
                                        double *param, int *nd, int *nstp, int *lrtrn);
void c_hacapk_bicgstab_cax_lfmtx_mgpu2_(stc_HACApK_leafmtxp *st_leafmtxp,
                                        stc_HACApK_lcontrol *st_ctl, double *u, double *b,
                                        double *param, int *nd, int *nstp, int *lrtrn);
void c_hacapk_bicgstab_cax_lfmtx_mgpu3_(stc_HACApK_leafmtxp *st_leafmtxp,
                                        stc_HACApK_lcontrol *st_ctl, double *u, double *b,
                                        double *param, int *nd, int *nstp, int *lrtrn);
/* GCR(m) on the GPU with the same arguments, for a Fortran driver that picks
 * GCR (param(85) = 2 in HACApK_solve, m_HACApK_use.f90:236-241): replaces the
 * call to the Fortran HACApK_gcrm_lfmtx (m_HACApK_solve.f90:506), which has
 * no C symbol in the reference.  param(87) is the restart length (8 when
 * outside 1..64). */
void c_hacapk_gcrm_lfmtx_gpu_(stc_HACApK_leafmtxp *st_leafmtxp, stc_HACApK_lcontrol *st_ctl,
                              double *u, double *b, double *param, int *nd, int *nstp, int *lrtrn);

#ifdef __cplusplus
}
#endif
#endif /* HACAPK_B200_H */
