// hbx_pipe.cu -- pipelined BiCGSTAB on the GPU (c_hacapk_bicgstab_cax_lfmtx_pipe_,
// HACApK_SOLVER_PIPE.c:144-600; _pipe2_ at :640-1148 is the same arithmetic).
//
// The products s = A p and z = A s are carried by recurrences, so a step is
// two H-matvecs (v = A z, t = A w) and two reduction points.  Each reduction
// point is one fused kernel: the element-wise updates, the compensated dot
// partials (hbx_dots.cuh order) and, in the block that finishes last, the
// totals and the scalar recurrences.  The state (alpha, beta, zeta, the step
// count, done/status) stays on the device, so a batch of steps
//   k_pipe_a, k_matvec(v = A z), k_pipe_b, k_matvec(t = A w)
// is captured once as a CUDA graph; after `done` is set every later kernel of
// the batch returns at once (the products through MatvecArgs::skip).
//
// The element-wise roundings follow the reference's BLAS-1 calls (daxpy
// y = y + a x, dlascl x = c x), written with __dmul_rn / __dadd_rn so that no
// multiply-add is contracted:
//   p = beta (p - zeta s) + r     s = beta (s - zeta z) + w     z = beta (z - zeta v) + t
//   q = r - alpha s               y = w - alpha z               zeta = (y.q) / (y.y)
//   u = (u + alpha p) + zeta q    r = q - zeta y                w = -zeta (t - alpha v) + y
//   beta = (alpha / zeta) (r.r0 / r.r0_old)
//   alpha = r.r0 / (w.r0 + beta s.r0 - beta zeta z.r0)
// The iterate accumulates in u: the reference adds the corrections to zx, a
// vector it never initialises, and copies the unchanged u back (:592).
#include <cuda_runtime.h>

#include "../../include/hacapk_b200.h"
#include "hbx_dots.cuh"

namespace hbx {
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }

__device__ __forceinline__ void finish(PipeState *st, int status) {
  st->done = 1;
  st->status = status;
}

// After r = b - H u, w = H r, t = H w: r0 = r; bnorm, r.r, w.r -> alpha.
__global__ void __launch_bounds__(kDotThreads) k_pipe_init(PipeVecs v, size_t n, PipeState *st, double *part,
                                                           double *hist, double tol, int max_iter) {
  Acc2 a[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double r = v.r[i], b = v.b[i];
    v.r0[i] = r;
    dot2_add(a[0], b, b);
    dot2_add(a[1], r, r);
    dot2_add(a[2], v.w[i], r);
  }
  block_partials<3>(a, part);
  if (!last_block(&st->ticket)) return;
  __shared__ double tot[3];
  const int w = threadIdx.x >> 5;
  if (w < 3) {
    const double t = pair_total(part, gridDim.x, w);
    if ((threadIdx.x & 31) == 0) tot[w] = t;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double bb = tot[0], rr = tot[1], wr = tot[2];
  const double bnorm = sqrt(bb);
  st->bnorm = bnorm;
  st->tol = tol;
  st->max_iter = max_iter;
  st->znorm = rr;
  st->alpha = rr / wr;
  st->beta = 0.0;
  st->zeta = 0.0;
  st->step = 0;
  st->done = 0;
  st->status = HBX_OK;
  const double rel = bnorm > 0.0 ? sqrt(rr) / bnorm : 0.0;
  st->relres = rel;
  hist[0] = rel;
  if (!isfinite(bb) || !isfinite(rr)) finish(st, HBX_ERR_NONFINITE);
  else if (rel < tol) finish(st, HBX_OK);
  else if (max_iter <= 0) finish(st, HBX_ERR_NOT_CONVERGED);
}

// p, s, z recurrences (copies on the first step), q, y, zeta = (y.q)/(y.y).
__global__ void __launch_bounds__(kDotThreads) k_pipe_a(PipeVecs v, size_t n, PipeState *st, double *part) {
  if (*(volatile int *)&st->done) return;
  const double alpha = st->alpha, beta = st->beta, zeta = st->zeta;
  const bool first = st->step == 0;
  Acc2 a[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double r = v.r[i], w = v.w[i], t = v.t[i];
    double p, s, z;
    if (first) {
      p = r;
      s = w;
      z = t;
    } else {
      const double s0 = v.s[i], z0 = v.z[i];
      p = add(mul(beta, add(v.p[i], mul(-zeta, s0))), r);
      s = add(mul(beta, add(s0, mul(-zeta, z0))), w);
      z = add(mul(beta, add(z0, mul(-zeta, v.v[i]))), t);
    }
    const double q = add(r, mul(-alpha, s)), y = add(w, mul(-alpha, z));
    v.p[i] = p;
    v.s[i] = s;
    v.z[i] = z;
    v.q[i] = q;
    v.y[i] = y;
    dot2_add(a[0], y, q);
    dot2_add(a[1], y, y);
  }
  block_partials<2>(a, part);
  if (!last_block(&st->ticket)) return;
  __shared__ double tot[2];
  const int w = threadIdx.x >> 5;
  if (w < 2) {
    const double t = pair_total(part, gridDim.x, w);
    if ((threadIdx.x & 31) == 0) tot[w] = t;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double zeta_new = tot[0] / tot[1];
  st->zeta = zeta_new;
  if (!isfinite(zeta_new)) finish(st, HBX_ERR_BREAKDOWN);  // y = 0 (HACApK_SOLVER_PIPE.c:433 divides unchecked)
}

// u, r, w updates; r.r0, w.r0, s.r0, z.r0, r.r -> beta, alpha, relres; stop test.
__global__ void __launch_bounds__(kDotThreads) k_pipe_b(PipeVecs v, size_t n, PipeState *st, double *part,
                                                        double *hist) {
  if (*(volatile int *)&st->done) return;
  const double alpha = st->alpha, zeta = st->zeta;
  Acc2 a[5] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double q = v.q[i], y = v.y[i], r0 = v.r0[i];
    v.u[i] = add(add(v.u[i], mul(alpha, v.p[i])), mul(zeta, q));
    const double r = add(q, mul(-zeta, y));
    const double w = add(mul(-zeta, add(v.t[i], mul(-alpha, v.v[i]))), y);
    v.r[i] = r;
    v.w[i] = w;
    dot2_add(a[0], r, r0);
    dot2_add(a[1], w, r0);
    dot2_add(a[2], v.s[i], r0);
    dot2_add(a[3], v.z[i], r0);
    dot2_add(a[4], r, r);
  }
  block_partials<5>(a, part);
  if (!last_block(&st->ticket)) return;
  __shared__ double tot[5];
  const int w = threadIdx.x >> 5;
  if (w < 5) {
    const double t = pair_total(part, gridDim.x, w);
    if ((threadIdx.x & 31) == 0) tot[w] = t;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const double znormold = st->znorm, znorm = tot[0];
  const double beta = mul(__ddiv_rn(alpha, zeta), __ddiv_rn(znorm, znormold));
  const double den = __dsub_rn(add(tot[1], mul(beta, tot[2])), mul(mul(beta, zeta), tot[3]));
  const double alpha_new = __ddiv_rn(znorm, den);
  const double rel = st->bnorm > 0.0 ? __ddiv_rn(__dsqrt_rn(tot[4]), st->bnorm) : 0.0;
  st->znorm = znorm;
  st->beta = beta;
  st->alpha = alpha_new;
  st->relres = rel;
  const int step = st->step + 1;
  st->step = step;
  hist[step] = rel;
  if (rel < st->tol) finish(st, HBX_OK);
  else if (!isfinite(rel) || !isfinite(alpha_new) || !isfinite(beta)) finish(st, HBX_ERR_BREAKDOWN);
  else if (step >= st->max_iter) finish(st, HBX_ERR_NOT_CONVERGED);
}

}  // namespace

cudaError_t pipe_launch_init(const PipeVecs &v, size_t n, PipeState *st, double *part, double *hist, double tol,
                             int max_iter, cudaStream_t s) {
  k_pipe_init<<<dot_blocks(n), kDotThreads, 0, s>>>(v, n, st, part, hist, tol, max_iter);
  return cudaGetLastError();
}

cudaError_t pipe_launch_a(const PipeVecs &v, size_t n, PipeState *st, double *part, cudaStream_t s) {
  k_pipe_a<<<dot_blocks(n), kDotThreads, 0, s>>>(v, n, st, part);
  return cudaGetLastError();
}

cudaError_t pipe_launch_b(const PipeVecs &v, size_t n, PipeState *st, double *part, double *hist, cudaStream_t s) {
  k_pipe_b<<<dot_blocks(n), kDotThreads, 0, s>>>(v, n, st, part, hist);
  return cudaGetLastError();
}

}  // namespace hbx
