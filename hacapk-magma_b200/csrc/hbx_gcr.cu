// hbx_gcr.cu -- GCR(m) on the GPU (HACApK_gcrm_lfmtx, m_HACApK_solve.f90:506-571).
//
// Every product is one k_matvec launch; the vectors stay on the device.  Dot
// products are compensated (Dot2) with the fixed reduction order of
// hbx_dots.cuh, so a solve is bit-reproducible; the vector updates are
// rounded as the reference writes them (a product, then a sum: no fma).  The
// state (alpha, |A p_l|^2, beta_l, the step count, done/status) lives on the
// device and each reduction is fused into the kernel that produces its
// vectors, the totals summed by the block that finishes last, so a whole
// restart cycle (m steps) is one captured CUDA graph:
//
//   k_gcr_update  u += alpha p_ik, r -= alpha A p_ik; r.r -> relres, stop test
//   k_matvec      A r (skipped once the stop test has fired)
//   k_gcr_proj    beta_l = -(A p_l . A r) / |A p_l|^2, l = 0..ik
//   k_gcr_orth    p_new = r + sum beta_l p_l, A p_new = A r + sum beta_l A p_l,
//                 l in order; then (A p_new . r), |A p_new|^2 -> the next alpha
//
// At a restart the new direction goes to slot 0 before the loop, so l = 0 is
// the new vector itself (its old |A p|^2 kept), as the Fortran does.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/hacapk_b200.h"
#include "hbx_dots.cuh"

namespace hbx {
namespace {

struct DotPairs {
  const double *x[kMaxDots];
  const double *y[kMaxDots];
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }

__global__ void __launch_bounds__(kDotThreads) k_dots(DotPairs d, int k, size_t n, double *part) {
  __shared__ double sh[kDotThreads / 32][2];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int j = 0; j < k; ++j) {
    Acc2 a{0.0, 0.0};
    const double *x = d.x[j], *y = d.y[j];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
      dot2_add(a, x[i], y[i]);
    a = warp_merge(a);
    if (lane == 0) {
      sh[w][0] = a.s;
      sh[w][1] = a.c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      Acc2 t{sh[0][0], sh[0][1]};
      for (int q = 1; q < kDotThreads / 32; ++q) t = acc2_merge(t, Acc2{sh[q][0], sh[q][1]});
      part[((size_t)blockIdx.x * kMaxDots + j) * 2] = t.s;
      part[((size_t)blockIdx.x * kMaxDots + j) * 2 + 1] = t.c;
    }
    __syncthreads();
  }
}

// out[j] = the sum of pair j's partials over nblk blocks, in block order
__global__ void k_dots_total(const double *part, int nblk, int k, double *out) {
  const int j = blockIdx.x;
  if (j >= k) return;
  const double t = pair_total(part, nblk, j);
  if (threadIdx.x == 0) out[j] = t;
}

__device__ __forceinline__ void finish(GcrState *st, int status) {
  st->done = 1;
  st->status = status;
}

// The totals of the block partials of K pairs, in the block that finished
// last (false elsewhere); on return tot[] holds them for thread 0.
template <int K>
__device__ __forceinline__ bool last_totals(GcrState *st, const double *part, double (&tot)[K]) {
  if (!last_block(&st->ticket)) return false;
  const int w = threadIdx.x >> 5;
  if (w < K) {
    const double t = pair_total(part, gridDim.x, w);
    if ((threadIdx.x & 31) == 0) tot[w] = t;
  }
  __syncthreads();
  return threadIdx.x == 0;
}

// After r = b - H u: p_0 = r; b.b, r.r -> bnorm, relres, the first stop test.
__global__ void __launch_bounds__(kDotThreads) k_gcr_init(GcrVecs v, size_t n, GcrState *st, double *part,
                                                          double tol, int max_iter) {
  Acc2 a[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double r = v.r[i], b = v.b[i];
    v.p[i] = r;
    dot2_add(a[0], b, b);
    dot2_add(a[1], r, r);
  }
  block_partials<2>(a, part);
  __shared__ double tot[2];
  if (!last_totals<2>(st, part, tot)) return;
  const double bnorm = sqrt(tot[0]), rn = sqrt(tot[1]);
  st->bnorm = bnorm;
  st->tol = tol;
  st->max_iter = max_iter;
  st->step = 0;
  st->done = 0;
  st->status = HBX_OK;
  const double rel = bnorm > 0.0 ? rn / bnorm : 0.0;
  st->relres = rel;
  if (!isfinite(rn) || !isfinite(bnorm)) finish(st, HBX_ERR_NONFINITE);
  else if (rel < tol) finish(st, HBX_OK);
  else if (max_iter <= 0) finish(st, HBX_ERR_NOT_CONVERGED);
}

// After A p_0: (A p_0 . r), |A p_0|^2 -> alpha, capap[0].
__global__ void __launch_bounds__(kDotThreads) k_gcr_alpha0(GcrVecs v, size_t n, GcrState *st, double *part) {
  if (*(volatile int *)&st->done) return;
  Acc2 a[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double q = v.ap[i];
    dot2_add(a[0], q, v.r[i]);
    dot2_add(a[1], q, q);
  }
  block_partials<2>(a, part);
  __shared__ double tot[2];
  if (!last_totals<2>(st, part, tot)) return;
  st->capap[0] = tot[1];
  st->alpha = tot[0] / tot[1];
}

// u += alpha p_ik, r -= alpha A p_ik; |r| -> relres; the stop test.
__global__ void __launch_bounds__(kDotThreads) k_gcr_update(GcrVecs v, size_t n, int ik, GcrState *st, double *part) {
  if (*(volatile int *)&st->done) return;
  const double alpha = st->alpha;
  const double *p = v.p + (size_t)ik * n, *q = v.ap + (size_t)ik * n;
  Acc2 a[1] = {{0.0, 0.0}};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    v.u[i] = add(v.u[i], mul(alpha, p[i]));
    const double r = __dsub_rn(v.r[i], mul(alpha, q[i]));
    v.r[i] = r;
    dot2_add(a[0], r, r);
  }
  block_partials<1>(a, part);
  __shared__ double tot[1];
  if (!last_totals<1>(st, part, tot)) return;
  const double rn = sqrt(tot[0]);
  const double rel = st->bnorm > 0.0 ? rn / st->bnorm : 0.0;
  const int step = st->step + 1;
  st->step = step;
  st->relres = rel;
  if (!isfinite(rn)) finish(st, HBX_ERR_BREAKDOWN);
  else if (rel < st->tol) finish(st, HBX_OK);
  else if (step >= st->max_iter) finish(st, HBX_ERR_NOT_CONVERGED);
}

// beta_l = -(A p_l . A r) / capap[l] for l = 0..ik; slot ikn already holds
// the new direction (A r) when ikn <= ik, as after the Fortran's copy.
__global__ void __launch_bounds__(kDotThreads) k_gcr_proj(GcrVecs v, size_t n, int ik, int ikn, GcrState *st,
                                                          double *part) {
  if (*(volatile int *)&st->done) return;
  __shared__ double sh[kDotThreads / 32][2];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int l = 0; l <= ik; ++l) {
    Acc2 a{0.0, 0.0};
    const double *x = l == ikn ? v.ar : v.ap + (size_t)l * n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
      dot2_add(a, x[i], v.ar[i]);
    a = warp_merge(a);
    if (lane == 0) {
      sh[w][0] = a.s;
      sh[w][1] = a.c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      Acc2 t{sh[0][0], sh[0][1]};
      for (int q = 1; q < kDotThreads / 32; ++q) t = acc2_merge(t, Acc2{sh[q][0], sh[q][1]});
      part[((size_t)blockIdx.x * kMaxDots + l) * 2] = t.s;
      part[((size_t)blockIdx.x * kMaxDots + l) * 2 + 1] = t.c;
    }
    __syncthreads();
  }
  if (!last_block(&st->ticket)) return;
  for (int l = w; l <= ik; l += kDotThreads / 32) {
    const double t = pair_total(part, gridDim.x, l);
    if (lane == 0) st->beta[l] = -t / st->capap[l];
  }
}

// p_ikn = r + sum_l beta_l p_l, A p_ikn likewise (l = 0..ik in order, the
// new slot read as its running value); then (A p_ikn . r), |A p_ikn|^2 ->
// alpha and capap[ikn] for the next step.
__global__ void __launch_bounds__(kDotThreads) k_gcr_orth(GcrVecs v, size_t n, int ik, int ikn, GcrState *st,
                                                          double *part) {
  if (*(volatile int *)&st->done) return;
  Acc2 a[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double r = v.r[i];
    double vp = r, va = v.ar[i];
    for (int l = 0; l <= ik; ++l) {
      const double bl = st->beta[l];
      const double sp = l == ikn ? vp : v.p[(size_t)l * n + i];
      const double sa = l == ikn ? va : v.ap[(size_t)l * n + i];
      vp = add(vp, mul(bl, sp));
      va = add(va, mul(bl, sa));
    }
    v.p[(size_t)ikn * n + i] = vp;
    v.ap[(size_t)ikn * n + i] = va;
    dot2_add(a[0], va, r);
    dot2_add(a[1], va, va);
  }
  block_partials<2>(a, part);
  __shared__ double tot[2];
  if (!last_totals<2>(st, part, tot)) return;
  st->capap[ikn] = tot[1];
  st->alpha = tot[0] / tot[1];
}

}  // namespace

int gcr_dot_blocks(size_t n) { return dot_blocks(n); }

cudaError_t gcr_launch_dots(int k, const double *const *x, const double *const *y, size_t n, double *part, double *out,
                            cudaStream_t s) {
  if (k < 1 || k > kMaxDots) return cudaErrorInvalidValue;
  DotPairs d{};
  for (int j = 0; j < k; ++j) {
    d.x[j] = x[j];
    d.y[j] = y[j];
  }
  const int nblk = gcr_dot_blocks(n);
  k_dots<<<nblk, kDotThreads, 0, s>>>(d, k, n, part);
  k_dots_total<<<k, 32, 0, s>>>(part, nblk, k, out);
  return cudaGetLastError();
}

cudaError_t gcr_launch_init(const GcrVecs &v, size_t n, GcrState *st, double *part, double tol, int max_iter,
                            cudaStream_t s) {
  k_gcr_init<<<dot_blocks(n), kDotThreads, 0, s>>>(v, n, st, part, tol, max_iter);
  return cudaGetLastError();
}

cudaError_t gcr_launch_alpha0(const GcrVecs &v, size_t n, GcrState *st, double *part, cudaStream_t s) {
  k_gcr_alpha0<<<dot_blocks(n), kDotThreads, 0, s>>>(v, n, st, part);
  return cudaGetLastError();
}

cudaError_t gcr_launch_update(const GcrVecs &v, size_t n, int ik, GcrState *st, double *part, cudaStream_t s) {
  k_gcr_update<<<dot_blocks(n), kDotThreads, 0, s>>>(v, n, ik, st, part);
  return cudaGetLastError();
}

cudaError_t gcr_launch_orth(const GcrVecs &v, size_t n, int ik, int ikn, GcrState *st, double *part,
                            cudaStream_t s) {
  if (ik < 0 || ik >= kMaxDots || ikn < 0 || ikn >= kMaxDots) return cudaErrorInvalidValue;
  k_gcr_proj<<<dot_blocks(n), kDotThreads, 0, s>>>(v, n, ik, ikn, st, part);
  k_gcr_orth<<<dot_blocks(n), kDotThreads, 0, s>>>(v, n, ik, ikn, st, part);
  return cudaGetLastError();
}

}  // namespace hbx
