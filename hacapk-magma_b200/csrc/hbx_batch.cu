// hbx_batch.cu -- vector kernels of the batched BiCGSTAB over many
// independent H-matrices packed as one block-diagonal H (no counterpart in
// the reference, which solves one body per run).  Instance k owns rows
// [off[k], off[k+1]) of every vector; each instance runs the recurrence of
// HACApK_SOLVER.c:602-732 with its own scalars (MrScal, one per instance) and
// its own stop test ||r||/||b|| < tol, checked before every step as
// HACApK_SOLVER.c:631 does.  A finished instance keeps u and r, and its p and
// t are zero so its rows of the block-diagonal products are zero.
//
// Dot products: one block per instance sums its rows with compensated
// (Dot2) accumulation, as the single-body solver does -- each thread in row
// order, then a fixed tree over the block -- so every run sums in the same
// order and the scalars match a body solved alone.
#include <cmath>

#include "../../include/hacapk_b200.h"
#include "hbx_device.cuh"
#include "hbx_engine.h"

namespace hbx {
namespace {

constexpr int kBt = 1024;  // threads of a per-body dot block

// out[k][q] = x_q . y_q over the rows of instance k
template <int NQ>
__global__ void __launch_bounds__(kBt) k_bt_dots(const int *off, const double *x0, const double *y0, const double *x1,
                                                 const double *y1, double *out) {
  const int k = blockIdx.x, tid = threadIdx.x;
  const int r0 = off[k], r1 = off[k + 1];
  Acc2 acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) acc[q] = Acc2{0.0, 0.0};
  for (int i = r0 + tid; i < r1; i += kBt) {
    dot2_add(acc[0], x0[i], y0[i]);
    if (NQ > 1) dot2_add(acc[NQ - 1], x1[i], y1[i]);
  }
  __shared__ Acc2 red[NQ][kBt];
#pragma unroll
  for (int q = 0; q < NQ; ++q) red[q][tid] = acc[q];
  __syncthreads();
  for (int w = kBt / 2; w > 0; w >>= 1) {
    if (tid < w) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) red[q][tid] = acc2_merge(red[q][tid], red[q][tid + w]);
    }
    __syncthreads();
  }
  if (tid < NQ) out[(size_t)k * NQ + tid] = red[tid][0].s + red[tid][0].c;
}

// Start of the solve: r = b - H u is formed; rh = r, p = Ap = 0 on every row.
__global__ void k_bt_setup(size_t n, const double *r, double *rh, double *p, double *ap) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    rh[i] = r[i];
    p[i] = 0.0;
    ap[i] = 0.0;
  }
}

// rho = rh.r = r.r, bnorm; an instance runs while ||r||/||b|| >= tol
__global__ void k_bt_init(int count, const double *dots /*[k][2]: r.r, b.b*/, double tol, const double *rtol,
                          int max_iter, MrScal *s, double *bnorm, int *any_active) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const double rr = dots[2 * k], bb = dots[2 * k + 1];
  const double bn = std::sqrt(bb);
  bnorm[k] = bn;
  MrScal q{};
  q.rho = rr;
  q.rr = rr;
  const double rel = bn > 0.0 ? std::sqrt(rr) / bn : 0.0;
  if (rtol) tol = rtol[k];  // per-instance tolerance (the inner solves of a refined batch)
  q.rtol = tol;
  q.status = 0;
  if (!isfinite(rel)) q.status = HBX_ERR_BREAKDOWN;
  else if (rel >= tol) q.active = max_iter > 0 ? 1 : 0;
  if (rel >= tol && max_iter <= 0) q.status = HBX_ERR_NOT_CONVERGED;
  s[k] = q;
  if (q.active) atomicOr(any_active, 1);
}

// p = r + beta (p - zeta Ap) (p = r on the first step); zero when finished
__global__ void k_bt_p(size_t n, const int *rinst, const MrScal *s, const double *r, double *p, const double *ap) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const MrScal &q = s[rinst[i]];
    if (!q.active) {
      p[i] = 0.0;
      continue;
    }
    p[i] = q.iters == 0 ? r[i] : fma(q.beta, fma(-q.zeta, ap[i], p[i]), r[i]);
  }
}

// alpha = rho / (rh . Ap)
__global__ void k_bt_alpha(int count, const double *dots, MrScal *s) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count || !s[k].active) return;
  const double d = dots[k];
  const double alpha = s[k].rho / d;
  if (d == 0.0 || !isfinite(alpha)) {
    s[k].active = 0;
    s[k].status = HBX_ERR_BREAKDOWN;
    return;
  }
  s[k].alpha = alpha;
}

// t = r - alpha Ap; zero when finished
__global__ void k_bt_t(size_t n, const int *rinst, const MrScal *s, const double *r, const double *ap, double *t) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const MrScal &q = s[rinst[i]];
    t[i] = q.active ? fma(-q.alpha, ap[i], r[i]) : 0.0;
  }
}

// zeta = (At . t) / (At . At).  At . At == 0 means At = 0: zeta = 0 keeps
// the step's BiCG half (u += alpha p, r = t); the stop test that follows
// (k_bt_beta) then ends the instance as converged when that r is below the
// tolerance and as a breakdown otherwise, before any further step.
__global__ void k_bt_zeta(int count, const double *dots, MrScal *s) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count || !s[k].active) return;
  const double tt = dots[2 * k], aa = dots[2 * k + 1];
  const double zeta = aa != 0.0 ? tt / aa : 0.0;
  if (!isfinite(zeta)) {
    s[k].active = 0;
    s[k].status = HBX_ERR_BREAKDOWN;
    return;
  }
  s[k].zeta = zeta;
}

// u += alpha p + zeta t;  r = t - zeta At  (running instances)
__global__ void k_bt_xr(size_t n, const int *rinst, const MrScal *s, const double *p, const double *t,
                        const double *at, double *u, double *r) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const MrScal &q = s[rinst[i]];
    if (!q.active) continue;
    const double tv = t[i];
    u[i] = fma(q.zeta, tv, fma(q.alpha, p[i], u[i]));
    r[i] = fma(-q.zeta, at[i], tv);
  }
}

// the step is done: rho_new = rh . r, rr = r . r; the stop test; beta
__global__ void k_bt_beta(int count, const double *dots, const double *bnorm, int max_iter, MrScal *s,
                          int *any_active) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count || !s[k].active) return;
  MrScal q = s[k];
  const double rho_new = dots[2 * k], rr = dots[2 * k + 1];
  q.iters += 1;
  q.rr = rr;
  const double rel = bnorm[k] > 0.0 ? std::sqrt(rr) / bnorm[k] : 0.0;
  if (!isfinite(rel)) {
    q.active = 0;
    q.status = HBX_ERR_BREAKDOWN;
  } else if (rel < q.rtol) {
    q.active = 0;
  } else if (q.iters >= max_iter) {
    q.active = 0;
    q.status = HBX_ERR_NOT_CONVERGED;
  } else {
    const double beta = (q.alpha / q.zeta) * (rho_new / q.rho);
    if (q.zeta == 0.0 || !isfinite(beta)) {
      q.active = 0;
      q.status = HBX_ERR_BREAKDOWN;
    } else {
      q.beta = beta;
      q.rho = rho_new;
    }
  }
  s[k] = q;
  if (q.active) atomicOr(any_active, 1);
}

int vgrid(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }

// pre[k] = active instances below k (count + 1 entries), one block: each
// thread counts a contiguous share, a block scan of the shares, then each
// thread writes its share's prefixes.
constexpr int kPreThreads = 1024;
__global__ void __launch_bounds__(kPreThreads) k_bt_prefix(int count, const MrScal *s, int *pre) {
  __shared__ int part[kPreThreads];
  const int t = threadIdx.x, per = (count + kPreThreads - 1) / kPreThreads;
  const int k0 = min(count, t * per), k1 = min(count, k0 + per);
  int c = 0;
  for (int k = k0; k < k1; ++k) c += s[k].active ? 1 : 0;
  part[t] = c;
  __syncthreads();
  for (int o = 1; o < kPreThreads; o <<= 1) {
    const int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - c;  // active instances below k0
  for (int k = k0; k < k1; ++k) {
    pre[k] = run;
    run += s[k].active ? 1 : 0;
  }
  if (t == kPreThreads - 1) pre[count] = part[t];
}

}  // namespace

cudaError_t bt_launch_prefix(int count, const MrScal *sc, int *pre, cudaStream_t s) {
  k_bt_prefix<<<1, kPreThreads, 0, s>>>(count, sc, pre);
  return cudaGetLastError();
}

cudaError_t bt_launch_dots(int nq, int count, const int *off, const double *x0, const double *y0, const double *x1,
                           const double *y1, double *out, cudaStream_t s) {
  if (nq == 1) k_bt_dots<1><<<count, kBt, 0, s>>>(off, x0, y0, nullptr, nullptr, out);
  else k_bt_dots<2><<<count, kBt, 0, s>>>(off, x0, y0, x1, y1, out);
  return cudaGetLastError();
}

cudaError_t bt_launch_setup(size_t n, const double *r, double *rh, double *p, double *ap, cudaStream_t s) {
  k_bt_setup<<<vgrid(n), 256, 0, s>>>(n, r, rh, p, ap);
  return cudaGetLastError();
}

cudaError_t bt_launch_init(int count, const double *dots, double tol, const double *rtol, int max_iter, MrScal *sc,
                           double *bnorm, int *any_active, cudaStream_t s) {
  cudaMemsetAsync(any_active, 0, sizeof(int), s);
  k_bt_init<<<(count + 127) / 128, 128, 0, s>>>(count, dots, tol, rtol, max_iter, sc, bnorm, any_active);
  return cudaGetLastError();
}

// r[i] = 0 for the rows of instances whose flag is 0
__global__ void k_bt_mask(size_t n, const int *rinst, const int *flag, double *r) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!flag[rinst[i]]) r[i] = 0.0;
}

cudaError_t bt_launch_mask(size_t n, const int *rinst, const int *flag, double *r, cudaStream_t s) {
  k_bt_mask<<<vgrid(n), 256, 0, s>>>(n, rinst, flag, r);
  return cudaGetLastError();
}

cudaError_t bt_launch_step(const BtStep &a, cudaStream_t s) {
  const int sg = (a.count + 127) / 128;
  cudaError_t e;
  k_bt_p<<<vgrid(a.n), 256, 0, s>>>(a.n, a.rinst, a.sc, a.r, a.p, a.ap);
  if (a.pre) k_bt_prefix<<<1, kPreThreads, 0, s>>>(a.count, a.sc, a.pre);
  if ((e = a.matvec(a.ctx, a.p, a.ap, s)) != cudaSuccess) return e;
  k_bt_dots<1><<<a.count, kBt, 0, s>>>(a.off, a.rh, a.ap, nullptr, nullptr, a.dots);
  k_bt_alpha<<<sg, 128, 0, s>>>(a.count, a.dots, a.sc);
  k_bt_t<<<vgrid(a.n), 256, 0, s>>>(a.n, a.rinst, a.sc, a.r, a.ap, a.t);
  if (a.pre) k_bt_prefix<<<1, kPreThreads, 0, s>>>(a.count, a.sc, a.pre);
  if ((e = a.matvec(a.ctx, a.t, a.at, s)) != cudaSuccess) return e;
  k_bt_dots<2><<<a.count, kBt, 0, s>>>(a.off, a.at, a.t, a.at, a.at, a.dots);
  k_bt_zeta<<<sg, 128, 0, s>>>(a.count, a.dots, a.sc);
  k_bt_xr<<<vgrid(a.n), 256, 0, s>>>(a.n, a.rinst, a.sc, a.p, a.t, a.at, a.u, a.r);
  k_bt_dots<2><<<a.count, kBt, 0, s>>>(a.off, a.rh, a.r, a.r, a.r, a.dots);
  cudaMemsetAsync(a.any_active, 0, sizeof(int), s);
  k_bt_beta<<<sg, 128, 0, s>>>(a.count, a.dots, a.bnorm, a.max_iter, a.sc, a.any_active);
  return cudaGetLastError();
}

}  // namespace hbx
