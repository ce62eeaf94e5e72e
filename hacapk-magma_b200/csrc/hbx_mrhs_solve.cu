// hbx_mrhs_solve.cu -- vector kernels of the multi-RHS BiCGSTAB (no
// counterpart in the reference).  Every vector is nd x kNrhs doubles,
// row-major (the kNrhs right-hand sides of a row adjacent); each right-hand
// side j runs its own BiCGSTAB recurrence of HACApK_SOLVER.c:602-732 with its
// own scalars and stops on its own (a convergence mask): a finished RHS keeps
// its x and r, and its p is fed to the product as zeros.
//
// Layout of the row-block kernels: block b covers rows [b*rpb, (b+1)*rpb),
// thread (rs = tid / 64, j = tid % 64) takes rows rs, rs + 4, ... of it, so a
// warp reads 32 consecutive doubles of a row.  Dot products are summed per
// thread, then over the 4 row lanes of the block, then over the blocks in
// block order (one thread per RHS): the same order on every run.
#include <algorithm>
#include <cmath>

#include "../../include/hacapk_b200.h"
#include "hbx_engine.h"

namespace hbx {
namespace {

constexpr int kRowLanes = 4;
constexpr int kVecThreads = kRowLanes * kNrhs;  // 256

template <int NQ>
__device__ __forceinline__ void block_partials(double (&acc)[NQ], double *part, int rhs) {
  __shared__ double red[NQ][kVecThreads];
  const int tid = threadIdx.x;
#pragma unroll
  for (int k = 0; k < NQ; ++k) red[k][tid] = acc[k];
  __syncthreads();
  if (tid < kNrhs) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      double v = red[k][tid];
#pragma unroll
      for (int l = 1; l < kRowLanes; ++l) v += red[k][l * kNrhs + tid];
      part[((size_t)blockIdx.x * NQ + k) * kNrhs + rhs] = v;
    }
  }
}

// part[b][k][j] = sum over the rows of block b of x_k(i, j) * y_k(i, j)
template <int NQ>
__global__ void __launch_bounds__(kVecThreads) k_mr_dots(int nd, int rpb, const double *x0, const double *y0,
                                                         const double *x1, const double *y1, double *part) {
  const int j = threadIdx.x % kNrhs, rs = threadIdx.x / kNrhs;
  const int r0 = blockIdx.x * rpb, r1 = min(nd, r0 + rpb);
  double acc[NQ];
#pragma unroll
  for (int k = 0; k < NQ; ++k) acc[k] = 0.0;
  for (int i = r0 + rs; i < r1; i += kRowLanes) {
    const size_t e = (size_t)i * kNrhs + j;
    acc[0] = fma(x0[e], y0[e], acc[0]);
    if (NQ > 1) acc[NQ - 1] = fma(x1[e], y1[e], acc[NQ - 1]);
  }
  block_partials<NQ>(acc, part, j);
}

// The scalar kernels run kScalThreads = 8 lanes per right-hand side: lane l
// of RHS j sums the partials of blocks l, l + 8, ... (two accumulators, so
// its loads overlap), then lane 0 adds the 8 lane sums in lane order -- a
// fixed order, the same on every run.
constexpr int kSumLanes = 8;
constexpr int kScalThreads = kSumLanes * kNrhs;  // 512

// out[q] (valid in lane 0 of each RHS, threads 0..kNrhs-1) = sum over the
// blocks of part[b][q0 + q][j] for q < NQ; j = threadIdx.x % kNrhs.
template <int NQ>
__device__ __forceinline__ void sum_parts(const double *part, int nblk, int nq, int q0, double (&out)[NQ]) {
  __shared__ double lanes[NQ][kScalThreads];
  const int j = threadIdx.x % kNrhs, l = threadIdx.x / kNrhs;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double a0 = 0.0, a1 = 0.0;
    int b = l;
    for (; b + kSumLanes < nblk; b += 2 * kSumLanes) {
      a0 += part[((size_t)b * nq + q0 + q) * kNrhs + j];
      a1 += part[((size_t)(b + kSumLanes) * nq + q0 + q) * kNrhs + j];
    }
    if (b < nblk) a0 += part[((size_t)b * nq + q0 + q) * kNrhs + j];
    lanes[q][threadIdx.x] = a0 + a1;
  }
  __syncthreads();
  if (l == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double v = lanes[q][j];
      for (int k = 1; k < kSumLanes; ++k) v += lanes[q][k * kNrhs + j];
      out[q] = v;
    }
  }
}

// r = rh = R, p = ap = x = 0
__global__ void __launch_bounds__(kVecThreads) k_mr_setup(size_t n, const double *R, double *r, double *rh, double *p,
                                                          double *ap, double *x) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const double v = R[e];
    r[e] = v;
    rh[e] = v;
    p[e] = 0.0;
    ap[e] = 0.0;
    x[e] = 0.0;
  }
}

// First scalars of an inner solve: rho = rh.r = r.r; an RHS runs while its
// mask is set and ||r|| is above its threshold.
__global__ void k_mr_init(const double *part, int nblk, const double *thresh, const int *mask, MrScal *s,
                          int *any_active) {
  const int j = threadIdx.x;
  __shared__ int any;
  if (j == 0) any = 0;
  double sums[1];
  sum_parts<1>(part, nblk, 1, 0, sums);
  if (j < kNrhs) {
    const double rr = sums[0];
    MrScal q{};
    q.rho = rr;
    q.rr = rr;
    q.rtol = thresh[j];
    q.active = (mask[j] && std::sqrt(rr) > q.rtol) ? 1 : 0;
    q.status = 0;
    s[j] = q;
    if (q.active) atomicOr(&any, 1);
  }
  __syncthreads();
  if (j == 0) *any_active = any;
}

// p = r + beta (p - zeta ap) (p = r on an RHS's first step); p32 = p as
// float, zero for a finished RHS.
__global__ void __launch_bounds__(kVecThreads) k_mr_p(size_t n, const MrScal *s, const double *r, double *p,
                                                      const double *ap, float *p32) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const MrScal &q = s[e % kNrhs];
    if (!q.active) {
      p32[e] = 0.0f;
      continue;
    }
    const double pv = q.iters == 0 ? r[e] : fma(q.beta, fma(-q.zeta, ap[e], p[e]), r[e]);
    p[e] = pv;
    p32[e] = (float)pv;
  }
}

// alpha = rho / (rh . Ap)
__global__ void k_mr_alpha(const double *part, int nblk, MrScal *s) {
  const int j = threadIdx.x;
  double sums[1];
  sum_parts<1>(part, nblk, 1, 0, sums);
  if (j >= kNrhs || !s[j].active) return;
  const double d = sums[0];
  const double alpha = s[j].rho / d;
  if (d == 0.0 || !isfinite(alpha)) {
    s[j].active = 0;
    s[j].status = HBX_ERR_BREAKDOWN;
    return;
  }
  s[j].alpha = alpha;
}

// t = r - alpha Ap; t32 = t as float (zero for a finished RHS)
__global__ void __launch_bounds__(kVecThreads) k_mr_t(size_t n, const MrScal *s, const double *r, const double *ap,
                                                      double *t, float *t32) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const MrScal &q = s[e % kNrhs];
    if (!q.active) {
      t32[e] = 0.0f;
      continue;
    }
    const double tv = fma(-q.alpha, ap[e], r[e]);
    t[e] = tv;
    t32[e] = (float)tv;
  }
}

// zeta = (At . t) / (At . At)
__global__ void k_mr_zeta(const double *part, int nblk, MrScal *s) {
  const int j = threadIdx.x;
  double sums[2];
  sum_parts<2>(part, nblk, 2, 0, sums);
  if (j >= kNrhs || !s[j].active) return;
  const double tt = sums[0], aa = sums[1];
  const double zeta = aa != 0.0 ? tt / aa : 0.0;
  if (!isfinite(zeta)) {
    s[j].active = 0;
    s[j].status = HBX_ERR_BREAKDOWN;
    return;
  }
  s[j].zeta = zeta;
}

// x += alpha p + zeta t;  r = t - zeta At;  partials of rh.r and r.r
__global__ void __launch_bounds__(kVecThreads) k_mr_xr(int nd, int rpb, const MrScal *s, const double *p,
                                                       const double *t, const double *at, const double *rh, double *x,
                                                       double *r, double *part) {
  const int j = threadIdx.x % kNrhs, rs = threadIdx.x / kNrhs;
  const int r0 = blockIdx.x * rpb, r1 = min(nd, r0 + rpb);
  const MrScal q = s[j];
  double acc[2] = {0.0, 0.0};
  if (q.active) {
    for (int i = r0 + rs; i < r1; i += kRowLanes) {
      const size_t e = (size_t)i * kNrhs + j;
      const double tv = t[e];
      x[e] = fma(q.zeta, tv, fma(q.alpha, p[e], x[e]));
      const double rv = fma(-q.zeta, at[e], tv);
      r[e] = rv;
      acc[0] = fma(rh[e], rv, acc[0]);
      acc[1] = fma(rv, rv, acc[1]);
    }
  }
  block_partials<2>(acc, part, j);
}

// rho_new = rh . r, rr = r . r; the stop test; beta for the next step
__global__ void k_mr_beta(const double *part, int nblk, int max_iter, MrScal *s, int *any_active) {
  const int j = threadIdx.x;
  __shared__ int any;
  if (j == 0) any = 0;
  double sums[2];
  sum_parts<2>(part, nblk, 2, 0, sums);
  if (j < kNrhs && s[j].active) {
    MrScal q = s[j];
    const double rho_new = sums[0], rr = sums[1];
    q.iters += 1;
    q.rr = rr;
    if (!isfinite(rr)) {
      q.active = 0;
      q.status = HBX_ERR_BREAKDOWN;
    } else if (std::sqrt(rr) <= q.rtol) {
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
    s[j] = q;
    if (q.active) atomicOr(&any, 1);
  }
  __syncthreads();
  if (j == 0) *any_active = any;
}

// out[j] = sum of part[.][0][j]  (norms of the outer loop)
__global__ void k_mr_colsum(const double *part, int nblk, double *out) {
  const int j = threadIdx.x;
  double sums[1];
  sum_parts<1>(part, nblk, 1, 0, sums);
  if (j < kNrhs) out[j] = sums[0];
}

// out (cols x rows) = in (rows x cols), 32 x 32 tiles
__global__ void k_mr_transpose(int rows, int cols, const double *in, double *out) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = by + k, c = bx + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = in[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = bx + k, r = by + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[threadIdx.x][k];
  }
}

// R (nd x kNrhs) = B - (HU)^T where HU is kNrhs x nd (one product per row)
__global__ void k_mr_resid(int nd, const double *B, const double *HU, double *R) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // bx: rows of R, by: RHS
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int j = by + k, i = bx + threadIdx.x;
    if (j < kNrhs && i < nd) tile[k][threadIdx.x] = HU[(size_t)j * nd + i];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int i = bx + k, j = by + threadIdx.x;
    if (i < nd && j < kNrhs) {
      const size_t e = (size_t)i * kNrhs + j;
      R[e] = B[e] - tile[threadIdx.x][k];
    }
  }
}

// U += D on the RHS whose mask is set
__global__ void __launch_bounds__(kVecThreads) k_mr_add(size_t n, const int *mask, const double *D, double *U) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    if (mask[e % kNrhs]) U[e] += D[e];
}

int grid_for(size_t n) { return (int)std::min<size_t>((n + kVecThreads - 1) / kVecThreads, 148 * 16); }

}  // namespace

int mr_row_blocks(int nd) { return std::max(1, std::min(2 * 148, (nd + 63) / 64)); }

cudaError_t mr_launch_dots(int nq, int nd, const double *x0, const double *y0, const double *x1, const double *y1,
                           double *part, cudaStream_t s) {
  const int nblk = mr_row_blocks(nd), rpb = (nd + nblk - 1) / nblk;
  if (nq == 1) k_mr_dots<1><<<nblk, kVecThreads, 0, s>>>(nd, rpb, x0, y0, nullptr, nullptr, part);
  else k_mr_dots<2><<<nblk, kVecThreads, 0, s>>>(nd, rpb, x0, y0, x1, y1, part);
  return cudaGetLastError();
}

cudaError_t mr_launch_setup(int nd, const double *R, double *r, double *rh, double *p, double *ap, double *x,
                            cudaStream_t s) {
  const size_t n = (size_t)nd * kNrhs;
  k_mr_setup<<<grid_for(n), kVecThreads, 0, s>>>(n, R, r, rh, p, ap, x);
  return cudaGetLastError();
}

cudaError_t mr_launch_init(int nd, const double *part, const double *thresh, const int *mask, MrScal *sc,
                           int *any_active, cudaStream_t s) {
  k_mr_init<<<1, kScalThreads, 0, s>>>(part, mr_row_blocks(nd), thresh, mask, sc, any_active);
  return cudaGetLastError();
}

cudaError_t mr_launch_step(const MrStep &a, cudaStream_t s) {
  const size_t n = (size_t)a.nd * kNrhs;
  const int nblk = mr_row_blocks(a.nd), rpb = (a.nd + nblk - 1) / nblk;
  cudaError_t e;
  k_mr_p<<<grid_for(n), kVecThreads, 0, s>>>(n, a.sc, a.r, a.p, a.ap, a.f32);
  if ((e = a.matmat(a.ctx, a.f32, a.ap, s)) != cudaSuccess) return e;
  k_mr_dots<1><<<nblk, kVecThreads, 0, s>>>(a.nd, rpb, a.rh, a.ap, nullptr, nullptr, a.part);
  k_mr_alpha<<<1, kScalThreads, 0, s>>>(a.part, nblk, a.sc);
  k_mr_t<<<grid_for(n), kVecThreads, 0, s>>>(n, a.sc, a.r, a.ap, a.t, a.f32);
  if ((e = a.matmat(a.ctx, a.f32, a.at, s)) != cudaSuccess) return e;
  k_mr_dots<2><<<nblk, kVecThreads, 0, s>>>(a.nd, rpb, a.at, a.t, a.at, a.at, a.part);
  k_mr_zeta<<<1, kScalThreads, 0, s>>>(a.part, nblk, a.sc);
  k_mr_xr<<<nblk, kVecThreads, 0, s>>>(a.nd, rpb, a.sc, a.p, a.t, a.at, a.rh, a.x, a.r, a.part);
  k_mr_beta<<<1, kScalThreads, 0, s>>>(a.part, nblk, a.max_iter, a.sc, a.any_active);
  return cudaGetLastError();
}

cudaError_t mr_launch_colsum(int nd, const double *part, double *out, cudaStream_t s) {
  k_mr_colsum<<<1, kScalThreads, 0, s>>>(part, mr_row_blocks(nd), out);
  return cudaGetLastError();
}

cudaError_t mr_launch_transpose(int rows, int cols, const double *in, double *out, cudaStream_t s) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  k_mr_transpose<<<grid, block, 0, s>>>(rows, cols, in, out);
  return cudaGetLastError();
}

cudaError_t mr_launch_resid(int nd, const double *B, const double *HU, double *R, cudaStream_t s) {
  dim3 grid((nd + 31) / 32, (kNrhs + 31) / 32), block(32, 8);
  k_mr_resid<<<grid, block, 0, s>>>(nd, B, HU, R);
  return cudaGetLastError();
}

cudaError_t mr_launch_add(int nd, const int *mask, const double *D, double *U, cudaStream_t s) {
  const size_t n = (size_t)nd * kNrhs;
  k_mr_add<<<grid_for(n), kVecThreads, 0, s>>>(n, mask, D, U);
  return cudaGetLastError();
}

}  // namespace hbx
