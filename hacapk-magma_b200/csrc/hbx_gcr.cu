// hbx_gcr.cu -- GCR(m) on the GPU (HACApK_gcrm_lfmtx, m_HACApK_solve.f90:506-571).
//
// Every product is one k_matvec launch; the vectors stay on the device.  Dot
// products are compensated (Dot2) per block and summed over the blocks in a
// fixed order, so a solve is bit-reproducible; the vector updates are
// rounded as the reference writes them (a product, then a sum: no fma).
//
//   k_dots       up to kMaxDots dot products of vector pairs, per-block
//                compensated partials
//   k_dots_total the partials of every pair summed in block order (one warp each)
//   k_gcr_alpha  alpha = (q . r) / (q . q); |A p_k|^2 kept for the later betas
//   k_gcr_step   u += alpha p_k,  r -= alpha q_k
//   k_gcr_betas  beta_l = -(A p_l . A r) / |A p_l|^2
//   k_gcr_orth   p_new += beta_l p_l, A p_new += beta_l A p_l, l in order --
//                at a restart the new direction lands in slot 0 before the
//                loop, so l = 0 is the new vector itself, as in the reference
#include <cuda_runtime.h>

#include <algorithm>

#include "hbx_dots.cuh"

namespace hbx {
namespace {

struct DotPairs {
  const double *x[kMaxDots];
  const double *y[kMaxDots];
};

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

// dots[0] = q . r, dots[1] = q . q  ->  alpha, capap[ik]
__global__ void k_gcr_alpha(const double *dots, int ik, double *capap, double *alpha) {
  capap[ik] = dots[1];
  *alpha = dots[0] / dots[1];
}

__global__ void k_gcr_step(size_t n, const double *alpha, const double *p, const double *q, double *u, double *r) {
  const double a = *alpha;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    u[i] = __dadd_rn(u[i], __dmul_rn(a, p[i]));
    r[i] = __dsub_rn(r[i], __dmul_rn(a, q[i]));
  }
}

__global__ void k_gcr_betas(const double *dots, const double *capap, int k, double *beta) {
  const int l = threadIdx.x;
  if (l < k) beta[l] = -dots[l] / capap[l];
}

__global__ void k_gcr_orth(size_t n, int k, int inew, const double *beta, double *p, double *ap) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double vp = p[(size_t)inew * n + i], va = ap[(size_t)inew * n + i];
    for (int l = 0; l < k; ++l) {
      const double sp = l == inew ? vp : p[(size_t)l * n + i];
      const double sa = l == inew ? va : ap[(size_t)l * n + i];
      vp = __dadd_rn(vp, __dmul_rn(beta[l], sp));
      va = __dadd_rn(va, __dmul_rn(beta[l], sa));
    }
    p[(size_t)inew * n + i] = vp;
    ap[(size_t)inew * n + i] = va;
  }
}

int vgrid(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }

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

cudaError_t gcr_launch_alpha(const double *dots, int ik, double *capap, double *alpha, cudaStream_t s) {
  k_gcr_alpha<<<1, 1, 0, s>>>(dots, ik, capap, alpha);
  return cudaGetLastError();
}

cudaError_t gcr_launch_step(size_t n, const double *alpha, const double *p, const double *q, double *u, double *r,
                            cudaStream_t s) {
  k_gcr_step<<<vgrid(n), 256, 0, s>>>(n, alpha, p, q, u, r);
  return cudaGetLastError();
}

cudaError_t gcr_launch_orth(size_t n, int k, int inew, const double *dots, const double *capap, double *beta,
                            double *p, double *ap, cudaStream_t s) {
  if (k < 1 || k > kMaxDots) return cudaErrorInvalidValue;
  k_gcr_betas<<<1, kMaxDots, 0, s>>>(dots, capap, k, beta);
  k_gcr_orth<<<vgrid(n), 256, 0, s>>>(n, k, inew, beta, p, ap);
  return cudaGetLastError();
}

}  // namespace hbx
