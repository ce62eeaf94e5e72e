// hbx_dots.cuh -- compensated dot products with a fixed reduction order,
// shared by the GCR(m) and pipelined BiCGSTAB kernels.
//
// Geometry: dot_blocks(n) blocks of kDotThreads threads; thread g of the grid
// accumulates elements g, g + G, g + 2G, ... (G the grid's thread count) in a
// Dot2 pair, the warps merge by butterfly (warp_merge), thread 0 of a block
// merges its warps in warp order and writes the block's partial
// part[(block * kMaxDots + j) * 2 + {0, 1}].  The total of pair j is summed
// over the blocks by one warp: lane l takes blocks l, l + 32, ..., each
// chunk of 32 is butterfly-merged and added to the running pair in chunk
// order.  The result therefore depends on n only, and a CPU replay that
// follows the same order reproduces it bit for bit.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>

#include "hbx_device.cuh"
#include "hbx_engine.h"

namespace hbx {

constexpr int kDotThreads = 256;

inline int dot_blocks(size_t n) { return (int)std::min<size_t>((n + kDotThreads - 1) / kDotThreads, 148 * 4); }

// Every thread of the block calls this with its K running pairs; thread 0
// writes the block's partials.
template <int K>
__device__ __forceinline__ void block_partials(Acc2 (&a)[K], double *part) {
  __shared__ double sh[kDotThreads / 32][K][2];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const Acc2 m = warp_merge(a[j]);
    if (lane == 0) {
      sh[w][j][0] = m.s;
      sh[w][j][1] = m.c;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      Acc2 t{sh[0][j][0], sh[0][j][1]};
      for (int q = 1; q < kDotThreads / 32; ++q) t = acc2_merge(t, Acc2{sh[q][j][0], sh[q][j][1]});
      part[((size_t)blockIdx.x * kMaxDots + j) * 2] = t.s;
      part[((size_t)blockIdx.x * kMaxDots + j) * 2 + 1] = t.c;
    }
  }
}

// The total of pair j over nblk block partials; called by a whole warp,
// returned on every lane.  The partials are read through L2 (written by
// other blocks of the same launch in the fused kernels).
__device__ __forceinline__ double pair_total(const double *part, int nblk, int j) {
  const int lane = threadIdx.x & 31;
  Acc2 a{0.0, 0.0};
  for (int b0 = 0; b0 < nblk; b0 += 32) {
    const int b = b0 + lane;
    Acc2 v{0.0, 0.0};
    if (b < nblk) v = Acc2{__ldcg(part + ((size_t)b * kMaxDots + j) * 2), __ldcg(part + ((size_t)b * kMaxDots + j) * 2 + 1)};
    a = acc2_merge(a, warp_merge(v));
  }
  return a.s + a.c;
}

// After block_partials: true in the block that finished last (the one that
// then sums every partial); it also re-arms the ticket for the next launch.
__device__ __forceinline__ bool last_block(unsigned *ticket) {
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(ticket, 1u);
    last = t == gridDim.x - 1;
    if (last) *ticket = 0;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

}  // namespace hbx
