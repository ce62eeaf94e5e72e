// hbx_device.cuh -- sm_100a device building blocks of the streaming H-matvec.
//
//  * mbarrier + cp.async.bulk (1D TMA) ring: one producer thread copies the
//    CTA's contiguous stream into NS shared-memory chunks; consumer warps
//    wait on a chunk's "full" barrier, read it, and arrive on its "empty"
//    barrier; the producer refills a slot once every consumer warp released
//    it.  Every wait is bounded by a %globaltimer deadline; a wait that runs
//    out sets an error bit and makes the waiter give up instead of hanging.
//  * A sense-reversing grid barrier (count, generation) for the persistent
//    cooperative grid, with split arrive / wait so work can be placed between
//    the two, and the same bounded wait.
//  * The block-row processor shared by the matvec and BiCGSTAB kernels.
#pragma once

#include <cstdint>

#include "hbx_plan.h"

namespace hbx {

constexpr uint32_t kRingBytes = (uint32_t)kRingChunks * kChunkBytes;
constexpr uint32_t kRingMask = kRingBytes - 1;
// consumer warps, then the bulk-copy producer warp, then the descriptor warp
constexpr int kProducerWarp = kConsumerWarps;
constexpr int kDescWarp = kConsumerWarps + 1;
constexpr int kThreads = (kConsumerWarps + 2) * 32;
// Chunks the producer prefetches into L2 beyond the ones in flight into the
// ring.  The ring alone keeps kRingBytes in flight per SM, about what HBM
// latency times the per-SM share of bandwidth needs, so any time consumers
// hold a chunk shows up as lost bandwidth; the L2 prefetch keeps HBM busy
// further ahead and turns the ring refills into L2 hits.
#ifndef HBX_L2_AHEAD
#define HBX_L2_AHEAD 0
#endif
constexpr uint32_t kL2Ahead = HBX_L2_AHEAD;

// error bits written to the device error word
enum : int { kErrPipeline = 1, kErrGridBarrier = 2, kErrProducer = 4 };

struct SharedLayout {
  static constexpr uint32_t ring = 0;
  static constexpr uint32_t full = kRingBytes;
  static constexpr uint32_t empty = full + 8 * kRingChunks;
  static constexpr uint32_t red = empty + 8 * kRingChunks;            // [2][NW][32] double
  static constexpr uint32_t scal = red + 2 * kConsumerWarps * 32 * 8;  // 64 doubles of scratch
  static constexpr uint32_t stage = scal + 64 * 8;                     // [2][kStageCap] double
  static constexpr uint32_t desc = stage + 2 * kStageCap * 8;          // [kDescSlots] run records
  static constexpr uint32_t dfull = desc + kDescSlots * kRecBytes;
  static constexpr uint32_t dempty = dfull + 8 * kDescSlots;
  static constexpr uint32_t bytes = dempty + 8 * kDescSlots;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// try_wait with a suspend-time hint: a waiting thread is parked (not
// spinning, so it takes no issue slots) until the phase completes or the
// hint (ns) elapses.
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(1000000u)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  while (!mbar_try_wait(bar, parity)) {
    if (gtimer() - t0 > timeout_ns) return false;
  }
  return true;
}

// Warp-uniform bounded wait: every lane observes the phase itself (so every
// lane acquires the bulk-copied bytes) and the outcome is agreed on.
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, uint64_t timeout_ns) {
  const bool ok = mbar_wait(bar, parity, timeout_ns);
  return __all_sync(0xffffffffu, ok);
}

// 1D bulk copy global -> shared, completion counted on `bar` (tx bytes).
// dst and src 16-byte aligned, bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Prefetch `bytes` (multiple of 16) of global memory into L2, no destination.
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// Ampere-style asynchronous gathers into shared memory (vector staging).
// 8-byte copies go through L1 (.ca); 16-byte copies bypass it (.cg).
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16cg(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ double ld_cg(const double *p) { return __ldcg(p); }

__device__ __forceinline__ double lds_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
  return v;
}

// 16-byte shared load (address 16-byte aligned).
__device__ __forceinline__ double2 lds_f64x2(uint32_t addr) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr));
  return v;
}

// ---- grid barrier: gbar[0] = arrivals, gbar[1] = generation ---------------
__device__ __forceinline__ void grid_arrive(unsigned *gbar, unsigned nblocks) {
  __threadfence();
  const unsigned old = atomicAdd(&gbar[0], 1u);
  if (old == nblocks - 1) {
    atomicExch(&gbar[0], 0u);
    __threadfence();
    atomicAdd(&gbar[1], 1u);
  }
}

// The trailing fence (as in cooperative groups' grid sync) orders every later
// load of the CTA -- after the caller's bar.sync -- behind the other CTAs'
// pre-barrier writes.
__device__ __forceinline__ bool grid_wait(const unsigned *gbar, unsigned gen, uint64_t timeout_ns) {
  if (ld_acquire(&gbar[1]) == gen) {
    const uint64_t t0 = gtimer();
    while (ld_acquire(&gbar[1]) == gen) {
      __nanosleep(64);
      if (gtimer() - t0 > timeout_ns) return false;
    }
  }
  __threadfence();
  return true;
}

// ---- producer: streams `npass` passes over the CTA's byte range ------------
__device__ __forceinline__ void producer_run(const uint8_t *src, uint32_t bytes, uint32_t npass,
                                             uint8_t *ring, uint64_t *full, uint64_t *empty, int *err,
                                             uint64_t timeout_ns) {
  const uint32_t K = (bytes + kChunkBytes - 1) >> kChunkLog;
  const uint32_t total = K * npass;
  auto prefetch = [&](uint32_t g) {
    const uint32_t off = (g % K) << kChunkLog;
    bulk_prefetch_l2(src + off, min((uint32_t)kChunkBytes, bytes - off));
  };
  for (uint32_t g = kRingChunks; g < min(total, (uint32_t)kRingChunks + kL2Ahead); ++g) prefetch(g);
  uint32_t issued = 0;
  for (uint32_t g = 0; g < total; ++g) {
    const uint32_t s = g & (kRingChunks - 1);
    if (g >= (uint32_t)kRingChunks) {
      if (!mbar_wait(&empty[s], ((g / kRingChunks) - 1) & 1, timeout_ns)) {
        atomicOr(err, kErrProducer);
        break;
      }
    }
    const uint32_t k = g % K;
    const uint32_t off = k << kChunkLog;
    const uint32_t nb = min((uint32_t)kChunkBytes, bytes - off);
    mbar_arrive_expect_tx(&full[s], nb);
    bulk_g2s(ring + ((size_t)s << kChunkLog), src + off, nb, &full[s]);
    issued = g + 1;
    if (kL2Ahead > 0 && g + kRingChunks + kL2Ahead < total) prefetch(g + kRingChunks + kL2Ahead);
  }
  // Copies still in flight must land before the CTA exits.
  const uint32_t g0 = issued > (uint32_t)kRingChunks ? issued - kRingChunks : 0;
  for (uint32_t g = g0; g < issued; ++g) mbar_wait(&full[g & (kRingChunks - 1)], (g / kRingChunks) & 1, timeout_ns);
}

// ---- descriptor warp: keeps the descriptor queue kDescSlots run records
// ahead of the consumers.  Records are fixed-size (kRecBytes) and contiguous
// per CTA, so each one is a single bulk copy with no dependent load.  Only
// lane 0 works.
__device__ __forceinline__ void desc_run(const RunRec *recs, uint32_t nruns, uint32_t npass, uint8_t *dbuf,
                                         uint64_t *dfull, uint64_t *dempty, int *err, uint64_t timeout_ns) {
  if ((threadIdx.x & 31) != 0) return;
  const uint32_t total = nruns * npass;
  for (uint32_t g = 0; g < total; ++g) {
    const uint32_t slot = g % kDescSlots;
    if (g >= (uint32_t)kDescSlots) {
      if (!mbar_wait(&dempty[slot], ((g / kDescSlots) - 1) & 1, timeout_ns)) {
        atomicOr(err, kErrProducer);
        return;
      }
    }
    mbar_arrive_expect_tx(&dfull[slot], (uint32_t)kRecBytes);
    bulk_g2s(dbuf + slot * kRecBytes, recs + (g % nruns), (uint32_t)kRecBytes, &dfull[slot]);
  }
  // the last slots' copies must land before the CTA exits
  const uint32_t g0 = total > (uint32_t)kDescSlots ? total - kDescSlots : 0;
  for (uint32_t g = g0; g < total; ++g) mbar_wait(&dfull[g % kDescSlots], (g / kDescSlots) & 1, timeout_ns);
}

// Consumer view of the descriptor queue; g counts runs across sections and passes.
struct DescQ {
  uint8_t *dbuf;
  uint64_t *dfull, *dempty;
  uint32_t g;
  uint64_t timeout_ns;
  int *err;
  __device__ __forceinline__ const RunRec *get(uint32_t i, bool &bad) {
    const uint32_t gi = g + i;
    const uint32_t slot = gi % kDescSlots;
    if (!bad && !warp_wait(&dfull[slot], (gi / kDescSlots) & 1, timeout_ns)) {
      bad = true;
      if ((threadIdx.x & 31) == 0) atomicOr(err, kErrPipeline);
    }
    return reinterpret_cast<const RunRec *>(dbuf + slot * kRecBytes);
  }
  __device__ __forceinline__ void release(uint32_t i) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(&dempty[(g + i) % kDescSlots]);
  }
};

// ---- consumer-side ring state (one per warp) ------------------------------
struct RingCounters {
  uint32_t waited, released;
  uint32_t bad;
};

// Releases every chunk below c0 (each only after it was observed full, so
// every release lands in the right barrier phase), then waits until chunk c1
// is full.  Out of line and by value, so the per-warp ring state stays in
// registers on the fast path.
__device__ __noinline__ RingCounters ring_advance(RingCounters rc, uint32_t c0, uint32_t c1, uint64_t *full,
                                                  uint64_t *empty, uint64_t timeout_ns, int *err) {
  const int lane = threadIdx.x & 31;
  while (!rc.bad && rc.released < c0) {
    if (rc.waited <= rc.released) {
      if (!warp_wait(&full[rc.released & (kRingChunks - 1)], (rc.released / kRingChunks) & 1, timeout_ns)) {
        rc.bad = 1;
        break;
      }
      rc.waited = rc.released + 1;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[rc.released & (kRingChunks - 1)]);
    ++rc.released;
  }
  while (!rc.bad && rc.waited <= c1) {
    if (!warp_wait(&full[rc.waited & (kRingChunks - 1)], (rc.waited / kRingChunks) & 1, timeout_ns)) {
      rc.bad = 1;
      break;
    }
    ++rc.waited;
  }
  if (rc.bad && lane == 0) atomicOr(err, kErrPipeline);
  return rc;
}

struct Ring {
  const uint8_t *buf;
  uint64_t *full, *empty;
  uint32_t waited;    // chunks [0, waited) observed full by this warp
  uint32_t released;  // chunks [0, released) released by this warp
  uint32_t base;      // absolute chunk index of position 0 of the current pass
  uint64_t timeout_ns;
  int *err;
  bool bad;           // a wait ran out: stop waiting, results are garbage

  __device__ __forceinline__ void advance(uint32_t c0, uint32_t c1) {
    if (bad) return;
    RingCounters rc{waited, released, 0u};
    rc = ring_advance(rc, c0, c1, full, empty, timeout_ns, err);
    waited = rc.waited;
    released = rc.released;
    bad = rc.bad != 0;
  }
  // Release every chunk below absolute index c.
  __device__ __forceinline__ void release_below(uint32_t c) {
    if (released < c) advance(c, 0);
  }
  // Make stream bytes [p0, p1) of the current pass readable (the span must
  // cover fewer than kRingChunks chunks).  The common case -- same chunk as
  // before, already full -- is two compares.
  __device__ __forceinline__ void ensure(uint32_t p0, uint32_t p1) {
    if (p1 <= p0) return;
    const uint32_t c0 = base + (p0 >> kChunkLog);
    const uint32_t c1 = base + ((p1 - 1) >> kChunkLog);
    if (c0 == released && c1 < waited) return;
    advance(c0, c1);
  }
  // Release everything below absolute chunk `end` (end of the last pass).
  __device__ __forceinline__ void drain(uint32_t end) { release_below(end); }
  __device__ __forceinline__ double ld(uint32_t p) const {
    const uint32_t c = base + (p >> kChunkLog);
    const double *q = reinterpret_cast<const double *>(buf + (((c & (kRingChunks - 1)) << kChunkLog) |
                                                              (p & (kChunkBytes - 1))));
    return *q;
  }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---- vector staging of one run: warp w gathers segments w, w+NW, ... with
// 8-byte cp.async (segments start anywhere); an odd-width block's zero
// column is written directly.  The record is in the descriptor queue.
__device__ __forceinline__ void gather_run(const RunRec &rec, const double *x, const double *zbu, double *stage) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const Run &run = rec.hdr;
  const double *vec = run_kind(run) == kRunU ? zbu : x;
  for (uint32_t q = w; q < run.nseg; q += kConsumerWarps) {
    const Seg sg = rec.seg[q];
    for (uint32_t e = lane; e < sg.len; e += 32) cp_async8(stage + sg.dst + e, vec + sg.src + e);
  }
  if ((run.flags & kPadCol) && w == 0 && lane == 0) stage[2u * run.npair - 1u] = 0.0;
  cp_async_commit();
}

// ---- one run of a block: acc(lane) += sum over the run's column pairs of
// B(lane, c) v(c).  Pair panel j (16h bytes, row i at 16i) is read by warp
// (rot + j) mod NW, four panels per iteration; lanes >= h repeat row h-1 and
// their sums are never used.
__device__ __forceinline__ void run_block(const Run &run, uint32_t stage_s, Ring &R, double &acc) {
  constexpr uint32_t NW = kConsumerWarps;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t h = run.nrow, np = run.npair;
  if (np == 0) return;
  const uint32_t pb = 16u * h;
  const uint32_t lrow = 16u * min((uint32_t)lane, h - 1u);
  const uint32_t ring_s = smem_u32(R.buf);
  const uint32_t q0 = (R.base << kChunkLog) + run.pos + lrow;
  uint32_t j = (uint32_t)((w - (int)run.rot) & (int)(NW - 1));
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  for (; j + 3 * NW < np; j += 4 * NW) {
    const uint32_t p0 = run.pos + j * pb;
    R.ensure(p0, p0 + 3 * NW * pb + pb);
    const uint32_t vq = stage_s + 16u * j;
    const double2 v0 = lds_f64x2(vq), v1 = lds_f64x2(vq + 16 * NW);
    const double2 v2 = lds_f64x2(vq + 32 * NW), v3 = lds_f64x2(vq + 48 * NW);
    const uint32_t q = (q0 + j * pb) & kRingMask;
    double2 m0, m1, m2, m3;
    if (q + 3 * NW * pb + 16u <= kRingBytes) {  // the four panels do not wrap around the ring end
      const uint32_t a = ring_s + q;
      m0 = lds_f64x2(a);
      m1 = lds_f64x2(a + NW * pb);
      m2 = lds_f64x2(a + 2 * NW * pb);
      m3 = lds_f64x2(a + 3 * NW * pb);
    } else {
      m0 = lds_f64x2(ring_s + q);
      m1 = lds_f64x2(ring_s + ((q + NW * pb) & kRingMask));
      m2 = lds_f64x2(ring_s + ((q + 2 * NW * pb) & kRingMask));
      m3 = lds_f64x2(ring_s + ((q + 3 * NW * pb) & kRingMask));
    }
    a0 = fma(m0.x, v0.x, a0);
    a1 = fma(m0.y, v0.y, a1);
    a2 = fma(m1.x, v1.x, a2);
    a3 = fma(m1.y, v1.y, a3);
    a0 = fma(m2.x, v2.x, a0);
    a1 = fma(m2.y, v2.y, a1);
    a2 = fma(m3.x, v3.x, a2);
    a3 = fma(m3.y, v3.y, a3);
  }
  for (; j < np; j += NW) {
    const uint32_t p0 = run.pos + j * pb;
    R.ensure(p0, p0 + pb);
    const double2 v = lds_f64x2(stage_s + 16u * j);
    const double2 m = lds_f64x2(ring_s + ((q0 + j * pb) & kRingMask));
    a0 = fma(m.x, v.x, a0);
    a1 = fma(m.y, v.y, a1);
  }
  acc += (a0 + a1) + (a2 + a3);
}

// ---- compensated (Dot2) accumulation ------------------------------------------
struct Acc2 {
  double s, c;
};
__device__ __forceinline__ void two_sum_add(Acc2 &a, double p) {
  const double s = a.s + p;
  const double z = s - a.s;
  a.c += (a.s - (s - z)) + (p - z);
  a.s = s;
}
__device__ __forceinline__ void dot2_add(Acc2 &a, double x, double y) {
  const double p = x * y;
  const double e = fma(x, y, -p);
  two_sum_add(a, p);
  a.c += e;
}
__device__ __forceinline__ Acc2 acc2_merge(Acc2 a, Acc2 b) {
  Acc2 r{a.s, a.c + b.c};
  two_sum_add(r, b.s);
  return r;
}
__device__ __forceinline__ Acc2 warp_merge(Acc2 a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Acc2 b{__shfl_xor_sync(0xffffffffu, a.s, o), __shfl_xor_sync(0xffffffffu, a.c, o)};
    // both lanes of a pair compute the same merge in the same operand order
    const int lane = threadIdx.x & 31;
    a = (lane & o) ? acc2_merge(b, a) : acc2_merge(a, b);
  }
  return a;
}

}  // namespace hbx
