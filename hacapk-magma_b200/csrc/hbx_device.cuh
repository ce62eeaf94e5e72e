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
// Run records in flight: the gather warp bulk-copies the records it will
// need this many runs ahead (they come from HBM: the matrix stream evicts
// them from L2 between two matvecs).
constexpr uint32_t kRecSlots = 8;
// Block ends are summed kGroup at a time, after one CTA barrier for the
// group; the partials of two groups fit in shared memory.
#ifndef HBX_GROUP
#define HBX_GROUP 2
#endif
constexpr uint32_t kGroup = HBX_GROUP;

// Shared-memory offset in the ring of stream byte p of absolute chunk c
// (c = pass base + p / kChunkBytes).  The ring need not be a power of two.
__device__ __forceinline__ uint32_t ring_off(uint32_t c, uint32_t p) {
  return (c % (uint32_t)kRingChunks) * (uint32_t)kChunkBytes + (p & (uint32_t)(kChunkBytes - 1));
}
// consumer warps, then the bulk-copy producer warp, then the gather warp
constexpr int kProducerWarp = kConsumerWarps;
constexpr int kGatherWarp = kConsumerWarps + 1;
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
  static constexpr uint32_t red = empty + 8 * kRingChunks;            // [2*kGroup][NW][64] double
  static constexpr uint32_t scal = red + 2 * kGroup * kConsumerWarps * 64 * 8;  // 64 doubles of scratch
  static constexpr uint32_t stage = scal + 64 * 8;                     // [kStages][kStageBytes]
  static constexpr uint32_t rec = stage + kStages * kStageBytes;       // [kRecSlots] run records
  static constexpr uint32_t rfull = rec + kRecSlots * kRecBytes;       // [kRecSlots] record landed
  static constexpr uint32_t hdr = rfull + 8 * kRecSlots;               // [kStages] Run
  static constexpr uint32_t sfull = hdr + kStages * 32;                // stage filled (gather warp)
  static constexpr uint32_t sempty = sfull + 8 * kStages;              // stage consumed (consumer warps)
  static constexpr uint32_t xready = sempty + 8 * kStages;             // a pass's x is complete grid-wide
  static constexpr uint32_t garrive = xready + 8;                      // this CTA arrived on the grid barrier
  static constexpr uint32_t gen = garrive + 8;                         // grid-barrier generation of that arrival
  static constexpr uint32_t binfo = gen + 16;                          // [2*kGroup] pending block ends
  static constexpr uint32_t bytes = binfo + 2 * kGroup * 8;
};
static_assert(SharedLayout::stage % 16 == 0 && SharedLayout::hdr % 16 == 0 && SharedLayout::sfull % 8 == 0 &&
                  SharedLayout::rec % 16 == 0,
              "shared-memory layout alignment");
static_assert(SharedLayout::bytes <= 227 * 1024, "shared memory per CTA");

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
#ifndef HBX_SUSPEND_NS
#define HBX_SUSPEND_NS 1000000
#endif
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
#if HBX_SUSPEND_NS > 0
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"((uint32_t)HBX_SUSPEND_NS)
      : "memory");
#else
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
#endif
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
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16cg(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// The mbarrier receives one arrival once every earlier cp.async of this
// thread has landed (the barrier's count includes it: .noinc).
__device__ __forceinline__ void cp_async_arrive(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

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
    const uint32_t s = g % kRingChunks;
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
  for (uint32_t g = g0; g < issued; ++g) mbar_wait(&full[g % kRingChunks], (g / kRingChunks) & 1, timeout_ns);
}

// ---- consumer-side ring state (one per warp) ------------------------------
struct RingCounters {
  uint32_t waited, released;
  uint32_t bad;
};

// Releases every chunk below c0 (each only after it was observed full, so
// every release lands in the right barrier phase), then waits until chunk c1
// is full.  Inlined: a chunk switch is frequent enough that a call costs.
__device__ __forceinline__ RingCounters ring_advance(RingCounters rc, uint32_t c0, uint32_t c1, uint64_t *full,
                                                  uint64_t *empty, uint64_t timeout_ns, int *err) {
  const int lane = threadIdx.x & 31;
  while (!rc.bad && rc.released < c0) {
    if (rc.waited <= rc.released) {
      if (!warp_wait(&full[rc.released % kRingChunks], (rc.released / kRingChunks) & 1, timeout_ns)) {
        rc.bad = 1;
        break;
      }
      rc.waited = rc.released + 1;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[rc.released % kRingChunks]);
    ++rc.released;
  }
  while (!rc.bad && rc.waited <= c1) {
    if (!warp_wait(&full[rc.waited % kRingChunks], (rc.waited / kRingChunks) & 1, timeout_ns)) {
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
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---- gather warp: for every run of the CTA, in order and for every pass,
// copies the run header into hdr[slot] and gathers the run's vector segments
// (x for P and D runs, zbu for U runs) into stage[slot] with 8-byte cp.async
// (segments start anywhere; the warp copies long segments together and
// short ones one per lane), kStages runs ahead of the consumers.  Lane l
// holds 16 bytes of the 512-byte record: lanes 0-1 the header, lane l >= 2
// segments 2(l-2) and 2(l-2)+1.  Before the first run of pass p it waits
// until that pass's x is complete grid-wide (xready), and before the first U
// run until every CTA's zbu is (this CTA's grid-barrier arrival, then the
// barrier).  Every wait is bounded; on a timeout the warp flags the error
// and stops, and the consumers' own bounded waits end the launch.
struct GatherCtx {
  const RunRec *recs;
  uint32_t nr_p, nr_d, nr_u, npass;
  const void *x0, *x1;  // x of pass 0 and pass 1 (float copies for FP32 engines)
  const void *zbu;       // zbu (float copy for FP32 engines)
  unsigned *gbar;
  int *err;
  uint64_t timeout_ns;
};

// Staging copies with cp.async: doubles for FP64 engines, the float copies
// of the vectors for FP32 engines.
template <bool kF32>
__device__ __forceinline__ void stage_elems(uint8_t *st, uint32_t dst, const void *src, uint32_t e0, uint32_t len,
                                            uint32_t step) {
  if (kF32) {
    float *sf = reinterpret_cast<float *>(st) + dst;
    const float *s = reinterpret_cast<const float *>(src);
    for (uint32_t e = e0; e < len; e += step) cp_async4(sf + e, s + e);
  } else {
    double *sd = reinterpret_cast<double *>(st) + dst;
    const double *s = reinterpret_cast<const double *>(src);
    for (uint32_t e = e0; e < len; e += step) cp_async8(sd + e, s + e);
  }
}

template <bool kF32, class SM>
__device__ __forceinline__ void gather_warp(const GatherCtx &c, const SM &sm) {
  const int lane = threadIdx.x & 31;
  const uint32_t nruns = c.nr_p + c.nr_d + c.nr_u, total = nruns * c.npass;
  if (total == 0) return;
  // records g .. g + kRecSlots - 1 are in flight into slots g % kRecSlots
  uint32_t issued = 0;
  auto issue = [&](uint32_t gg) {
    const uint32_t rs = gg % kRecSlots;
    mbar_arrive_expect_tx(&sm.rfull[rs], (uint32_t)kRecBytes);
    bulk_g2s(sm.rec + rs * kRecBytes, c.recs + (gg % nruns), (uint32_t)kRecBytes, &sm.rfull[rs]);
  };
  if (lane == 0)
    for (uint32_t gg = 0; gg < min(total, kRecSlots); ++gg) issue(gg);
  issued = min(total, kRecSlots);
  uint32_t g = 0;
  for (; g < total; ++g) {
    const uint32_t k = g % nruns, pass = g / nruns;
    const uint32_t rs = g % kRecSlots;
    if (!warp_wait(&sm.rfull[rs], (g / kRecSlots) & 1, c.timeout_ns)) {
      if (lane == 0) atomicOr(c.err, kErrProducer);
      break;
    }
    const uint4 cur = reinterpret_cast<const uint4 *>(sm.rec + rs * kRecBytes)[lane];
    __syncwarp();  // every lane has read the slot before it is refilled
    if (g + kRecSlots < total) {
      if (lane == 0) issue(g + kRecSlots);
      issued = g + kRecSlots + 1;
    }
    bool ok = true;
    if (k == 0) ok = warp_wait(sm.xready, pass & 1, c.timeout_ns);
    if (ok && k == c.nr_p + c.nr_d) {  // first U run of the pass: zbu must be complete grid-wide
      ok = warp_wait(sm.garrive, pass & 1, c.timeout_ns);
      if (ok) {
        int gok = 1;
        if (lane == 0) gok = grid_wait(c.gbar, *sm.gen, c.timeout_ns) ? 1 : 0;
        ok = __shfl_sync(0xffffffffu, gok, 0) != 0;
        __syncwarp();
        __threadfence();
      }
    }
    const uint32_t slot = g % kStages;
    if (ok && g >= (uint32_t)kStages) ok = warp_wait(&sm.sempty[slot], ((g / kStages) - 1) & 1, c.timeout_ns);
    if (!ok) {
      if (lane == 0) atomicOr(c.err, kErrProducer);
      ++g;  // this record was consumed
      break;
    }
    if (lane < 2) reinterpret_cast<uint4 *>(sm.hdr + slot)[lane] = cur;
    const uint32_t w2 = __shfl_sync(0xffffffffu, cur.z, 0);  // nrow | npanel << 16
    const uint32_t w3 = __shfl_sync(0xffffffffu, cur.w, 0);  // flags | rot << 16
    const uint32_t w4 = __shfl_sync(0xffffffffu, cur.x, 1);  // nseg | vlen << 16
    const uint32_t nseg = w4 & 0xffffu, vlen = w4 >> 16;
    const void *vec = (w3 & 0xffu) == kRunU ? c.zbu : ((pass & 1) ? c.x1 : c.x0);
    const uint32_t esz = kF32 ? 4u : 8u;
    uint8_t *st = sm.stage + slot * kStageBytes;
    const uint32_t nlong = __shfl_sync(0xffffffffu, cur.w, 1);
    // long segments: the whole warp copies each one (segment s sits in lane
    // 2 + s/2 of the record, fields (x, y) for even s and (z, w) for odd s)
    for (uint32_t q = 0; q < nlong; ++q) {
      const int holder = 2 + (int)(q >> 1);
      const uint32_t src = __shfl_sync(0xffffffffu, (q & 1) ? cur.z : cur.x, holder);
      const uint32_t ld = __shfl_sync(0xffffffffu, (q & 1) ? cur.w : cur.y, holder);
      const uint32_t len = ld & 0xffffu, dst = ld >> 16;
      stage_elems<kF32>(st, dst, static_cast<const uint8_t *>(vec) + (size_t)src * esz, (uint32_t)lane, len, 32);
    }
    // short segments: lane i copies segment nlong + i (and nlong + 32 + i)
    for (uint32_t base = nlong; base < nseg; base += 32) {
      const uint32_t q = base + (uint32_t)lane;
      const int holder = 2 + (int)((q >> 1) & 31u);  // only q < nseg <= 60 is used
      const uint32_t sx = __shfl_sync(0xffffffffu, cur.x, holder);
      const uint32_t sy = __shfl_sync(0xffffffffu, cur.y, holder);
      const uint32_t sz = __shfl_sync(0xffffffffu, cur.z, holder);
      const uint32_t sw = __shfl_sync(0xffffffffu, cur.w, holder);
      if (q < nseg) {
        const uint32_t src = (q & 1) ? sz : sx, ld = (q & 1) ? sw : sy;
        const uint32_t len = ld & 0xffffu, dst = ld >> 16;
        stage_elems<kF32>(st, dst, static_cast<const uint8_t *>(vec) + (size_t)src * esz, 0, len, 1);
      }
    }
    // the zero columns that fill the last panel
    const uint32_t vend = (w2 >> 16) * (kF32 ? 4u : 2u);
    for (uint32_t e = vlen + (uint32_t)lane; e < vend; e += 32) {
      if (kF32) reinterpret_cast<float *>(st)[e] = 0.0f;
      else reinterpret_cast<double *>(st)[e] = 0.0;
    }
    cp_async_arrive(&sm.sfull[slot]);
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.sfull[slot]);  // releases the header and the plain stores
  }
  // record copies still in flight (only after an error) must land before exit
  if (lane == 0)
    for (uint32_t gg = g; gg < issued; ++gg) mbar_wait(&sm.rfull[gg % kRecSlots], (gg / kRecSlots) & 1, c.timeout_ns);
  cp_async_wait_all();
}

// ---- one run of a block: acc(lane) += sum over the run's panels of
// B(lane, c) v(c).  Panel j (16h bytes, row i at 16i: two double columns or
// four float columns) is read by warp (rot + j) mod NW, kUnroll panels per
// iteration, so the 16 warps together hold a window of NW*kUnroll panels of
// the ring; lanes >= h repeat row h-1 and their sums are never used.  FP32
// panels are multiplied in float (four accumulators per row) and added to the
// row's double accumulator at the end of the run.
#ifndef HBX_UNROLL
#define HBX_UNROLL 4
#endif
constexpr uint32_t kUnroll = HBX_UNROLL;

__device__ __forceinline__ float4 lds_f32x4(uint32_t addr) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
  return v;
}

// Per-precision panel arithmetic: load a 16-byte stage group / panel row and
// multiply-accumulate it.
template <bool kF32>
struct PanelMath;
template <>
struct PanelMath<false> {
  using V = double2;
  struct Acc {
    double a0 = 0.0, a1 = 0.0;
    __device__ __forceinline__ double sum() const { return a0 + a1; }
  };
  static __device__ __forceinline__ V ld(uint32_t addr) { return lds_f64x2(addr); }
  static __device__ __forceinline__ void fma(Acc &a, const V &m, const V &v) {
    a.a0 = ::fma(m.x, v.x, a.a0);
    a.a1 = ::fma(m.y, v.y, a.a1);
  }
};
template <>
struct PanelMath<true> {
  using V = float4;
  struct Acc {
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    __device__ __forceinline__ double sum() const { return ((double)a0 + (double)a1) + ((double)a2 + (double)a3); }
  };
  static __device__ __forceinline__ V ld(uint32_t addr) { return lds_f32x4(addr); }
  static __device__ __forceinline__ void fma(Acc &a, const V &m, const V &v) {
    a.a0 = fmaf(m.x, v.x, a.a0);
    a.a1 = fmaf(m.y, v.y, a.a1);
    a.a2 = fmaf(m.z, v.z, a.a2);
    a.a3 = fmaf(m.w, v.w, a.a3);
  }
};

// (18 warps of 576 threads leave 96 registers a thread: the two-row form
// unrolls by 2 to stay within them.)
template <bool kTwoRows, bool kF32>
__device__ __forceinline__ void run_block_rows(const Run &run, uint32_t stage_s, Ring &R, double &acc, double &acc2) {
  using PM = PanelMath<kF32>;
  using V = typename PM::V;
  constexpr uint32_t NW = kConsumerWarps, U = kTwoRows ? 2 : kUnroll;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t h = run.nrow, np = run.npanel;
  if (np == 0) return;
  const uint32_t pb = 16u * h;
  const uint32_t lrow = 16u * min((uint32_t)lane, h - 1u);
  const uint32_t lrow2 = 16u * min((uint32_t)lane + 32u, h - 1u) - lrow;  // second row, relative
  const uint32_t ring_s = smem_u32(R.buf);
  uint32_t j = (uint32_t)((w - (int)run.rot) & (int)(NW - 1));
  typename PM::Acc a[U], b[kTwoRows ? U : 1];
  for (; j + (U - 1) * NW < np; j += U * NW) {
    const uint32_t p0 = run.pos + j * pb;
    R.ensure(p0, p0 + (U - 1) * NW * pb + pb);
    V v[U], m[U], m2[kTwoRows ? U : 1];
#pragma unroll
    for (uint32_t u = 0; u < U; ++u) v[u] = PM::ld(stage_s + 16u * (j + u * NW));
    const uint32_t pl = p0 + lrow;
    const uint32_t q = ring_off(R.base + (pl >> kChunkLog), pl);
    if (q + (U - 1) * NW * pb + (kTwoRows ? lrow2 : 0u) + 16u <= kRingBytes) {  // no wrap around the ring end
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        m[u] = PM::ld(ring_s + q + u * NW * pb);
        if (kTwoRows) m2[u] = PM::ld(ring_s + q + u * NW * pb + lrow2);
      }
    } else {
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        const uint32_t pu = pl + u * NW * pb;
        m[u] = PM::ld(ring_s + ring_off(R.base + (pu >> kChunkLog), pu));
        if (kTwoRows) m2[u] = PM::ld(ring_s + ring_off(R.base + ((pu + lrow2) >> kChunkLog), pu + lrow2));
      }
    }
#pragma unroll
    for (uint32_t u = 0; u < U; ++u) {
      PM::fma(a[u], m[u], v[u]);
      if (kTwoRows) PM::fma(b[u], m2[u], v[u]);
    }
  }
  for (; j < np; j += NW) {
    const uint32_t p0 = run.pos + j * pb;
    R.ensure(p0, p0 + pb);
    const V vv = PM::ld(stage_s + 16u * j);
    const uint32_t pl = p0 + lrow;
    PM::fma(a[0], PM::ld(ring_s + ring_off(R.base + (pl >> kChunkLog), pl)), vv);
    if (kTwoRows) {
      const uint32_t p2 = pl + lrow2;
      PM::fma(b[0], PM::ld(ring_s + ring_off(R.base + (p2 >> kChunkLog), p2)), vv);
    }
  }
  double t = 0.0;
#pragma unroll
  for (uint32_t u = 0; u < U; ++u) t += a[u].sum();
  acc += t;
  if (kTwoRows) {
    double t2 = 0.0;
#pragma unroll
    for (uint32_t u = 0; u < U; ++u) t2 += b[u].sum();
    acc2 += t2;
  }
}

// acc: row `lane` of the block; acc2: row lane + 32 (P slabs taller than 32).
template <bool kF32>
__device__ __forceinline__ void run_block(const Run &run, uint32_t stage_s, Ring &R, double &acc, double &acc2) {
  if (run.nrow > 32) run_block_rows<true, kF32>(run, stage_s, R, acc, acc2);
  else run_block_rows<false, kF32>(run, stage_s, R, acc, acc2);
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
