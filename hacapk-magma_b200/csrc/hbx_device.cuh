// hbx_device.cuh -- sm_100a device building blocks of the streaming H-matvec.
//
//  * mbarrier + cp.async.bulk (1D TMA) ring: one producer thread copies the
//    CTA's contiguous stream into kRingChunks shared-memory chunks, as far
//    ahead as the ring allows; consumer warps wait on a chunk's "full"
//    barrier, read it and arrive on its "empty" barrier, so the copies go on
//    while the consumers do the bookkeeping of a run.
//  * Gather warps fill a ring of vector stage buffers (the x or zbu segments
//    of a run) with cp.async; mbarriers hand a buffer to the consumers and
//    back.
//  * Every wait is bounded by a %globaltimer deadline; a wait that runs out
//    sets an error bit and makes the waiter give up instead of hanging.
//  * A sense-reversing grid barrier (count, generation) for the persistent
//    cooperative grid, with split arrive / wait and the same bounded wait.
#pragma once

#include <cstdint>

#include "hbx_plan.h"

namespace hbx {

constexpr uint32_t kRingBytes = (uint32_t)kRingChunks * kChunkBytes;
#ifndef HBX_GATHER_WARPS
#define HBX_GATHER_WARPS 2
#endif
constexpr int kGatherWarps = HBX_GATHER_WARPS;  // warps that stage run vectors
#ifndef HBX_REC_SLOTS
#define HBX_REC_SLOTS 8
#endif
constexpr uint32_t kRecSlots = HBX_REC_SLOTS;   // run records in flight per gather warp
constexpr uint32_t kRedSlots = 4;               // block ends parked at once
static_assert(kStages % kGatherWarps == 0, "a stage slot is always filled by the same gather warp");
// consumer warps, the bulk-copy producer warp, the gather warps, the
// grid-barrier warp and the block-sum warp
constexpr int kProducerWarp = kConsumerWarps;
constexpr int kGatherWarp0 = kConsumerWarps + 1;
constexpr int kSyncWarp = kGatherWarp0 + kGatherWarps;
constexpr int kSumWarp = kSyncWarp + 1;
constexpr int kThreads = (kSumWarp + 1) * 32;

// Shared-memory offset in the ring of stream byte p of absolute chunk c
// (c = pass base + p / kChunkBytes).  The ring need not be a power of two.
__device__ __forceinline__ uint32_t ring_off(uint32_t c, uint32_t p) {
  return (c % (uint32_t)kRingChunks) * (uint32_t)kChunkBytes + (p & (uint32_t)(kChunkBytes - 1));
}

// error bits written to the device error word
enum : int { kErrPipeline = 1, kErrGridBarrier = 2, kErrProducer = 4 };

struct SharedLayout {
  static constexpr uint32_t ring = 0;
  static constexpr uint32_t full = kRingBytes;                               // [kRingChunks] chunk landed
  static constexpr uint32_t empty = full + 8 * kRingChunks;                  // [kRingChunks] chunk consumed
  static constexpr uint32_t red = empty + 8 * kRingChunks;                   // [kRedSlots][NW][64] double
  static constexpr uint32_t stage = red + kRedSlots * kConsumerWarps * 64 * 8;  // [kStages][kStageBytes]
  static constexpr uint32_t lite = stage + kStages * kStageBytes;            // [kMaxCtaRuns] RunLite
  static constexpr uint32_t rec = lite + kMaxCtaRuns * 16;                   // [kGatherWarps][kRecSlots] records
  static constexpr uint32_t scal = rec + kGatherWarps * kRecSlots * kRecBytes;  // 64 doubles of scratch
  static constexpr uint32_t sfull = scal + 64 * 8;                           // [kStages] stage filled
  static constexpr uint32_t sempty = sfull + 8 * kStages;                    // [kStages] stage consumed
  static constexpr uint32_t rfull = sempty + 8 * kStages;                    // [kGatherWarps][kRecSlots]
  static constexpr uint32_t xready = rfull + 8 * kGatherWarps * kRecSlots;   // a pass's x is complete grid-wide
  static constexpr uint32_t pdone = xready + 8;                              // the CTA's P blocks are summed
  static constexpr uint32_t gdone = pdone + 8;                               // every CTA's zbu is complete
  static constexpr uint32_t redfull = gdone + 8;                             // [kRedSlots] a block's partials parked
  static constexpr uint32_t rdone = redfull + 8 * kRedSlots;                 // a pass's block sums are written
  // [0] block ends summed so far; [1] the launch's first grid-barrier
  // generation; [2] passes whose x is ready; [3] passes whose zbu is
  // complete grid-wide (the gather warps wait on these two counters, not on
  // xready / gdone: a gather warp can reach its first wait of a kind after
  // both of the launch's phases completed, where a parity wait would take
  // the finished second phase for the one it wants and never return)
  static constexpr uint32_t rsum = rdone + 8;
  static constexpr uint32_t bytes = rsum + 16 + 16;
};
static_assert(SharedLayout::red % 16 == 0 && SharedLayout::stage % 16 == 0 && SharedLayout::lite % 16 == 0 &&
                  SharedLayout::rec % 16 == 0 && SharedLayout::sfull % 8 == 0,
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
// lane acquires the copied bytes) and the outcome is agreed on.
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

// The same with an L2 cache-eviction hint (a createpolicy value).
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

// L2 policies of the streamed factors: the part of a CTA's stream that is
// kept in L2 from one pass to the next (evict_last), and the rest, which
// passes through L2 without displacing it or the vectors (evict_first).
__device__ __forceinline__ uint64_t l2_policy_keep() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_stream() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
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

// CTA-scope acquire load / release store of a shared-memory word.
__device__ __forceinline__ unsigned ld_acquire_s(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.cta.shared.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_s(unsigned *p, unsigned v) {
  asm volatile("st.release.cta.shared.u32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}

// Bounded wait until a CTA counter in shared memory reaches `need`; every
// lane acquires it.  Warp-uniform outcome.
__device__ __forceinline__ bool count_wait(const unsigned *cnt, unsigned need, uint64_t timeout_ns) {
  bool ok = true;
  if (ld_acquire_s(cnt) < need) {
    const uint64_t t0 = gtimer();
    while (ld_acquire_s(cnt) < need) {
      __nanosleep(64);
      if (gtimer() - t0 > timeout_ns) {
        ok = false;
        break;
      }
    }
  }
  return __all_sync(0xffffffffu, ok);
}

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

// ---- grid barrier -----------------------------------------------------------
// gbar[0] counts arrivals and gbar[1] completed barrier instances, both since
// the words were last cleared and modulo 2^32.  A launch reads gbar[1] once
// at its start (grid_gen0; no instance of the launch can complete before
// every CTA has started), numbers its instances k = 0, 1, ... in the same
// order in every CTA, and instance k is complete once gbar[0] has reached
// nblocks * (gen0 + k + 1).  The last arriver also advances gbar[1] for the
// next launch; nobody waits for that.  A CTA arrives on instance k + 1 only
// after it has seen instance k complete.
__device__ __forceinline__ unsigned grid_gen0(const unsigned *gbar) { return ld_acquire(&gbar[1]); }
__device__ __forceinline__ unsigned grid_target(unsigned gen0, unsigned k, unsigned nblocks) {
  return nblocks * (gen0 + k + 1u);
}
//
// Memory order: the arrival is a release at GPU scope and the polls are
// acquires, with no separate fences.  Release and acquire are cumulative over
// causality order, and the CTA's other threads reach the arriving thread (and
// leave the waiting one) through bar.sync or an mbarrier, so the writes of
// every thread of every CTA before the barrier happen before the reads of
// every thread after it.  (Full fences on both sides and a sleep in the poll
// cost 1.5 us per BiCGSTAB step of C1.)
__device__ __forceinline__ void grid_arrive(unsigned *gbar, unsigned target) {
  unsigned old;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(&gbar[0]) : "memory");
  if (old + 1u == target) atomicAdd(&gbar[1], 1u);
}

__device__ __forceinline__ bool grid_wait(const unsigned *gbar, unsigned target, uint64_t timeout_ns) {
  if ((int)(ld_acquire(&gbar[0]) - target) < 0) {
    const uint64_t t0 = gtimer();
    while ((int)(ld_acquire(&gbar[0]) - target) < 0)
      if (gtimer() - t0 > timeout_ns) return false;
  }
  return true;
}

// ---- producer: streams `npass` passes over the CTA's byte range ------------
// Chunk g of the launch (g = pass * K + k) covers stream bytes k * kChunkBytes
// on, in ring slot g % kRingChunks.  `keep` > 0: the chunks that start below
// byte `keep` of the CTA's stream are read with the evict_last policy (they
// stay in L2 for the next pass), the others with evict_first; keep == 0
// issues plain copies.
// With `cinst` set (a block-diagonal engine inside a batched solve), a
// chunk none of whose instances is active is not copied: its full barrier
// completes on the producer's arrival alone and the consumers read whatever
// the slot holds (the rows of inactive instances are left undefined).
struct StreamSrc {
  const uint8_t *src;
  uint32_t bytes, keep;
  const uint32_t *cinst;  // [K] instance range of each chunk (lo | hi << 16), or null
  const int *pre;         // prefix counts of active instances
};
__device__ __forceinline__ void producer_issue(const StreamSrc &ss, uint32_t K, uint32_t g, uint8_t *ring,
                                               uint64_t *full) {
  const uint32_t s = g % kRingChunks;
  if (ss.cinst) {
    const uint32_t e = ss.cinst[g % K], lo = e & 0xffffu, hi = e >> 16;
    if (lo > hi || ss.pre[hi + 1] == ss.pre[lo]) {
      mbar_arrive(&full[s]);
      return;
    }
  }
  const uint32_t off = (g % K) << kChunkLog;
  const uint32_t nb = min((uint32_t)kChunkBytes, ss.bytes - off);
  mbar_arrive_expect_tx(&full[s], nb);
  if (ss.keep == 0) bulk_g2s(ring + ((size_t)s << kChunkLog), ss.src + off, nb, &full[s]);
  else
    bulk_g2s_hint(ring + ((size_t)s << kChunkLog), ss.src + off, nb, &full[s],
                  off < ss.keep ? l2_policy_keep() : l2_policy_stream());
}

// The producer thread's part of the CTA set-up, before the CTA's first
// barrier: it sets up the ring's barriers and issues the first chunks (one
// per ring slot, which needs no empty wait), so the stream is under way while
// the other threads load the run summaries and reduce scalars.  Returns the
// number of chunks issued; producer_run goes on from there.
__device__ __forceinline__ uint32_t producer_start(const StreamSrc &ss, uint32_t npass, uint8_t *ring,
                                                  uint64_t *full, uint64_t *empty) {
  for (int i = 0; i < kRingChunks; ++i) {
    mbar_init(&full[i], 1);
    mbar_init(&empty[i], kConsumerWarps);
  }
  mbar_fence_init();
  const uint32_t K = (ss.bytes + kChunkBytes - 1) >> kChunkLog;
  const uint32_t n = min(K * npass, (uint32_t)kRingChunks);
  for (uint32_t g = 0; g < n; ++g) producer_issue(ss, K, g, ring, full);
  return n;
}

// Bounded wait for chunks [g0, issued) -- copies still in flight must land
// before the CTA exits.
__device__ __forceinline__ void producer_drain(uint64_t *full, uint32_t issued, uint64_t timeout_ns) {
  const uint32_t g0 = issued > (uint32_t)kRingChunks ? issued - kRingChunks : 0;
  for (uint32_t g = g0; g < issued; ++g) mbar_wait(&full[g % kRingChunks], (g / kRingChunks) & 1, timeout_ns);
}

// The rest of the stream: chunk g once the consumers emptied chunk
// g - kRingChunks.
__device__ __forceinline__ void producer_run(const StreamSrc &ss, uint32_t npass, uint32_t issued0, uint8_t *ring,
                                             uint64_t *full, uint64_t *empty, int *err, uint64_t timeout_ns) {
  const uint32_t K = (ss.bytes + kChunkBytes - 1) >> kChunkLog;
  const uint32_t total = K * npass;
  uint32_t issued = issued0;
  for (uint32_t g = issued0; g < total; ++g) {
    const uint32_t s = g % kRingChunks;
    if (g >= (uint32_t)kRingChunks) {
      if (!mbar_wait(&empty[s], ((g / kRingChunks) - 1) & 1, timeout_ns)) {
        atomicOr(err, kErrProducer);
        break;
      }
    }
    producer_issue(ss, K, g, ring, full);
    issued = g + 1;
  }
  producer_drain(full, issued, timeout_ns);
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

// ---- gather warps ----------------------------------------------------------
// Staging copies with cp.async: doubles for FP64 engines, the float copies of
// the vectors for FP32 engines.
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

struct GatherCtx {
  const RunRec *recs;   // the CTA's records
  uint32_t nr, nr_pd;   // runs of a pass; P + D runs (index of the first U run)
  uint32_t npass;
  const void *x0, *x1;  // the gathered vector of pass 0 and pass 1 (float copies for FP32 engines)
  const void *z0, *z1;  // zbu of pass 0 and pass 1 (float copies for FP32 engines)
  int *err;
  uint64_t timeout_ns;
};

// Gather warp gi stages runs g = gi, gi + kGatherWarps, ... (g counted over
// the passes) into stage slot g % kStages: it waits until the consumers have
// given the slot back, copies each long segment with the whole warp and each
// short one with one lane, clears the zero columns of the last panel, and
// completes the slot's sfull barrier (32 cp.async arrivals + one plain
// arrival).  Before its first run of a pass it waits for that pass's x
// (the x-ready count), and before its first U run of a pass for the grid
// barrier that completes zbu (the zbu-ready count).  Run records arrive
// kRecSlots runs ahead by cp.async.
template <int kPrec, class SM>
__device__ __forceinline__ void gather_warp(const GatherCtx &c, const SM &sm, uint32_t gi) {
  constexpr bool kF32 = kPrec != kFP64;  // float copies of the vectors (FP32 and BF16 storage)
  const int lane = threadIdx.x & 31;
  const uint32_t total = c.nr * c.npass;
  uint8_t *recs = sm.rec + gi * kRecSlots * kRecBytes;
  uint64_t *rfull = sm.rfull + gi * kRecSlots;
  // the i-th run of this warp is g = gi + i * kGatherWarps
  auto fetch = [&](uint32_t i) {
    const uint32_t g = gi + i * kGatherWarps;
    const uint8_t *src = reinterpret_cast<const uint8_t *>(c.recs + (g % c.nr));
#pragma unroll
    for (uint32_t o = 0; o < (uint32_t)kRecBytes; o += 512)
      cp_async16cg(recs + (i % kRecSlots) * kRecBytes + o + lane * 16, src + o + lane * 16);
    cp_async_arrive(&rfull[i % kRecSlots]);
  };
  const uint32_t nmine = total > gi ? (total - gi + kGatherWarps - 1) / kGatherWarps : 0;
  for (uint32_t i = 0; i < nmine && i < kRecSlots; ++i) fetch(i);
  int xpass = -1, upass = -1;  // passes whose x / zbu readiness this warp has observed
  bool ok = true;
  for (uint32_t i = 0; i < nmine && ok; ++i) {
    const uint32_t g = gi + i * kGatherWarps, k = g % c.nr, pass = g / c.nr;
    ok = warp_wait(&rfull[i % kRecSlots], (i / kRecSlots) & 1, c.timeout_ns);
    if (ok && xpass < (int)pass) {
      ok = count_wait(&sm.rsum[2], pass + 1, c.timeout_ns);
      xpass = (int)pass;
    }
    const bool is_u = k >= c.nr_pd;
    if (ok && is_u && upass < (int)pass) {
      ok = count_wait(&sm.rsum[3], pass + 1, c.timeout_ns);
      upass = (int)pass;
      __threadfence();
    }
    const uint32_t slot = g % kStages;
    if (ok && g >= (uint32_t)kStages) ok = warp_wait(&sm.sempty[slot], ((g / kStages) - 1) & 1, c.timeout_ns);
    if (!ok) break;
    const uint8_t *rec = recs + (i % kRecSlots) * kRecBytes;
    const Run h = *reinterpret_cast<const Run *>(rec);
    const Seg *seg = reinterpret_cast<const Seg *>(rec + sizeof(Run));
    const uint8_t *xv = static_cast<const uint8_t *>((pass & 1) ? c.x1 : c.x0);
    const uint8_t *zv = static_cast<const uint8_t *>((pass & 1) ? c.z1 : c.z0);
    constexpr uint32_t esz = kF32 ? 4u : 8u;
    uint8_t *st = sm.stage + slot * kStageBytes;
    // a segment's source: zbu for U runs, x for P and D runs, and for the
    // merged D+U runs of an atom zbu when kSegZbu is set in its src
    const bool du = (h.flags & 0xffu) == kRunDU;
    auto src_of = [&](const Seg &sg) -> const uint8_t * {
      if (du) return (sg.src & kSegZbu) ? zv + (size_t)(sg.src & ~kSegZbu) * esz : xv + (size_t)sg.src * esz;
      return (is_u ? zv : xv) + (size_t)sg.src * esz;
    };
    for (uint32_t q = 0; q < h.nlong; ++q) {
      const Seg sg = seg[q];
      stage_elems<kF32>(st, sg.dst, src_of(sg), (uint32_t)lane, sg.len, 32);
    }
    for (uint32_t q = h.nlong + lane; q < h.nseg; q += 32) {
      const Seg sg = seg[q];
      stage_elems<kF32>(st, sg.dst, src_of(sg), 0, sg.len, 1);
    }
    const uint32_t vend = (uint32_t)h.npanel * group_cols(kPrec);
    for (uint32_t e = h.vlen + lane; e < vend; e += 32) {
      if (kF32) reinterpret_cast<float *>(st)[e] = 0.0f;
      else reinterpret_cast<double *>(st)[e] = 0.0;
    }
    cp_async_arrive(&sm.sfull[slot]);
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.sfull[slot]);  // releases the plain stores
    __syncwarp();  // every lane has read the record before its slot is refilled
    if (i + kRecSlots < nmine) fetch(i + kRecSlots);
  }
  if (!ok && lane == 0) atomicOr(c.err, kErrProducer);
  cp_async_wait_all();  // copies in flight land before the warp exits
}

// ---- panel arithmetic --------------------------------------------------------
__device__ __forceinline__ float4 lds_f32x4(uint32_t addr) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
  return v;
}

// A lane's accumulator for a row: FP64 panels (two double columns) add into
// two doubles; FP32 panels (four float columns) and BF16 panels (eight
// bfloat16 columns) into four floats, folded into the double total at the end
// of every run.  V is a panel's slice of the staged vector (ldv: panel j),
// M one 16-byte panel row (ldm).
template <int kPrec>
struct PanelMath;
template <>
struct PanelMath<kFP64> {
  using V = double2;
  using M = double2;
  struct Acc {
    double a0 = 0.0, a1 = 0.0;
    __device__ __forceinline__ double take() {
      const double s = a0 + a1;
      a0 = 0.0;
      a1 = 0.0;
      return s;
    }
  };
  static __device__ __forceinline__ V ldv(uint32_t stage_s, uint32_t j) { return lds_f64x2(stage_s + 16u * j); }
  static __device__ __forceinline__ M ldm(uint32_t addr) { return lds_f64x2(addr); }
  static __device__ __forceinline__ void fma(Acc &a, const M &m, const V &v) {
    a.a0 = ::fma(m.x, v.x, a.a0);
    a.a1 = ::fma(m.y, v.y, a.a1);
  }
};
template <>
struct PanelMath<kFP32> {
  using V = float4;
  using M = float4;
  struct Acc {
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    __device__ __forceinline__ double take() {
      const double s = ((double)a0 + (double)a1) + ((double)a2 + (double)a3);
      a0 = a1 = a2 = a3 = 0.f;
      return s;
    }
  };
  static __device__ __forceinline__ V ldv(uint32_t stage_s, uint32_t j) { return lds_f32x4(stage_s + 16u * j); }
  static __device__ __forceinline__ M ldm(uint32_t addr) { return lds_f32x4(addr); }
  static __device__ __forceinline__ void fma(Acc &a, const M &m, const V &v) {
    a.a0 = fmaf(m.x, v.x, a.a0);
    a.a1 = fmaf(m.y, v.y, a.a1);
    a.a2 = fmaf(m.z, v.z, a.a2);
    a.a3 = fmaf(m.w, v.w, a.a3);
  }
};
// A 32-bit word of a BF16 panel row holds columns 2k (low half) and 2k + 1
// (high half); a bfloat16 is the high half of a float, so widening is a
// shift or a mask.  Panel j's eight staged floats lie at 32 j bytes.
template <>
struct PanelMath<kBF16> {
  struct V {
    float4 lo, hi;
  };
  using M = uint4;
  using Acc = PanelMath<kFP32>::Acc;
  static __device__ __forceinline__ V ldv(uint32_t stage_s, uint32_t j) {
    return V{lds_f32x4(stage_s + 32u * j), lds_f32x4(stage_s + 32u * j + 16u)};
  }
  static __device__ __forceinline__ M ldm(uint32_t addr) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(addr));
    return v;
  }
  static __device__ __forceinline__ float lo(uint32_t w) { return __uint_as_float(w << 16); }
  static __device__ __forceinline__ float hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }
  static __device__ __forceinline__ void fma(Acc &a, const M &m, const V &v) {
    a.a0 = fmaf(lo(m.x), v.lo.x, a.a0);
    a.a1 = fmaf(hi(m.x), v.lo.y, a.a1);
    a.a2 = fmaf(lo(m.y), v.lo.z, a.a2);
    a.a3 = fmaf(hi(m.y), v.lo.w, a.a3);
    a.a0 = fmaf(lo(m.z), v.hi.x, a.a0);
    a.a1 = fmaf(hi(m.z), v.hi.y, a.a1);
    a.a2 = fmaf(lo(m.w), v.hi.z, a.a2);
    a.a3 = fmaf(hi(m.w), v.hi.w, a.a3);
  }
};

// ---- one run of a consumer warp ------------------------------------------
// The warp reads panels j = (w - rot) mod NW, j + NW, ... of the run (16h
// bytes each; lane i reads row min(i, h-1), and row min(i + 32, h-1) of P
// slabs taller than 32, 16 bytes each: two double, four float or eight
// bfloat16 columns) from the ring, kUnroll panels per iteration (BF16:
// kUnroll / 2; two-row form: 2), and adds their products with the staged
// vector into its accumulators; it adds the run's sums of its rows to t0
// (row i) and t1 (row i + 32).  Lanes past the last row repeat it; their
// sums are never used.
#ifndef HBX_UNROLL
#define HBX_UNROLL 4
#endif
constexpr uint32_t kUnroll = HBX_UNROLL;

template <bool kTwoRows, int kPrec, int kGroupWarps>
__device__ __forceinline__ void run_rows(const RunLite &L, uint32_t stage_s, Ring &R, uint32_t w, double &t0,
                                         double &t1) {
  using PM = PanelMath<kPrec>;
  using V = typename PM::V;
  using M = typename PM::M;
  // panels per iteration: BF16 panels are twice as wide as FP32 ones, so
  // half as many give the same columns per iteration
#ifndef HBX_UNROLL_BF16
#define HBX_UNROLL_BF16 (HBX_UNROLL / 2)
#endif
#ifndef HBX_UNROLL_F32
#define HBX_UNROLL_F32 HBX_UNROLL
#endif
  // NW: the warps that share this run (a consumer group); w: the warp's index in it
  constexpr uint32_t NW = kGroupWarps,
                     U = kTwoRows ? 2 : (kPrec == kBF16 ? HBX_UNROLL_BF16 : kPrec == kFP32 ? HBX_UNROLL_F32 : kUnroll);
  const int lane = threadIdx.x & 31;
  const uint32_t h = L.nrow, np = L.npanel;
  const uint32_t pb = 16u * h;
  const uint32_t lrow = 16u * min((uint32_t)lane, h - 1u);
  const uint32_t lrow2 = 16u * min((uint32_t)lane + 32u, h - 1u) - lrow;  // second row, relative
  const uint32_t ring_s = smem_u32(R.buf);
  // the planned rotation for this warp count (another count: any rotation
  // covers every panel once)
  const uint32_t rot = NW == (uint32_t)kStepWarps ? (uint32_t)L.rot_step
                       : NW == (uint32_t)kProductWarps ? (uint32_t)L.rot : (uint32_t)L.rot % NW;
  uint32_t j = (w + NW - rot) % NW;
  typename PM::Acc a[U], b[kTwoRows ? U : 1];
  for (; j + (U - 1) * NW < np; j += U * NW) {
    const uint32_t p0 = L.pos + j * pb;
    R.ensure(p0, p0 + (U - 1) * NW * pb + pb);
    V v[U];
    M m[U], m2[kTwoRows ? U : 1];
#pragma unroll
    for (uint32_t u = 0; u < U; ++u) v[u] = PM::ldv(stage_s, j + u * NW);
    const uint32_t pl = p0 + lrow;
    const uint32_t q = ring_off(R.base + (pl >> kChunkLog), pl);
    if (q + (U - 1) * NW * pb + (kTwoRows ? lrow2 : 0u) + 16u <= kRingBytes) {  // no wrap around the ring end
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        m[u] = PM::ldm(ring_s + q + u * NW * pb);
        if (kTwoRows) m2[u] = PM::ldm(ring_s + q + u * NW * pb + lrow2);
      }
    } else {
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        const uint32_t pu = pl + u * NW * pb;
        m[u] = PM::ldm(ring_s + ring_off(R.base + (pu >> kChunkLog), pu));
        if (kTwoRows) m2[u] = PM::ldm(ring_s + ring_off(R.base + ((pu + lrow2) >> kChunkLog), pu + lrow2));
      }
    }
#pragma unroll
    for (uint32_t u = 0; u < U; ++u) {
      PM::fma(a[u], m[u], v[u]);
      if (kTwoRows) PM::fma(b[u], m2[u], v[u]);
    }
  }
  for (; j < np; j += NW) {
    const uint32_t p0 = L.pos + j * pb;
    R.ensure(p0, p0 + pb);
    const V vv = PM::ldv(stage_s, j);
    const uint32_t pl = p0 + lrow;
    PM::fma(a[0], PM::ldm(ring_s + ring_off(R.base + (pl >> kChunkLog), pl)), vv);
    if (kTwoRows) {
      const uint32_t p2 = pl + lrow2;
      PM::fma(b[0], PM::ldm(ring_s + ring_off(R.base + (p2 >> kChunkLog), p2)), vv);
    }
  }
#pragma unroll
  for (uint32_t u = 0; u < U; ++u) t0 += a[u].take();
  if (kTwoRows) {
#pragma unroll
    for (uint32_t u = 0; u < U; ++u) t1 += b[u].take();
  }
}

template <int kPrec, int kGroupWarps>
__device__ __forceinline__ void run_panels(const RunLite &L, uint32_t stage_s, Ring &R, uint32_t w, double &t0,
                                           double &t1) {
  if (L.nrow > 32) run_rows<true, kPrec, kGroupWarps>(L, stage_s, R, w, t0, t1);
  else run_rows<false, kPrec, kGroupWarps>(L, stage_s, R, w, t0, t1);
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
