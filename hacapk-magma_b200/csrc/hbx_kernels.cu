// hbx_kernels.cu -- persistent sm_100a kernels of the H-matvec / BiCGSTAB path.
//
// k_matvec      one H-matvec: y = alpha*H*x + beta*yin (HACApK_BATCH.c:47-255
//               replaced: one launch instead of ceil(n/5000) vbatched GEMVs per
//               phase, no atomics, no zeroing of zbu/zau).
// k_bicg_setup  r = b - H u has been formed by k_matvec; sets rh = r, p = Ap = 0
//               and the first reduction partials (HACApK_SOLVER.c:533-594).
// k_bicg_iter   one BiCGSTAB step of HACApK_SOLVER.c:602-732 in one launch:
//               both H-matvecs, the vector updates and all dot products, with
//               compensated (Dot2) partial sums reduced in a fixed order.
//
// The file is compiled three times: as itself (k_matvec and the small vector
// kernels, 16 consumer warps), with HBX_STEP_TU and HBX_CONSUMER_WARPS=13
// (k_bicg_setup, the FP64 k_bicg_iter and the dot kernels): with fewer
// threads per CTA the step kernel gets the registers it needs without
// spilling, and its scalar phases synchronise fewer warps (C1 step 121.4 ->
// 115 us, while the standalone product is fastest with 16); and with
// HBX_STEP_TU, HBX_STEP_LP and HBX_CONSUMER_WARPS=kStepWarpsLp (the FP32 and
// BF16 k_bicg_iter, whose consumer warps form two groups like the FP32 and
// BF16 products').
//
// All kernels run one CTA per SM: consumer warps, a bulk-copy producer
// warp, kGatherWarps gather warps, a grid-barrier warp and a block-sum warp.
// The producer streams the CTA's packed runs through a shared-memory ring
// with cp.async.bulk; the consumers take every 16th panel of every run
// (rotated so the work stays balanced), multiply it by the run's staged
// vector and accumulate in registers; at a block end they park their partial
// sums and go on, and the block-sum warp adds them in a fixed order and
// writes the rows.  Grid-wide dependencies (zbu complete, dot products
// complete) use a bounded grid barrier; the launch is cooperative so every
// CTA is resident.
#include "hbx_device.cuh"
#include "hbx_engine.h"

namespace hbx {
namespace {

constexpr int NW = kConsumerWarps;
[[maybe_unused]] constexpr int kConsumerThreads = NW * 32;
// Consumer groups: the FP32 and BF16 product kernels split their warps into
// kProductGroups groups taking alternate runs; the FP64 product (whose
// summation order the drop-in's iteration counts follow, and which a CPU
// replay reproduces bit for bit) and the step kernels keep one group.
template <int kPrec>
constexpr int groups_of() {
  return ((NW == kProductWarps || NW == kStepWarpsLp) && kPrec != kFP64) ? kProductGroups : 1;
}
static_assert(kStages % kProductGroups == 0, "a stage slot always serves the same consumer group");
#ifdef HBX_STEP_LP
static_assert(NW == kStepWarpsLp, "the FP32 / BF16 step unit is built with kStepWarpsLp consumer warps");
#elif defined(HBX_STEP_TU)
static_assert(NW == kStepWarps, "the FP64 step unit is built with kStepWarps consumer warps");
#else
static_assert(NW == kProductWarps, "the product unit is built with kProductWarps consumer warps");
#endif

struct Smem {
  uint8_t *ring;
  uint64_t *full, *empty;
  double *red;     // [kRedSlots][NW][64] partial sums of a block end
  uint8_t *stage;  // [kStages][kStageBytes]
  RunLite *lite;   // the CTA's run summaries
  uint8_t *rec;    // [kGatherWarps][kRecSlots] run records
  double *scal;    // 64 doubles
  uint64_t *sfull, *sempty, *rfull;
  uint64_t *xready, *pdone, *gdone, *redfull, *rdone;
  unsigned *rsum;
};

__device__ __forceinline__ Smem smem_layout(uint8_t *base) {
  Smem s;
  s.ring = base + SharedLayout::ring;
  s.full = reinterpret_cast<uint64_t *>(base + SharedLayout::full);
  s.empty = reinterpret_cast<uint64_t *>(base + SharedLayout::empty);
  s.red = reinterpret_cast<double *>(base + SharedLayout::red);
  s.stage = base + SharedLayout::stage;
  s.lite = reinterpret_cast<RunLite *>(base + SharedLayout::lite);
  s.rec = base + SharedLayout::rec;
  s.scal = reinterpret_cast<double *>(base + SharedLayout::scal);
  s.sfull = reinterpret_cast<uint64_t *>(base + SharedLayout::sfull);
  s.sempty = reinterpret_cast<uint64_t *>(base + SharedLayout::sempty);
  s.rfull = reinterpret_cast<uint64_t *>(base + SharedLayout::rfull);
  s.xready = reinterpret_cast<uint64_t *>(base + SharedLayout::xready);
  s.pdone = reinterpret_cast<uint64_t *>(base + SharedLayout::pdone);
  s.gdone = reinterpret_cast<uint64_t *>(base + SharedLayout::gdone);
  s.redfull = reinterpret_cast<uint64_t *>(base + SharedLayout::redfull);
  s.rdone = reinterpret_cast<uint64_t *>(base + SharedLayout::rdone);
  s.rsum = reinterpret_cast<unsigned *>(base + SharedLayout::rsum);
  return s;
}

// Barriers (but the ring's: producer_start), the block-sum counter, the
// launch's first grid-barrier generation and the CTA's run summaries (`lite`,
// nr of them) in shared memory.  Thread t0 sets up the barriers; threads t0
// and up copy the summaries.  The caller synchronises the CTA afterwards.
__device__ __forceinline__ void init_cta_part(const Smem &s, const RunLite *lite, uint32_t nr, const unsigned *gbar,
                                              uint32_t t0, uint32_t group_warps) {
  if (threadIdx.x == t0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&s.sfull[i], 33);  // 32 cp.async arrivals of a gather warp + its lane 0
      mbar_init(&s.sempty[i], group_warps);  // the slot's runs belong to one consumer group
    }
    for (int i = 0; i < kGatherWarps * (int)kRecSlots; ++i) mbar_init(&s.rfull[i], 32);
    mbar_init(s.xready, 1);
    mbar_init(s.pdone, 1);
    mbar_init(s.gdone, 1);
    for (uint32_t i = 0; i < kRedSlots; ++i) mbar_init(&s.redfull[i], NW);
    mbar_init(s.rdone, 1);
    s.rsum[0] = 0;
    s.rsum[1] = grid_gen0(gbar);
    s.rsum[2] = 0;
    s.rsum[3] = 0;
    mbar_fence_init();
  }
  if (threadIdx.x < t0 || s.lite == lite) return;  // summaries read where they lie (see cta_smem)
  const uint4 *src = reinterpret_cast<const uint4 *>(lite);
  uint4 *dst = reinterpret_cast<uint4 *>(s.lite);
  for (uint32_t k = threadIdx.x - t0; k < nr; k += blockDim.x - t0) dst[k] = __ldg(src + k);
}

// The CTA's shared-memory layout; a CTA with more runs than the summary
// array holds reads its run summaries from global memory instead.
__device__ __forceinline__ Smem cta_smem(uint8_t *base, const RunLite *lite, uint32_t nr) {
  Smem s = smem_layout(base);
  if (nr > (uint32_t)kMaxCtaRuns) s.lite = const_cast<RunLite *>(lite);
  return s;
}

#ifndef HBX_STEP_TU
__device__ __forceinline__ void init_cta(const Smem &s, const RunLite *lite, uint32_t nr, const unsigned *gbar,
                                         uint32_t group_warps) {
  init_cta_part(s, lite, nr, gbar, 0, group_warps);
  __syncthreads();
}
#endif

// ---- grid-barrier warp: once per pass, after the CTA's P blocks are summed
// (pdone), arrive on the grid barrier, wait for it and release the U runs
// (gdone).  The barrier latency stays off the consumer and gather warps.
// Pass p uses grid-barrier instance k0 + p * kstep of the launch.
// `beyond` > 0 (a test hook) waits for an instance that no launch of this
// grid completes, so the bounded waits of the whole CTA expire.
__device__ __forceinline__ void sync_warp(unsigned *gbar, uint32_t npass, uint32_t k0, uint32_t kstep, const Smem &sm,
                                          int *err, uint64_t tmo, uint32_t beyond = 0) {
  for (uint32_t p = 0; p < npass; ++p) {
    if (!mbar_wait(sm.pdone, p & 1, tmo)) {
      atomicOr(err, kErrPipeline);
      return;  // the waits on gdone are bounded too
    }
    const unsigned target = grid_target(sm.rsum[1], k0 + p * kstep + beyond, gridDim.x);
    grid_arrive(gbar, target);  // a release: the CTA's zbu stores (before pdone) are visible grid-wide
    if (!grid_wait(gbar, target, tmo)) {
      atomicOr(err, kErrGridBarrier);
      return;
    }
    st_release_s(&sm.rsum[3], p + 1);  // the gather warps' U runs of pass p may start
    mbar_arrive(sm.gdone);
  }
}

// x of the launch's pass `pass` is ready: the gather warps' count, then the
// block-sum warp's barrier.  One thread.
__device__ __forceinline__ void signal_xready(const Smem &sm, unsigned pass) {
  st_release_s(&sm.rsum[2], pass + 1);
  mbar_arrive(sm.xready);
}

// Where the block sums of one H-matvec pass go.
struct PassOut {
  double alpha, beta;
  const double *yin;
  double *y, *zbu;
  float *zbu32;     // FP32 engines: zbu rounded to float (what the U runs gather)
  uint32_t pass;    // pass index within the launch (barrier parities)
  uint32_t nblk_p;  // P blocks of the CTA
};

// End of a block for a consumer warp: park its row sums (rows lane and
// lane + 32) in red slot nb mod kRedSlots, once the block-sum warp has
// emptied it, and arrive on the slot's barrier.  Returns false after a
// timed-out wait.
__device__ __forceinline__ bool block_end(double t0, double t1, uint32_t &nb, const Smem &sm, int *err,
                                          uint64_t tmo) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t slot = nb % kRedSlots;
  int ok = 1;
  if (nb >= kRedSlots && lane == 0 && ld_acquire_s(sm.rsum) + kRedSlots <= nb) {
    const uint64_t ts = gtimer();
    while (ld_acquire_s(sm.rsum) + kRedSlots <= nb) {
      if (gtimer() - ts > tmo) {
        ok = 0;
        atomicOr(err, kErrPipeline);
        break;
      }
    }
  }
  ++nb;
  if (!__shfl_sync(0xffffffffu, ok, 0)) return false;
  double *rb = sm.red + slot * (NW * 64) + w * 64;
  rb[lane] = t0;
  rb[32 + lane] = t1;
  __syncwarp();
  if (lane == 0) mbar_arrive(&sm.redfull[slot]);
  return true;
}

// ---- block-sum warp: for every block end of every pass, in order, wait
// until all consumer warps parked their partial sums, add them in warp order
// and write the rows -- P: zbu = s;  D: y = alpha*s + beta*yin;  U: y +=
// alpha*s (the atom's D block was summed before, in this same order) --
// then free the slot.  After the pass's last P block it signals pdone (the
// CTA's zbu rows are complete), after the pass's last block rdone.
__device__ __forceinline__ void sum_warp(uint32_t nr, uint32_t npass, uint32_t nblk_p, const PassOut *outs,
                                         const Smem &sm, int *err, uint64_t tmo) {
  const int lane = threadIdx.x & 31;
  uint32_t nb = 0;
  for (uint32_t pass = 0; pass < npass; ++pass) {
    const PassOut &o = outs[pass];
    // Not before the pass has started: rdone must not run a phase ahead of
    // the consumers' wait on it (a CTA without blocks would otherwise
    // complete both passes' phases at once).
    if (!warp_wait(sm.xready, pass & 1, tmo)) {
      if (lane == 0) atomicOr(err, kErrPipeline);
      return;
    }
    uint32_t np_done = 0;
    for (uint32_t r = 0; r < nr; ++r) {
      const RunLite L = sm.lite[r];
      if (!(L.flags & kLast)) continue;
      const uint32_t slot = nb % kRedSlots;
      if (!warp_wait(&sm.redfull[slot], (nb / kRedSlots) & 1, tmo)) {
        if (lane == 0) atomicOr(err, kErrPipeline);
        return;  // the consumers' bounded waits end the launch
      }
      const uint32_t kind = L.flags & 0xffu;
      const double *rb = sm.red + slot * (NW * 64);
      for (uint32_t i = lane; i < L.nrow; i += 32) {
        double s = rb[i];
#pragma unroll
        for (int k = 1; k < NW; ++k) s += rb[k * 64 + i];
        const uint32_t row = L.out + i;
        if (kind == kRunP) {
          o.zbu[row] = s;
          if (o.zbu32) o.zbu32[row] = (float)s;
        } else if (kind == kRunD || kind == kRunDU) {  // an atom's first (a merged one: only) block
          double v = o.alpha * s;
          if (o.beta != 0.0) v = fma(o.beta, o.yin[row], v);
          o.y[row] = v;
        } else {
          o.y[row] = fma(o.alpha, s, o.y[row]);
        }
      }
      ++nb;
      __syncwarp();
      if (lane == 0) {
        __threadfence_block();
        st_release_s(sm.rsum, nb);  // the slot may be refilled
        if (kind == kRunP && ++np_done == nblk_p) mbar_arrive(sm.pdone);  // the CTA's zbu rows are complete
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(sm.rdone);
  }
}

// One H-matvec pass of a consumer warp over the CTA's runs (the pass starts
// at absolute ring chunk R.base and is K chunks long).  For every run the
// warp waits for its staged vector, multiplies its panels (every 16th,
// rotated), gives the stage slot back and, at a block end, parks its row
// sums for the block-sum warp.  Before it can block, a warp gives back every
// ring chunk below the run it is about to process, so no wait holds a chunk
// another warp needs.  nb counts the block ends over the launch.
template <int kPrec>
__device__ __forceinline__ void consume_pass(Ring &R, uint32_t K, uint32_t nr, uint32_t &nb, uint32_t pass,
                                             const Smem &sm, int *err, uint64_t tmo) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool bad = R.bad;
  double t0 = 0.0, t1 = 0.0;  // this lane's block sums: rows lane and lane + 32
  constexpr int kGroups = groups_of<kPrec>(), kGroupWarps = NW / kGroups;
  const uint32_t grp = kGroups == 1 ? 0u : (uint32_t)w / kGroupWarps;
  const uint32_t wl = kGroups == 1 ? (uint32_t)w : (uint32_t)w % kGroupWarps;
  for (uint32_t r = 0; r < nr; ++r) {
    const RunLite L = sm.lite[r];
    const uint32_t g = pass * nr + r, slot = g % kStages;
    R.release_below(R.base + (L.pos >> kChunkLog));
    if (kGroups == 1 || g % kGroups == grp) {  // a run of this warp's group (the other group's: parking only)
      // Every warp of the group observes every phase of the slot's barrier,
      // panels or not: a warp that skipped phases could take an older
      // completed phase for the one it waits on.
      if (!bad && !warp_wait(&sm.sfull[slot], (g / kStages) & 1, tmo)) {
        bad = true;
        if (lane == 0) atomicOr(err, kErrPipeline);
      }
      if (!bad) run_panels<kPrec, kGroupWarps>(L, smem_u32(sm.stage + slot * kStageBytes), R, wl, t0, t1);
      bad = bad || R.bad;
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.sempty[slot]);
    }
    if (L.flags & kLast) {
      R.release_below(R.base + ((L.pos + 16u * L.nrow * L.npanel) >> kChunkLog));
      if (bad) ++nb;
      else if (!block_end(t0, t1, nb, sm, err, tmo)) bad = true;
      t0 = 0.0;
      t1 = 0.0;
    }
  }
  R.release_below(R.base + K);
}

// The consumer warps' part of one H-matvec pass: the P-done signal of a CTA
// without P blocks, the pass, then the wait for the block-sum warp (every
// row of the pass is written) and, in warp 0, for the pass's grid barrier
// (the caller's next grid barrier must not start before it completes).
template <int kPrec>
__device__ __forceinline__ void matvec_pass(Ring &R, uint32_t K, uint32_t nr, uint32_t &nb, const PassOut &o,
                                            const Smem &sm, int *err, uint64_t tmo) {
  if (o.nblk_p == 0 && threadIdx.x == 0) mbar_arrive(sm.pdone);
  consume_pass<kPrec>(R, K, nr, nb, o.pass, sm, err, tmo);
  if (!warp_wait(sm.rdone, o.pass & 1, tmo) && (threadIdx.x & 31) == 0) atomicOr(err, kErrPipeline);
  if (threadIdx.x < 32 && !warp_wait(sm.gdone, o.pass & 1, tmo) && threadIdx.x == 0) atomicOr(err, kErrGridBarrier);
}

// Bytes at the head of a CTA's stream read with the evict_last policy: a
// fraction keep_frac / 2^16 of the stream, whole chunks (0: no cache hints).
__device__ __forceinline__ uint32_t keep_bytes(uint32_t stream_bytes, uint32_t keep_frac) {
  if (keep_frac == 0) return 0;
  const uint64_t b = ((uint64_t)stream_bytes * keep_frac) >> 16;
  const uint64_t r = (b + kChunkBytes - 1) & ~(uint64_t)(kChunkBytes - 1);
  return r > 0xffffffffull ? 0xffffffffu : (uint32_t)r;
}

// kPrec: storage precision of the factors; FP32 and BF16 engines gather the
// float copies of the vectors.
#ifndef HBX_STEP_TU
template <int kPrec>
__global__ void __launch_bounds__(kThreads, 1) k_matvec(MatvecArgs a) {
  constexpr bool kF32 = kPrec != kFP64;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  if (a.skip && *(volatile const int *)a.skip) return;  // set by an earlier launch: the same on every CTA
  const CtaInfo ci = a.ctas[blockIdx.x];
  const uint32_t nr = ci.nr_p + ci.nr_d + ci.nr_u;
  const Smem sm = cta_smem(smem_raw, a.lite + ci.rec_begin, nr);
  const uint64_t t_start = a.prof ? gtimer() : 0;
  uint32_t issued0 = 0;
  const StreamSrc ss{a.stream + ci.stream_off, ci.stream_bytes, keep_bytes(ci.stream_bytes, a.keep_frac),
                     a.chunk_inst ? a.chunk_inst + a.chunk_base[blockIdx.x] : nullptr, a.inst_pre};
  if (threadIdx.x == kProducerWarp * 32) issued0 = producer_start(ss, 1, sm.ring, sm.full, sm.empty);
  init_cta(sm, a.lite + ci.rec_begin, nr, a.gbar, NW / groups_of<kPrec>());
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t K = (ci.stream_bytes + kChunkBytes - 1) >> kChunkLog;
  if (w == kProducerWarp) {
    if (lane == 0 && K > 0)
      producer_run(ss, 1, issued0, sm.ring, sm.full, sm.empty, a.err, a.timeout_ns);
    return;
  }
  if (w >= kGatherWarp0 && w < kSyncWarp) {
    const void *xs = kF32 ? static_cast<const void *>(a.x32) : static_cast<const void *>(a.x);
    const void *zs = kF32 ? static_cast<const void *>(a.zbu32) : static_cast<const void *>(a.zbu);
    const GatherCtx c{a.recs + ci.rec_begin, nr, ci.nr_p + ci.nr_d, 1, xs, xs, zs, zs, a.err, a.timeout_ns};
    gather_warp<kPrec>(c, sm, (uint32_t)(w - kGatherWarp0));
    return;
  }
  if (w == kSyncWarp) {
    if (lane == 0) sync_warp(a.gbar, 1, 0, 0, sm, a.err, a.timeout_ns, a.stall ? 1u : 0u);
    return;
  }
  const PassOut o{a.alpha, a.beta, a.yin, a.y, a.zbu, kF32 ? a.zbu32 : nullptr, 0, ci.nblk_p};
  if (w == kSumWarp) {
    sum_warp(nr, 1, ci.nblk_p, &o, sm, a.err, a.timeout_ns);
    return;
  }
  if (threadIdx.x == 0) signal_xready(sm, 0);  // x is an input: ready from the start
  uint32_t nb = 0;
  Ring R{sm.ring, sm.full, sm.empty, 0, 0, 0, a.timeout_ns, a.err, false};
  matvec_pass<kPrec>(R, K, nr, nb, o, sm, a.err, a.timeout_ns);
  if (a.prof && threadIdx.x == 0) {
    a.prof[blockIdx.x * 16 + 0] = t_start;
    a.prof[blockIdx.x * 16 + 5] = gtimer();
  }
}

#endif  // !HBX_STEP_TU

#ifdef HBX_STEP_TU
// ---------------------------------------------------------------- BiCGSTAB
template <class F>
__device__ __forceinline__ void for_own_rows(const Atom *atoms, const CtaInfo &ci, F f) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t q = w; q < ci.n_atoms; q += NW) {
    const Atom A = atoms[ci.atom_begin + q];
    if ((uint32_t)lane < A.h) f(A.r0 + lane);
  }
}

// The same over the warp's atoms after its first one (index w + NW, ...).
template <class F>
__device__ __forceinline__ void for_more_rows(const Atom *atoms, const CtaInfo &ci, F f) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t q = w + NW; q < ci.n_atoms; q += NW) {
    const Atom A = atoms[ci.atom_begin + q];
    if ((uint32_t)lane < A.h) f(A.r0 + lane);
  }
}

// Per-CTA compensated partial sums of NS dot products over the owned rows.
// acc[] holds the calling thread's partials; the result goes to part[cta][slot0+k].
template <int NSL>
__device__ __forceinline__ void cta_partials(Acc2 (&acc)[NSL], double *part, int slot0, const Smem &sm) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NSL; ++k) acc[k] = warp_merge(acc[k]);
  double *sc = sm.red;  // reuse: [NW][NSL][2]
  named_bar(1, kConsumerThreads);  // red may still be read by an atom reduction
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NSL; ++k) {
      sc[(w * NSL + k) * 2 + 0] = acc[k].s;
      sc[(w * NSL + k) * 2 + 1] = acc[k].c;
    }
  }
  named_bar(1, kConsumerThreads);
  if (w == 0 && lane < NSL) {
    Acc2 t{sc[lane * 2], sc[lane * 2 + 1]};
    for (int q = 1; q < NW; ++q) t = acc2_merge(t, Acc2{sc[(q * NSL + lane) * 2], sc[(q * NSL + lane) * 2 + 1]});
    double *dst = part + ((size_t)blockIdx.x * kSlots + slot0 + lane) * 2;
    dst[0] = t.s;
    dst[1] = t.c;
    __threadfence();
  }
  named_bar(1, kConsumerThreads);
}

// Total of one slot over all CTAs, same operation order in every CTA (full warp).
// (The loads of a lane are issued together, then merged in CTA order; a
// merge with a zero pair leaves the sum unchanged.)
__device__ __forceinline__ double reduce_slot(const double *part, int ncta, int slot) {
  constexpr int kBatch = 5;
  const int lane = threadIdx.x & 31;
  Acc2 a{0.0, 0.0};
  for (int c0 = 0; c0 < ncta; c0 += 32 * kBatch) {
    Acc2 v[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
      const int c = c0 + lane + 32 * k;
      v[k] = Acc2{0.0, 0.0};
      if (c < ncta) {
        const double *src = part + ((size_t)c * kSlots + slot) * 2;
        v[k] = Acc2{__ldcg(src), __ldcg(src + 1)};
      }
    }
#pragma unroll
    for (int k = 0; k < kBatch; ++k) a = acc2_merge(a, v[k]);
  }
  a = warp_merge(a);
  return a.s + a.c;
}

// Grid-barrier instances of one BiCGSTAB step, in order: p complete, zbu of
// the first H-matvec complete, the r^.Ap partials, t complete, zbu of the
// second H-matvec, the At.t / At.At partials.
enum : unsigned { kGridP = 0, kGridPass0 = 1, kGridAlpha = 2, kGridT = 3, kGridPass1 = 4, kGridZeta = 5 };

// Full grid barrier (instance k of the launch) among the consumer warps of
// every CTA.
__device__ __forceinline__ bool grid_sync(unsigned *gbar, unsigned k, int *err, uint64_t timeout_ns, const Smem &sm) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  named_bar(1, kConsumerThreads);
  if (w == 0 && lane == 0) {
    const unsigned target = grid_target(sm.rsum[1], k, gridDim.x);
    grid_arrive(gbar, target);
    const bool ok = grid_wait(gbar, target, timeout_ns);
    if (!ok) atomicOr(err, kErrGridBarrier);
    sm.scal[62] = ok ? 1.0 : 0.0;
  }
  named_bar(1, kConsumerThreads);
  return sm.scal[62] != 0.0;
}

#ifndef HBX_STEP_LP
__global__ void __launch_bounds__(kThreads, 1) k_bicg_setup(BicgArgs a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const Smem sm = smem_layout(smem_raw);
  if ((threadIdx.x >> 5) >= NW) return;
  const CtaInfo ci = a.ctas[blockIdx.x];
  Acc2 acc[3] = {{0, 0}, {0, 0}, {0, 0}};
  for_own_rows(a.atoms, ci, [&](uint32_t r) {
    const double rv = a.r[r];
    a.rh[r] = rv;
    a.p[r] = 0.0;
    a.ap[r] = 0.0;
    dot2_add(acc[0], rv, rv);
    dot2_add(acc[1], rv, rv);
    const double bv = a.b[r];
    dot2_add(acc[2], bv, bv);
  });
  // slots 0,1 then 5
  Acc2 a01[2] = {acc[0], acc[1]};
  cta_partials<2>(a01, a.part, kSlotRhoR, sm);
  Acc2 a5[1] = {acc[2]};
  cta_partials<1>(a5, a.part, kSlotBB, sm);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    BicgState st{};
    *a.state = st;
  }
}
#endif

template <int kPrec>
__global__ void __launch_bounds__(kThreads, 1) k_bicg_iter(BicgArgs a) {
  constexpr bool kF32 = kPrec != kFP64;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const CtaInfo ci = a.ctas[blockIdx.x];
  const uint32_t nr = ci.nr_p + ci.nr_d + ci.nr_u;
  const Smem sm = cta_smem(smem_raw, a.lite + ci.rec_begin, nr);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ncta = gridDim.x;
  auto stamp = [&](int k) {
    if (a.prof && threadIdx.x == 0) a.prof[blockIdx.x * 16 + 8 + k] = gtimer();
  };
  const uint64_t t_start = a.prof ? gtimer() : 0;
  // A consumer warp's first owned atom and this lane's row of it: its vector
  // entries stay in registers through the step, loaded while the step's
  // scalars are reduced (the rows of further atoms are read where needed).
  const Atom a0 = (w < NW && (uint32_t)w < ci.n_atoms) ? a.atoms[ci.atom_begin + w] : Atom{0, 0};
  const bool own0 = (uint32_t)lane < a0.h;
  const uint32_t row0 = a0.r0 + lane;
  double c_r = 0.0, c_rh = 0.0, c_p = 0.0, c_ap = 0.0, c_u = 0.0, c_t = 0.0, c_at = 0.0;
  if (own0) {
    c_r = a.r[row0];
    c_rh = a.rh[row0];
    c_p = __ldcg(&a.p[row0]);  // see S1
    c_ap = a.ap[row0];
    c_u = a.u[row0];
  }
  // the producer starts the stream of the first H-matvec, warps 4 and up set
  // up the CTA and warps 0-3 reduce the scalars
  const StreamSrc ss{a.stream + ci.stream_off, ci.stream_bytes, keep_bytes(ci.stream_bytes, a.keep_frac)};
  uint32_t issued0 = 0;
  if (threadIdx.x == kProducerWarp * 32) issued0 = producer_start(ss, 2, sm.ring, sm.full, sm.empty);
  init_cta_part(sm, a.lite + ci.rec_begin, nr, a.gbar, 128, NW / groups_of<kPrec>());

  // ---- S0: scalars of the previous step; stop test at the top of the loop
  // (HACApK_SOLVER.c:602-603).  Every CTA computes identical values: warps
  // 0-2 reduce the three dot products side by side, warp 3 reads the state.
  if (w < 3) {
    const double v = reduce_slot(a.part, ncta, w == 0 ? kSlotRhoR : (w == 1 ? kSlotRR : kSlotBB));
    if (lane == 0) sm.scal[10 + w] = v;
  } else if (w == 3 && lane == 0) {
    sm.scal[13] = __ldcg(&a.state->alpha);
    sm.scal[14] = __ldcg(&a.state->zeta);
    sm.scal[15] = __ldcg(&a.state->rho);
    sm.scal[16] = (double)__ldcg(&a.state->iter);
    sm.scal[17] = (double)__ldcg(&a.state->done);
    sm.scal[18] = (double)__ldcg(&a.state->status);
    sm.scal[19] = (double)__ldcg(&a.state->breakdown);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double rho_new = sm.scal[10], rr = sm.scal[11], bb = sm.scal[12];
    BicgState st;
    st.alpha = sm.scal[13];
    st.zeta = sm.scal[14];
    st.rho = sm.scal[15];
    st.iter = (int)sm.scal[16];
    st.done = (int)sm.scal[17];
    st.status = (int)sm.scal[18];
    st.breakdown = (int)sm.scal[19];
    const double bnorm = sqrt(bb);
    const double relres = (bnorm > 0.0) ? sqrt(rr) / bnorm : 0.0;
    int done = st.done, status = st.status;
    double beta = 0.0;
    if (!done) {
      if (st.breakdown) { done = 1; status = HBX_ERR_BREAKDOWN; }
      // NaN or Inf in b or x0 shows in b.b or r.r before the first step
      else if (!isfinite(bb) || !isfinite(rr)) { done = 1; status = st.iter == 0 ? HBX_ERR_NONFINITE : HBX_ERR_BREAKDOWN; }
      else if (relres < a.tol) { done = 1; status = HBX_OK; }
      else if (!isfinite(relres)) { done = 1; status = HBX_ERR_BREAKDOWN; }
      else if (st.iter >= a.max_iter) { done = 1; status = HBX_ERR_NOT_CONVERGED; }
      else if (st.iter > 0) {
        // beta = -alpha/zeta * (rh.r_new)/znormold with the reference's sign
        // flips (HACApK_SOLVER.c:650-655, :699, :724) = (alpha/zeta) rho_new/rho_old
        beta = (st.alpha / st.zeta) * (rho_new / st.rho);
        if (!isfinite(beta)) { done = 1; status = HBX_ERR_BREAKDOWN; }
      }
    }
    sm.scal[0] = done;
    sm.scal[1] = status;
    sm.scal[2] = beta;
    sm.scal[3] = st.zeta;
    sm.scal[4] = rho_new;
    sm.scal[5] = relres;
    sm.scal[6] = st.iter;
    sm.scal[7] = bnorm;
    if (done && blockIdx.x == 0) {
      a.state->done = 1;
      a.state->status = status;
      a.state->relres = relres;
      a.state->bnorm = bnorm;
    }
  }
  __syncthreads();
  if (sm.scal[0] != 0.0) {
    if (threadIdx.x == kProducerWarp * 32) producer_drain(sm.full, issued0, a.timeout_ns);
    return;
  }
  if (a.prof && threadIdx.x == 0) a.prof[blockIdx.x * 16 + 8] = t_start;  // stamps of working steps only
  const double beta = sm.scal[2], zeta_prev = sm.scal[3], rho = sm.scal[4];
  const double relres = sm.scal[5], bnorm = sm.scal[7];
  const int iter = (int)sm.scal[6];

  const uint32_t K = (ci.stream_bytes + kChunkBytes - 1) >> kChunkLog;
  if (w == kProducerWarp) {
    if (lane == 0 && K > 0)
      producer_run(ss, 2, issued0, sm.ring, sm.full, sm.empty, a.err, a.timeout_ns);
    return;
  }
  if (w >= kGatherWarp0 && w < kSyncWarp) {
    const void *x0 = kF32 ? static_cast<const void *>(a.p32) : static_cast<const void *>(a.p);
    const void *x1 = kF32 ? static_cast<const void *>(a.t32) : static_cast<const void *>(a.t);
    const void *z0 = kF32 ? static_cast<const void *>(a.zbu32) : static_cast<const void *>(a.zbu);
    const void *z1 =
        kF32 ? static_cast<const void *>(a.zbu32 + a.zbu_len) : static_cast<const void *>(a.zbu + a.zbu_len);
    const GatherCtx c{a.recs + ci.rec_begin, nr, ci.nr_p + ci.nr_d, 2, x0, x1, z0, z1, a.err, a.timeout_ns};
    gather_warp<kPrec>(c, sm, (uint32_t)(w - kGatherWarp0));
    return;
  }
  if (w == kSyncWarp) {
    if (lane == 0) sync_warp(a.gbar, 2, kGridPass0, kGridPass1 - kGridPass0, sm, a.err, a.timeout_ns);
    return;
  }
  // The two H-matvecs write separate zbu copies, so a U run of the second
  // never reads a line of the first from L1.
  const PassOut outs[2] = {{1.0, 0.0, nullptr, a.ap, a.zbu, kF32 ? a.zbu32 : nullptr, 0, ci.nblk_p},
                           {1.0, 0.0, nullptr, a.at, a.zbu + a.zbu_len, kF32 ? a.zbu32 + a.zbu_len : nullptr, 1,
                            ci.nblk_p}};
  if (w == kSumWarp) {
    sum_warp(nr, 2, ci.nblk_p, outs, sm, a.err, a.timeout_ns);
    return;
  }
  Ring R{sm.ring, sm.full, sm.empty, 0, 0, 0, a.timeout_ns, a.err, false};
  uint32_t nb = 0;

  // ---- S1: p = r + beta*(p - zeta*Ap)  (p = r on the first step)
  if (own0) {
    c_p = (beta == 0.0) ? c_r : fma(-zeta_prev, c_ap, c_p) * beta + c_r;
    a.p[row0] = c_p;
    if (kF32) a.p32[row0] = (float)c_p;
  }
  if (beta == 0.0) {
    for_more_rows(a.atoms, ci, [&](uint32_t r) {
      const double v = a.r[r];
      a.p[r] = v;
      if (kF32) a.p32[r] = (float)v;
    });
  } else {
    for_more_rows(a.atoms, ci, [&](uint32_t r) {
      // p through L2 only: a line of p cached in L1 here could hold rows of
      // another CTA that the gather warps read after it rewrote them
      const double v = fma(-zeta_prev, a.ap[r], __ldcg(&a.p[r])) * beta;
      const double pv = v + a.r[r];
      a.p[r] = pv;
      if (kF32) a.p32[r] = (float)pv;
    });
  }
  __threadfence();
  grid_sync(a.gbar, kGridP, a.err, a.timeout_ns, sm);
  if (threadIdx.x == 0) signal_xready(sm, 0);  // p complete grid-wide: pass 0 may be gathered
  stamp(1);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.state->iter = iter + 1;
    a.state->beta = beta;
    a.state->rho = rho;
    a.state->relres = relres;
    a.state->bnorm = bnorm;
    a.hist[iter] = relres;
  }

  // ---- S2: Ap = H p;  rh . Ap
  matvec_pass<kPrec>(R, K, nr, nb, outs[0], sm, a.err, a.timeout_ns);
  stamp(2);
  {
    Acc2 acc[1] = {{0, 0}};
    named_bar(1, kConsumerThreads);
    if (own0) {
      c_ap = a.ap[row0];
      dot2_add(acc[0], c_rh, c_ap);
    }
    for_more_rows(a.atoms, ci, [&](uint32_t r) { dot2_add(acc[0], a.rh[r], a.ap[r]); });
    cta_partials<1>(acc, a.part, kSlotRhAp, sm);
  }
  grid_sync(a.gbar, kGridAlpha, a.err, a.timeout_ns, sm);
  if (w == 0) {
    const double zden = reduce_slot(a.part, ncta, kSlotRhAp);
    if (lane == 0) sm.scal[8] = rho / zden;
  }
  named_bar(1, kConsumerThreads);
  const double alpha = sm.scal[8];
  stamp(3);

  // ---- S3: t = r - alpha*Ap
  if (own0) {
    c_t = fma(-alpha, c_ap, c_r);
    a.t[row0] = c_t;
    if (kF32) a.t32[row0] = (float)c_t;
  }
  for_more_rows(a.atoms, ci, [&](uint32_t r) {
    const double v = fma(-alpha, a.ap[r], a.r[r]);
    a.t[r] = v;
    if (kF32) a.t32[r] = (float)v;
  });
  __threadfence();
  grid_sync(a.gbar, kGridT, a.err, a.timeout_ns, sm);
  if (threadIdx.x == 0) signal_xready(sm, 1);  // t complete grid-wide: pass 1 may be gathered
  stamp(4);

  // ---- S4: At = H t;  At . t,  At . At
  R.base = K;
  matvec_pass<kPrec>(R, K, nr, nb, outs[1], sm, a.err, a.timeout_ns);
  stamp(5);
  {
    Acc2 acc[2] = {{0, 0}, {0, 0}};
    named_bar(1, kConsumerThreads);
    if (own0) {
      c_at = a.at[row0];
      dot2_add(acc[0], c_at, c_t);
      dot2_add(acc[1], c_at, c_at);
    }
    for_more_rows(a.atoms, ci, [&](uint32_t r) {
      const double atv = a.at[r];
      dot2_add(acc[0], atv, a.t[r]);
      dot2_add(acc[1], atv, atv);
    });
    cta_partials<2>(acc, a.part, kSlotAtT, sm);
  }
  grid_sync(a.gbar, kGridZeta, a.err, a.timeout_ns, sm);
  if (w < 2) {  // the two sums side by side
    const double v = reduce_slot(a.part, ncta, w == 0 ? kSlotAtT : kSlotAtAt);
    if (lane == 0) sm.scal[10 + w] = v;
  }
  named_bar(1, kConsumerThreads);
  if (w == 0) {
    const double s3 = sm.scal[10], s4 = sm.scal[11];
    if (lane == 0) {
      const double zeta = (s4 != 0.0) ? s3 / s4 : 0.0;
      sm.scal[9] = zeta;
      const bool bad = !isfinite(alpha) || !isfinite(zeta);
      if (blockIdx.x == 0) {
        a.state->alpha = alpha;
        a.state->zeta = zeta;
        if (bad) a.state->breakdown = 1;
      }
    }
  }
  named_bar(1, kConsumerThreads);
  const double zeta = sm.scal[9];
  stamp(6);

  // ---- S5: u += alpha*p + zeta*t;  r = t - zeta*At;  rh . r,  r . r
  // A breakdown (alpha or zeta not finite: r^.Ap or At.At zero or
  // overflowing, which HACApK_SOLVER.c:650, :694 divide by unchecked) keeps
  // u and r of the previous step; the next launch ends the solve with
  // HBX_ERR_BREAKDOWN.
  if (!isfinite(alpha) || !isfinite(zeta)) {
    stamp(7);
    return;
  }
  {
    Acc2 acc[2] = {{0, 0}, {0, 0}};
    if (own0) {
      a.u[row0] = fma(zeta, c_t, fma(alpha, c_p, c_u));
      const double rv = fma(-zeta, c_at, c_t);
      a.r[row0] = rv;
      dot2_add(acc[0], c_rh, rv);
      dot2_add(acc[1], rv, rv);
    }
    for_more_rows(a.atoms, ci, [&](uint32_t r) {
      const double uv = fma(alpha, a.p[r], a.u[r]);
      a.u[r] = fma(zeta, a.t[r], uv);
      const double rv = fma(-zeta, a.at[r], a.t[r]);
      a.r[r] = rv;
      dot2_add(acc[0], a.rh[r], rv);
      dot2_add(acc[1], rv, rv);
    });
    cta_partials<2>(acc, a.part, kSlotRhoR, sm);
  }
  stamp(7);
}

// part[cta][slot] over own rows, then (block 0 of a second launch) the total.
#ifndef HBX_STEP_LP
__global__ void __launch_bounds__(kThreads, 1) k_dot_partial(BicgArgs a, const double *x, const double *y, int slot) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const Smem sm = smem_layout(smem_raw);
  if ((threadIdx.x >> 5) >= NW) return;
  const CtaInfo ci = a.ctas[blockIdx.x];
  Acc2 acc[1] = {{0, 0}};
  for_own_rows(a.atoms, ci, [&](uint32_t r) { dot2_add(acc[0], x[r], y[r]); });
  cta_partials<1>(acc, a.part, slot, sm);
}
#endif

// y = (float)x: the input of an FP32 engine's matvec.
#endif  // HBX_STEP_TU

#ifndef HBX_STEP_TU
__global__ void k_to_float(const double *x, float *y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

// y += a * x (the refinement update of the mixed-precision solve).
__global__ void k_axpy(double a, const double *x, double *y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}

#endif  // !HBX_STEP_TU

#ifdef HBX_STEP_TU
#ifndef HBX_STEP_LP
__global__ void k_dot_total(const double *part, int ncta, int slot, double *out) {
  const double v = reduce_slot(part, ncta, slot);
  if (threadIdx.x == 0) *out = v;
}
#endif

#endif  // HBX_STEP_TU

}  // namespace

#ifndef HBX_STEP_TU
// ---- fixed scratch for hbx_matvec_noalloc -------------------------------
// One 1 MiB array per device, held by every GPU that loads this library until
// the process exits: [0, 256) barrier words, [256, end) the zbu segments.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// Host side: the device address of g_noalloc_scratch on the current device.
cudaError_t noalloc_scratch_address(void **ptr) { return cudaGetSymbolAddress(ptr, g_noalloc_scratch); }

size_t kernel_smem_bytes() { return SharedLayout::bytes; }

cudaError_t configure_kernels() {
  const int smem = (int)SharedLayout::bytes;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_matvec<kFP64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_matvec<kFP32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_matvec<kBF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  return configure_step_kernels();
}

#endif  // !HBX_STEP_TU

template <class Args>
static cudaError_t launch_coop(void (*kern)(Args), const Args &a, int num_ctas, cudaStream_t s) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(num_ctas);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = SharedLayout::bytes;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, a);
}

#ifndef HBX_STEP_TU
cudaError_t launch_matvec(const MatvecArgs &a, int num_ctas, cudaStream_t s, int precision) {
  if (precision == kBF16) return launch_coop(k_matvec<kBF16>, a, num_ctas, s);
  return precision == kFP32 ? launch_coop(k_matvec<kFP32>, a, num_ctas, s) : launch_coop(k_matvec<kFP64>, a, num_ctas, s);
}

cudaError_t launch_to_float(const double *x, float *y, size_t n, cudaStream_t s) {
  k_to_float<<<296, 256, 0, s>>>(x, y, n);
  return cudaGetLastError();
}

cudaError_t launch_axpy(double alpha, const double *x, double *y, size_t n, cudaStream_t s) {
  k_axpy<<<296, 256, 0, s>>>(alpha, x, y, n);
  return cudaGetLastError();
}
#elif !defined(HBX_STEP_LP)
cudaError_t configure_step_kernels() {
  const int smem = (int)SharedLayout::bytes;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_bicg_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_bicg_iter<kFP64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_dot_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  return configure_step_kernels_lp();
}

cudaError_t launch_bicg_setup(const BicgArgs &a, int num_ctas, cudaStream_t s) {
  k_bicg_setup<<<num_ctas, kThreads, SharedLayout::bytes, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bicg_iter(const BicgArgs &a, int num_ctas, cudaStream_t s, int precision) {
  if (precision != kFP64) return launch_bicg_iter_lp(a, num_ctas, s, precision);
  return launch_coop(k_bicg_iter<kFP64>, a, num_ctas, s);
}

cudaError_t launch_dot(const BicgArgs &a, const double *x, const double *y, int slot, double *out, int num_ctas,
                       cudaStream_t s) {
  k_dot_partial<<<num_ctas, kThreads, SharedLayout::bytes, s>>>(a, x, y, slot);
  k_dot_total<<<1, 32, 0, s>>>(a.part, num_ctas, slot, out);
  return cudaGetLastError();
}
#else
// The FP32 and BF16 step kernels: kStepWarpsLp consumer warps in two groups.
cudaError_t configure_step_kernels_lp() {
  const int smem = (int)SharedLayout::bytes;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_bicg_iter<kFP32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_bicg_iter<kBF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  return cudaSuccess;
}

cudaError_t launch_bicg_iter_lp(const BicgArgs &a, int num_ctas, cudaStream_t s, int precision) {
  return precision == kBF16 ? launch_coop(k_bicg_iter<kBF16>, a, num_ctas, s)
                            : launch_coop(k_bicg_iter<kFP32>, a, num_ctas, s);
}
#endif  // HBX_STEP_TU

}  // namespace hbx
