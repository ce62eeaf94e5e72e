// hbx_mrhs.cu -- H-matrix product with many right-hand sides on the sm_100a
// tensor cores: Y = alpha * H X + beta * Yin for kNrhs = 64 right-hand sides.
//
// The packed stream is the FP32 engine's (panels of 4 columns x h rows, 16
// bytes a row) with every run an even number of panels, so two panels make
// the K = 8 of one TF32 step.  Per CTA (one per SM), 16 warps:
//
//   warps 0-3   epilogue: TMEM accumulator -> zbu (P blocks) or Y (D, U)
//   warp 4      tcgen05: allocates TMEM; one thread issues the MMAs of the
//               even blocks
//   warp 5      bulk-copy producer of the stream ring (16 KB chunks)
//   warps 6-13  gather: X (or zbu) columns of a run, 64 at a time, into a
//               K-major operand stage [4-column chunk][rhs][4] (16 KB), one
//               stage per warp
//   warp 14     grid barrier between the P blocks and the U runs
//   warp 15     one thread issues the MMAs of the odd blocks
//
// Two issuers because one thread's issue loop (descriptors, ring and stage
// waits, commits: ~170 cycles an MMA of M = 64, N <= 64, K = 8) paced the
// whole CTA; each has its own two accumulators, waits for its own slices'
// stages, and hands every ring chunk back (the empty barriers count both).
//
// One MMA: D[rhs][row] += Xs[rhs][k..k+8] * Panel[row][k..k+8]^T with
// M = 64 right-hand sides, N = the block's rows rounded up to 8, A (the
// staged X) and B (two panels straight from the ring) both K-major in the
// canonical no-swizzle layout: 8-row core matrices of 16-byte rows, the next
// 8 rows 128 bytes on (SBO), the next 4 columns LBO on (1 KB for A, 16h for
// B).  D lives in TMEM (M = 64: rhs m in lane (m mod 16) + 32 (m / 16)); two
// 64-column accumulators let the epilogue of one block overlap the MMAs of
// the next.  The ring is smaller than k_matvec's (the product is bound by
// the X stages, not by the stream) and MMAs read it in place: a panel pair
// that runs past the
// ring's end reads a mirror of the first bytes of slot 0 that the producer
// keeps behind the ring.  Rows of D past h come from bytes after the pair
// and are never stored.
//
// No counterpart in the reference (its batched GEMV takes one vector).
#include "hbx_device.cuh"
#include "hbx_engine.h"

namespace hbx {
namespace {

constexpr int kSliceCols = 64;                         // stage columns per slice
constexpr int kSliceChunks = kSliceCols / 4;           // 4-column K chunks per slice
constexpr int kChunkXBytes = kNrhs * 16;               // one chunk, all right-hand sides: 1 KB
constexpr int kSliceBytes = kSliceChunks * kChunkXBytes;  // 16 KB
constexpr int kMChunkLog = 14;  // ring chunk: 16 KB
constexpr int kMChunkBytes = 1 << kMChunkLog;
constexpr int kMRingChunks = 4;
constexpr uint32_t kMRingBytes = (uint32_t)kMRingChunks * kMChunkBytes;
constexpr int kXStages = 8;
constexpr int kMirrorBytes = 2304;  // >= 2 panels of 64 rows + 7 rows past them
constexpr int kAccCols = 64;        // TMEM columns per accumulator (rows of a block <= 64)
constexpr int kIssuers = 2;  // MMA-issuing threads (warps kMmaWarp and kMmaWarp2), alternate blocks
constexpr int kTmemCols = 2 * kIssuers * kAccCols;  // two accumulators per issuer
constexpr int kEpiWarps = 4, kMmaWarp = 4, kProdWarpM = 5, kGathWarp0 = 6, kGathWarps = 8, kSyncWarpM = 14,
              kMmaWarp2 = 15;
static_assert(kXStages == kGathWarps, "gather warp gi always fills stage gi");
constexpr int kThreadsM = (kMmaWarp2 + 1) * 32;

struct MLayout {
  static constexpr uint32_t ring = 0;
  static constexpr uint32_t xst = (kMRingBytes + kMirrorBytes + 1023) / 1024 * 1024;  // [kXStages] slices
  static constexpr uint32_t rec = xst + kXStages * kSliceBytes;                       // [kGathWarps][2] records
  static constexpr uint32_t lite = rec + 2 * kGathWarps * kRecBytes;                  // [kMaxPairRuns] summaries
  static constexpr uint32_t full = lite + kMaxPairRuns * 16;
  static constexpr uint32_t empty = full + 8 * kMRingChunks;
  static constexpr uint32_t xfull = empty + 8 * kMRingChunks;
  static constexpr uint32_t xempty = xfull + 8 * kXStages;
  static constexpr uint32_t accfull = xempty + 8 * kXStages;
  static constexpr uint32_t accempty = accfull + 8 * 2 * kIssuers;
  static constexpr uint32_t pdone = accempty + 8 * 2 * kIssuers;
  static constexpr uint32_t gdone = pdone + 8;
  static constexpr uint32_t mdone = gdone + 8;
  static constexpr uint32_t tmem = mdone + 8;  // TMEM base address (tcgen05.alloc writes it)
  static constexpr uint32_t gen0 = tmem + 4;   // first grid-barrier generation of the launch
  static constexpr uint32_t xcnt = (gen0 + 4 + 15) / 16 * 16;  // [kXStages] slices staged per slot
  static constexpr uint32_t bytes = xcnt + 4 * kXStages;
};
static_assert(MLayout::bytes <= 227 * 1024, "shared memory per CTA");
static_assert(MLayout::xst % 1024 == 0 && MLayout::rec % 16 == 0 && MLayout::full % 8 == 0, "layout alignment");

// ---- tcgen05 ----------------------------------------------------------------
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, no swizzle, K-major canonical layout.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3fffu);
  d |= (uint64_t)((lbo >> 4) & 0x3fffu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3fffu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, absolute LBO, layout SWIZZLE_NONE
}

// Instruction descriptor: kind::tf32, D f32, A and B K-major, M x N.
__device__ __forceinline__ uint32_t idesc_tf32(uint32_t m, uint32_t n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

// The barrier receives one arrival once every MMA this thread issued so far
// has completed.
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// ---- producer with the ring-end mirror ------------------------------------
__device__ __forceinline__ void mr_issue(const uint8_t *src, uint32_t bytes, uint32_t g, uint8_t *ring,
                                         uint64_t *full) {
  const uint32_t s = g % kMRingChunks;
  const uint32_t off = g << kMChunkLog;
  const uint32_t nb = min((uint32_t)kMChunkBytes, bytes - off);
  const uint32_t nm = s == 0 ? min(nb, (uint32_t)kMirrorBytes) : 0u;
  mbar_arrive_expect_tx(&full[s], nb + nm);
  bulk_g2s(ring + ((size_t)s << kMChunkLog), src + off, nb, &full[s]);
  if (nm) bulk_g2s(ring + kMRingBytes, src + off, nm, &full[s]);
}

__device__ __forceinline__ void mr_producer(const uint8_t *src, uint32_t bytes, uint8_t *ring, uint64_t *full,
                                            uint64_t *empty, int *err, uint64_t tmo) {
  const uint32_t K = (bytes + kMChunkBytes - 1) >> kMChunkLog;
  uint32_t issued = 0;
  for (uint32_t g = 0; g < K; ++g) {
    if (g >= (uint32_t)kMRingChunks && !mbar_wait(&empty[g % kMRingChunks], ((g / kMRingChunks) - 1) & 1, tmo)) {
      atomicOr(err, kErrProducer);
      break;
    }
    mr_issue(src, bytes, g, ring, full);
    issued = g + 1;
  }
  // copies still in flight land before the CTA exits
  const uint32_t g0 = issued > (uint32_t)kMRingChunks ? issued - kMRingChunks : 0;
  for (uint32_t g = g0; g < issued; ++g) mbar_wait(&full[g % kMRingChunks], (g / kMRingChunks) & 1, tmo);
}

struct MSmem {
  uint8_t *ring, *xst, *rec;
  RunLite *lite;
  uint64_t *full, *empty, *xfull, *xempty, *accfull, *accempty, *pdone, *gdone, *mdone;
  uint32_t *tmem, *gen0, *xcnt;
};

__device__ __forceinline__ MSmem mlayout(uint8_t *b) {
  MSmem s;
  s.ring = b + MLayout::ring;
  s.xst = b + MLayout::xst;
  s.rec = b + MLayout::rec;
  s.lite = reinterpret_cast<RunLite *>(b + MLayout::lite);
  s.full = reinterpret_cast<uint64_t *>(b + MLayout::full);
  s.empty = reinterpret_cast<uint64_t *>(b + MLayout::empty);
  s.xfull = reinterpret_cast<uint64_t *>(b + MLayout::xfull);
  s.xempty = reinterpret_cast<uint64_t *>(b + MLayout::xempty);
  s.accfull = reinterpret_cast<uint64_t *>(b + MLayout::accfull);
  s.accempty = reinterpret_cast<uint64_t *>(b + MLayout::accempty);
  s.pdone = reinterpret_cast<uint64_t *>(b + MLayout::pdone);
  s.gdone = reinterpret_cast<uint64_t *>(b + MLayout::gdone);
  s.mdone = reinterpret_cast<uint64_t *>(b + MLayout::mdone);
  s.tmem = reinterpret_cast<uint32_t *>(b + MLayout::tmem);
  s.gen0 = reinterpret_cast<uint32_t *>(b + MLayout::gen0);
  s.xcnt = reinterpret_cast<uint32_t *>(b + MLayout::xcnt);
  return s;
}

// A block without columns (a D block of an atom that no dense leaf touches)
// is one run of no panels: nothing is multiplied for it.
__device__ __forceinline__ bool empty_block(const RunLite &L) {
  return L.npanel == 0 && (L.flags & kFirst) && (L.flags & kLast);
}

__device__ __forceinline__ uint32_t run_slices(const RunLite &L) {
  return (4u * L.npanel + kSliceCols - 1) / kSliceCols;
}

// ---- gather warp gi: slices q = gi, gi + kGathWarps, ... of the launch ----
// Lane (c = lane & 3, m0 = lane >> 2) copies column c of every 4-column chunk
// for right-hand sides m0, m0 + 8, ...: consecutive lanes write consecutive
// words of the stage.  A stage column past the run's real columns is zero.
// The record of the next run with a slice of this warp is fetched into the
// other of the warp's two record buffers while it stages the current one.
__device__ __forceinline__ void mr_gather(const MatmatArgs &a, const CtaInfo &ci, uint32_t nr, const MSmem &sm,
                                          uint32_t gi) {
  const int lane = threadIdx.x & 31;
  const uint32_t c4 = lane & 3, m0 = lane >> 2;
  const RunRec *recs = a.recs + ci.rec_begin;
  uint8_t *rbuf = sm.rec + gi * 2 * kRecBytes;
  // the next run at or after r (slice counter q at r) that holds a slice of this warp
  auto next_own = [&](uint32_t &r, uint32_t &q) {
    for (; r < nr; ++r) {
      const uint32_t nsl = run_slices(sm.lite[r]);
      if ((gi + kGathWarps - q % kGathWarps) % kGathWarps < nsl) return;
      q += nsl;
    }
  };
  auto fetch = [&](uint32_t r, uint32_t b) {
    const uint8_t *src = reinterpret_cast<const uint8_t *>(recs + r);
#pragma unroll
    for (uint32_t o = 0; o < (uint32_t)kRecBytes; o += 512)
      cp_async16cg(rbuf + b * kRecBytes + o + lane * 16, src + o + lane * 16);
  };
  bool ok = true, zbu_ready = false;
  uint32_t r = 0, q = 0, b = 0;
  next_own(r, q);
  if (r < nr) fetch(r, 0);
  while (ok && r < nr) {
    const RunLite L = sm.lite[r];
    const uint32_t nsl = run_slices(L), mine0 = (gi + kGathWarps - q % kGathWarps) % kGathWarps;
    cp_async_wait_all();  // this run's record has landed
    __syncwarp();
    uint32_t rn = r + 1, qn = q + nsl;
    next_own(rn, qn);
    if (rn < nr) fetch(rn, b ^ 1u);
    const uint8_t *rec = rbuf + b * kRecBytes;
    const Run &hdr = *reinterpret_cast<const Run *>(rec);
    const Seg *seg = reinterpret_cast<const Seg *>(rec + sizeof(Run));
    const uint32_t kind = L.flags & 0xffu, vlen = hdr.vlen, nseg = hdr.nseg;
    const float *vec = kind == kRunU ? a.zbu : a.x;
    if (kind == kRunU && !zbu_ready) {
      ok = warp_wait(sm.gdone, 0, a.timeout_ns);  // every CTA's zbu rows are written
      __threadfence();
      zbu_ready = true;
      if (!ok) break;
    }
    uint32_t si = 0;  // this lane's segment cursor (segments are in stage order)
    for (uint32_t s = mine0; s < nsl && ok; s += kGathWarps) {
      const uint32_t qs = q + s, slot = qs % kXStages;
      if (qs >= (uint32_t)kXStages) ok = warp_wait(&sm.xempty[slot], ((qs / kXStages) - 1) & 1, a.timeout_ns);
      if (!ok) break;
      float *st = reinterpret_cast<float *>(sm.xst + slot * kSliceBytes);
      const uint32_t ncol = min((uint32_t)kSliceCols, 4u * L.npanel - s * kSliceCols);
      for (uint32_t k = 0; k < ncol / 4; ++k) {
        const uint32_t sc = s * kSliceCols + 4 * k + c4;  // stage column of this lane
        while (si < nseg && (uint32_t)seg[si].dst + seg[si].len <= sc) ++si;
        float *dst = st + k * (kChunkXBytes / 4) + c4;
        if (sc < vlen && si < nseg && seg[si].dst <= sc) {
          const float *src = vec + (size_t)(seg[si].src + (sc - seg[si].dst)) * kNrhs;
#pragma unroll
          for (uint32_t t = 0; t < 8; ++t) cp_async4(dst + (m0 + 8 * t) * 4, src + m0 + 8 * t);
        } else {
#pragma unroll
          for (uint32_t t = 0; t < 8; ++t) dst[(m0 + 8 * t) * 4] = 0.0f;
        }
      }
      cp_async_wait_all();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor cores
      __syncwarp();
      if (lane == 0) {
        st_release_s(&sm.xcnt[slot], qs / kXStages + 1);
        mbar_arrive(&sm.xfull[slot]);
      }
    }
    r = rn;
    q = qn;
    b ^= 1u;
  }
  if (!ok && lane == 0) atomicOr(a.err, kErrPipeline);
  cp_async_wait_all();
}

// One thread's bounded wait until a shared counter reaches `need`.
__device__ __forceinline__ bool thread_count_wait(const unsigned *cnt, unsigned need, uint64_t timeout_ns) {
  if (ld_acquire_s(cnt) >= need) return true;
  const uint64_t t0 = gtimer();
  while (ld_acquire_s(cnt) < need)
    if (gtimer() - t0 > timeout_ns) return false;
  return true;
}

// ---- MMA thread ---------------------------------------------------------------
// Per slice: wait for its X stage and for every ring chunk its panel pairs
// touch (at most 16 KB of pairs, two chunks), then issue its MMAs back to
// back with the descriptors advanced in place, and commit the stage back.
__device__ __forceinline__ void mr_mma(const MatmatArgs &a, uint32_t nr, uint32_t K, const MSmem &sm, uint32_t me) {
  const RunLite *lite = sm.lite;
  const uint64_t tmo = a.timeout_ns;
  const uint32_t tbase = *sm.tmem;
  const uint32_t ring_s = smem_u32(sm.ring), xst_s = smem_u32(sm.xst);
  uint32_t waited = 0, released = 0, q = 0, nb = 0, nbk = 0;  // nb: blocks so far, nbk: this issuer's
  bool ok = true, first = true;
  // Releases ring chunks below c once the MMAs issued so far are done with
  // them; a chunk is waited for (full) before its release, so the empty
  // phases stay in order.
  auto release_below = [&](uint32_t c) {
    while (ok && released < c) {
      if (waited <= released) {
        ok = mbar_wait(&sm.full[released % kMRingChunks], (released / kMRingChunks) & 1, tmo);
        if (!ok) return;
        waited = released + 1;
      }
      tc_commit(&sm.empty[released % kMRingChunks]);
      ++released;
    }
  };
  for (uint32_t r = 0; r < nr && ok; ++r) {
    const RunLite L = lite[r];
    if (empty_block(L)) continue;
    if ((nb & 1u) != me) {  // the other issuer's block: count its slices
      q += run_slices(L);
      if (L.flags & kLast) ++nb;
      continue;
    }
    const uint32_t h = L.nrow, n8 = (h + 7u) & ~7u, pb = 16u * h;
    const uint32_t idesc = idesc_tf32(kNrhs, n8);
    const uint32_t buf = 2u * me + (nbk & 1u);
    const uint32_t dtm = tbase + buf * kAccCols;
    if (L.flags & kFirst) {
      // Hand back the ring chunks below this block first: the epilogue takes
      // the blocks in order, so the other issuer's earlier block (which may
      // still need those chunks refilled) must not wait on this issuer.
      release_below(L.pos >> kMChunkLog);
      // the epilogue has read this accumulator's previous block
      if (nbk >= 2 && !(ok = mbar_wait(&sm.accempty[buf], ((nbk >> 1) - 1) & 1, tmo))) break;
      tc_fence_after();  // the epilogue's TMEM reads come before these MMAs' writes
      first = true;
    }
    const uint32_t nsl = run_slices(L), npair = L.npanel / 2u;
    for (uint32_t s = 0; s < nsl && ok; ++s, ++q) {
      const uint32_t slot = q % kXStages;
      const uint32_t p0 = s * (kSliceCols / 8), p1 = min(npair, p0 + kSliceCols / 8);
      const uint32_t pos0 = L.pos + 2u * p0 * pb, pos1 = L.pos + 2u * p1 * pb;
      release_below(pos0 >> kMChunkLog);
      const uint32_t clast = (pos1 - 1u) >> kMChunkLog;
      while (ok && waited <= clast) {
        ok = mbar_wait(&sm.full[waited % kMRingChunks], (waited / kMRingChunks) & 1, tmo);
        waited += ok ? 1u : 0u;
      }
      // The stage's fill count first: the other issuer may not have taken
      // the slot's previous slice yet, and a parity wait two phases ahead
      // would return at once.
      if (ok) ok = thread_count_wait(&sm.xcnt[slot], q / kXStages + 1, tmo);
      if (ok) ok = mbar_wait(&sm.xfull[slot], (q / kXStages) & 1, tmo);
      if (!ok) break;
      uint64_t adesc = smem_desc(xst_s + slot * kSliceBytes, kChunkXBytes, 128);
      uint32_t baddr = ring_s + ((pos0 >> kMChunkLog) % kMRingChunks) * kMChunkBytes + (pos0 & (kMChunkBytes - 1));
      const uint64_t bhi = smem_desc(0, pb, 128);  // the descriptor without its address
      for (uint32_t p = p0; p < p1; ++p) {
        mma_tf32(dtm, adesc, bhi | (uint64_t)((baddr >> 4) & 0x3fffu), idesc, first ? 0u : 1u);
        first = false;
        adesc += (2u * kChunkXBytes) >> 4;  // the next two K chunks of the stage
        baddr += 2u * pb;
        if (baddr >= ring_s + kMRingBytes) baddr -= kMRingBytes;  // a pair that starts past the ring's end
      }
      tc_commit(&sm.xempty[slot]);  // the stage slot is free once these MMAs are done
    }
    if (ok && (L.flags & kLast)) {
      tc_commit(&sm.accfull[buf]);
      ++nbk;
      ++nb;
    }
  }
  release_below(K);
  if (!ok) atomicOr(a.err, kErrPipeline);
  // every MMA has completed before TMEM is handed back
  tc_commit(sm.mdone);
  mbar_wait(sm.mdone, 0, tmo);
}

// ---- epilogue warps -----------------------------------------------------------
// Warp w reads TMEM lanes 32w..32w+31 (rhs 16w + lane for lane < 16): all of
// a block's columns (its rows) first, then, for D and U blocks, all the Y
// values it updates, so each block costs one round trip of each kind.
__device__ __forceinline__ void tmem_ld8_async(uint32_t taddr, uint32_t *r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

__device__ __forceinline__ void mr_epilogue(const MatmatArgs &a, uint32_t nr, uint32_t nblk_p, const MSmem &sm) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t m = 16u * w + lane;  // right-hand side of this thread's TMEM lane (lane < 16)
  const uint32_t tlane = (32u * (uint32_t)w) << 16;  // this warp's TMEM lane quarter
  uint32_t nb = 0, np_done = 0;
  if (nblk_p == 0 && lane == 0) mbar_arrive(sm.pdone);
  bool ok = true;
  for (uint32_t r = 0; r < nr && ok; ++r) {
    const RunLite L = sm.lite[r];
    if (!(L.flags & kLast)) continue;
    const uint32_t h = L.nrow, kind = L.flags & 0xffu;
    if (empty_block(L)) {
      // no columns: D rows are beta * yin, P rows zero, U rows unchanged
      if (lane < 16)
        for (uint32_t i = 0; i < h; ++i) {
          const size_t o = (size_t)(L.out + i) * kNrhs + m;
          if (kind == kRunD) a.y[o] = a.beta != 0.0 ? a.beta * a.yin[o] : 0.0;
          else if (kind == kRunP) a.zbu[o] = 0.0f;
        }
      __syncwarp();
      if (kind == kRunP && ++np_done == nblk_p && lane == 0) mbar_arrive(sm.pdone);
      continue;
    }
    // block nb: issuer nb & 1, that issuer's block nbk = nb >> 1 in its accumulator nbk & 1
    const uint32_t nbk = nb >> 1, buf = 2u * (nb & 1u) + (nbk & 1u);
    ok = warp_wait(&sm.accfull[buf], (nbk >> 1) & 1, a.timeout_ns);
    if (!ok) break;
    tc_fence_after();
    const uint32_t taddr = *sm.tmem + tlane + buf * kAccCols;
    // 16 rows at a time: their columns from TMEM, then (D with beta, U) the
    // Y values they update, then the stores
    const bool add = kind == kRunU || (kind == kRunD && a.beta != 0.0);
    const double *src = kind == kRunU ? a.y : a.yin;
    const double c = kind == kRunU ? 1.0 : a.beta;
    for (uint32_t r0 = 0; r0 < h; r0 += 16) {
      uint32_t v[16];
      tmem_ld8_async(taddr + r0, v);
      if (r0 + 8 < h) tmem_ld8_async(taddr + r0 + 8, v + 8);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (lane < 16) {
        const size_t o0 = (size_t)(L.out + r0) * kNrhs + m;
        const uint32_t n = min(16u, h - r0);
        if (kind == kRunP) {
#pragma unroll
          for (uint32_t i = 0; i < 16; ++i)
            if (i < n) a.zbu[o0 + (size_t)i * kNrhs] = __uint_as_float(v[i]);
        } else {
          double old[16];
#pragma unroll
          for (uint32_t i = 0; i < 16; ++i) old[i] = (add && i < n) ? src[o0 + (size_t)i * kNrhs] : 0.0;
#pragma unroll
          for (uint32_t i = 0; i < 16; ++i)
            if (i < n) a.y[o0 + (size_t)i * kNrhs] = fma(a.alpha, (double)__uint_as_float(v[i]), c * old[i]);
        }
      }
    }
    tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.accempty[buf]);
    if (kind == kRunP && ++np_done == nblk_p && lane == 0) mbar_arrive(sm.pdone);  // this warp's zbu rows are out
    ++nb;
  }
  if (!ok && lane == 0) atomicOr(a.err, kErrPipeline);
}

__global__ void __launch_bounds__(kThreadsM, 1) k_matmat(MatmatArgs a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const MSmem sm = mlayout(smem_raw);
  const CtaInfo ci = a.ctas[blockIdx.x];
  const uint32_t nr = ci.nr_p + ci.nr_d + ci.nr_u;
  const uint32_t K = (ci.stream_bytes + kMChunkBytes - 1) >> kMChunkLog;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kMRingChunks; ++i) {
      mbar_init(&sm.full[i], 1);
      mbar_init(&sm.empty[i], kIssuers);  // both issuers hand every chunk back
    }
    for (int i = 0; i < kXStages; ++i) {
      mbar_init(&sm.xfull[i], 1);
      mbar_init(&sm.xempty[i], 1);
      sm.xcnt[i] = 0;
    }
    for (int i = 0; i < 2 * kIssuers; ++i) {
      mbar_init(&sm.accfull[i], 1);
      mbar_init(&sm.accempty[i], kEpiWarps);
    }
    mbar_init(sm.pdone, kEpiWarps);
    mbar_init(sm.gdone, 1);
    mbar_init(sm.mdone, kIssuers);
    *sm.gen0 = grid_gen0(a.gbar);
    mbar_fence_init();
  }
  {  // the CTA's run summaries
    const uint4 *src = reinterpret_cast<const uint4 *>(a.lite + ci.rec_begin);
    uint4 *dst = reinterpret_cast<uint4 *>(sm.lite);
    for (uint32_t k = threadIdx.x; k < nr; k += blockDim.x) dst[k] = __ldg(src + k);
  }
  if (w == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(sm.tmem)),
                 "r"((uint32_t)kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  if (w == kProdWarpM) {
    if (lane == 0 && K > 0) mr_producer(a.stream + ci.stream_off, ci.stream_bytes, sm.ring, sm.full, sm.empty, a.err, a.timeout_ns);
    return;
  }
  if (w >= kGathWarp0 && w < kGathWarp0 + kGathWarps) {
    mr_gather(a, ci, nr, sm, (uint32_t)(w - kGathWarp0));
    return;
  }
  if (w == kSyncWarpM) {
    if (lane == 0) {
      if (!mbar_wait(sm.pdone, 0, a.timeout_ns)) {
        atomicOr(a.err, kErrPipeline);
        return;
      }
      const unsigned target = grid_target(*sm.gen0, 0, gridDim.x);
      grid_arrive(a.gbar, target);
      if (!grid_wait(a.gbar, target, a.timeout_ns)) {
        atomicOr(a.err, kErrGridBarrier);
        return;
      }
      mbar_arrive(sm.gdone);
    }
    return;
  }
  if (w == kMmaWarp2) {
    if (lane == 0) mr_mma(a, nr, K, sm, 1);
    return;  // its MMAs are complete (mdone) before warp kMmaWarp frees TMEM
  }
  if (w == kMmaWarp) {
    if (lane == 0) mr_mma(a, nr, K, sm, 0);
    __syncwarp();
  } else {
    mr_epilogue(a, nr, ci.nblk_p, sm);
  }
  // TMEM goes back once the MMAs are complete and the epilogue has read it
  tc_fence_before();
  named_bar(2, (kEpiWarps + 1) * 32);
  tc_fence_after();
  if (w == kMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*sm.tmem), "r"((uint32_t)kTmemCols)
                 : "memory");
}

}  // namespace

size_t matmat_smem_bytes() { return MLayout::bytes; }

cudaError_t configure_matmat() {
  return cudaFuncSetAttribute(k_matmat, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLayout::bytes);
}

cudaError_t launch_matmat(const MatmatArgs &a, int num_ctas, cudaStream_t s) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(num_ctas);
  cfg.blockDim = dim3(kThreadsM);
  cfg.dynamicSmemBytes = MLayout::bytes;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_matmat, a);
}

}  // namespace hbx
