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
// All kernels run one CTA per SM: 16 consumer warps, one producer warp and
// one descriptor warp.  The producer streams the CTA's packed runs through a
// shared-memory ring with cp.async.bulk; consumer warps own interleaved
// column pairs of every run (rotated so the work stays balanced) and
// accumulate in registers.  Grid-wide dependencies (zbu complete, dot
// products complete) use a bounded grid barrier; the launch is cooperative so
// every CTA is resident.
#include "hbx_device.cuh"
#include "hbx_engine.h"

namespace hbx {
namespace {

constexpr int NW = kConsumerWarps;
constexpr int kConsumerThreads = NW * 32;

struct Smem {
  uint8_t *ring;
  uint64_t *full, *empty;
  double *red;    // [2*kGroup][NW][64]
  uint2 *binfo;   // [2*kGroup] (out, h | kind << 16) of the pending block ends
  double *scal;   // 64 doubles
  uint8_t *stage; // [kStages][kStageBytes]
  uint8_t *rec;   // [kRecSlots] run records
  uint64_t *rfull;
  Run *hdr;       // [kStages] headers of the staged runs
  uint64_t *sfull, *sempty;
  uint64_t *xready, *garrive;
  unsigned *gen;
};

__device__ __forceinline__ Smem smem_layout(uint8_t *base) {
  Smem s;
  s.ring = base + SharedLayout::ring;
  s.full = reinterpret_cast<uint64_t *>(base + SharedLayout::full);
  s.empty = reinterpret_cast<uint64_t *>(base + SharedLayout::empty);
  s.red = reinterpret_cast<double *>(base + SharedLayout::red);
  s.scal = reinterpret_cast<double *>(base + SharedLayout::scal);
  s.stage = base + SharedLayout::stage;
  s.rec = base + SharedLayout::rec;
  s.rfull = reinterpret_cast<uint64_t *>(base + SharedLayout::rfull);
  s.hdr = reinterpret_cast<Run *>(base + SharedLayout::hdr);
  s.sfull = reinterpret_cast<uint64_t *>(base + SharedLayout::sfull);
  s.sempty = reinterpret_cast<uint64_t *>(base + SharedLayout::sempty);
  s.xready = reinterpret_cast<uint64_t *>(base + SharedLayout::xready);
  s.garrive = reinterpret_cast<uint64_t *>(base + SharedLayout::garrive);
  s.gen = reinterpret_cast<unsigned *>(base + SharedLayout::gen);
  s.binfo = reinterpret_cast<uint2 *>(base + SharedLayout::binfo);
  return s;
}

__device__ __forceinline__ void init_barriers(const Smem &s) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < kRingChunks; ++i) {
      mbar_init(&s.full[i], 1);
      mbar_init(&s.empty[i], NW);
    }
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&s.sfull[i], 33);  // 32 cp.async arrivals of the gather warp + its lane 0
      mbar_init(&s.sempty[i], NW);
    }
    for (uint32_t i = 0; i < kRecSlots; ++i) mbar_init(&s.rfull[i], 1);
    mbar_init(s.xready, 1);
    mbar_init(s.garrive, 1);
    mbar_fence_init();
  }
  __syncthreads();
}

__device__ __forceinline__ uint32_t run_end(const Run &r) { return r.pos + run_bytes(r); }

// Cross-warp sums of the finished blocks.  A warp that finishes its part of
// a block writes its 64 partial sums (rows lane and lane + 32) to red buffer
// nae % (2 kGroup); after
// every kGroup blocks (and at the end of a section) one CTA barrier makes
// them visible and warp (block mod NW) sums each pending block in warp order
// and writes its rows:  kind P: zbu[out+i] = s;  D: y = alpha*s + beta*yin;
// U: y += alpha*s.  A group's buffers are refilled only after the next
// group's barrier, which its summing warps pass after they have summed.
struct BlockEnds {
  uint32_t nae = 0;   // blocks finished so far (the same in every warp)
  uint32_t pend = 0;  // finished but not yet summed
};

__device__ __forceinline__ void flush_block_ends(BlockEnds &B, const Smem &sm, double alpha, double beta,
                                                 const double *yin, double *y, double *zbu, float *zbu32,
                                                 const Ring &R) {
  if (B.pend == 0) return;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  named_bar(2, kConsumerThreads);
  for (uint32_t q = B.nae - B.pend; q < B.nae; ++q) {
    if ((uint32_t)w != q % NW || R.bad) continue;
    const uint32_t b = q % (2 * kGroup);
    const uint2 bi = sm.binfo[b];
    const uint32_t h = bi.y & 0xffffu, kind = bi.y >> 16;
    const double *rb = sm.red + b * (NW * 64);
    for (uint32_t row = lane; row < h; row += 32) {
      double s = rb[row];
#pragma unroll
      for (int k = 1; k < NW; ++k) s += rb[k * 64 + row];
      const uint32_t r = bi.x + row;
      if (kind == kRunP) {
        zbu[r] = s;
        if (zbu32) zbu32[r] = (float)s;
        continue;
      }
      if (kind == kRunD) {
        double v = alpha * s;
        if (beta != 0.0) v = fma(beta, yin[r], v);
        y[r] = v;
      } else {
        y[r] = fma(alpha, s, y[r]);
      }
    }
  }
  B.pend = 0;
}

// End of a block: park this warp's partials; sum the group when it is full.
// Before the barrier a warp gives back every ring chunk it will not read
// again, so no warp waits at a barrier while holding chunks others need.
__device__ __forceinline__ void block_end(const Run &run, double &acc, double &acc2, BlockEnds &B, const Smem &sm,
                                          double alpha, double beta, const double *yin, double *y, double *zbu,
                                          float *zbu32, Ring &R) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  R.release_below(R.base + (run_end(run) >> kChunkLog));
  const uint32_t b = B.nae % (2 * kGroup);
  sm.red[b * (NW * 64) + w * 64 + lane] = acc;
  sm.red[b * (NW * 64) + w * 64 + 32 + lane] = acc2;
  if (w == 0 && lane == 0) sm.binfo[b] = make_uint2(run.out, (uint32_t)run.nrow | (run_kind(run) << 16));
  acc = 0.0;
  acc2 = 0.0;
  ++B.nae;
  if (++B.pend == kGroup) flush_block_ends(B, sm, alpha, beta, yin, y, zbu, zbu32, R);
}

// Consumer view of the stage ring: run g (counted over sections and passes)
// is in slot g % kStages.
struct StageQ {
  uint32_t g;
};

// Runs a section: waits for each run's staged vector, processes it, and
// gives the slot back.  Before a wait the warp gives back the ring chunks of
// the previous run, so no warp blocks while holding chunks the others need.
// process(run, stage) returns the stream position where the run ends.
template <class F>
__device__ __forceinline__ void run_section(uint32_t nruns, StageQ &Q, const Smem &sm, Ring &R, int *err,
                                            F &&process) {
  uint32_t rend = 0;
  for (uint32_t k = 0; k < nruns; ++k) {
    const uint32_t g = Q.g + k, slot = g % kStages;
    if (k > 0) R.release_below(R.base + (rend >> kChunkLog));
    if (!R.bad && !warp_wait(&sm.sfull[slot], (g / kStages) & 1, R.timeout_ns)) {
      R.bad = true;
      if ((threadIdx.x & 31) == 0) atomicOr(err, kErrPipeline);
    }
    Run run = sm.hdr[slot];
    if (R.bad) run.npanel = 0;  // after a timed-out wait: touch neither the stage nor the ring
    rend = process(run, smem_u32(sm.stage + slot * kStageBytes));
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(&sm.sempty[slot]);
  }
  Q.g += nruns;
}

// One H-matvec over this CTA's stream (pass starting at absolute chunk R.base,
// K chunks long).  The CTA arrives on the grid barrier after its P runs; the
// gather warp waits for the barrier before it stages the first U run, so the
// D runs hide the barrier latency.  Every warp has released the whole pass
// when it returns.
template <bool kF32>
__device__ __forceinline__ void matvec_body(Ring &R, StageQ &Q, uint32_t K, const CtaInfo &ci, double alpha,
                                            double beta, const double *yin, double *y, double *zbu, float *zbu32,
                                            unsigned *gbar, int *err, const Smem &sm, BlockEnds &B,
                                            unsigned long long *prof = nullptr) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto stamp = [&](int k) {
    if (prof && w == 0 && lane == 0) prof[blockIdx.x * 16 + k] = gtimer();
  };
  stamp(0);
  double acc = 0.0, acc2 = 0.0;
  auto block = [&](const Run &run, uint32_t stage_s) {
    run_block<kF32>(run, stage_s, R, acc, acc2);
    if (run.flags & kLast) block_end(run, acc, acc2, B, sm, alpha, beta, yin, y, zbu, zbu32, R);
    return run_end(run);
  };
  // ---- P: zbu = V^T x for this CTA's slabs
  uint32_t pend = 0;
  run_section(ci.nr_p, Q, sm, R, err, [&](const Run &run, uint32_t st) { return pend = block(run, st); });
  R.release_below(R.base + (pend >> kChunkLog));
  flush_block_ends(B, sm, alpha, beta, yin, y, zbu, zbu32, R);
  stamp(1);
  if (lane == 0) __threadfence();
  named_bar(1, kConsumerThreads);
  stamp(2);
  unsigned gen = 0;
  if (w == 0 && lane == 0) {
    gen = ld_acquire(&gbar[1]);
    *sm.gen = gen;
    grid_arrive(gbar, gridDim.x);
    mbar_arrive(sm.garrive);
  }
  // ---- D: dense rows of the owned atoms
  uint32_t dend = pend;
  run_section(ci.nr_d, Q, sm, R, err, [&](const Run &run, uint32_t st) { return dend = block(run, st); });
  R.release_below(R.base + (dend >> kChunkLog));
  flush_block_ends(B, sm, alpha, beta, yin, y, zbu, zbu32, R);
  stamp(3);
  stamp(4);
  // ---- U: U rows of the owned atoms times zbu (staged after the grid barrier)
  run_section(ci.nr_u, Q, sm, R, err, [&](const Run &run, uint32_t st) { return block(run, st); });
  R.release_below(R.base + K);
  flush_block_ends(B, sm, alpha, beta, yin, y, zbu, zbu32, R);
  // The barrier counts arrivals per instance: this CTA may arrive on the
  // next instance only once this one is complete (a CTA without U runs has
  // not waited for it yet).
  if (w == 0 && lane == 0 && !grid_wait(gbar, gen, R.timeout_ns)) atomicOr(err, kErrGridBarrier);
  stamp(5);
}

template <bool kF32>
__global__ void __launch_bounds__(kThreads, 1) k_matvec(MatvecArgs a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const Smem sm = smem_layout(smem_raw);
  const CtaInfo ci = a.ctas[blockIdx.x];
  init_barriers(sm);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t K = (ci.stream_bytes + kChunkBytes - 1) >> kChunkLog;
  if (w == kProducerWarp) {
    if (lane == 0 && K > 0)
      producer_run(a.stream + ci.stream_off, ci.stream_bytes, 1, sm.ring, sm.full, sm.empty, a.err, a.timeout_ns);
    return;
  }
  if (w == kGatherWarp) {
    const void *xs = kF32 ? static_cast<const void *>(a.x32) : static_cast<const void *>(a.x);
    const void *zs = kF32 ? static_cast<const void *>(a.zbu32) : static_cast<const void *>(a.zbu);
    const GatherCtx c{a.recs + ci.rec_begin, ci.nr_p, ci.nr_d, ci.nr_u, 1, xs, xs, zs, a.gbar, a.err,
                      a.timeout_ns};
    gather_warp<kF32>(c, sm);
    return;
  }
  if (threadIdx.x == 0) mbar_arrive(sm.xready);  // x is an input: ready from the start
  Ring R{sm.ring, sm.full, sm.empty, 0, 0, 0, a.timeout_ns, a.err, false};
  StageQ Q{0};
  BlockEnds B;
  matvec_body<kF32>(R, Q, K, ci, a.alpha, a.beta, a.yin, a.y, a.zbu, kF32 ? a.zbu32 : nullptr, a.gbar, a.err, sm, B,
                    a.prof);
  R.drain(K);
}

// ---------------------------------------------------------------- BiCGSTAB
template <class F>
__device__ __forceinline__ void for_own_rows(const Atom *atoms, const CtaInfo &ci, F f) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t q = w; q < ci.n_atoms; q += NW) {
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
__device__ __forceinline__ double reduce_slot(const double *part, int ncta, int slot) {
  const int lane = threadIdx.x & 31;
  Acc2 a{0.0, 0.0};
  for (int c = lane; c < ncta; c += 32) {
    const double *src = part + ((size_t)c * kSlots + slot) * 2;
    a = acc2_merge(a, Acc2{__ldcg(src), __ldcg(src + 1)});
  }
  a = warp_merge(a);
  return a.s + a.c;
}

// Full grid barrier among the consumer warps of every CTA.
__device__ __forceinline__ bool grid_sync(unsigned *gbar, int *err, uint64_t timeout_ns, const Smem &sm) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  named_bar(1, kConsumerThreads);
  if (w == 0 && lane == 0) {
    const unsigned gen = ld_acquire(&gbar[1]);
    grid_arrive(gbar, gridDim.x);
    const bool ok = grid_wait(gbar, gen, timeout_ns);
    if (!ok) atomicOr(err, kErrGridBarrier);
    sm.scal[62] = ok ? 1.0 : 0.0;
  }
  named_bar(1, kConsumerThreads);
  return sm.scal[62] != 0.0;
}

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

template <bool kF32>
__global__ void __launch_bounds__(kThreads, 1) k_bicg_iter(BicgArgs a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const Smem sm = smem_layout(smem_raw);
  const CtaInfo ci = a.ctas[blockIdx.x];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ncta = gridDim.x;
  auto stamp = [&](int k) {
    if (a.prof && threadIdx.x == 0) a.prof[blockIdx.x * 16 + 8 + k] = gtimer();
  };
  const uint64_t t_start = a.prof ? gtimer() : 0;
  init_barriers(sm);

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
  if (sm.scal[0] != 0.0) return;
  if (a.prof && threadIdx.x == 0) a.prof[blockIdx.x * 16 + 8] = t_start;  // stamps of working steps only
  const double beta = sm.scal[2], zeta_prev = sm.scal[3], rho = sm.scal[4];
  const double relres = sm.scal[5], bnorm = sm.scal[7];
  const int iter = (int)sm.scal[6];

  const uint32_t K = (ci.stream_bytes + kChunkBytes - 1) >> kChunkLog;
  if (w == kProducerWarp) {
    if (lane == 0 && K > 0)
      producer_run(a.stream + ci.stream_off, ci.stream_bytes, 2, sm.ring, sm.full, sm.empty, a.err, a.timeout_ns);
    return;
  }
  if (w == kGatherWarp) {
    const void *x0 = kF32 ? static_cast<const void *>(a.p32) : static_cast<const void *>(a.p);
    const void *x1 = kF32 ? static_cast<const void *>(a.t32) : static_cast<const void *>(a.t);
    const void *zs = kF32 ? static_cast<const void *>(a.zbu32) : static_cast<const void *>(a.zbu);
    const GatherCtx c{a.recs + ci.rec_begin, ci.nr_p, ci.nr_d, ci.nr_u, 2, x0, x1, zs, a.gbar, a.err,
                      a.timeout_ns};
    gather_warp<kF32>(c, sm);
    return;
  }
  Ring R{sm.ring, sm.full, sm.empty, 0, 0, 0, a.timeout_ns, a.err, false};
  StageQ Q{0};
  BlockEnds B;

  // ---- S1: p = r + beta*(p - zeta*Ap)  (p = r on the first step)
  if (beta == 0.0) {
    for_own_rows(a.atoms, ci, [&](uint32_t r) {
      const double v = a.r[r];
      a.p[r] = v;
      if (kF32) a.p32[r] = (float)v;
    });
  } else {
    for_own_rows(a.atoms, ci, [&](uint32_t r) {
      const double v = fma(-zeta_prev, a.ap[r], a.p[r]) * beta;
      const double pv = v + a.r[r];
      a.p[r] = pv;
      if (kF32) a.p32[r] = (float)pv;
    });
  }
  __threadfence();
  grid_sync(a.gbar, a.err, a.timeout_ns, sm);
  if (threadIdx.x == 0) mbar_arrive(sm.xready);  // p complete grid-wide: pass 1 may be staged
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
  matvec_body<kF32>(R, Q, K, ci, 1.0, 0.0, nullptr, a.ap, a.zbu, kF32 ? a.zbu32 : nullptr, a.gbar, a.err, sm, B);
  stamp(2);
  {
    Acc2 acc[1] = {{0, 0}};
    named_bar(1, kConsumerThreads);
    for_own_rows(a.atoms, ci, [&](uint32_t r) { dot2_add(acc[0], a.rh[r], a.ap[r]); });
    cta_partials<1>(acc, a.part, kSlotRhAp, sm);
  }
  grid_sync(a.gbar, a.err, a.timeout_ns, sm);
  if (w == 0) {
    const double zden = reduce_slot(a.part, ncta, kSlotRhAp);
    if (lane == 0) sm.scal[8] = rho / zden;
  }
  named_bar(1, kConsumerThreads);
  const double alpha = sm.scal[8];
  stamp(3);

  // ---- S3: t = r - alpha*Ap
  for_own_rows(a.atoms, ci, [&](uint32_t r) {
    const double v = fma(-alpha, a.ap[r], a.r[r]);
    a.t[r] = v;
    if (kF32) a.t32[r] = (float)v;
  });
  __threadfence();
  grid_sync(a.gbar, a.err, a.timeout_ns, sm);
  if (threadIdx.x == 0) mbar_arrive(sm.xready);  // t complete grid-wide: pass 2 may be staged
  stamp(4);

  // ---- S4: At = H t;  At . t,  At . At
  R.base = K;
  matvec_body<kF32>(R, Q, K, ci, 1.0, 0.0, nullptr, a.at, a.zbu, kF32 ? a.zbu32 : nullptr, a.gbar, a.err, sm, B);
  stamp(5);
  {
    Acc2 acc[2] = {{0, 0}, {0, 0}};
    named_bar(1, kConsumerThreads);
    for_own_rows(a.atoms, ci, [&](uint32_t r) {
      const double atv = a.at[r];
      dot2_add(acc[0], atv, a.t[r]);
      dot2_add(acc[1], atv, atv);
    });
    cta_partials<2>(acc, a.part, kSlotAtT, sm);
  }
  grid_sync(a.gbar, a.err, a.timeout_ns, sm);
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
  {
    Acc2 acc[2] = {{0, 0}, {0, 0}};
    for_own_rows(a.atoms, ci, [&](uint32_t r) {
      const double uv = fma(alpha, a.p[r], a.u[r]);
      a.u[r] = fma(zeta, a.t[r], uv);
      const double rv = fma(-zeta, a.at[r], a.t[r]);
      a.r[r] = rv;
      dot2_add(acc[0], a.rh[r], rv);
      dot2_add(acc[1], rv, rv);
    });
    cta_partials<2>(acc, a.part, kSlotRhoR, sm);
  }
  R.drain(2 * K);
  stamp(7);
}

// part[cta][slot] over own rows, then (block 0 of a second launch) the total.
__global__ void __launch_bounds__(kThreads, 1) k_dot_partial(BicgArgs a, const double *x, const double *y, int slot) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const Smem sm = smem_layout(smem_raw);
  if ((threadIdx.x >> 5) >= NW) return;
  const CtaInfo ci = a.ctas[blockIdx.x];
  Acc2 acc[1] = {{0, 0}};
  for_own_rows(a.atoms, ci, [&](uint32_t r) { dot2_add(acc[0], x[r], y[r]); });
  cta_partials<1>(acc, a.part, slot, sm);
}

// y = (float)x: the input of an FP32 engine's matvec.
__global__ void k_to_float(const double *x, float *y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

// y += a * x (the refinement update of the mixed-precision solve).
__global__ void k_axpy(double a, const double *x, double *y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}

__global__ void k_dot_total(const double *part, int ncta, int slot, double *out) {
  const double v = reduce_slot(part, ncta, slot);
  if (threadIdx.x == 0) *out = v;
}

}  // namespace

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
  if ((e = cudaFuncSetAttribute(k_matvec<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_matvec<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_bicg_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_bicg_iter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_bicg_iter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_dot_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
  return cudaSuccess;
}

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

cudaError_t launch_matvec(const MatvecArgs &a, int num_ctas, cudaStream_t s, int precision) {
  return precision == kFP32 ? launch_coop(k_matvec<true>, a, num_ctas, s) : launch_coop(k_matvec<false>, a, num_ctas, s);
}

cudaError_t launch_bicg_setup(const BicgArgs &a, int num_ctas, cudaStream_t s) {
  k_bicg_setup<<<num_ctas, kThreads, SharedLayout::bytes, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bicg_iter(const BicgArgs &a, int num_ctas, cudaStream_t s, int precision) {
  return precision == kFP32 ? launch_coop(k_bicg_iter<true>, a, num_ctas, s)
                            : launch_coop(k_bicg_iter<false>, a, num_ctas, s);
}

cudaError_t launch_to_float(const double *x, float *y, size_t n, cudaStream_t s) {
  k_to_float<<<296, 256, 0, s>>>(x, y, n);
  return cudaGetLastError();
}

cudaError_t launch_axpy(double alpha, const double *x, double *y, size_t n, cudaStream_t s) {
  k_axpy<<<296, 256, 0, s>>>(alpha, x, y, n);
  return cudaGetLastError();
}

cudaError_t launch_dot(const BicgArgs &a, const double *x, const double *y, int slot, double *out, int num_ctas,
                       cudaStream_t s) {
  k_dot_partial<<<num_ctas, kThreads, SharedLayout::bytes, s>>>(a, x, y, slot);
  k_dot_total<<<1, 32, 0, s>>>(a.part, num_ctas, slot, out);
  return cudaGetLastError();
}

}  // namespace hbx
