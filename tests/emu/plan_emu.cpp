// Test-only CPU interpreter of the engine's packed layout.  It links the
// product's planner/packer (hbx_plan.cpp), walks every CTA's run records the
// way the sm_100a kernel does (P slabs -> zbu, D/U atom blocks -> y), checks
// the layout invariants the kernel relies on (16-byte aligned streams, runs
// back to back inside their CTA stream, gather segments covering each run's
// stage exactly, heights <= 32 (64 for P slabs), atoms partitioning the rows
// exactly once, zbu written once before it is read), and returns y = H x.
// With FP32 or BF16 storage it multiplies the float (bfloat16) factors by
// the float-rounded vector, as the kernel does, but sums in double.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../hacapk-magma_b200/csrc/hbx_plan.h"

using namespace hbx;

static int emu_run(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, int precision, bool pairs, const double *x,
                   double *y, long long *stats, char *msg, int msglen, const PlanCosts &costs = PlanCosts(),
                   int merge_keep = -1) {
  auto bad = [&](const std::string &s) {
    std::snprintf(msg, msglen, "%s", s.c_str());
    return 1;
  };
  Plan plan;
  std::string err;
  int rc = make_plan(st, nd, num_ctas, plan, err, precision, pairs, costs, merge_keep);
  if (rc != 0) return bad("make_plan: " + err);
  std::vector<uint8_t> buf(plan.total_bytes, 0xAB);
  pack_plan(st, plan, buf.data());
  std::vector<double> zbu(plan.zbu_len, NAN);
  std::vector<char> zset(plan.zbu_len, 0);
  std::vector<int> owner(nd, -1);
  std::fill(y, y + nd, NAN);
  long long nruns = 0;
  const uint32_t G = group_cols(precision);
  std::vector<double> stage(kStageBytes / stage_elem_bytes(precision)), acc(kSlabMax);

  // structural checks of one CTA's records; returns "" when fine
  auto check_cta = [&](int c) -> std::string {
    const CtaInfo &ci = plan.ctas[c];
    if (ci.stream_off % 256 != 0 || ci.stream_bytes % 16 != 0) return "stream alignment";
    if (ci.stream_off + ci.stream_bytes > plan.total_bytes) return "stream outside buffer";
    const uint32_t nr = ci.nr_p + ci.nr_d + ci.nr_u;
    if ((uint64_t)ci.rec_begin + nr > plan.recs.size() || plan.lite.size() != plan.recs.size())
      return "records outside the record array";
    uint32_t pos = 0;
    for (uint32_t k = 0; k < nr; ++k) {
      const Run &r = plan.recs[ci.rec_begin + k].hdr;
      uint32_t want = k < ci.nr_p ? kRunP : (k < ci.nr_p + ci.nr_d ? kRunD : kRunU);
      if (want == kRunU && run_kind(r) == kRunDU) want = kRunDU;  // merged blocks sit in the U section
      if (run_kind(r) != want) return "run kind out of section order";
      if (r.nrow == 0 || r.nrow > (want == kRunP ? kSlabMax : kAtomMax)) return "run height outside 1..32 (1..64 for P)";
      const RunLite &L = plan.lite[ci.rec_begin + k];
      if (L.pos != r.pos || L.out != r.out || L.npanel != r.npanel || L.nrow != r.nrow || L.rot != r.rot ||
          L.flags != r.flags)
        return "run summary does not match its record";
      // pair-panel runs (multi-RHS layout) are whole panel pairs
      const uint32_t RG = pairs ? 2 * G : G;
      if (G * r.npanel * stage_elem_bytes(precision) > (uint32_t)kStageBytes || r.vlen > G * r.npanel ||
          (r.npanel > 0 && r.vlen + RG <= G * r.npanel) || (pairs && r.npanel % 2 != 0))
        return "run width";
      if (r.nseg > kRunSegs) return "too many segments";
      if (r.rot >= kProductWarps || L.rot_step >= kStepWarps) return "bad rotation";
      if (r.pos != pos || r.pos % 16 != 0) return "runs not back to back";
      pos += run_bytes(r);
      if (r.vlen != G * r.npanel && !(r.flags & kLast)) return "zero columns outside a block's last run";
      const uint32_t real = r.vlen;
      const uint64_t vmax = want == kRunU ? plan.zbu_len : (uint64_t)nd;
      const bool du = want == kRunDU;
      std::vector<char> cov(real, 0);
      uint32_t d = 0;
      if (r.nlong > r.nseg) return "nlong > nseg";
      for (uint32_t q = 0; q < r.nseg; ++q) {
        const Seg &s = plan.recs[ci.rec_begin + k].seg[q];
        if (s.len == 0 || (uint32_t)s.dst + s.len > real) return "segment outside the stage";
        if (pairs ? (r.nlong != 0 || s.dst != d) : ((q < r.nlong) != (s.len > (uint32_t)kSegShort)))
          return pairs ? "pair-panel segments not in stage order" : "long segments not first";
        const bool z = du && (s.src & kSegZbu);
        const uint64_t src = du ? (s.src & ~kSegZbu) : s.src;
        if (src + s.len > (du ? (z ? plan.zbu_len : (uint64_t)nd) : vmax)) return "segment source out of range";
        for (uint32_t e = 0; e < s.len; ++e) {
          if (cov[s.dst + e]) return "segments overlap";
          cov[s.dst + e] = 1;
        }
        d += s.len;
      }
      if (d != real) return "segments cover " + std::to_string(d) + " of " + std::to_string(real) + " columns";
      if (want == kRunP && (uint64_t)r.out + r.nrow > plan.zbu_len) return "P rows outside zbu";
      if (want != kRunP && (uint64_t)r.out + r.nrow > (uint64_t)nd) return "atom rows outside [0, nd)";
    }
    if (pos != ci.stream_bytes) return "stream length mismatch";
    return "";
  };
  // one run: gather, multiply its pair panels, finish the block on its last run
  // vec: the run's vector; a kRunDU run picks x or zbu per segment
  auto run_one = [&](const CtaInfo &ci, uint32_t k, const double *vec) {
    const RunRec &R = plan.recs[ci.rec_begin + k];
    const Run &r = R.hdr;
    const bool du = run_kind(r) == kRunDU;
    for (uint32_t q = 0; q < r.nseg; ++q)
      for (uint32_t e = 0; e < R.seg[q].len; ++e) {
        const uint32_t sv = R.seg[q].src;
        const double v = du ? ((sv & kSegZbu) ? zbu[(sv & ~kSegZbu) + e] : x[sv + e]) : vec[sv + e];
        stage[R.seg[q].dst + e] = precision != kFP64 ? (double)(float)v : v;
      }
    for (uint32_t c = r.vlen; c < G * r.npanel; ++c) stage[c] = 0.0;
    if (r.flags & kFirst) std::fill(acc.begin(), acc.end(), 0.0);
    const double *d = reinterpret_cast<const double *>(buf.data() + ci.stream_off + r.pos);
    const float *f = reinterpret_cast<const float *>(buf.data() + ci.stream_off + r.pos);
    const uint16_t *hb = reinterpret_cast<const uint16_t *>(buf.data() + ci.stream_off + r.pos);
    for (uint32_t j = 0; j < r.npanel; ++j)
      for (uint32_t i = 0; i < r.nrow; ++i)
        for (uint32_t c = 0; c < G; ++c) {
          const size_t k = ((size_t)j * r.nrow + i) * G + c;
          const double m = precision == kBF16 ? (double)bf16_to_float(hb[k])
                                              : (precision == kFP32 ? (double)f[k] : d[k]);
          acc[i] += m * stage[G * j + c];
        }
    ++nruns;
  };

  for (int c = 0; c < plan.num_ctas; ++c) {
    std::string e = check_cta(c);
    if (!e.empty()) return bad("cta " + std::to_string(c) + ": " + e);
  }
  // pass 1: P runs of every CTA
  for (int c = 0; c < plan.num_ctas; ++c) {
    const CtaInfo &ci = plan.ctas[c];
    for (uint32_t k = 0; k < ci.nr_p; ++k) {
      run_one(ci, k, x);
      const Run &r = plan.recs[ci.rec_begin + k].hdr;
      if (r.flags & kLast)
        for (uint32_t i = 0; i < r.nrow; ++i) {
          if (zset[r.out + i]) return bad("zbu entry written twice");
          zbu[r.out + i] = acc[i];
          zset[r.out + i] = 1;
        }
    }
  }
  for (uint64_t i = 0; i < plan.zbu_len; ++i)
    if (!zset[i]) return bad("zbu entry never written");
  // pass 2: D then U runs
  for (int c = 0; c < plan.num_ctas; ++c) {
    const CtaInfo &ci = plan.ctas[c];
    uint32_t owned = 0;
    for (uint32_t k = ci.nr_p; k < ci.nr_p + ci.nr_d + ci.nr_u; ++k) {
      const Run &r = plan.recs[ci.rec_begin + k].hdr;
      const bool is_du = run_kind(r) == kRunDU;
      const bool is_u = k >= ci.nr_p + ci.nr_d && !is_du;  // adds to rows an earlier D block wrote
      run_one(ci, k, is_u ? zbu.data() : x);
      if (!(r.flags & kLast)) continue;
      for (uint32_t i = 0; i < r.nrow; ++i) {
        const uint32_t row = r.out + i;
        if (!is_u) {
          if (owner[row] != -1) return bad("row written by two atoms");
          owner[row] = c;
          y[row] = acc[i];
        } else {
          if (owner[row] != c) return bad("U run writes a row the CTA does not own");
          y[row] += acc[i];
        }
      }
      if (!is_u) {
        if (owned >= ci.n_atoms) return bad("more D blocks than owned atoms");
        const Atom &A = plan.atoms[ci.atom_begin + owned];
        if (A.r0 != r.out || A.h != r.nrow) return bad("owned-atom list does not match the D blocks");
        ++owned;
      }
    }
    if (owned != ci.n_atoms) return bad("owned atoms without a D block");
  }
  for (int r = 0; r < nd; ++r)
    if (owner[r] < 0) return bad("row " + std::to_string(r) + " not owned by any atom");
  if (stats) {
    stats[0] = (long long)plan.total_bytes;
    stats[1] = nruns;
    stats[2] = (long long)plan.atoms.size();
    stats[3] = (long long)plan.zbu_len;
    stats[4] = (long long)plan.alg_bytes;
    uint64_t mx = 0, sum = 0;
    for (auto &ci : plan.ctas) { mx = std::max<uint64_t>(mx, ci.stream_bytes); sum += ci.stream_bytes; }
    stats[5] = (long long)mx;
    stats[6] = (long long)sum;
    stats[7] = (long long)plan.pad_bytes;
  }
  return 0;
}

extern "C" int emu_matvec_prec(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, int precision, const double *x,
                               double *y, long long *stats, char *msg, int msglen) {
  return emu_run(st, nd, num_ctas, precision, false, x, y, stats, msg, msglen);
}

// The multi-RHS engine's layout (FP32 factors, runs of whole panel pairs,
// segments in stage order), one right-hand side at a time.
extern "C" int emu_matvec_pairs(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, const double *x, double *y,
                                long long *stats, char *msg, int msglen) {
  return emu_run(st, nd, num_ctas, kFP32, true, x, y, stats, msg, msglen);
}

// The layout under another balancing cost model (what hbx_autotune tries).
extern "C" int emu_matvec_costs(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, long long block_cost,
                                long long run_cost, const double *x, double *y, long long *stats, char *msg,
                                int msglen) {
  PlanCosts c;
  c.block = (uint64_t)block_cost;
  c.run = (uint64_t)run_cost;
  return emu_run(st, nd, num_ctas, kFP64, false, x, y, stats, msg, msglen, c);
}

// Several independent H-matrices as one block-diagonal engine layout.
extern "C" int emu_matvec_batch(const stc_HACApK_leafmtxp *const *st, const int *nd, int count, int num_ctas,
                                const double *x, double *y, long long *stats, char *msg, int msglen) {
  CombinedLeaves cl;
  std::string err;
  if (combine_leaves(st, nd, count, cl, err) != 0) {
    std::snprintf(msg, msglen, "combine_leaves: %s", err.c_str());
    return 1;
  }
  return emu_run(&cl.container, cl.off[count], num_ctas, kFP64, false, x, y, stats, msg, msglen);
}

extern "C" int emu_matvec(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, const double *x, double *y,
                          long long *stats, char *msg, int msglen) {
  return emu_matvec_prec(st, nd, num_ctas, kFP64, x, y, stats, msg, msglen);
}

// The same walk over the packed layout of H^T (hbx_plan.cpp:transpose_leaves).
extern "C" int emu_matvec_transposed(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, const double *x, double *y,
                                     long long *stats, char *msg, int msglen) {
  TransposedLeaves tl;
  std::string err;
  if (transpose_leaves(st, nd, tl, err) != 0) {
    std::snprintf(msg, msglen, "transpose_leaves: %s", err.c_str());
    return 1;
  }
  return emu_matvec(&tl.container, nd, num_ctas, x, y, stats, msg, msglen);
}

// bfloat16 rounding of the packer, one value at a time (checked against an
// independent restatement in the tests).
extern "C" unsigned emu_bf16_from_double(double v) { return bf16_from_double(v); }

// FNV-1a digest of everything a plan hands to the device: run records, run
// summaries, CTA table, owned atoms and the packed stream.
extern "C" unsigned long long emu_plan_digest(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, int precision,
                                              int pairs) {
  Plan plan;
  std::string err;
  if (make_plan(st, nd, num_ctas, plan, err, precision, pairs != 0) != 0) return 0;
  std::vector<uint8_t> buf(plan.total_bytes, 0);
  pack_plan(st, plan, buf.data());
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&](const void *p, size_t n) {
    const uint8_t *b = static_cast<const uint8_t *>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  };
  mix(plan.recs.data(), plan.recs.size() * sizeof(RunRec));
  mix(plan.lite.data(), plan.lite.size() * sizeof(RunLite));
  mix(plan.ctas.data(), plan.ctas.size() * sizeof(CtaInfo));
  mix(plan.atoms.data(), plan.atoms.size() * sizeof(Atom));
  mix(buf.data(), buf.size());
  return h;
}

// The layout with merged D+U blocks (make_plan's merge_keep), FP64 or any
// storage precision.
extern "C" int emu_matvec_merged(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, int precision, int merge_keep,
                                 const double *x, double *y, long long *stats, char *msg, int msglen) {
  return emu_run(st, nd, num_ctas, precision, false, x, y, stats, msg, msglen, PlanCosts(), merge_keep);
}

// Per-CTA stream bytes and run counts of a plan (merge_keep as make_plan's).
extern "C" int emu_plan_cta_table(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, int precision, int merge_keep,
                                  long long *bytes, int *runs) {
  Plan plan;
  std::string err;
  if (make_plan(st, nd, num_ctas, plan, err, precision, false, PlanCosts(), merge_keep) != 0) return 1;
  for (int c = 0; c < num_ctas; ++c) {
    bytes[c] = plan.ctas[c].stream_bytes;
    runs[c] = (int)(plan.ctas[c].nr_p + plan.ctas[c].nr_d + plan.ctas[c].nr_u);
  }
  return 0;
}

// Per-CTA run counts by section (P, D, U) of a plan.
extern "C" int emu_plan_cta_sections(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, int precision,
                                     int merge_keep, int *np, int *ndr, int *nu, int *natoms) {
  Plan plan;
  std::string err;
  if (make_plan(st, nd, num_ctas, plan, err, precision, false, PlanCosts(), merge_keep) != 0) return 1;
  for (int c = 0; c < num_ctas; ++c) {
    np[c] = (int)plan.ctas[c].nr_p;
    ndr[c] = (int)plan.ctas[c].nr_d;
    nu[c] = (int)plan.ctas[c].nr_u;
    natoms[c] = (int)plan.ctas[c].n_atoms;
  }
  return 0;
}

// y = alpha H x + beta yin in the FP64 kernel's own operation order, so that
// it equals k_matvec bit for bit (merge_keep as make_plan's; merged D+U runs
// gather x or zbu per segment and write like D blocks): consumer warp w takes panels
// j = (w - rot) mod 16, j + 16, ... of every run, four at a time (two for P
// slabs taller than 32 rows, whose lanes also carry row lane + 32) into
// accumulator pairs (one fma per column), folds them into its block sum at
// the end of the run (a0 + a1, accumulators in order), and the block-sum
// warp adds the 16 warps' sums in warp order; P blocks write zbu, D blocks
// y = alpha s (+ beta yin), U blocks y = fma(alpha, s, y).
extern "C" int emu_matvec_kernel_order_mk(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, int merge_keep,
                                          double alpha, const double *x, double beta, const double *yin, double *y) {
  Plan plan;
  std::string err;
  if (make_plan(st, nd, num_ctas, plan, err, kFP64, false, PlanCosts(), merge_keep) != 0) return 1;
  std::vector<uint8_t> buf(plan.total_bytes, 0);
  pack_plan(st, plan, buf.data());
  std::vector<double> zbu(plan.zbu_len, 0.0), stage(kStageBytes / 8);
  constexpr int NW = kConsumerWarps;
  std::vector<double> t0(NW * 32), t1(NW * 32);
  auto do_pass = [&](int phase) {  // phase 0: P runs; 1: D then U runs
    for (int c = 0; c < plan.num_ctas; ++c) {
      const CtaInfo &ci = plan.ctas[c];
      const uint32_t k0 = phase == 0 ? 0 : ci.nr_p, k1 = phase == 0 ? ci.nr_p : ci.nr_p + ci.nr_d + ci.nr_u;
      std::fill(t0.begin(), t0.end(), 0.0);
      std::fill(t1.begin(), t1.end(), 0.0);
      for (uint32_t k = k0; k < k1; ++k) {
        const RunRec &R = plan.recs[ci.rec_begin + k];
        const Run &r = R.hdr;
        const bool du = run_kind(r) == kRunDU;  // merged D+U: writes like a D block
        const bool is_u = k >= ci.nr_p + ci.nr_d && !du;
        const double *vec = is_u ? zbu.data() : x;
        for (uint32_t q = 0; q < r.nseg; ++q) {
          const uint32_t sv = R.seg[q].src;
          for (uint32_t e = 0; e < R.seg[q].len; ++e)
            stage[R.seg[q].dst + e] = du ? ((sv & kSegZbu) ? zbu[(sv & ~kSegZbu) + e] : x[sv + e]) : vec[sv + e];
        }
        for (uint32_t e = r.vlen; e < 2u * r.npanel; ++e) stage[e] = 0.0;
        const double *d = reinterpret_cast<const double *>(buf.data() + ci.stream_off + r.pos);
        const uint32_t h = r.nrow, np = r.npanel;
        const bool two = h > 32;
        const uint32_t U = two ? 2 : 4;
        // the FP64 product keeps one consumer group: warp w takes panel j
        // with j = (w - rot) mod 16
        constexpr int GW = NW;
        const int grp = 0;
        for (int w = 0; w < NW; ++w)
          for (uint32_t lane = 0; lane < 32; ++lane) {
            const uint32_t ra = std::min(lane, h - 1), rb = std::min(lane + 32, h - 1);
            double a0[4] = {0, 0, 0, 0}, a1[4] = {0, 0, 0, 0}, b0[4] = {0, 0, 0, 0}, b1[4] = {0, 0, 0, 0};
            auto panel = [&](uint32_t j, uint32_t u) {
              const double vx = stage[2 * j], vy = stage[2 * j + 1];
              const double *ma = d + ((size_t)j * h + ra) * 2, *mb = d + ((size_t)j * h + rb) * 2;
              a0[u] = std::fma(ma[0], vx, a0[u]);
              a1[u] = std::fma(ma[1], vy, a1[u]);
              if (two) {
                b0[u] = std::fma(mb[0], vx, b0[u]);
                b1[u] = std::fma(mb[1], vy, b1[u]);
              }
            };
            const uint32_t wl = (uint32_t)(w - grp * GW);
            uint32_t j = (wl + GW - r.rot % GW) % GW;
            for (; j + (U - 1) * GW < np; j += U * GW)
              for (uint32_t u = 0; u < U; ++u) panel(j + u * GW, u);
            for (; j < np; j += GW) panel(j, 0);
            for (uint32_t u = 0; u < U; ++u) t0[w * 32 + lane] += a0[u] + a1[u];
            if (two)
              for (uint32_t u = 0; u < U; ++u) t1[w * 32 + lane] += b0[u] + b1[u];
          }
        if (!(r.flags & kLast)) continue;
        for (uint32_t i = 0; i < h; ++i) {
          auto part = [&](int w) { return i < 32 ? t0[w * 32 + i] : t1[w * 32 + i - 32]; };
          double s = part(0);
          for (int w = 1; w < NW; ++w) s += part(w);
          const uint32_t row = r.out + i;
          if (phase == 0) {
            zbu[row] = s;
          } else if (!is_u) {
            double v = alpha * s;
            if (beta != 0.0) v = std::fma(beta, yin[row], v);
            y[row] = v;
          } else {
            y[row] = std::fma(alpha, s, y[row]);
          }
        }
        std::fill(t0.begin(), t0.end(), 0.0);
        std::fill(t1.begin(), t1.end(), 0.0);
      }
    }
  };
  do_pass(0);
  do_pass(1);
  return 0;
}

extern "C" int emu_matvec_kernel_order(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, double alpha,
                                       const double *x, double beta, const double *yin, double *y) {
  return emu_matvec_kernel_order_mk(st, nd, num_ctas, -1, alpha, x, beta, yin, y);
}

// ---- compensated dot products in the device's reduction order -------------
// The grid of hbx_dots.cuh: min(ceil(n/256), 592) blocks of 256 threads;
// thread g accumulates elements g, g + G, ... as a Dot2 pair; butterfly merge
// inside each warp, warps merged in order per block, blocks summed by one
// warp in chunks of 32 (butterfly-merged), chunks added in order.
namespace {
struct A2 {
  double s, c;
};
inline void a2_add(A2 &a, double p) {
  const double s = a.s + p;
  const double z = s - a.s;
  a.c += (a.s - (s - z)) + (p - z);
  a.s = s;
}
inline void a2_dot(A2 &a, double x, double y) {
  const double p = x * y;
  const double e = std::fma(x, y, -p);
  a2_add(a, p);
  a.c += e;
}
inline A2 a2_merge(A2 a, A2 b) {
  A2 r{a.s, a.c + b.c};
  a2_add(r, b.s);
  return r;
}
A2 a2_warp(const A2 *in) {
  A2 v[32], nv[32];
  for (int l = 0; l < 32; ++l) v[l] = in[l];
  for (int o = 16; o > 0; o >>= 1) {
    for (int l = 0; l < 32; ++l) nv[l] = (l & o) ? a2_merge(v[l ^ o], v[l]) : a2_merge(v[l], v[l ^ o]);
    for (int l = 0; l < 32; ++l) v[l] = nv[l];
  }
  return v[0];
}
}  // namespace

extern "C" void emu_dots(int k, const double *const *x, const double *const *y, size_t n, double *out) {
  const size_t nblk = std::min<size_t>((n + 255) / 256, 148 * 4), G = nblk * 256;
  std::vector<A2> part(nblk);
  for (int j = 0; j < k; ++j) {
    for (size_t b = 0; b < nblk; ++b) {
      A2 wm[8];
      for (int w = 0; w < 8; ++w) {
        A2 lanes[32];
        for (int l = 0; l < 32; ++l) {
          A2 a{0.0, 0.0};
          for (size_t i = b * 256 + w * 32 + l; i < n; i += G) a2_dot(a, x[j][i], y[j][i]);
          lanes[l] = a;
        }
        wm[w] = a2_warp(lanes);
      }
      A2 t = wm[0];
      for (int w = 1; w < 8; ++w) t = a2_merge(t, wm[w]);
      part[b] = t;
    }
    A2 a{0.0, 0.0};
    for (size_t b0 = 0; b0 < nblk; b0 += 32) {
      A2 lanes[32];
      for (int l = 0; l < 32; ++l) lanes[l] = b0 + l < nblk ? part[b0 + l] : A2{0.0, 0.0};
      a = a2_merge(a, a2_warp(lanes));
    }
    out[j] = a.s + a.c;
  }
}

// The chunk -> instance-range table of a block-diagonal engine checked
// against its runs: every chunk a run's bytes touch must list the run's
// instance.  stats: [chunks, chunks holding one instance, chunks holding
// none, runs].  Returns the number of violations, or -1 when no table is built.
extern "C" int emu_chunk_table(const stc_HACApK_leafmtxp *const *st, const int *nd, int count, int num_ctas,
                               int precision, int merge_keep, long long *stats) {
  CombinedLeaves cl;
  std::string err;
  if (combine_leaves(st, nd, count, cl, err) != 0) return -2;
  Plan plan;
  if (make_plan(&cl.container, cl.off[count], num_ctas, plan, err, precision, false, PlanCosts(), merge_keep) != 0)
    return -3;
  std::vector<int> rinst((size_t)cl.off[count]);
  for (int k = 0; k < count; ++k)
    for (int i = cl.off[k]; i < cl.off[k + 1]; ++i) rinst[i] = k;
  std::vector<uint32_t> cinst, cbase;
  if (!chunk_instances(plan, rinst, cinst, cbase)) return -1;
  int bad = 0;
  long long runs = 0, one = 0, none = 0, chunks = 0;
  for (size_t c = 0; c < plan.ctas.size(); ++c) {
    const CtaInfo &ci = plan.ctas[c];
    const uint32_t K = (ci.stream_bytes + kChunkBytes - 1) >> kChunkLog;
    chunks += K;
    for (uint32_t g = 0; g < K; ++g) {
      const uint32_t e = cinst[cbase[c] + g], lo = e & 0xffffu, hi = e >> 16;
      one += lo == hi;
      none += lo > hi;
    }
    for (uint32_t r = 0; r < ci.nr_p + ci.nr_d + ci.nr_u; ++r) {
      const Run &hd = plan.recs[ci.rec_begin + r].hdr;
      const uint32_t bytes = run_bytes(hd);
      if (!bytes) continue;
      ++runs;
      // the run's instance from first principles: its rows, or for P runs its first column
      const int k = run_kind(hd) == kRunP ? rinst[plan.recs[ci.rec_begin + r].seg[0].src] : rinst[hd.out];
      for (uint32_t g = hd.pos >> kChunkLog; g <= (hd.pos + bytes - 1) >> kChunkLog; ++g) {
        if (g >= K) { ++bad; continue; }
        const uint32_t e = cinst[cbase[c] + g], lo = e & 0xffffu, hi = e >> 16;
        if (!(lo <= (uint32_t)k && (uint32_t)k <= hi)) ++bad;
      }
    }
  }
  if (stats) {
    stats[0] = chunks;
    stats[1] = one;
    stats[2] = none;
    stats[3] = runs;
  }
  return bad;
}
