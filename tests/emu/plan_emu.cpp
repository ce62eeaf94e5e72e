// Test-only CPU interpreter of the engine's packed layout.  It links the
// product's planner/packer (hbx_plan.cpp), walks every CTA's term list the
// way the sm_100a kernel does (P panels -> zbu, D/U atom terms -> y), checks
// the layout invariants the kernel relies on (16-byte aligned streams, term
// data inside its CTA stream, atoms partitioning the rows exactly once,
// panel width <= 64, atom height <= 32), and returns y = H x.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../hacapk-magma_b200/csrc/hbx_plan.h"

using namespace hbx;

extern "C" int emu_matvec(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, const double *x, double *y,
                          long long *stats, char *msg, int msglen) {
  auto bad = [&](const std::string &s) {
    std::snprintf(msg, msglen, "%s", s.c_str());
    return 1;
  };
  Plan plan;
  std::string err;
  int rc = make_plan(st, nd, num_ctas, plan, err);
  if (rc != 0) return bad("make_plan: " + err);
  std::vector<uint8_t> buf(plan.total_bytes, 0xAB);
  pack_plan(st, plan, buf.data());
  std::vector<double> zbu(plan.zbu_len, 0.0);
  std::vector<char> zset(plan.zbu_len, 0);
  std::vector<int> owner(nd, -1);
  std::fill(y, y + nd, NAN);
  long long nterms = 0;
  // pass 1: P sections of every CTA (chunk terms; a panel's chunks are consecutive)
  for (int c = 0; c < plan.num_ctas; ++c) {
    const CtaInfo &ci = plan.ctas[c];
    if (ci.stream_off % 256 != 0 || ci.stream_bytes % 16 != 0) return bad("stream alignment");
    if (ci.stream_off + ci.stream_bytes > plan.total_bytes) return bad("stream outside buffer");
    // runs cover the three sections exactly, in order
    uint32_t expect = ci.term_begin;
    const uint32_t nsec[3] = {ci.nr_p, ci.nr_d, ci.nr_u};
    const uint32_t tsec[3] = {ci.n_p, ci.n_d, ci.n_u};
    uint32_t ri = ci.run_begin;
    for (int sec = 0; sec < 3; ++sec) {
      uint32_t covered = 0;
      for (uint32_t k = 0; k < nsec[sec]; ++k, ++ri) {
        const Run &R = plan.runs[ri];
        if (R.term_first != expect || R.nterm == 0 || R.nterm > (uint32_t)kRunTerms || R.vlen > (uint32_t)kStageCap)
          return bad("bad run");
        uint32_t v = 0;
        for (uint32_t q = 0; q < R.nterm; ++q) {
          const Term &T = plan.terms[R.term_first + q];
          if (T.voff != v) return bad("voff mismatch");
          v += term_vlen(T);
          if (sec > 0) {
            const Term &T0 = plan.terms[R.term_first];
            if (T.nrow != R.nrow || T.out != R.out || T.pos != R.pos + T.voff * R.nrow * 8 ||
                T.rot != (uint16_t)((R.rot + T.voff) % kConsumerWarps) || T0.pos != R.pos)
              return bad("D/U run is not one contiguous h x W block");
          }
          if (sec > 0 && (T.kind & kAtomEnd) && q + 1 != R.nterm) return bad("run crosses an atom end");
        }
        if (v != R.vlen) return bad("run vlen mismatch");
        if (sec > 0 && (R.ncol != R.vlen || (R.flags & kAtomEnd) != (plan.terms[R.term_first + R.nterm - 1].kind & kAtomEnd)))
          return bad("D/U run header mismatch");
        expect += R.nterm;
        covered += R.nterm;
      }
      if (covered != tsec[sec]) return bad("runs do not cover the section");
    }
    std::vector<double> acc(kPanelCols, 0.0);
    for (uint32_t i = 0; i < ci.n_p; ++i) {
      const Term &T = plan.terms[ci.term_begin + i];
      if ((T.kind & 0xff) != kTermP || T.ncol == 0 || T.ncol > (uint32_t)kPanelCols || T.rot >= kConsumerWarps ||
          T.nrow == 0 || T.nrow > (uint32_t)kPanelRows)
        return bad("bad P term");
      if ((uint64_t)T.pos + (uint64_t)T.nrow * T.ncol * 8 > ci.stream_bytes) return bad("P term outside stream");
      if (T.vec + T.nrow > (uint32_t)nd || T.out + T.ncol > plan.zbu_len) return bad("P term vector range");
      if (T.kind & kPanelFirst) std::fill(acc.begin(), acc.end(), 0.0);
      const double *d = reinterpret_cast<const double *>(buf.data() + ci.stream_off + T.pos);
      for (uint32_t l = 0; l < T.ncol; ++l)
        for (uint32_t t = 0; t < T.nrow; ++t) acc[l] += d[(size_t)l * T.nrow + t] * x[T.vec + t];
      if (T.kind & kPanelLast)
        for (uint32_t l = 0; l < T.ncol; ++l) { zbu[T.out + l] = acc[l]; zset[T.out + l] = 1; }
      ++nterms;
    }
  }
  // pass 2: D then U sections
  for (int c = 0; c < plan.num_ctas; ++c) {
    const CtaInfo &ci = plan.ctas[c];
    std::vector<double> acc(kAtomMax, 0.0);
    for (int pass = 0; pass < 2; ++pass) {
      const uint32_t t0 = ci.term_begin + ci.n_p + (pass ? ci.n_d : 0);
      const uint32_t nt = pass ? ci.n_u : ci.n_d;
      for (uint32_t i = 0; i < nt; ++i) {
        const Term &T = plan.terms[t0 + i];
        const int kind = T.kind & 0xff;
        if (kind != (pass ? kTermU : kTermD) || T.nrow == 0 || T.nrow > (uint32_t)kAtomMax || T.rot >= kConsumerWarps)
          return bad("bad D/U term");
        if ((uint64_t)T.pos + (uint64_t)T.nrow * T.ncol * 8 > ci.stream_bytes) return bad("D/U term outside stream");
        if (T.out + T.nrow > (uint32_t)nd) return bad("atom rows outside [0, nd)");
        if (pass == 0 && T.vec + T.ncol > (uint32_t)nd) return bad("D term column range");
        if (pass == 1 && T.vec + T.ncol > plan.zbu_len) return bad("U term zbu range");
        const double *d = reinterpret_cast<const double *>(buf.data() + ci.stream_off + T.pos);
        const double *v = pass ? zbu.data() : x;
        for (uint32_t col = 0; col < T.ncol; ++col)
          for (uint32_t r = 0; r < T.nrow; ++r) acc[r] += d[(size_t)col * T.nrow + r] * v[T.vec + col];
        if (T.kind & kAtomEnd) {
          for (uint32_t r = 0; r < T.nrow; ++r) {
            const uint32_t row = T.out + r;
            if (pass == 0) {
              if (owner[row] != -1) return bad("row written by two atoms");
              owner[row] = c;
              y[row] = acc[r];
            } else {
              if (owner[row] != c) return bad("U pass writes a row the CTA does not own");
              y[row] += acc[r];
            }
            acc[r] = 0.0;
          }
        }
        ++nterms;
      }
    }
  }
  for (int r = 0; r < nd; ++r)
    if (owner[r] < 0) return bad("row " + std::to_string(r) + " not owned by any atom");
  for (int c = 0; c < plan.num_ctas; ++c) {
    const CtaInfo &ci = plan.ctas[c];
    for (uint32_t i = 0; i < ci.n_u; ++i) {
      const Term &T = plan.terms[ci.term_begin + ci.n_p + ci.n_d + i];
      for (uint32_t l = 0; l < T.ncol; ++l)
        if (!zset[T.vec + l]) return bad("U term reads a zbu entry no panel writes");
    }
  }
  if (stats) {
    stats[0] = (long long)plan.total_bytes;
    stats[1] = nterms;
    stats[2] = (long long)plan.atoms.size();
    stats[3] = (long long)plan.zbu_len;
    stats[4] = (long long)plan.alg_bytes;
    uint64_t mx = 0, sum = 0;
    for (auto &ci : plan.ctas) { mx = std::max<uint64_t>(mx, ci.stream_bytes); sum += ci.stream_bytes; }
    stats[5] = (long long)mx;
    stats[6] = (long long)sum;
  }
  return 0;
}
