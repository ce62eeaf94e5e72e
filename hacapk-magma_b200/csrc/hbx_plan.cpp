// hbx_plan.cpp -- host planner and packer for the per-CTA streaming layout.
//
// Replaces the setup of c_hacapk_adot_body_lfcpy_batch_sorted_
// (HACApK_BATCH_SORT.c:86-858): where the reference sorts the GEMVs of the
// two phases by size (:269-369) and uploads each transposed panel padded to
// lda=roundup(M,32) (:541-811), this planner splits the leaves into V-panels
// and row-atom terms, balances them over the persistent CTAs by bytes
// (longest-processing-time first), and packs every CTA's terms back to back
// with no padding.
#include "hbx_plan.h"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <queue>

#include <omp.h>

namespace hbx {
namespace {

const stc_HACApK_leafmtx *leaf_at(const stc_HACApK_leafmtxp *st, int ip) {
  return reinterpret_cast<const stc_HACApK_leafmtx *>(
      reinterpret_cast<const char *>(st->st_lf) + (size_t)st->st_lf_stride * ip);
}

const double *a2_of(const stc_HACApK_leafmtx *s) {
  return reinterpret_cast<const double *>(reinterpret_cast<const char *>(s->a1) + s->a1size);
}

constexpr uint64_t kTermOverhead = 256;  // bytes-equivalent fixed cost of a term

struct Panel {
  int leaf, l0, kc;
  uint64_t bytes;
};

// Min-heap load balancer (longest processing time first).
struct Bins {
  std::vector<uint64_t> load;
  std::priority_queue<std::pair<uint64_t, int>, std::vector<std::pair<uint64_t, int>>,
                      std::greater<std::pair<uint64_t, int>>> heap;
  explicit Bins(int n) : load(n, 0) {
    for (int i = 0; i < n; ++i) heap.push({0, i});
  }
  int take(uint64_t cost) {
    auto top = heap.top();
    heap.pop();
    load[top.second] += cost;
    heap.push({load[top.second], top.second});
    return top.second;
  }
};

}  // namespace

int make_plan(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, Plan &plan, std::string &err) {
  plan = Plan();
  if (!st || nd <= 0 || num_ctas <= 0) { err = "null container, nd <= 0 or no CTAs"; return HBX_ERR_INVALID; }
  const int nlf = st->nlf;
  if (nlf < 0 || (nlf > 0 && (!st->st_lf || st->st_lf_stride < (int)sizeof(stc_HACApK_leafmtx)))) {
    err = "bad leaf array (nlf, st_lf or st_lf_stride)";
    return HBX_ERR_INVALID;
  }
  plan.nd = nd;
  plan.nlf = nlf;
  plan.num_ctas = num_ctas;

  // ---- validation, zbu offsets
  std::vector<uint64_t> zoff(nlf, 0);
  uint64_t zlen = 0;
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    if (s->ltmtx != 1 && s->ltmtx != 2) { err = "leaf " + std::to_string(ip) + ": ltmtx not 1 or 2"; return HBX_ERR_INVALID; }
    if (s->ndl < 0 || s->ndt < 0 || s->nstrtl < 1 || s->nstrtt < 1 ||
        (long long)s->nstrtl - 1 + s->ndl > nd || (long long)s->nstrtt - 1 + s->ndt > nd) {
      err = "leaf " + std::to_string(ip) + ": row/column range outside [1, nd]";
      return HBX_ERR_INVALID;
    }
    if (s->ltmtx == 1) {
      if (s->kt < 0) { err = "leaf " + std::to_string(ip) + ": negative kt"; return HBX_ERR_INVALID; }
      if (s->kt > 0 && s->ndl > 0 && s->ndt > 0) {
        if (!s->a1) { err = "leaf " + std::to_string(ip) + ": null a1"; return HBX_ERR_INVALID; }
        if (s->a1size < (long long)s->ndt * s->kt * 8) { err = "leaf " + std::to_string(ip) + ": a1size smaller than ndt*kt*8"; return HBX_ERR_INVALID; }
        zoff[ip] = zlen;
        zlen += (uint64_t)s->kt;
        plan.lowrank_words += (uint64_t)s->kt * (uint64_t)(s->ndl + s->ndt);
        plan.nlfkt++;
        plan.ktmax = std::max(plan.ktmax, s->kt);
      }
    } else if (s->ndl > 0 && s->ndt > 0) {
      if (!s->a1) { err = "leaf " + std::to_string(ip) + ": null a1"; return HBX_ERR_INVALID; }
      plan.dense_words += (uint64_t)s->ndl * (uint64_t)s->ndt;
    }
  }
  plan.zbu_len = zlen;
  uint64_t ktsum = 0;
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    if (s->ltmtx == 1 && s->kt > 0 && s->ndl > 0 && s->ndt > 0) ktsum += (uint64_t)s->kt;
  }
  plan.alg_bytes = 8 * (plan.dense_words + plan.lowrank_words) + 16ull * nd + 16ull * ktsum;
  plan.alg_flops = 2 * (plan.dense_words + plan.lowrank_words);

  // ---- row atoms
  std::vector<int> bnd;
  bnd.reserve(2 * (size_t)nlf + 2);
  bnd.push_back(0);
  bnd.push_back(nd);
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    if (s->ndl <= 0) continue;
    bnd.push_back(s->nstrtl - 1);
    bnd.push_back(s->nstrtl - 1 + s->ndl);
  }
  std::sort(bnd.begin(), bnd.end());
  bnd.erase(std::unique(bnd.begin(), bnd.end()), bnd.end());
  std::vector<Atom> atoms;
  for (size_t i = 0; i + 1 < bnd.size(); ++i) {
    int len = bnd[i + 1] - bnd[i];
    int pieces = (len + kAtomMax - 1) / kAtomMax;
    int base = len / pieces, rem = len % pieces, r = bnd[i];
    for (int p = 0; p < pieces; ++p) {
      int h = base + (p < rem ? 1 : 0);
      atoms.push_back(Atom{(uint32_t)r, (uint32_t)h});
      r += h;
    }
  }
  const int natoms = (int)atoms.size();
  std::vector<int> row_atom(nd);
  for (int a = 0; a < natoms; ++a)
    for (uint32_t r = atoms[a].r0; r < atoms[a].r0 + atoms[a].h; ++r) row_atom[r] = a;

  // ---- per-atom D and U term lists (CSR, leaf order inside an atom)
  std::vector<uint32_t> dcnt(natoms + 1, 0), ucnt(natoms + 1, 0);
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    if (s->ndl <= 0 || s->ndt <= 0) continue;
    if (s->ltmtx == 1 && s->kt <= 0) continue;
    int a0 = row_atom[s->nstrtl - 1], a1 = row_atom[s->nstrtl - 2 + s->ndl];
    for (int a = a0; a <= a1; ++a) (s->ltmtx == 2 ? dcnt : ucnt)[a + 1]++;
  }
  std::partial_sum(dcnt.begin(), dcnt.end(), dcnt.begin());
  std::partial_sum(ucnt.begin(), ucnt.end(), ucnt.begin());
  std::vector<uint32_t> dleaf(dcnt[natoms]), uleaf(ucnt[natoms]);
  {
    std::vector<uint32_t> dfill(dcnt.begin(), dcnt.end() - 1), ufill(ucnt.begin(), ucnt.end() - 1);
    for (int ip = 0; ip < nlf; ++ip) {
      const stc_HACApK_leafmtx *s = leaf_at(st, ip);
      if (s->ndl <= 0 || s->ndt <= 0) continue;
      if (s->ltmtx == 1 && s->kt <= 0) continue;
      int a0 = row_atom[s->nstrtl - 1], a1 = row_atom[s->nstrtl - 2 + s->ndl];
      for (int a = a0; a <= a1; ++a) {
        if (s->ltmtx == 2) dleaf[dfill[a]++] = (uint32_t)ip;
        else uleaf[ufill[a]++] = (uint32_t)ip;
      }
    }
  }
  std::vector<uint64_t> acost(natoms, 0);
  for (int a = 0; a < natoms; ++a) {
    uint64_t c = kTermOverhead;
    for (uint32_t q = dcnt[a]; q < dcnt[a + 1]; ++q)
      c += (uint64_t)atoms[a].h * leaf_at(st, dleaf[q])->ndt * 8 + kTermOverhead;
    for (uint32_t q = ucnt[a]; q < ucnt[a + 1]; ++q)
      c += (uint64_t)atoms[a].h * leaf_at(st, uleaf[q])->kt * 8 + kTermOverhead;
    acost[a] = c;
  }

  // ---- V-panels
  const uint64_t total_est = 8 * (plan.dense_words + plan.lowrank_words);
  const uint64_t budget = total_est / (uint64_t)num_ctas + 1;
  const uint64_t panel_cap = std::max<uint64_t>(64 * 1024, budget / 3);
  std::vector<Panel> panels;
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    if (s->ltmtx != 1 || s->kt <= 0 || s->ndl <= 0 || s->ndt <= 0) continue;
    int np = (s->kt + kPanelCols - 1) / kPanelCols;
    while (np < s->kt && (uint64_t)s->ndt * ((s->kt + np - 1) / np) * 8 > panel_cap) np *= 2;
    np = std::min(np, s->kt);
    int base = s->kt / np, rem = s->kt % np, l0 = 0;
    for (int p = 0; p < np; ++p) {
      int kc = base + (p < rem ? 1 : 0);
      panels.push_back(Panel{ip, l0, kc, (uint64_t)s->ndt * kc * 8 + kTermOverhead});
      l0 += kc;
    }
  }

  // ---- balance: panels first (they gate the grid barrier), then atoms
  Bins bins(num_ctas);
  std::vector<int> porder(panels.size());
  std::iota(porder.begin(), porder.end(), 0);
  std::stable_sort(porder.begin(), porder.end(), [&](int a, int b) { return panels[a].bytes > panels[b].bytes; });
  std::vector<std::vector<int>> cta_panels(num_ctas), cta_atoms(num_ctas);
  for (int q : porder) cta_panels[bins.take(panels[q].bytes)].push_back(q);
  std::vector<int> aorder(natoms);
  std::iota(aorder.begin(), aorder.end(), 0);
  std::stable_sort(aorder.begin(), aorder.end(), [&](int a, int b) { return acost[a] > acost[b]; });
  for (int a : aorder) cta_atoms[bins.take(acost[a])].push_back(a);

  // ---- emit terms, runs and stream offsets per CTA
  plan.ctas.resize(num_ctas);
  uint64_t off = 0;
  for (int c = 0; c < num_ctas; ++c) {
    auto &pl = cta_panels[c];
    auto &al = cta_atoms[c];
    std::sort(pl.begin(), pl.end(), [&](int a, int b) {
      return panels[a].leaf != panels[b].leaf ? panels[a].leaf < panels[b].leaf : panels[a].l0 < panels[b].l0;
    });
    std::sort(al.begin(), al.end());
    CtaInfo info{};
    info.stream_off = off;
    info.term_begin = (uint32_t)plan.terms.size();
    info.atom_begin = (uint32_t)plan.atoms.size();
    info.n_atoms = (uint32_t)al.size();
    uint64_t pos = 0, rot = 0;
    auto push = [&](uint64_t bytes, uint32_t nrow, uint32_t ncol, uint32_t vec, uint32_t out, uint16_t kind,
                    uint32_t leaf, uint64_t trot) {
      Term t{};
      t.pos = (uint32_t)pos;
      t.nrow = nrow; t.ncol = ncol; t.vec = vec; t.out = out;
      t.kind = kind;
      t.rot = (uint16_t)(trot % kConsumerWarps);
      t.leaf = leaf;
      plan.terms.push_back(t);
      pos += bytes;
    };
    // P: one term per panel chunk; a panel keeps one warp rotation
    for (int q : pl) {
      const Panel &P = panels[q];
      const stc_HACApK_leafmtx *s = leaf_at(st, P.leaf);
      for (int r0 = 0; r0 < s->ndt; r0 += kPanelRows) {
        const int hv = std::min(kPanelRows, s->ndt - r0);
        uint16_t k = kTermP | (r0 == 0 ? kPanelFirst : 0) | (r0 + hv == s->ndt ? kPanelLast : 0);
        push((uint64_t)hv * P.kc * 8, (uint32_t)hv, (uint32_t)P.kc, (uint32_t)(s->nstrtt - 1 + r0),
             (uint32_t)(zoff[P.leaf] + P.l0), k, (uint32_t)P.leaf, rot);
        info.n_p++;
      }
      rot += (uint64_t)P.kc;
    }
    // D: dense rows of every owned atom, split into column pieces <= kStageCap
    for (int a : al) {
      const Atom &A = atoms[a];
      plan.atoms.push_back(A);
      if (dcnt[a + 1] == dcnt[a]) {
        push(0, A.h, 0, 0, A.r0, kTermD | kAtomEnd, 0xffffffffu, rot);
        info.n_d++;
      }
      for (uint32_t q = dcnt[a]; q < dcnt[a + 1]; ++q) {
        const stc_HACApK_leafmtx *s = leaf_at(st, dleaf[q]);
        for (int c0 = 0; c0 < s->ndt; c0 += kStageCap) {
          const int wc = std::min(kStageCap, s->ndt - c0);
          const bool last = (q + 1 == dcnt[a + 1]) && (c0 + wc == s->ndt);
          push((uint64_t)A.h * wc * 8, A.h, (uint32_t)wc, (uint32_t)(s->nstrtt - 1 + c0), A.r0,
               kTermD | (last ? kAtomEnd : 0), dleaf[q], rot);
          rot += (uint64_t)wc;
          info.n_d++;
        }
      }
    }
    // U: U rows of every owned atom, split into column pieces <= kStageCap
    for (int a : al) {
      const Atom &A = atoms[a];
      for (uint32_t q = ucnt[a]; q < ucnt[a + 1]; ++q) {
        const stc_HACApK_leafmtx *s = leaf_at(st, uleaf[q]);
        for (int c0 = 0; c0 < s->kt; c0 += kStageCap) {
          const int wc = std::min(kStageCap, s->kt - c0);
          const bool last = (q + 1 == ucnt[a + 1]) && (c0 + wc == s->kt);
          push((uint64_t)A.h * wc * 8, A.h, (uint32_t)wc, (uint32_t)(zoff[uleaf[q]] + c0), A.r0,
               kTermU | (last ? kAtomEnd : 0), uleaf[q], rot);
          rot += (uint64_t)wc;
          info.n_u++;
        }
      }
    }
    // runs: consecutive terms whose vector segments fit one stage buffer
    info.run_begin = (uint32_t)plan.runs.size();
    auto build_runs = [&](uint32_t first, uint32_t count, bool split_at_atoms) {
      uint32_t nr = 0, i = first;
      while (i < first + count) {
        Run r{};
        r.term_first = i;
        while (i < first + count) {
          Term &t = plan.terms[i];
          const uint32_t len = term_vlen(t);
          if (r.nterm > 0 && (r.vlen + len > (uint32_t)kStageCap || r.nterm == (uint32_t)kRunTerms)) break;
          t.voff = r.vlen;
          r.vlen += len;
          r.nterm++;
          i++;
          if (split_at_atoms && (t.kind & kAtomEnd)) break;
        }
        if (split_at_atoms) {
          const Term &t0 = plan.terms[r.term_first];
          const Term &tl = plan.terms[r.term_first + r.nterm - 1];
          r.pos = t0.pos;
          r.nrow = t0.nrow;
          r.ncol = r.vlen;
          r.out = t0.out;
          r.flags = (uint16_t)(tl.kind & kAtomEnd);
          r.rot = t0.rot;
        }
        plan.runs.push_back(r);
        nr++;
      }
      return nr;
    };
    info.nr_p = build_runs(info.term_begin, info.n_p, false);
    info.nr_d = build_runs(info.term_begin + info.n_p, info.n_d, true);
    info.nr_u = build_runs(info.term_begin + info.n_p + info.n_d, info.n_u, true);
    uint64_t bytes = (pos + 15) & ~uint64_t(15);
    if (bytes > 0xffffffffull) {
      err = "a CTA stream exceeds 4 GiB; use more CTAs";
      return HBX_ERR_INVALID;
    }
    info.stream_bytes = (uint32_t)bytes;
    plan.ctas[c] = info;
    off += (bytes + 255) & ~uint64_t(255);
  }
  plan.total_bytes = std::max<uint64_t>(off, 256);
  return HBX_OK;
}

void pack_plan(const stc_HACApK_leafmtxp *st, const Plan &plan, uint8_t *dst) {
  // zbu offset of each low-rank leaf, to recover a panel's first column
  std::vector<uint64_t> zoff(plan.nlf, 0);
  uint64_t z = 0;
  for (int ip = 0; ip < plan.nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    if (s->ltmtx == 1 && s->kt > 0 && s->ndl > 0 && s->ndt > 0) { zoff[ip] = z; z += (uint64_t)s->kt; }
  }
  const int nc = plan.num_ctas;
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nc; ++c) {
    const CtaInfo &info = plan.ctas[c];
    uint8_t *base = dst + info.stream_off;
    std::memset(base, 0, info.stream_bytes);
    const uint32_t nt = info.n_p + info.n_d + info.n_u;
    for (uint32_t i = 0; i < nt; ++i) {
      const Term &t = plan.terms[info.term_begin + i];
      if (t.leaf == 0xffffffffu) continue;
      const stc_HACApK_leafmtx *s = leaf_at(st, (int)t.leaf);
      double *d = reinterpret_cast<double *>(base + t.pos);
      const int kind = t.kind & 0xff;
      if (kind == kTermP) {
        const int ndt = s->ndt, kc = (int)t.ncol, hv = (int)t.nrow;
        const int r0 = (int)t.vec - (s->nstrtt - 1);
        const int l0 = (int)(t.out - zoff[t.leaf]);
        const double *V = s->a1;  // V(t, l) = a1[t + l*ndt]
        for (int l = 0; l < kc; ++l)
          std::memcpy(d + (size_t)l * hv, V + (size_t)(l0 + l) * ndt + r0, (size_t)hv * 8);
      } else if (kind == kTermD) {
        const int h = (int)t.nrow, w = (int)t.ncol, ndt = s->ndt;
        const int ro = (int)t.out - (s->nstrtl - 1);
        const int c0 = (int)t.vec - (s->nstrtt - 1);
        const double *A = s->a1;  // A(il, it) = a1[it + il*ndt]
        for (int i = 0; i < h; ++i) {
          const double *row = A + (size_t)(ro + i) * ndt + c0;
          for (int cc = 0; cc < w; ++cc) d[(size_t)cc * h + i] = row[cc];
        }
      } else {
        const int h = (int)t.nrow, w = (int)t.ncol, ndl = s->ndl;
        const int ro = (int)t.out - (s->nstrtl - 1);
        const int c0 = (int)(t.vec - zoff[t.leaf]);
        const double *U = a2_of(s);  // U(i, l) = a2[i + l*ndl]
        for (int l = 0; l < w; ++l) std::memcpy(d + (size_t)l * h, U + (size_t)(c0 + l) * ndl + ro, (size_t)h * 8);
      }
    }
  }
}

}  // namespace hbx
