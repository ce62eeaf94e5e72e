// hbx_plan.cpp -- host planner and packer for the per-CTA streaming layout.
//
// Replaces the setup of c_hacapk_adot_body_lfcpy_batch_sorted_
// (HACApK_BATCH_SORT.c:86-858): where the reference sorts the GEMVs of the
// two phases by size (:269-369) and uploads each transposed panel padded to
// lda=roundup(M,32) (:541-811), this planner stacks the V factors of every
// column cluster into P slabs, cuts the dense and U factors into row-atom
// blocks, balances the blocks over the persistent CTAs by bytes (longest
// processing time first), and packs every CTA's runs back to back as panels
// of 16-byte rows (two double or four float columns; zero columns fill a
// block's last panel, nothing else).
#include "hbx_plan.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <queue>
#include <utility>

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

bool lowrank_active(const stc_HACApK_leafmtx *s) { return s->ltmtx == 1 && s->kt > 0 && s->ndl > 0 && s->ndt > 0; }
bool dense_active(const stc_HACApK_leafmtx *s) { return s->ltmtx == 2 && s->ndl > 0 && s->ndt > 0; }

// Bytes-equivalent fixed costs of a block and of a run, for balancing only
// (the latency of a block end or a run switch, at the per-SM share of HBM
// bandwidth).


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

uint64_t block_cost(uint32_t h, uint32_t W, int prec, const PlanCosts &c) {
  const uint64_t g = group_cols(prec), wp = (W + g - 1) / g * g;
  return (uint64_t)elem_bytes(prec) * h * wp + c.block + c.run * (1 + wp * stage_elem_bytes(prec) / kStageBytes);
}

// Vector index of block column c (c < W): P -> x index, D -> x index, U -> zbu index.
struct ColumnMap {
  const Plan &plan;
  const Block &b;
  uint32_t p_x0;  // P: x index of column 0
  // walks the pieces of a D/U block; returns vsrc of column c and the number
  // of following columns (c included) that stay contiguous in the same piece
  std::pair<uint32_t, uint32_t> at(uint32_t c, uint32_t &piece, uint32_t &piece_c0) const {
    if (b.kind == kRunP) return {p_x0 + c, b.W - c};
    while (piece < b.npiece && c >= piece_c0 + plan.pieces[b.piece_begin + piece].n) {
      piece_c0 += plan.pieces[b.piece_begin + piece].n;
      ++piece;
    }
    const Piece &P = plan.pieces[b.piece_begin + piece];
    return {P.vsrc + (c - piece_c0), P.n - (c - piece_c0)};
  }
};

// Gather segments of block columns [c0, c1) (c1 <= W): contiguous vector
// ranges merged, in stage order; with long_first the ones longer than
// kSegShort are moved to the front (the single-RHS gather copies those with
// the whole warp).
void segments(const ColumnMap &M, uint32_t c0, uint32_t c1, std::vector<Seg> &out, bool long_first) {
  out.clear();
  uint32_t piece = 0, piece_c0 = 0;
  uint32_t c = c0;
  while (c < c1) {
    auto [src, avail] = M.at(c, piece, piece_c0);
    uint32_t n = std::min(avail, c1 - c);
    if (!out.empty()) {
      Seg &L = out.back();
      if (L.src + L.len == src) {
        L.len = (uint16_t)(L.len + n);
        c += n;
        continue;
      }
    }
    out.push_back(Seg{src, (uint16_t)n, (uint16_t)(c - c0)});
    c += n;
  }
  if (long_first)
    std::stable_partition(out.begin(), out.end(), [](const Seg &s) { return s.len > (uint32_t)kSegShort; });
}

uint32_t count_long(const std::vector<Seg> &segs) {
  uint32_t n = 0;
  for (const Seg &s : segs) n += s.len > (uint32_t)kSegShort ? 1u : 0u;
  return n;
}

}  // namespace

int make_plan(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, Plan &plan, std::string &err, int precision,
              bool pair_panels, const PlanCosts &costs, int merge_keep) {
  plan = Plan();
  plan.costs = costs;
  if (precision != kFP64 && precision != kFP32 && precision != kBF16) {
    err = "unknown storage precision";
    return HBX_ERR_INVALID;
  }
  if (pair_panels && precision != kFP32) { err = "panel pairs need FP32 storage"; return HBX_ERR_INVALID; }
  if (pair_panels && merge_keep >= 0) { err = "merged D+U blocks need the single-vector layout"; return HBX_ERR_INVALID; }
  plan.precision = precision;
  plan.pair_panels = pair_panels;
  const uint32_t G = group_cols(precision);
  // run widths are multiples of RG columns: whole panels, or whole panel
  // pairs (the K = 8 of one TF32 tensor-core step) for the multi-RHS engine
  const uint32_t RG = pair_panels ? 2 * G : G;
  const uint32_t stage_cols = (pair_panels ? kPairStageBytes : kStageBytes) / stage_elem_bytes(precision);
  if (!st || nd <= 0 || num_ctas <= 0) { err = "null container, nd <= 0 or no CTAs"; return HBX_ERR_INVALID; }
  const int nlf = st->nlf;
  if (nlf < 0 || (nlf > 0 && (!st->st_lf || st->st_lf_stride < (int)sizeof(stc_HACApK_leafmtx)))) {
    err = "bad leaf array (nlf, st_lf or st_lf_stride)";
    return HBX_ERR_INVALID;
  }
  plan.nd = nd;
  plan.nlf = nlf;
  plan.num_ctas = num_ctas;

  // ---- validation and storage counts
  uint64_t ktsum = 0;
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
      if (lowrank_active(s)) {
        if (!s->a1) { err = "leaf " + std::to_string(ip) + ": null a1"; return HBX_ERR_INVALID; }
        if (s->a1size < (long long)s->ndt * s->kt * 8) { err = "leaf " + std::to_string(ip) + ": a1size smaller than ndt*kt*8"; return HBX_ERR_INVALID; }
        ktsum += (uint64_t)s->kt;
        plan.lowrank_words += (uint64_t)s->kt * (uint64_t)(s->ndl + s->ndt);
        plan.nlfkt++;
        plan.ktmax = std::max(plan.ktmax, s->kt);
      }
    } else if (dense_active(s)) {
      if (!s->a1) { err = "leaf " + std::to_string(ip) + ": null a1"; return HBX_ERR_INVALID; }
      plan.dense_words += (uint64_t)s->ndl * (uint64_t)s->ndt;
    }
  }
  plan.zbu_len = ktsum;
  plan.alg_bytes = 8 * (plan.dense_words + plan.lowrank_words) + 16ull * nd + 16ull * ktsum;
  plan.alg_flops = 2 * (plan.dense_words + plan.lowrank_words);

  // ---- P column groups (low-rank leaves with the same nstrtt and ndt), zbu order
  std::map<std::pair<int, int>, uint32_t> gid;
  std::vector<std::vector<uint32_t>> gl;
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    if (!lowrank_active(s)) continue;
    auto key = std::make_pair(s->nstrtt, s->ndt);
    auto it = gid.find(key);
    if (it == gid.end()) {
      it = gid.emplace(key, (uint32_t)gl.size()).first;
      gl.emplace_back();
    }
    gl[it->second].push_back((uint32_t)ip);
  }
  const uint32_t ngroups = (uint32_t)gl.size();
  plan.zoff.assign(nlf, 0);
  plan.group_leaf_begin.assign(ngroups + 1, 0);
  std::vector<uint64_t> gz(ngroups, 0), grows(ngroups, 0);
  {
    uint64_t z = 0;
    for (uint32_t g = 0; g < ngroups; ++g) {
      plan.group_leaf_begin[g] = (uint32_t)plan.group_leaves.size();
      gz[g] = z;
      for (uint32_t ip : gl[g]) {
        plan.group_leaves.push_back(ip);
        plan.zoff[ip] = z;
        z += (uint64_t)leaf_at(st, (int)ip)->kt;
      }
      grows[g] = z - gz[g];
    }
    plan.group_leaf_begin[ngroups] = (uint32_t)plan.group_leaves.size();
  }
  if (ktsum > 0xffffffffull || (uint64_t)nd > 0xffffffffull) { err = "zbu length exceeds 2^32"; return HBX_ERR_INVALID; }
  if (merge_keep >= 0 && ktsum >= kSegZbu) { err = "zbu length reaches 2^31 (merged blocks)"; return HBX_ERR_INVALID; }

  // ---- P blocks: slabs of <= 64 stacked rows
  std::vector<uint32_t> pblocks;
  for (uint32_t g = 0; g < ngroups; ++g) {
    const uint32_t R = (uint32_t)grows[g];
    const uint32_t pieces = (R + kSlabMax - 1) / kSlabMax;
    const uint32_t base = R / pieces, rem = R % pieces;
    const uint32_t W = (uint32_t)leaf_at(st, (int)gl[g][0])->ndt;
    uint32_t r = 0;
    for (uint32_t p = 0; p < pieces; ++p) {
      const uint32_t h = base + (p < rem ? 1 : 0);
      pblocks.push_back((uint32_t)plan.blocks.size());
      plan.blocks.push_back(Block{kRunP, (uint16_t)h, g, r, W, 0, 0});
      r += h;
    }
  }

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

  // ---- per-atom dense and low-rank leaf lists (CSR)
  std::vector<uint32_t> dcnt(natoms + 1, 0), ucnt(natoms + 1, 0);
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    const bool d = dense_active(s), u = lowrank_active(s);
    if (!d && !u) continue;
    int a0 = row_atom[s->nstrtl - 1], a1 = row_atom[s->nstrtl - 2 + s->ndl];
    for (int a = a0; a <= a1; ++a) (d ? dcnt : ucnt)[a + 1]++;
  }
  std::partial_sum(dcnt.begin(), dcnt.end(), dcnt.begin());
  std::partial_sum(ucnt.begin(), ucnt.end(), ucnt.begin());
  std::vector<uint32_t> dleaf(dcnt[natoms]), uleaf(ucnt[natoms]);
  {
    std::vector<uint32_t> dfill(dcnt.begin(), dcnt.end() - 1), ufill(ucnt.begin(), ucnt.end() - 1);
    for (int ip = 0; ip < nlf; ++ip) {
      const stc_HACApK_leafmtx *s = leaf_at(st, ip);
      const bool d = dense_active(s), u = lowrank_active(s);
      if (!d && !u) continue;
      int a0 = row_atom[s->nstrtl - 1], a1 = row_atom[s->nstrtl - 2 + s->ndl];
      for (int a = a0; a <= a1; ++a) {
        if (d) dleaf[dfill[a]++] = (uint32_t)ip;
        else uleaf[ufill[a]++] = (uint32_t)ip;
      }
    }
  }
  // D blocks (one per atom, possibly empty) and U blocks (atoms with low-rank rows)
  std::vector<uint32_t> dblock(natoms), ublock(natoms, 0xffffffffu);
  std::vector<uint64_t> acost(natoms, 0);
  for (int a = 0; a < natoms; ++a) {
    Block b{kRunD, (uint16_t)atoms[a].h, (uint32_t)a, 0, 0, (uint32_t)plan.pieces.size(), 0};
    for (uint32_t q = dcnt[a]; q < dcnt[a + 1]; ++q) {
      const stc_HACApK_leafmtx *s = leaf_at(st, (int)dleaf[q]);
      plan.pieces.push_back(Piece{dleaf[q], 0, (uint32_t)s->ndt, (uint32_t)(s->nstrtt - 1)});
      b.W += (uint32_t)s->ndt;
      b.npiece++;
    }
    dblock[a] = (uint32_t)plan.blocks.size();
    plan.blocks.push_back(b);
    acost[a] = block_cost(b.h, b.W, precision, costs);
    if (ucnt[a + 1] > ucnt[a]) {
      // zbu order, so that the segments of one column group merge
      std::sort(uleaf.begin() + ucnt[a], uleaf.begin() + ucnt[a + 1],
                [&](uint32_t x, uint32_t y) { return plan.zoff[x] < plan.zoff[y]; });
      Block u{kRunU, (uint16_t)atoms[a].h, (uint32_t)a, 0, 0, (uint32_t)plan.pieces.size(), 0};
      for (uint32_t q = ucnt[a]; q < ucnt[a + 1]; ++q) {
        const stc_HACApK_leafmtx *s = leaf_at(st, (int)uleaf[q]);
        plan.pieces.push_back(Piece{uleaf[q], 0, (uint32_t)s->kt, (uint32_t)plan.zoff[uleaf[q]]});
        u.W += (uint32_t)s->kt;
        u.npiece++;
      }
      ublock[a] = (uint32_t)plan.blocks.size();
      plan.blocks.push_back(u);
      acost[a] += block_cost(u.h, u.W, precision, costs);
    }
  }

  // ---- balance: P slabs first (they gate the grid barrier), then atoms
  Bins bins(num_ctas);
  std::vector<std::vector<uint32_t>> cta_p(num_ctas), cta_atoms(num_ctas);
  {
    std::vector<uint32_t> order(pblocks);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
      return block_cost(plan.blocks[x].h, plan.blocks[x].W, precision, costs) >
             block_cost(plan.blocks[y].h, plan.blocks[y].W, precision, costs);
    });
    for (uint32_t b : order) cta_p[bins.take(block_cost(plan.blocks[b].h, plan.blocks[b].W, precision, costs))].push_back(b);
    std::vector<int> aorder(natoms);
    std::iota(aorder.begin(), aorder.end(), 0);
    std::stable_sort(aorder.begin(), aorder.end(), [&](int x, int y) { return acost[x] > acost[y]; });
    for (int a : aorder) cta_atoms[bins.take(acost[a])].push_back((uint32_t)a);
  }

  // ---- emit run records and stream offsets per CTA
  plan.ctas.resize(num_ctas);
  uint64_t off = 0;
  std::vector<Seg> segs;
  for (int c = 0; c < num_ctas; ++c) {
    auto &pl = cta_p[c];
    auto &al = cta_atoms[c];
    std::sort(pl.begin(), pl.end());
    std::sort(al.begin(), al.end());
    CtaInfo info{};
    info.stream_off = off;
    info.rec_begin = (uint32_t)plan.recs.size();
    info.atom_begin = (uint32_t)plan.atoms.size();
    info.n_atoms = (uint32_t)al.size();
    // merge_keep >= 0: atoms with low-rank rows past the first merge_keep
    // take one kRunDU block; the atom list follows the blocks' order
    std::vector<uint32_t> split, merged;
    {
      uint32_t with_u = 0;
      for (uint32_t a : al) {
        const bool has_u = ublock[a] != 0xffffffffu;
        if (merge_keep >= 0 && has_u && with_u++ >= (uint32_t)merge_keep) merged.push_back(a);
        else split.push_back(a);
      }
    }
    for (uint32_t a : split) plan.atoms.push_back(atoms[a]);
    for (uint32_t a : merged) plan.atoms.push_back(atoms[a]);
    uint64_t pos = 0;
    uint32_t rot = 0, rot_step = 0;
    auto emit_block = [&](uint32_t bi) -> uint32_t {
      const Block &b = plan.blocks[bi];
      const uint32_t Wp = (b.W + RG - 1) / RG * RG;
      ColumnMap M{plan, b, 0};
      uint32_t out = 0;
      if (b.kind == kRunP) {
        const stc_HACApK_leafmtx *s = leaf_at(st, (int)plan.group_leaves[plan.group_leaf_begin[b.a]]);
        M.p_x0 = (uint32_t)(s->nstrtt - 1);
        out = (uint32_t)(gz[b.a] + b.r0);
      } else {
        out = atoms[b.a].r0;
      }
      uint32_t nr = 0, col = 0;
      do {
        uint32_t nc = std::min<uint32_t>(stage_cols, Wp - col);
        segments(M, col, std::min(col + nc, b.W), segs, !pair_panels);
        if (segs.size() > (size_t)kRunSegs) {
          // too many pieces: the widest run (a multiple of RG columns) whose
          // segments fit the record (the count grows with the width)
          uint32_t lo = RG, hi = nc - RG;
          while (lo < hi) {
            const uint32_t mid = ((lo + hi + RG) / 2) / RG * RG;
            segments(M, col, std::min(col + mid, b.W), segs, !pair_panels);
            if (segs.size() <= (size_t)kRunSegs) lo = mid;
            else hi = mid - RG;
          }
          nc = lo;
          segments(M, col, std::min(col + nc, b.W), segs, !pair_panels);
        }
        RunRec rec{};
        Run &r = rec.hdr;
        r.pos = (uint32_t)pos;
        r.out = out;
        r.nrow = b.h;
        r.npanel = (uint16_t)(nc / G);
        const bool last = (col + nc == Wp);
        r.flags = (uint16_t)(b.kind | (col == 0 ? kFirst : 0) | (last ? kLast : 0));
        r.rot = (uint16_t)rot;
        r.nseg = (uint16_t)segs.size();
        r.nlong = pair_panels ? 0 : count_long(segs);
        r.vlen = (uint16_t)(std::min(col + nc, b.W) - col);
        r.block = bi;
        r.col0 = col;
        std::copy(segs.begin(), segs.end(), rec.seg);
        plan.recs.push_back(rec);
        RunLite L{};
        L.pos = r.pos;
        L.out = r.out;
        L.npanel = r.npanel;
        L.nrow = (uint8_t)r.nrow;
        L.rot = (uint8_t)r.rot;
        L.rot_step = (uint16_t)rot_step;
        L.flags = r.flags;
        plan.lite.push_back(L);
        plan.pad_bytes += (uint64_t)elem_bytes(precision) * b.h * (nc - r.vlen);
        pos += 16ull * b.h * r.npanel;
        rot = (rot + r.npanel) % kProductWarps;
        rot_step = (rot_step + r.npanel) % kStepWarps;
        col += nc;
        ++nr;
      } while (col < Wp);
      return nr;
    };
    for (uint32_t b : pl) info.nr_p += emit_block(b);
    info.nblk_p = (uint32_t)pl.size();
    for (uint32_t a : split) info.nr_d += emit_block(dblock[a]);
    for (uint32_t a : split)
      if (ublock[a] != 0xffffffffu) info.nr_u += emit_block(ublock[a]);
    for (uint32_t a : merged) {
      const Block d = plan.blocks[dblock[a]], u = plan.blocks[ublock[a]];
      Block m{kRunDU, d.h, d.a, 0, d.W + u.W, (uint32_t)plan.pieces.size(), d.npiece + u.npiece};
      for (uint32_t q = 0; q < d.npiece; ++q) {
        const Piece pc = plan.pieces[d.piece_begin + q];
        plan.pieces.push_back(pc);
      }
      for (uint32_t q = 0; q < u.npiece; ++q) {
        Piece pc = plan.pieces[u.piece_begin + q];
        pc.vsrc |= kSegZbu;
        plan.pieces.push_back(pc);
      }
      plan.blocks.push_back(m);
      info.nr_u += emit_block((uint32_t)plan.blocks.size() - 1);
    }
    if (pos > 0xfffffff0ull) {
      err = "a CTA stream exceeds 4 GiB; use more CTAs";
      return HBX_ERR_INVALID;
    }
    // the multi-RHS kernel keeps every run summary in shared memory; the
    // single-RHS kernels read them from global memory past kMaxCtaRuns
    if (pair_panels && info.nr_p + info.nr_d + info.nr_u > (uint32_t)kMaxPairRuns) {
      err = "a CTA holds more than " + std::to_string(kMaxPairRuns) + " runs; use more CTAs";
      return HBX_ERR_INVALID;
    }
    info.stream_bytes = (uint32_t)pos;  // a multiple of 16 by construction
    plan.ctas[c] = info;
    off += (pos + 255) & ~uint64_t(255);
  }
  plan.total_bytes = std::max<uint64_t>(off, 256);
  return HBX_OK;
}

void pack_plan(const stc_HACApK_leafmtxp *st, const Plan &plan, uint8_t *dst) {
  const int nc = plan.num_ctas;
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nc; ++c) {
    const CtaInfo &info = plan.ctas[c];
    uint8_t *base = dst + info.stream_off;
    std::memset(base, 0, info.stream_bytes);
    const uint32_t nr = info.nr_p + info.nr_d + info.nr_u;
    std::vector<std::pair<uint32_t, uint32_t>> prow;  // P: (leaf, rank) of each slab row
    for (uint32_t k = 0; k < nr; ++k) {
      const Run &r = plan.recs[info.rec_begin + k].hdr;
      const Block &b = plan.blocks[r.block];
      const uint32_t h = r.nrow, G = group_cols(plan.precision), ncol = G * r.npanel;
      const int prec = plan.precision;
      double *d = reinterpret_cast<double *>(base + r.pos);
      float *f = reinterpret_cast<float *>(base + r.pos);
      uint16_t *hb = reinterpret_cast<uint16_t *>(base + r.pos);
      // element (row i, run column cc): panel cc/G, row i, slot cc%G (16-byte rows)
      auto put = [&](uint32_t i, uint32_t cc, double v) {
        const size_t k = ((size_t)(cc / G) * h + i) * G + cc % G;
        if (prec == kBF16) hb[k] = bf16_from_double(v);
        else if (prec == kFP32) f[k] = (float)v;
        else d[k] = v;
      };
      if (b.kind == kRunP) {
        // slab rows -> (leaf, rank); V_L(t, k) = a1[t + k*ndt]
        prow.clear();
        uint32_t row = 0;
        for (uint32_t q = plan.group_leaf_begin[b.a]; q < plan.group_leaf_begin[b.a + 1] && prow.size() < h; ++q) {
          const uint32_t ip = plan.group_leaves[q];
          const int kt = leaf_at(st, (int)ip)->kt;
          for (int kk = 0; kk < kt && prow.size() < h; ++kk, ++row)
            if (row >= b.r0) prow.push_back({ip, (uint32_t)kk});
        }
        for (uint32_t cc = 0; cc < ncol; ++cc) {
          const uint32_t col = r.col0 + cc;
          if (col >= b.W) continue;  // zero pad column
          for (uint32_t i = 0; i < h; ++i) {
            const stc_HACApK_leafmtx *s = leaf_at(st, (int)prow[i].first);
            put(i, cc, s->a1[(size_t)col + (size_t)prow[i].second * s->ndt]);
          }
        }
        continue;
      }
      // D / U: walk the pieces of the run's columns
      uint32_t piece = 0, piece_c0 = 0;
      for (uint32_t cc = 0; cc < ncol; ++cc) {
        const uint32_t col = r.col0 + cc;
        if (col >= b.W) continue;
        while (col >= piece_c0 + plan.pieces[b.piece_begin + piece].n) {
          piece_c0 += plan.pieces[b.piece_begin + piece].n;
          ++piece;
        }
        const Piece &P = plan.pieces[b.piece_begin + piece];
        const stc_HACApK_leafmtx *s = leaf_at(st, (int)P.leaf);
        const uint32_t lc = P.c0 + (col - piece_c0);
        // the block's atom rows, relative to the leaf's first row
        const uint32_t atom_r0 = r.out;
        const int ro = (int)atom_r0 - (s->nstrtl - 1);
        for (uint32_t i = 0; i < h; ++i) {
          double v;
          if (b.kind == kRunD || (b.kind == kRunDU && s->ltmtx == 2))
            v = s->a1[(size_t)lc + (size_t)(ro + (int)i) * s->ndt];  // A(il, it) = a1[it + il*ndt]
          else v = a2_of(s)[(size_t)(ro + (int)i) + (size_t)lc * s->ndl];              // U(i, l) = a2[i + l*ndl]
          put(i, cc, v);
        }
      }
    }
  }
}

int transpose_leaves(const stc_HACApK_leafmtxp *st, int nd, TransposedLeaves &out, std::string &err) {
  out = TransposedLeaves();
  if (!st || nd <= 0) { err = "null container or nd <= 0"; return HBX_ERR_INVALID; }
  const int nlf = st->nlf;
  if (nlf < 0 || (nlf > 0 && (!st->st_lf || st->st_lf_stride < (int)sizeof(stc_HACApK_leafmtx)))) {
    err = "bad leaf array (nlf, st_lf or st_lf_stride)";
    return HBX_ERR_INVALID;
  }
  // sizes first (one allocation), then the copies
  std::vector<size_t> off(nlf + 1, 0);
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    size_t words = 0;
    if (s->ndl > 0 && s->ndt > 0 && s->a1) {
      if (s->ltmtx == 2) words = (size_t)s->ndl * s->ndt;
      else if (s->ltmtx == 1 && s->kt > 0) words = (size_t)s->kt * (s->ndl + s->ndt);
    }
    off[ip + 1] = off[ip] + words;
  }
  out.data.resize(std::max<size_t>(1, off[nlf]));
  out.leaves.resize(std::max(1, nlf));
  for (int ip = 0; ip < nlf; ++ip) {
    const stc_HACApK_leafmtx *s = leaf_at(st, ip);
    stc_HACApK_leafmtx t = *s;
    t.nstrtl = s->nstrtt;
    t.ndl = s->ndt;
    t.nstrtt = s->nstrtl;
    t.ndt = s->ndl;
    t.a1 = nullptr;
    t.a2 = nullptr;
    t.a1size = 0;
    double *d = out.data.data() + off[ip];
    if (off[ip + 1] > off[ip]) {
      if (s->ltmtx == 2) {
        // A(il, it) = a1[it + il*ndt];  A^T(it, il) = a1'[il + it*ndl]
        for (int il = 0; il < s->ndl; ++il)
          for (int it = 0; it < s->ndt; ++it) d[(size_t)il + (size_t)it * s->ndl] = s->a1[(size_t)it + (size_t)il * s->ndt];
        t.a1 = d;
        t.a1size = (long long)s->ndl * s->ndt * 8;
      } else {
        // new V (ndt' x kt = ndl x kt) is the old U, new U is the old V
        const size_t nu = (size_t)s->ndl * s->kt, nv = (size_t)s->ndt * s->kt;
        std::memcpy(d, a2_of(s), nu * 8);
        std::memcpy(d + nu, s->a1, nv * 8);
        t.a1 = d;
        t.a1size = (long long)nu * 8;
        t.a2 = d + nu;
      }
    }
    out.leaves[ip] = t;
  }
  out.container = *st;
  out.container.st_lf = out.leaves.data();
  out.container.st_lf_stride = (int)sizeof(stc_HACApK_leafmtx);
  return HBX_OK;
}

int combine_leaves(const stc_HACApK_leafmtxp *const *st, const int *nd, int count, CombinedLeaves &out,
                   std::string &err) {
  out = CombinedLeaves();
  if (!st || !nd || count <= 0) { err = "no instances"; return HBX_ERR_INVALID; }
  out.off.assign(count + 1, 0);
  size_t nleaves = 0;
  int nlfkt = 0, ktmax = 0;
  for (int k = 0; k < count; ++k) {
    const stc_HACApK_leafmtxp *c = st[k];
    if (!c || nd[k] <= 0) { err = "instance " + std::to_string(k) + ": null container or nd <= 0"; return HBX_ERR_INVALID; }
    if (c->nlf < 0 || (c->nlf > 0 && (!c->st_lf || c->st_lf_stride < (int)sizeof(stc_HACApK_leafmtx)))) {
      err = "instance " + std::to_string(k) + ": bad leaf array (nlf, st_lf or st_lf_stride)";
      return HBX_ERR_INVALID;
    }
    if ((long long)out.off[k] + nd[k] > 0x7fffffffLL) { err = "combined size exceeds 2^31"; return HBX_ERR_INVALID; }
    out.off[k + 1] = out.off[k] + nd[k];
    nleaves += (size_t)c->nlf;
    nlfkt += c->nlfkt;
    ktmax = std::max(ktmax, c->ktmax);
  }
  out.leaves.reserve(std::max<size_t>(1, nleaves));
  for (int k = 0; k < count; ++k) {
    const stc_HACApK_leafmtxp *c = st[k];
    for (int ip = 0; ip < c->nlf; ++ip) {
      stc_HACApK_leafmtx t = *leaf_at(c, ip);
      if (t.nstrtl < 1 || t.nstrtt < 1 || t.nstrtl - 1 + t.ndl > nd[k] || t.nstrtt - 1 + t.ndt > nd[k]) {
        err = "instance " + std::to_string(k) + ", leaf " + std::to_string(ip) + ": outside [1, nd]";
        return HBX_ERR_INVALID;
      }
      t.nstrtl += out.off[k];
      t.nstrtt += out.off[k];
      out.leaves.push_back(t);
    }
  }
  if (out.leaves.empty()) out.leaves.resize(1);
  std::memset(&out.container, 0, sizeof(out.container));
  out.container.nd = out.off[count];
  out.container.nlf = (int)nleaves;
  out.container.nlfkt = nlfkt;
  out.container.ktmax = ktmax;
  out.container.st_lf_stride = (int)sizeof(stc_HACApK_leafmtx);
  out.container.st_lf = out.leaves.data();
  return HBX_OK;
}

// The instance range [lo, hi] of every stream chunk of every CTA of a
// block-diagonal engine (cinst, lo | hi << 16; lo > hi: no run bytes), and
// each CTA's first entry (cbase).  A run belongs to the instance of its
// output rows (D, U, merged D+U) or of its columns (P); false when a run's
// rows or x columns reach into two instances, which a block-diagonal leaf
// list never gives, and the engine then streams every chunk.
bool chunk_instances(const Plan &plan, const std::vector<int> &rinst, std::vector<uint32_t> &cinst,
                            std::vector<uint32_t> &cbase) {
  const size_t nrow = rinst.size();
  cinst.clear();
  cbase.assign(plan.ctas.size(), 0);
  for (size_t c = 0; c < plan.ctas.size(); ++c) {
    const CtaInfo &ci = plan.ctas[c];
    const uint32_t K = (ci.stream_bytes + kChunkBytes - 1) >> kChunkLog;
    cbase[c] = (uint32_t)cinst.size();
    std::vector<uint32_t> lo(K, 0xffffu), hi(K, 0u);
    const uint32_t nr = ci.nr_p + ci.nr_d + ci.nr_u;
    if ((size_t)ci.rec_begin + nr > plan.recs.size()) return false;
    for (uint32_t r = 0; r < nr; ++r) {
      const RunRec &rec = plan.recs[ci.rec_begin + r];
      const Run &hd = rec.hdr;
      const uint32_t bytes = run_bytes(hd);
      if (bytes == 0) continue;
      const uint32_t kind = run_kind(hd);
      int k = -1;
      auto same = [&](size_t row0, size_t len) {
        if (len == 0) return true;
        if (row0 + len > nrow) return false;
        if (k < 0) k = rinst[row0];
        return rinst[row0] == k && rinst[row0 + len - 1] == k;
      };
      if (kind != kRunP && !same(hd.out, hd.nrow)) return false;
      for (uint32_t q = 0; q < hd.nseg; ++q) {
        const Seg &sg = rec.seg[q];
        if (kind == kRunU || (kind == kRunDU && (sg.src & kSegZbu))) continue;  // zbu
        if (!same(sg.src, sg.len)) return false;
      }
      if (k < 0) continue;
      for (uint32_t g = hd.pos >> kChunkLog; g <= (hd.pos + bytes - 1) >> kChunkLog && g < K; ++g) {
        lo[g] = std::min(lo[g], (uint32_t)k);
        hi[g] = std::max(hi[g], (uint32_t)k);
      }
    }
    for (uint32_t g = 0; g < K; ++g) cinst.push_back(lo[g] | (hi[g] << 16));
  }
  if (cinst.empty()) cinst.push_back(0xffffu);
  return true;
}


}  // namespace hbx
