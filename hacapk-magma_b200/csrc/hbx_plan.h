// hbx_plan.h -- device layout of a packed H-matrix and the host planner.
//
// The leaf list is re-laid out once, at setup, into one byte stream per
// persistent CTA.  A CTA's stream is contiguous in HBM, so the kernel moves
// it into shared memory with plain 1D bulk copies (cp.async.bulk) through a
// ring of fixed-size chunks, and every byte of H crosses HBM exactly once per
// matvec.  The stream holds three sections, each a list of terms:
//
//   P  V-panels: columns [l0, l0+kc) of a low-rank leaf's V (ndt x kt),
//      stored as row chunks of <= PANEL_ROWS rows, column-major inside a
//      chunk; one term per chunk (flags mark a panel's first and last
//      chunk).  Output: zbu[out + l] = sum_t V(t, l0+l) x(nstrtt-1+t).
//   D  dense terms: the rows of a dense leaf that fall in one row atom,
//      h x ndt column-major.  Output accumulated into the atom's rows.
//   U  low-rank terms: the rows of U (ndl x kt) that fall in one row atom,
//      h x kt column-major, multiplied by the leaf's zbu segment.
//
// Row atoms partition [0, nd) so that every leaf's row range is a union of
// atoms and no atom is taller than 32 rows.  Each atom belongs to exactly
// one CTA, which sums all its D and U terms in a fixed order and writes the
// rows once: no atomics, bit-reproducible results.  The P section of every
// CTA must complete (grid barrier) before any CTA reads zbu in its U section;
// the D section sits between the two so the barrier latency is hidden.
//
// Every term reads one contiguous vector segment (P: x over its rows, D: x
// over its columns, U: zbu over its columns).  Consecutive terms of a section
// are grouped into runs whose segments fit a shared-memory stage buffer; the
// consumers gather run k+1's segments with cp.async while they compute run k,
// so no vector load is on the critical path.  A D or U run holds terms of one
// atom only; their data is back to back in the stream and their segments back
// to back in the stage, so the kernel treats the whole run as one h x W
// column-major block times one staged vector.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/hacapk_b200.h"

namespace hbx {

constexpr int kAtomMax = 32;       // rows per atom (one lane per row)
constexpr int kPanelRows = 256;    // rows per V-panel chunk (8 per lane)
constexpr int kConsumerWarps = 16; // warps that compute (+ a producer and a descriptor warp)
constexpr int kPanelCols = kConsumerWarps;  // columns per V-panel (one per consumer warp)
constexpr int kChunkLog = 15;      // ring chunk = 32 KB (bulk copies this size stream at HBM rate)
constexpr int kChunkBytes = 1 << kChunkLog;
constexpr int kRingChunks = 4;     // 128 KB ring per CTA
constexpr int kStageCap = 1024;    // doubles per vector stage buffer (x2)
constexpr int kRunTerms = 64;      // terms per run (descriptor queue slot)
constexpr int kDescSlots = 4;      // runs staged ahead by the descriptor warp

enum TermKind : uint16_t { kTermP = 0, kTermD = 1, kTermU = 2 };
enum TermFlags : uint16_t { kAtomEnd = 0x100, kPanelFirst = 0x200, kPanelLast = 0x400 };

// 32-byte term descriptor.
struct alignas(16) Term {
  uint32_t pos;    // byte offset of the term's data inside the CTA stream
  uint32_t nrow;   // P: chunk rows (<= kPanelRows);  D/U: atom height h
  uint32_t ncol;   // P: kc;  D: columns (of ndt);  U: columns (of kt)
  uint32_t vec;    // start of the vector segment: P, D: x index;  U: zbu index
  uint32_t out;    // P: zbu offset of the panel's column 0;  D/U: first atom row
  uint16_t kind;   // TermKind | TermFlags
  uint16_t rot;    // consumer warp that takes column 0 of this term
  uint32_t leaf;   // leaf index (packing and diagnostics)
  uint32_t voff;   // offset of the vector segment in the run's stage buffer
};

#ifdef __CUDACC__
#define HBX_HD __host__ __device__
#else
#define HBX_HD
#endif

HBX_HD inline uint32_t term_vlen(const Term &t) {
  return (t.kind & 0xff) == kTermP ? t.nrow : t.ncol;
}

struct alignas(16) Run {
  uint32_t term_first;  // absolute index into the term array
  uint32_t nterm;
  uint32_t vlen;        // doubles gathered into the stage buffer
  uint32_t pos;         // D/U: byte offset of the run's h x W block
  uint32_t nrow;        // D/U: atom height h
  uint32_t ncol;        // D/U: W = total columns of the run's terms
  uint32_t out;         // D/U: first row of the atom
  uint16_t flags;       // kAtomEnd when the run closes its atom
  uint16_t rot;         // consumer warp that takes column 0
};
static_assert(sizeof(Run) == 32, "Run must stay 32 bytes");
static_assert(sizeof(Term) == 32, "Term must stay 32 bytes");

struct CtaInfo {
  uint64_t stream_off;   // byte offset of the CTA stream in the packed buffer
  uint32_t stream_bytes; // multiple of 16
  uint32_t term_begin;
  uint32_t n_p, n_d, n_u;
  uint32_t atom_begin, n_atoms;  // owned atoms (rows written by this CTA)
  uint32_t run_begin;            // runs of the P, D, U sections, in order
  uint32_t nr_p, nr_d, nr_u;
  uint32_t pad[3];
};
static_assert(sizeof(CtaInfo) == 64, "CtaInfo layout");

struct Atom {
  uint32_t r0, h;
};

// Host-side plan: everything needed to pack and launch.
struct Plan {
  int nd = 0, nlf = 0, nlfkt = 0, ktmax = 0;
  int num_ctas = 0;
  std::vector<Atom> atoms;          // in CTA order (atom_begin indexes this)
  std::vector<Term> terms;          // in CTA order
  std::vector<Run> runs;            // in CTA order
  std::vector<CtaInfo> ctas;
  uint64_t total_bytes = 0;         // packed buffer size
  uint64_t zbu_len = 0;
  uint64_t dense_words = 0, lowrank_words = 0;
  uint64_t alg_bytes = 0, alg_flops = 0;
};

// Validates the leaf list and builds the plan.  Returns HBX_OK or an error
// (message in `err`).
int make_plan(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, Plan &plan, std::string &err);

// Writes the packed stream of every CTA into `dst` (plan.total_bytes bytes).
void pack_plan(const stc_HACApK_leafmtxp *st, const Plan &plan, uint8_t *dst);

}  // namespace hbx
