// hbx_plan.h -- device layout of a packed H-matrix and the host planner.
//
// Every part of the H-matvec is re-laid out, once at setup, as BLOCKS: a
// block is h <= 32 output rows times W columns, multiplied by a vector of W
// entries gathered from x or zbu.  Three kinds of blocks make up a matvec:
//
//   P  zbu = V^T x.  Low-rank leaves that share a column range (same nstrtt
//      and ndt: one column cluster) are stacked, so their V^T form one tall
//      matrix (sum of kt rows) over the same x segment; it is cut into slabs
//      of <= 64 rows.  zbu is numbered in this stacking order, so a slab
//      writes a contiguous zbu range.
//   D  the rows of the dense leaves that fall in one row atom, side by side
//      (W = sum of their ndt), times their x segments.
//   U  the rows of the U factors that fall in one row atom, side by side
//      (W = sum of their kt), times their zbu segments.
//
// Row atoms partition [0, nd) so that every leaf's row range is a union of
// atoms and no atom is taller than 32 rows.  An atom's D and U blocks belong
// to one CTA, which sums them in a fixed order and writes each row itself:
// no atomics, bit-reproducible results.  Every CTA's P blocks must finish
// (grid barrier) before any CTA reads zbu in its U blocks; the D blocks sit
// between the two so that the barrier latency is hidden.
//
// A block is stored as panels of column groups, each h x G row-major with
// 16-byte rows: G = 2 double columns (FP64 storage), G = 4 float columns
// (FP32 storage) or G = 8 bfloat16 columns (BF16 storage).  One 16-byte
// shared-memory load then gives a lane one row of G columns (and a second
// load row i + 32 in P slabs taller than 32), and
// the 32 lanes of a warp read h*16 consecutive bytes, free of bank
// conflicts.  A block's last panel is filled with zero columns.  A block's
// columns are cut into RUNS that fit the 8 KB vector stage buffer (1024
// doubles, or 2048 floats for FP32 and BF16 storage, whose vectors are
// staged as float) and a run record; all CTA data is one contiguous
// byte stream (P runs, then D runs, then U runs) that the kernel moves into
// shared memory with 1D bulk copies, so every byte of H crosses HBM once per
// matvec.
//
// Each run has a fixed-size record (header + gather segments) and a 16-byte
// summary (RunLite).  Gather warps read the records and fill a ring of
// kStages vector stage buffers with cp.async, runs ahead of the consumer
// warps; the consumer warps keep the CTA's summaries in shared memory.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hacapk_b200.h"

namespace hbx {

#ifdef __CUDACC__
#define HBX_HD __host__ __device__
#else
#define HBX_HD
#endif

constexpr int kAtomMax = 32;       // rows per D/U block (one lane per row)
constexpr int kSlabMax = 64;       // rows per P slab (two rows per lane)
// Consumer warps of the product kernels (k_matvec) and of the BiCGSTAB step
// kernel (k_bicg_iter, compiled in its own translation unit with fewer
// threads, so that it keeps its registers); the planner rotates the panels of
// consecutive runs for both counts.
constexpr int kProductWarps = 16;
constexpr int kStepWarps = 13;
// the FP32 / BF16 step kernels (a third translation unit): two groups of 6
#ifndef HBX_STEP_LP_WARPS
#define HBX_STEP_LP_WARPS 12
#endif
constexpr int kStepWarpsLp = HBX_STEP_LP_WARPS;
// The FP32 and BF16 product kernels split their consumer warps into groups
// that take alternate runs (warps [g*8, g*8+8) take runs r with r % 2 == g),
// so that the fixed work of one run overlaps the next run's; the FP64 product
// and the step kernels keep one group.
#ifndef HBX_PRODUCT_GROUPS
#define HBX_PRODUCT_GROUPS 2
#endif
constexpr int kProductGroups = HBX_PRODUCT_GROUPS;
static_assert(kProductWarps % kProductGroups == 0, "equal consumer groups");
#ifndef HBX_CONSUMER_WARPS
#define HBX_CONSUMER_WARPS 16
#endif
constexpr int kConsumerWarps = HBX_CONSUMER_WARPS; // warps that multiply (+ producer, gather, grid-barrier and block-sum warps)

#ifndef HBX_CHUNK_LOG
#define HBX_CHUNK_LOG 15
#endif
#ifndef HBX_RING_CHUNKS
#define HBX_RING_CHUNKS 4
#endif
constexpr int kChunkLog = HBX_CHUNK_LOG;      // ring chunk = 32 KB (bulk copies this size stream at HBM rate)
constexpr int kChunkBytes = 1 << kChunkLog;
constexpr int kRingChunks = HBX_RING_CHUNKS;  // 128 KB ring per CTA
#ifndef HBX_STAGE_BYTES
#define HBX_STAGE_BYTES 8192
#endif
constexpr int kStageBytes = HBX_STAGE_BYTES;  // one vector stage buffer: 1024 doubles or 2048 floats (8 KB)
constexpr int kPairStageBytes = 8192;         // run width of the multi-RHS layout (2048 float columns)
static_assert(kStageBytes % 16 == 0 && kStageBytes >= kPairStageBytes && kStageBytes / 4 <= 65535,
              "stage size: 16-byte multiple, at least the multi-RHS run width, columns within 16-bit offsets");
constexpr int kStageCap = kStageBytes / 8;  // doubles per stage buffer
constexpr int kRunSegs = 124;      // gather segments per run record
constexpr int kSegShort = 32;      // a segment this long or shorter is copied by one gather lane;
                                   // a longer one by the whole gather warp
constexpr int kRecBytes = 1024;    // one run record: 32-byte header + kRunSegs segments
#ifndef HBX_STAGES
#define HBX_STAGES 4
#endif
constexpr int kStages = HBX_STAGES;  // vector stage buffers: runs gathered ahead of the consumers
constexpr int kMaxCtaRuns = 1024;    // run summaries a CTA keeps in shared memory (more: read from global memory)
constexpr int kMaxPairRuns = 512;    // the same for the multi-RHS engine (pair-panel plans)

// kRunDU: an atom's dense and low-rank columns in one block (x segments,
// then zbu segments marked by kSegZbu), placed in the U section (its gather
// waits for zbu); only plans made with merge_keep >= 0 hold it.
enum RunKind : uint16_t { kRunP = 0, kRunD = 1, kRunU = 2, kRunDU = 3 };
constexpr uint32_t kSegZbu = 0x80000000u;  // kRunDU segment source: zbu (else x)
enum RunFlags : uint16_t { kFirst = 0x100, kLast = 0x200 };

// Storage precision of the packed factors.  A panel row is always 16 bytes:
// two double, four float or eight bfloat16 columns.  The gathered vectors
// are double for FP64 storage and float otherwise.
enum Precision : int { kFP64 = 0, kFP32 = 1, kBF16 = 2 };
HBX_HD constexpr uint32_t group_cols(int prec) { return prec == kBF16 ? 8u : (prec == kFP32 ? 4u : 2u); }
HBX_HD constexpr uint32_t elem_bytes(int prec) { return prec == kBF16 ? 2u : (prec == kFP32 ? 4u : 8u); }
HBX_HD constexpr uint32_t stage_elem_bytes(int prec) { return prec == kFP64 ? 8u : 4u; }

// bfloat16: the high half of a float.  Storage rounds a double to the
// nearest bfloat16, ties to even, in one step (no intermediate float
// rounding); bfloat16 has float's exponent range, so every factor keeps 8
// significant bits whatever its magnitude.  Below 2^-126 the bfloat16
// values are subnormal, multiples of 2^-133: the double is scaled to units
// of 2^-133 (exactly) and rounded to the nearest integer, ties to even.
inline uint16_t bf16_from_double(double v) {
  uint64_t b;
  std::memcpy(&b, &v, sizeof b);
  const uint64_t mag = b & 0x7fffffffffffffffull;
  const uint16_t sign = (uint16_t)((b >> 48) & 0x8000u);
  if (mag >= 0x7ff0000000000000ull) {  // inf / nan
    const float f = (float)v;
    uint32_t u;
    std::memcpy(&u, &f, sizeof u);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);  // quiet nan
    return (uint16_t)(u >> 16);
  }
  if (mag < 0x3810000000000000ull) {  // below 2^-126
    double m;
    std::memcpy(&m, &mag, sizeof m);
    const double q = std::ldexp(m, 133);  // < 128, exact
    double k = std::floor(q);
    const double f = q - k;                // exact
    if (f > 0.5 || (f == 0.5 && std::fmod(k, 2.0) != 0.0)) k += 1.0;
    return (uint16_t)(sign | (uint16_t)k);  // k == 128 is the smallest normal, 2^-126
  }
  // keep 7 fraction bits of the 52: round the low 45 bits to nearest, ties to even
  b += (1ull << 44) - 1ull + ((b >> 45) & 1ull);
  b &= ~((1ull << 45) - 1ull);
  double r;
  std::memcpy(&r, &b, sizeof r);
  const float f = (float)r;  // exact, or +-inf past float's range
  uint32_t u;
  std::memcpy(&u, &f, sizeof u);
  return (uint16_t)(u >> 16);
}
inline float bf16_to_float(uint16_t h) {  // host side (the kernels shift in registers)
  const uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, sizeof f);
  return f;
}

// Gather segment: stage[dst + e] = vec[src + e], e < len (vec = x or zbu).
struct Seg {
  uint32_t src;
  uint16_t len;
  uint16_t dst;
};
static_assert(sizeof(Seg) == 8, "Seg layout");

// 32-byte run header; its segments follow it in the run record.
struct alignas(16) Run {
  uint32_t pos;    // byte offset of the run's pair panels in the CTA stream (16-aligned)
  uint32_t out;    // first output row: zbu index (P) or y row (D, U)
  uint16_t nrow;   // h: 1..32 for D/U, 1..64 for P
  uint16_t npanel; // column-group panels (2 columns each for FP64, 4 for FP32)
  uint16_t flags;  // RunKind | RunFlags
  uint16_t rot;    // consumer warp that takes panel 0
  uint16_t nseg;   // gather segments (<= kRunSegs)
  uint16_t vlen;   // real columns; the stage is zero from vlen to the end of the last panel
  uint32_t block;  // block index (host-side packing and checks)
  uint32_t col0;   // first block column of the run
  uint32_t nlong;  // the first nlong segments are longer than kSegShort
};
static_assert(sizeof(Run) == 32, "Run must stay 32 bytes");

// What the consumer and block-sum warps need of a run (16 bytes, kept in
// shared memory for the whole launch).
struct alignas(16) RunLite {
  uint32_t pos;     // byte offset of the run's panels in the CTA stream
  uint32_t out;     // first output row: zbu index (P) or y row (D, U)
  uint16_t npanel;  // column-group panels
  uint8_t nrow;     // h: 1..32 (1..64 for P)
  uint8_t rot;      // consumer warp that takes panel 0 (kProductWarps consumers)
  uint16_t flags;   // RunKind | RunFlags
  uint16_t rot_step;  // the same for kStepWarps consumers
};
static_assert(sizeof(RunLite) == 16, "RunLite layout");

struct alignas(16) RunRec {
  Run hdr;
  Seg seg[kRunSegs];
};
static_assert(sizeof(RunRec) == kRecBytes, "RunRec must be kRecBytes");

HBX_HD inline uint32_t run_kind(const Run &r) { return r.flags & 0xffu; }
HBX_HD inline uint32_t run_bytes(const Run &r) { return 16u * r.nrow * r.npanel; }

struct CtaInfo {
  uint64_t stream_off;    // byte offset of the CTA stream in the packed buffer
  uint32_t stream_bytes;  // multiple of 16
  uint32_t rec_begin;     // first run record (and summary) of the CTA (P, D, U runs in order)
  uint32_t nr_p, nr_d, nr_u;
  uint32_t atom_begin, n_atoms;  // owned atoms (rows written by this CTA)
  uint32_t nblk_p;               // P blocks (slabs) of the CTA
  uint32_t pad[6];
};
static_assert(sizeof(CtaInfo) == 64, "CtaInfo layout");

struct Atom {
  uint32_t r0, h;
};

// Host-only description of a block, used by the packer and the checks.
// kind P: `a` = column group, rows [r0, r0+h) of the group's stacked rows.
// kind D/U: `a` = row atom; columns are the pieces [piece_begin, +npiece).
struct Block {
  uint16_t kind, h;
  uint32_t a, r0, W;
  uint32_t piece_begin, npiece;
};
// A run of block columns taken from one leaf: D -> leaf columns [c0, c0+n)
// (x index vsrc); U -> ranks [c0, c0+n) of the leaf (zbu index vsrc).
struct Piece {
  uint32_t leaf, c0, n, vsrc;
};

// The balancing cost model: a block costs its bytes plus `block` plus `run`
// per stage-full of columns (the fixed work of a block end and of a run).
#ifndef HBX_BLOCK_COST
#define HBX_BLOCK_COST 8192
#endif
#ifndef HBX_RUN_COST
#define HBX_RUN_COST 4096
#endif
struct PlanCosts {
  uint64_t block = HBX_BLOCK_COST;
  uint64_t run = HBX_RUN_COST;
};

// Host-side plan: everything needed to pack and launch.
struct Plan {
  int nd = 0, nlf = 0, nlfkt = 0, ktmax = 0;
  int num_ctas = 0;
  int precision = kFP64;
  bool pair_panels = false;         // multi-RHS layout (even panel counts, segments in stage order)
  PlanCosts costs;                  // the balancing cost model the plan was made with
  std::vector<Atom> atoms;          // in CTA order (atom_begin indexes this)
  std::vector<RunRec> recs;         // in CTA order
  std::vector<RunLite> lite;        // one summary per record, same order
  std::vector<CtaInfo> ctas;
  std::vector<Block> blocks;
  std::vector<Piece> pieces;
  std::vector<uint32_t> group_leaf_begin, group_leaves;  // P column groups (CSR over leaf indices)
  std::vector<uint64_t> zoff;       // zbu offset of each low-rank leaf
  uint64_t total_bytes = 0;         // packed buffer size
  uint64_t zbu_len = 0;
  uint64_t dense_words = 0, lowrank_words = 0;
  uint64_t pad_bytes = 0;           // zero columns that fill a block's last panel
  uint64_t alg_bytes = 0, alg_flops = 0;
};

// Validates the leaf list and builds the plan.  Returns HBX_OK or an error
// (message in `err`).
// pair_panels (FP32 only): every run holds an even number of panels and its
// segments stay in stage order -- the layout of the multi-RHS engine.
// merge_keep >= 0 (single-vector layouts only): every atom with low-rank
// rows, except the first merge_keep such atoms of each CTA, gets one kRunDU
// block in place of its D and U blocks; the CTA's atom list then holds the
// atoms of its D blocks, then those of its kRunDU blocks.  The default, -1,
// keeps every atom split.
int make_plan(const stc_HACApK_leafmtxp *st, int nd, int num_ctas, Plan &plan, std::string &err,
              int precision = kFP64, bool pair_panels = false, const PlanCosts &costs = PlanCosts(),
              int merge_keep = -1);

// Writes the packed stream of every CTA into `dst` (plan.total_bytes bytes).
void pack_plan(const stc_HACApK_leafmtxp *st, const Plan &plan, uint8_t *dst);

// Block-diagonal engines: the instance range of every stream chunk of every
// CTA (cinst[cbase[c] + g] = lo | hi << 16, lo > hi when the chunk holds no
// run bytes), from the host run records and the instance of every row.
// False when a run reaches into two instances.
bool chunk_instances(const Plan &plan, const std::vector<int> &rinst, std::vector<uint32_t> &cinst,
                     std::vector<uint32_t> &cbase);

// The leaf list of H^T, in host memory owned by the object: a dense leaf
// (ndl x ndt) becomes its transpose (ndt x ndl); a low-rank leaf U V^T becomes
// V U^T (the factors swap places, no arithmetic), so the packed H^T streams
// exactly the bytes of H.  The reference has no transposed product
// (HACApK_BATCH_SORT.c:123 only changes the storage orientation of A*x).
struct TransposedLeaves {
  std::vector<stc_HACApK_leafmtx> leaves;
  std::vector<double> data;
  stc_HACApK_leafmtxp container{};
};
int transpose_leaves(const stc_HACApK_leafmtxp *st, int nd, TransposedLeaves &out, std::string &err);

// The leaves of `count` independent H-matrices as one block-diagonal leaf
// list: instance k's rows and columns move by off[k] = nd[0] + ... +
// nd[k-1] (off[count] = the total size).  The factors are not copied: the
// combined leaves point at the instances' own data.
struct CombinedLeaves {
  std::vector<stc_HACApK_leafmtx> leaves;
  std::vector<int> off;
  stc_HACApK_leafmtxp container{};
};
int combine_leaves(const stc_HACApK_leafmtxp *const *st, const int *nd, int count, CombinedLeaves &out,
                   std::string &err);

}  // namespace hbx
