// Host-side layout builder for the streamed H-matrix matvec.
//
// The reference applies y = sum_FR A x + sum_LR A (B x) block by block
// (src/hmat/hmatrix/hmat.cc:472-537).  On the device the same product runs as
// two streaming passes over re-laid-out block data:
//
//  phase 1 ("B stage"):   t = B_b x[cols_b] for every low-rank block b.
//      The B factors of all low-rank blocks that share one column cluster are
//      stacked into one tall matrix (they multiply the same slice of x); the
//      stack is cut into items of at most kHMax rows.  t is ordered by stack.
//  phase 2 ("row panels"): y[p] = sum over the blocks that cover row panel p of
//      (slice of A_b or of the full block) times (t_b or x[cols]).
//      Row panels are the finest partition of the rows by block boundaries, so
//      every block covers whole panels.  One item per panel: the slices of all
//      covering blocks side by side.
//
// Every item is a dense h x n matrix times a gathered vector, owned by one
// CTA, so outputs are written once, without atomics.  Rows are padded to a
// multiple of 8.  FP64 and FP32 items are column-major (ld = padded rows);
// BF16 items are stored as 8x8 tiles (column group, then row group, then
// 8 columns x 8 contiguous rows) so that tensor-core fragment loads from shared
// memory are 128-byte contiguous.  An item is cut into chunks of at most
// kStageBytes; a chunk is what one TMA bulk copy stages into shared memory
// (plus one more for its contiguous run of vector values).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace bw {

constexpr int kStageBytes = 32768;   // bytes of block data per pipeline stage
constexpr int kMaxCols = 512;        // columns per chunk (size of a stage's gather buffer)
constexpr int kHMax = 512;           // max padded rows of one item
constexpr int kRowAlign = 8;         // padded rows are a multiple of this
constexpr int kItemAlign = 64;       // item start alignment, in elements
constexpr int kItemsPerCta = 8;      // minimum items per CTA share (load balance)

// Chunk flags
constexpr uint32_t kFirst = 1u;      // first chunk of an item: reset accumulators
constexpr uint32_t kLast = 2u;       // last chunk of an item: reduce and write the output
constexpr uint32_t kEnd = 4u;        // no more chunks for this CTA (written by the producer, never stored)

// One chunk descriptor, 32 bytes, read by the producer warp and copied into
// shared memory for the consumer warps.  The vector values of the chunk's
// columns are the contiguous run gsrc[g_off .. g_off + ncols), where gsrc is
// the gathered x for phase 1 (stacked B rows multiply one slice of x) and the
// per-matvec gather array G2 for phase 2.
struct alignas(16) Chunk {
  int64_t data_off;  // element offset of the chunk's first column in the data array
  int32_t ncols;     // columns in this chunk
  int32_t hpad;      // padded row count of the item (multiple of 8)
  int32_t rows;      // rows of the item to write (<= hpad)
  int32_t out_off;   // first output index: t offset (phase 1) or row (phase 2)
  uint32_t flags;    // kFirst | kLast
  int32_t g_off;     // first vector value in the phase's gather source
};
static_assert(sizeof(Chunk) == 32, "chunk descriptor must be 32 bytes");
constexpr int kChunkWords = sizeof(Chunk) / 4;

// One run of G2: G2[dst .. dst + cols) = scale * src[src_off .. src_off + cols)
// with src = x (gathered) or t.  Built once per matvec before phase 2.
struct GatherSeg {
  int32_t dst;
  int32_t src_off;
  uint32_t cols_src;  // cols | src << 31
  float scale;        // BF16: the full block's scale; 1 elsewhere
};
static_assert(sizeof(GatherSeg) == 16, "gather segment must be 16 bytes");

// A read-only view of a column-major block (or of its transpose).
struct View {
  const double *p = nullptr;
  int64_t ld = 0;
  bool trans = false;
  double at(int64_t i, int64_t j) const { return trans ? p[i * ld + j] : p[i + j * ld]; }
};

struct FullBlock {
  int64_t i0, j0, m, n;
  View a;
};
struct LowRankBlock {
  int64_t i0, j0, m, n, r;
  View A, B;  // A: m x r, B: r x n
};

// Column segment of an item: where its vector values come from and, for
// phase 2, which block slice fills its data.
struct Segment {
  int kind;        // 0: FR slice, 1: LR A slice, 2: LR B stack (rows from Item::pieces)
  int64_t block;   // block index (kinds 0, 1)
  int64_t row0;    // first row of the block in this item (kinds 0, 1)
  int64_t ncols;   // columns
  int src;         // 0: x, 1: t
  int64_t src_off; // offset in x or t
};

// Rows [r0, r0 + n) of the B factor of low-rank block `block` (phase 1).
struct RowPiece {
  int64_t block, r0, n;
};

struct Item {
  int64_t off[3] = {0, 0, 0};  // element offset in the phase's data array, per precision
  int32_t h = 0, hpad = 0;     // rows, padded rows
  int64_t ncols = 0;           // total columns
  int32_t out_off = 0;
  std::vector<Segment> segs;
  std::vector<RowPiece> pieces;  // phase 1 only
};

// Per precision: the chunks item by item, items in the order the CTAs take
// them (decreasing cost), the chunk ranges of the queue units (runs of
// consecutive items, Tuning::unit_bytes), and (phase 2) the runs that fill
// the gather array G2 of g_len values.
struct ChunkPlan {
  std::vector<Chunk> chunks;
  std::vector<int32_t> item_ptr;  // queue units + 1 (chunk index of each unit's first chunk)
  std::vector<GatherSeg> gsegs;   // phase 2 only
  int64_t g_len = 0;
};

struct PhasePlan {
  std::vector<Item> items;
  int64_t n_elems[3] = {0, 0, 0};  // size of the data array in elements, per precision
  ChunkPlan cp[3];                 // FP64, FP32, BF16
};

struct OperatorPlan {
  int64_t n_out = 0, n_in = 0;  // rows of the operator, columns
  int64_t t_len = 0;            // sum of ranks
  std::vector<int64_t> t_off;   // per LR block
  std::vector<float> scale_fr;  // BF16 scales per FR block
  std::vector<float> scale_a, scale_b;  // BF16 scales per LR block
  std::vector<float> t_scale;   // BF16: per t entry, scale_a * scale_b of its block
  PhasePlan ph[2];
  int64_t n_panels = 0;
  int64_t n_stacks = 0;
};

// Queue units: consecutive items (in the queue's longest-first order) are
// handed out together until the unit's cost reaches this many bytes, so a
// CTA makes one queue round trip (atomic + chunk-range loads) per unit
// rather than per item.  0 (the default): one item per unit.  Measured on the
// 48 x 2DS0-H batch (items of ~10 KB): 64 KB units change FP64 phase 1 from
// 163 to 150 us but BF16 phase 1 from 163 to 181 us (coarser units balance
// worse); the queue round trip is not what limits small items.
constexpr int kUnitBytes = 0;

// Plan parameters a tuner may change (bw_set_tuning); the defaults are the
// compiled-in choices.
struct Tuning {
  int items_per_cta[2] = {kItemsPerCta, kItemsPerCta};  // per phase: items per CTA share (granularity)
  int chunk_bytes = kStageBytes;                        // block data per chunk (<= kStageBytes)
  int mm_items_per_cta = kItemsPerCta;                  // matmat phase 1
  int unit_bytes = kUnitBytes;                          // streaming queue: minimum cost of a unit
  int narrow_rows = 64;   // items of at most this many padded rows skip the staging (0: never) ...
  int narrow_cols = 512;  // ... warp per item up to this many columns, CTA-cooperatively above
  int narrow_coop = 0;    // 1: items above narrow_cols columns run a CTA each in the unstaged kernel
};

// Queue units [0, wide) of a phase run in the CTA-wide kernel; of the rest,
// [wide, coop) CTA-cooperatively and [coop, end) warp per item.
struct NarrowSplit {
  int64_t wide = 0, coop = 0;
};

struct Problem {
  Tuning tune;
  int dof = 1;
  int64_t n_rows = 0, n_cols = 0;
  std::vector<FullBlock> fr;
  std::vector<LowRankBlock> lr;
  // Batch members (block-diagonal problem): member k owns rows
  // [row_off[k], row_off[k+1]) and columns [col_off[k], col_off[k+1]); blocks
  // must tile each member's diagonal block.  Empty: one member.
  std::vector<int64_t> row_off, col_off;
};

// Validates the pattern and builds the structural plan (items) of the operator
// (transposed = true builds H^T from the same blocks).  Throws std::runtime_error
// with a message on a malformed pattern.
// Items are cut so that none holds more than 1/kItemsPerCta of the average
// per-CTA share of `grid` CTAs (static scheduling needs fine grains).
void build_operator(const Problem &p, bool transposed, int grid, OperatorPlan &op);

// Computes BF16 per-block scales (max |entry|, 1 if the block is zero) and the
// per-t-entry scales, and checks that every entry is finite when check_finite.
void compute_scales(const Problem &p, bool transposed, bool check_finite, OperatorPlan &op);

// Lays out every item for one precision (0 FP64, 1 FP32, 2 BF16), splits it
// into chunks, and orders the items longest first (cost = bytes + a per-chunk
// overhead): the kernel's CTAs take them in that order from a device queue.
void build_chunks(const Problem &p, bool transposed, int prec, int grid, OperatorPlan &op);

// Writes the data of items [i_begin, i_end) of one phase, converted to the
// precision and in its layout, into dst (dst[0] is element `base` of the
// phase's array).
void fill_items(const Problem &p, bool transposed, const OperatorPlan &op, int phase, int prec, int64_t i_begin,
                int64_t i_end, int64_t base, void *dst);

// Element index of (row i, column c) of an item inside the item's data.
inline int64_t item_index(int prec, int64_t hpad, int64_t i, int64_t c) {
  if (prec == 2) return (c >> 3) * (8 * hpad) + (i >> 3) * 64 + (c & 7) * 8 + (i & 7);
  return c * hpad + i;
}
// Elements an item occupies.
inline int64_t item_elems(int prec, int64_t hpad, int64_t ncols) {
  if (prec == 2) return ((ncols + 7) / 8) * 8 * hpad;
  return ncols * hpad;
}

int esize_of(int prec);
uint16_t to_bf16(float f);
float from_bf16(uint16_t b);

// ----------------------------------------------------------------------------
// Multi-right-hand-side layout: Y = H X on the tcgen05 tensor cores.
//
// The same two phases as the matvec, but every chunk is a small GEMM
// D(rows x 64) += A(rows x kc) * B(kc x 64):
//  * A is the chunk's block data in BF16 8x8 tiles (the layout above);
//  * B is a run of rows of an 8x8-tiled BF16 operand with kMmRhs columns.
//    That operand is X (the gathered right-hand sides) in phase 1 and for
//    full-rank slices, and T8 (the phase-1 products) for low-rank slices.
//  * The 8x8 tiles are the MN-major, no-swizzle canonical operand layout of
//    tcgen05.mma.
// Runs of operand rows must start on an 8-row tile boundary, so:
//  * every column segment of an item is widened to the 8-aligned window of
//    operand rows around it, with zeros in the widened columns;
//  * T8 numbers the products of each low-rank block from an 8-aligned
//    offset, its rank rounded up to a multiple of 8 with zero rows;
//  * items are padded to a multiple of 16 columns (one MMA K-step) and to at
//    least 32 (the K-steps of an item alternate between two MMA issuers);
//  * items have at most 256 rows (two M = 128 tiles).
// The phases:
//  * phase 1: stacks of B factors per column cluster, as for the matvec, with
//    rows on T8's numbering;
//  * phase 2: row panels, with FR and A slices on their widened windows.
// Block data is stored unscaled: BF16 has FP32's exponent range, so a
// per-block scale would leave every rounded mantissa unchanged.
constexpr int kMmRhs = 64;             // right-hand sides per pass (MMA N)
constexpr int kMmStageBytes = 49152;   // block data + operand rows of one pipeline stage
constexpr int kMmMaxRuns = 4;          // operand runs per chunk (a chunk ends early to keep this)
constexpr int kMmMaxCols = 512;        // columns per chunk
constexpr int kMmHMax = 256;           // rows per item (two M = 128 tiles)
constexpr int kMmMinCols = 32;         // columns per item (two K-steps: one per MMA issuer)
constexpr int kMmPadRows = 32;         // zero operand rows after X and T8 that widened windows may reach

struct MmRun {
  uint32_t src;   // first operand row (multiple of 8) | operand << 31 (0: X, 1: T8)
  uint32_t rows;  // operand rows (multiple of 8)
};
// One chunk descriptor, 64 bytes, with its operand runs inline.
struct alignas(16) MmChunk {
  int64_t data_off;  // element offset of the chunk's first column group
  int32_t kc;        // columns (multiple of 16); the runs cover exactly kc operand rows
  int32_t hpad;      // rows of the item's tiles (multiple of 8, <= kHMax)
  int32_t rows;      // rows of the item to write
  int32_t out_off;   // first output row: T8 row (phase 1) or y row (phase 2)
  uint32_t flags;    // kFirst | kLast | (number of runs << 8)
  uint32_t pad_;
  MmRun run[kMmMaxRuns];
};
static_assert(sizeof(MmChunk) == 64, "matmat chunk descriptor must be 64 bytes");
constexpr int kMmChunkWords = sizeof(MmChunk) / 4;

// Column segment of a matmat item: operand rows [src_row, src_row + ncols),
// the block's real columns at [lead, lead + width) of the window.
struct MmSeg {
  int kind;          // 0: FR slice, 1: LR A slice, 2: LR B stack
  int64_t block;     // kinds 0, 1
  int64_t row0;      // first row of the block in this item (kinds 0, 1)
  int64_t lead, width, ncols;
  int src;           // 0: X, 1: T8
  int64_t src_row;
};

struct MmStack {
  int64_t j0, n;                // column cluster
  std::vector<int64_t> blocks;  // low-rank blocks, in T8 order
  int64_t t8_base;              // T8 row of the stack's first row
};

struct MmItem {
  int64_t off = 0;               // element offset in the phase's data array
  int32_t h = 0, hpad = 0, out_off = 0;
  int64_t ncols = 0;             // multiple of 16
  std::vector<MmSeg> segs;
  int64_t stack = -1, srow0 = 0;  // phase 1: stack and its first row in this item
};

struct MmPhase {
  std::vector<MmItem> items;
  int64_t n_elems = 0;
  std::vector<MmChunk> chunks;    // item by item
  std::vector<int32_t> item_ptr;  // chunk ranges of the items, longest first (items + 1)
};

struct MmPlan {
  int64_t n_in = 0, n_out = 0;
  int64_t t8_len = 0;              // rows of T8 (multiple of 8)
  std::vector<int64_t> t8_off;     // per low-rank block
  std::vector<MmStack> stacks;
  MmPhase ph[2];
};

// Builds the matmat plan of the operator (transposed: H^T) from the problem
// and the operator's matvec plan (its row panels are reused).
void build_mm_plan(const Problem &p, bool transposed, int grid, const OperatorPlan &op, MmPlan &mm);

// compute_scales from per-block maxima instead of the data: max_fr[k] =
// max |entry| of stored full-rank block k, max_a[k] / max_b[k] of low-rank
// block k's A / B factors, and nonfinite_fr[k] / nonfinite_lr[k] = 1 when the
// block (or either factor) holds an entry that is not <= 1e300 in magnitude.
// The results equal compute_scales' bit for bit (a maximum does not depend on
// the order it is taken in), for H and H^T.
void scales_from_maxima(const Problem &p, bool transposed, bool check_finite, const double *max_fr,
                        const double *max_a, const double *max_b, const int *nonfinite_fr, const int *nonfinite_lr,
                        OperatorPlan &op);

// The layout fill (fill_items) as column-block copies, for packing on the
// device from flat block arrays: run k copies rows [src_r0, src_r0 + n) x
// columns [src_c0, src_c0 + ncols) of a block view (array 0: the full-rank
// data, 1: the low-rank data; element (i, j) at src_off + i + j ld, or
// src_off + i ld + j when trans) into item rows [dst_r0, dst_r0 + n) x columns
// [dst_c0, dst_c0 + ncols) of the item at element item_off, in the storage of
// one precision (bw_pack.h).  inv: 1 / the block's BF16 scale (1 otherwise).
struct PackRun {
  int64_t item_off, src_off, ld;
  double inv;
  int32_t hpad, dst_r0, dst_c0, src_r0, src_c0, n, ncols;
  int8_t trans, array;
  int16_t pad;
};

// Runs of one phase and precision, in item order.  The blocks' views must
// point into [fr_base, fr_base + fr_len) or [lr_base, lr_base + lr_len)
// (std::invalid_argument otherwise).
void build_pack_runs(const Problem &p, bool transposed, const OperatorPlan &op, int phase, int prec,
                     const double *fr_base, int64_t fr_len, const double *lr_base, int64_t lr_len,
                     std::vector<PackRun> &out);

// Writes the BF16 data of items [i_begin, i_end) of one matmat phase into dst
// (dst[0] is element `base` of the phase's array; dst must be zeroed).
void fill_mm_items(const Problem &p, bool transposed, const MmPlan &mm, int phase, int64_t i_begin, int64_t i_end,
                   int64_t base, uint16_t *dst);

}  // namespace bw
