// hm_mixed.h -- the mixed-precision (BF16 hi + lo) form of the H-matvec.
//
// Every cluster that owns low-rank factors gets one "panel": the factors of
// all its blocks side by side (rows = the cluster's points, columns = the sum
// of the blocks' ranks).  The projection of a whole block column is then one
// dense panel^T X product, and the expansion of a block row one panel x T
// product, so no block pays rank padding: the panel is padded once, to whole
// 8-column tiles.  Columns whose BF16 rounding the tolerance cannot absorb
// (the leading singular directions of each block) sit in the panel's first
// tiles and carry a BF16 low part; the trailing ones are stored as BF16 only.
//
// Rows are padded per leaf to whole 32-row tiles ("global tiles"), so each
// 32-row tile lies inside one leaf.  A tile of 32 rows x 8 columns is stored
// in the order the mma.sync fragments want it: lane L of a warp loads one
// 16-byte word and has its four fragment registers, 512 contiguous bytes per
// warp load.  Two such orders exist per factor:
//   P1 (phase 1, the factor is the B operand of X^T V, pairs along rows):
//     lane (g,t) = {V[2t,2t+1][g], V[2t+8,2t+9][g], V[16+2t,17+2t][g], V[24+2t,25+2t][g]}
//     at word 4 g + (t ^ ((g >> 1) & 3)) (the 64-byte-swizzled core-matrix
//     order, so that runs of tiles are tcgen05 operand images)
//   P2 (phase 2, the factor is the A operand of U T, pairs along columns):
//     lane (g,t) = {U[g][2t,2t+1], U[g+8][2t,2t+1], U[g+16][2t,2t+1], U[g+24][2t,2t+1]}
// (g = lane / 4, t = lane % 4; each pair is bf16x2 with the lower index in the
// low half).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "hm_internal.h"

struct hm_hmatrix_s;

namespace hm {

struct MxPanel {
  long long hi1, lo1, hi2, lo2;  // 512-byte tile offsets into MxPlan::store, [row tile][col tile]
  long long s0;                  // first phase-1 output tile (nchunk x nct tiles)
  long long t0;                  // first global factor column tile (nct tiles)
  long long tw0;                 // first 32-bit word of the panel's T (nctl tiles of 128 words, then 64 each)
  long long tb0;                 // 128-column passes on tcgen05: first 2 KB block of its T (nct hi blocks, nctl lo)
  int nct, nctl;                 // 8-column tiles; the first nctl carry low parts
  int tile0, nrt;                // first global row tile, row tiles
  int nchunk;                    // row chunks of the projection
  int nchunkt;                   // the same in a 128-column pass on tcgen05 (its own chunk size)
  long long s0t;                 // its first chunk-partial tile there
  int r0;                        // first (tree-order) row of the cluster
};

struct MxUnit {  // phase-1 work item, one warp: up to 8 column tiles x up to 64 row tiles
  int panel, ct0, nct, rt0, nrt, chunk;
};

// A phase-1 unit of the tcgen05 kernel with the panel fields it needs (one
// load per unit): up to 16 column tiles of one kind (with or without low parts).
struct TcUnit {
  long long vhi;  // P1 hi tile (512-byte units) of its first column tile at its first row tile
  long long vlo;  // the same for the low parts (units with low parts)
  long long out;  // T (panel in one row chunk): its first global column tile; else its first S tile
  int shi, slo;   // tiles per row tile of the panel: nct, nctl
  int nct, nrt;   // column tiles (<= 16), row tiles
  int xtile;      // global row tile of its first row (X's image)
  int flags;      // 1: columns with low parts; 2: T (else chunk partials S)
};

// Phase 2 of a 128-column pass on tcgen05 works on blocks of 4 global row
// tiles (128 rows).  Each block's sources, in the order they are added --
// the ancestors' panels level by level, then the leaves' dense blocks -- are
// cut into steps (host-built):
//   kind 0: up to 4 column tiles of a panel with low parts (A hi + lo, T hi + lo)
//   kind 1: up to 8 column tiles of a panel without (A hi, T hi)
//   kind 2: 4 column tiles (32 columns) of a dense block (A hi + lo, X's image)
//   kind 3: nothing (a block without sources: its rows of Y are zero)
// A rows of the block's tiles that the source does not cover (mask bit k
// clear) are zero.
struct P2Step {
  long long a_hi, a_lo;  // P2 tile (512-byte units) of the block's tile 0 at the step's first column tile
  long long b_hi, b_lo;  // 16-byte offset of B: T blocks (kinds 0, 1) or X's image (kind 2)
  int a_stride, a_stride_lo;  // tiles per row tile of the source (hi, lo)
  int info;                   // kind | column tiles << 2 | mask << 8
  int pad;
};

struct MxDense {  // a dense block in P2 order, hi + lo, [row tile][col tile]
  long long hi, lo;
  int row_tile0, col_tile0;  // global row tiles of its row and column clusters
  int nrt, nct;              // nct: 8-column tiles, a multiple of 4
  int r0, c0, m, n;
  const float* src;          // the FP32 block (m x n, column-major); read only while converting
};

// Where one FP32 factor (or dense block) of the matrix sits in the panels:
// the columns of a pair's side in its cluster's panel (the first khi of them
// in the low-part group at colL, the others at colH), or a dense block.
struct MxLoc {
  const float* key;  // the FP32 array it was converted from (its identity, also after that array is freed)
  int kind;          // 0 factor, 1 dense block
  int idx;           // panel, or dense block
  int rows, cols;    // rows x columns, column-major, as the FP32 array was
  int khi, colL, colH;
};

struct MxPlan {
  bool enabled = false;  // the product runs on the panels (else the FP32 per-block kernels)
  int fmt = 0;           // tile format: 0 BF16 hi + lo (mixed form), 1 FP32 in TF32 fragment order (FP32 form)
  DevBuf<uint4> store;  // all BF16 tiles
  long long store_tiles = 0;
  DevBuf<MxPanel> panels;
  int num_panels = 0;
  DevBuf<int> pan_of;      // heap-ordered cluster (2^l - 1 + a) -> panel or -1
  DevBuf<MxUnit> units;
  int num_units = 0;
  DevBuf<int> tile_leaf;   // global row tile -> leaf
  DevBuf<int> leaf_tile0;  // leaf -> first global row tile (num_leaves + 1)
  int num_tiles = 0;
  int p2_tile0 = 0, p2_tiles = 0;  // row tiles phase 2 writes (all, or a block-row shard's)
  // global factor column (8 * t0 + c) -> where its projection goes in T:
  // (word << 1) | h, word = the column's first 32-bit word at lane row 0 (row
  // g adds 16 g words in a tile with low parts, 8 g in one without), h = 1
  // for a tile without low parts.  A data column goes to its mirror column
  // (the mirror map is an involution on the factor columns); a padding column
  // is stored as -1 - (its own entry) and fills its own words with zeros.
  DevBuf<int> tslot;
  DevBuf<int2> mtiles;     // (panel, column tile) of panels projected in several row chunks
  long long nmt = 0;
  long long s_tiles = 0, t_tiles = 0, t_words = 0;
  DevBuf<MxDense> dense;
  int num_dense = 0;
  DevBuf<int> leaf_dptr, leaf_dblk;  // dense blocks covering each leaf's rows
  long long bytes_p1 = 0, bytes_p2 = 0;  // BF16 bytes of the factors (unpadded) and dense blocks
  std::vector<MxPanel> h_panels;          // host copy (the schedule rebuilds units and S offsets)
  std::vector<MxDense> h_dense;           // host copy
  std::vector<MxLoc> h_locs;              // every factor and dense block converted into the panels
  std::vector<std::pair<const float*, int>> loc_index;  // h_locs by key, sorted (built on first use)
  int chunk_tiles = 128, group_tiles = 8;  // phase-1 unit shape (schedule parameters; measured best at 16 RHS)
  bool p1_ring = false;                    // phase 1 by persistent warps with a cp.async ring
  int num_sms = 148;
  // 128-column passes (BF16 format) on tcgen05 (hm_mixed_tc.cu): phase-1
  // units of up to 16 column tiles, split where a panel's low-part tiles end;
  // T in 2 KB blocks (per 8 columns: 128 right-hand sides x 8 BF16, the
  // K-major core-matrix layout); tslot_tc: per global factor column the
  // destination's {hi, lo} position (block * 8 + column; lo -1 without a low
  // part; a padding column: {-1 - own hi, own lo}); phase-2 blocks of 4 row
  // tiles with their steps (p2_step_ptr: CSR over p2_blocks blocks).
  bool wide_tc = true;
  int tc_chunk_tiles = 32;         // row tiles per tcgen05 phase-1 unit
  DevBuf<int2> mtiles_tc;          // (panel, column tile) of panels of several tcgen05 row chunks
  long long nmt_tc = 0, s_tiles_tc = 0;
  DevBuf<TcUnit> tc_units;
  int num_tc_units = 0;
  DevBuf<int2> tslot_tc;
  DevBuf<P2Step> p2_steps;
  DevBuf<int> p2_step_ptr;
  int p2_blocks = 0;
  DevBuf<int> tc_err;  // set when a bounded wait of those kernels gave up
  bool tc_pass(int halves) const { return wide_tc && fmt == 0 && halves == 8; }
  // scratch of one 16-column panel of right-hand sides, in floats: X
  // fragments, chunk partials, T (the projections by expanding column: BF16
  // hi + lo for the columns with low parts, hi for the others)
  // of a pass of `halves` such panels (1, 2, 4 or 8: up to 128 right-hand sides)
  // (FP32 format: X as TF32 hi + lo, 8 words per lane and tile instead of 4)
  // (a tcgen05 pass keeps X's image, 16 KB per row tile, where the eight
  // parts' fragments would be, its chunk partials, 4 KB per tile, where the
  // parts' partials would be, and T in blocks where the parts' T would be)
  long long scratch_floats(int halves = 1) const {
    const long long st = tc_pass(halves) ? std::max(s_tiles, s_tiles_tc) : s_tiles;
    return (((long long)num_tiles * (fmt ? 8 : 4) + st) * 128 + t_words) * halves;
  }
};

struct MxPair {  // one stored low-rank pair (u rows, v columns) = fu fv^T, and its mirror
  int level, r0, m, c0, n, k, khi;
  const float* fu;  // m x k, column-major
  const float* fv;  // n x k, column-major
};

struct MxDenseIn {
  int r0, m, c0, n;
  const float* D;  // m x n, column-major
};

// Builds the panels, converts the FP32 factors and dense blocks, and lays out
// the phase-1 units and the column map of the projection.
hm_status mixed_build(hm_hmatrix_s* h, const std::vector<MxPair>& pairs, const std::vector<MxDenseIn>& dense,
                      cudaStream_t s);

// A 128-column pass on tcgen05 after k_mx_split_x wrote Xtc (16 KB per row
// tile): phase 1 (T as blocks, or chunk partials S: 128 floats per column),
// the chunk reduction, phase 2 (Y, tree order, nr <= 128 columns).
struct KernelMarks;
hm_status mixed_tc_pass(hm_hmatrix_s* h, int nr, const uint4* Xtc, float* S, uint4* Tb, float* Y, int ldy,
                        cudaStream_t s, KernelMarks* km);

struct KernelMarks;

// Phase-1 units of chunk_tiles row tiles x group_tiles (<= 8) column tiles,
// the projection's S layout that goes with them, and the phase-1 kernel
// (p1_ring: persistent warps with a cp.async ring, else one warp per unit).  The caller rebuilds the
// matvec plan afterwards (the scratch size changes).
hm_status mixed_schedule(hm_hmatrix_s* h, int chunk_tiles, int group_tiles, int p1_ring, cudaStream_t s);

// One pass of nr <= 128 right-hand sides in tree order (two, four or eight parts of 16
// when nr > 16: every factor tile is read once for all of them); scratch holds
// scratch_floats(h) floats, h = 1, 2, 4 or 8 parts.  km (optional) receives an event
// after each kernel.
hm_status mixed_run_panel(hm_hmatrix_s* h, int nr, const float* X, int ldx, float* Y, int ldy, float* scratch,
                          cudaStream_t s, KernelMarks* km);

// The FP32 values of the BF16 panels: for each (h_locs index, device
// destination), the factor or dense block rebuilt column-major from its hi
// (+ lo) tiles.  A value is hi + lo (exact in FP32), moved one FP32 ulp toward
// hi where hi + lo would round to another BF16 hi, so that converting the
// result again gives the same tiles bit for bit.
hm_status mixed_unpack(hm_hmatrix_s* h, const std::vector<std::pair<int, float*>>& jobs, cudaStream_t s);

// Index into h_locs of the factor or dense block converted from `key`, or -1.
int mixed_find_loc(hm_hmatrix_s* h, const float* key);

// The FP32 format (hm_fp32.cu): tile conversion of the panels and dense
// blocks, and one pass of nr <= 16 right-hand sides.
hm_status fp32_convert(hm_hmatrix_s* h, const std::vector<const float*>& colsrc, const std::vector<MxDense>& dense,
                       cudaStream_t s);
hm_status fp32_run_panel(hm_hmatrix_s* h, int nr, const float* X, int ldx, float* Y, int ldy, float* scratch,
                         cudaStream_t s, KernelMarks* km);

}  // namespace hm
