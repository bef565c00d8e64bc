// hm_hmatrix.h -- the H-matrix handle and its matvec plan.
#pragma once
#include <vector>

#include "hm_internal.h"
#include "hm_kernels.cuh"
#include "hm_mixed.h"

namespace hm {

// Events recorded after each kernel of one product, for per-kernel device
// times (profiling entry points only; the hot path passes nullptr).
struct KernelMarks {
  static constexpr int kMax = 8;
  cudaEvent_t ev[kMax + 1];
  const char* name[kMax];
  long long bytes[kMax];  // algorithmic bytes of each kernel
  int n = 0;
  void mark(const char* nm, long long b, cudaStream_t s) {
    if (n >= kMax) return;
    name[n] = nm;
    bytes[n] = b;
    cudaEventRecord(ev[n + 1], s);
    ++n;
  }
};

// Y[leaf rows] += K(leaf, leaf) X[leaf rows] for every leaf, entries from the
// coordinates (the diagonal blocks of a matrix built with diag_fly).
hm_status diag_fly_panel(hm_hmatrix_s* h, int nr, const float* X, int ldx, float* Y, int ldy, cudaStream_t s,
                         KernelMarks* km);

// One block of the matrix as the matvec sees it (both orientations of a stored
// pair appear, the mirror one with U and V exchanged).
struct LRBlock {
  int r0, m, c0, n, k;
  int level;
  int khi;         // leading columns that keep a BF16 low part in the mixed form
  const float* U;  // m x k, column-major (ld m)
  const float* V;  // n x k, column-major (ld n)
  long long toff;  // offset of this block's k x nrhs_max projection in the T workspace
};

struct DenseBlock {
  int r0, m, c0, n;
  int trans;       // always 0: D is m x n, column-major (ld m); mirrors are stored transposed
  const float* D;
};

struct P1Item {
  int block;       // index into the low-rank block list
  int chunk;       // 512-row chunk of the block's V
  long long part;  // -1: the block has one chunk and stores T_b; else offset of this chunk's partial
};

struct MultiItem {  // a block whose projection is the sum of several chunk partials
  long long toff;   // T_b
  long long poff;   // first partial
  int kpad, nch;
};

struct MatvecPlan {
  DevBuf<LRBlock> lr;        // low-rank blocks, both orientations
  DevBuf<P1Item> p1;         // phase 1 work items (one warp each)
  int num_p1 = 0;
  DevBuf<MultiItem> multi;  // projections summed over several chunk partials
  int num_multi = 0;
  long long part_floats = 0;  // partials, stored after the projections in T
  DevBuf<int2> groups;       // phase 2 work items: (leaf, first row of a 32-row group)
  int num_groups = 0;
  DevBuf<int> leaf_ptr;      // 2^depth + 1
  DevBuf<int> leaf_blk;      // low-rank blocks covering each leaf row
  DevBuf<DenseBlock> dense;  // dense blocks
  DevBuf<int> leaf_dptr;     // 2^depth + 1
  DevBuf<int> leaf_dblk;     // dense blocks of each leaf row
  DevBuf<float> T;           // projections: per block 16 x kpad_b, then the chunk partials
  long long t_floats = 0;    // sum_b 16 * kpad_b
  long long t_per_rhs = 0;   // sum_b kpad_b
  int nrhs_cap = 0;
  int num_leaves = 0;
  int maxleaf = 1;
  DevBuf<float> Xp, Yp;      // permuted copies for original-order calls (n * nrhs_cap)
  int p1_rows = 1024;         // rows of V per phase-1 item (schedule parameter)
  long long bytes_p1 = 0, bytes_p2 = 0;  // FP32 factor bytes read by each phase (+ dense in phase 2)
  long long multi_t_floats = 0;          // projections written by the chunk reduction
};

}  // namespace hm

struct hm_hmatrix_s;
namespace hm {
long long device_bytes(const hm_hmatrix_s* h);
// Frees the FP32 factor and dense storage of a mixed-form matrix whose panels
// are built (their address ranges stay in chunk_meta).
void release_fp32(hm_hmatrix_s* h);
}  // namespace hm

struct hm_hmatrix_s {
  hm_kdtree tree = nullptr;        // not owned
  hm_structure structure = nullptr;  // not owned
  int n = 0, d = 0, depth = 0;
  hm_build_opts opts{};
  hm::KernelParams kp{};
  std::vector<hm::DevBuf<float>> storage;  // factor / dense chunks
  // The mixed form releases its FP32 chunks once its BF16 panels are built
  // (the product reads the panels only); what the chunks held is then rebuilt
  // from the panels when asked for (export, files).  chunk_meta keeps each
  // released chunk's address range, the identity of the arrays in it.
  bool fp32_released = false;
  std::vector<std::pair<const float*, size_t>> chunk_meta;
  hm_hmatrix_stats stats{};
  hm::MatvecPlan plan;
  hm::MxPlan mx;                     // mixed precision form (panels of BF16 hi + lo tiles)
  bool diag_fly = false;             // diagonal leaf blocks recomputed from the coordinates per product
  int leaf_lo = 0, leaf_hi = 0;      // block-row shard: the product's rows are those of leaves [leaf_lo, leaf_hi)
  int plan_gen = 0;                  // bumped whenever the product's plan is rebuilt
  // host mirror of the block list (for export / tests)
  std::vector<hm::LRBlock> h_lr;
  std::vector<hm::DenseBlock> h_dense;
};
