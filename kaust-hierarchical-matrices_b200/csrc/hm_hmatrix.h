// hm_hmatrix.h -- the H-matrix handle and its matvec plan.
#pragma once
#include <vector>

#include "hm_internal.h"
#include "hm_kernels.cuh"

namespace hm {

// One block of the matrix as the matvec sees it (both orientations of a stored
// pair appear, the mirror one with U and V exchanged).
struct LRBlock {
  int r0, m, c0, n, k;
  int level;
  const float* U;  // m x k, column-major (ld m)
  const float* V;  // n x k, column-major (ld n)
  long long toff;  // offset of this block's k x nrhs_max projection in the T workspace
};

struct DenseBlock {
  int r0, m, c0, n;
  int trans;       // 0: D is m x n (ld m); 1: D is stored n x m (ld n), use D^T
  const float* D;
};

struct MatvecPlan {
  // low-rank blocks, and for phase 2 the CSR of low-rank blocks per leaf row:
  // every block whose row cluster contains the leaf
  DevBuf<LRBlock> lr;
  DevBuf<int> p1_items;      // phase 1 work items: block index << 8 | chunk (see hm_matvec.cu)
  int num_p1 = 0;
  DevBuf<int> leaf_ptr;      // 2^depth + 1
  DevBuf<int> leaf_blk;      // low-rank blocks covering each leaf row
  DevBuf<DenseBlock> dense;  // dense blocks
  DevBuf<int> leaf_dptr;     // 2^depth + 1
  DevBuf<int> leaf_dblk;     // dense blocks of each leaf row
  DevBuf<float> T;           // projections workspace (sum_b k_b * nrhs_cap)
  long long t_per_rhs = 0;   // sum_b k_b
  int nrhs_cap = 0;
  int num_leaves = 0;
  int maxleaf = 1;
  DevBuf<float> Xp, Yp;      // permuted copies for original-order calls (n * nrhs_cap)
};

}  // namespace hm

struct hm_hmatrix_s {
  hm_kdtree tree = nullptr;        // not owned
  hm_structure structure = nullptr;  // not owned
  int n = 0, d = 0, depth = 0;
  hm_build_opts opts{};
  hm::KernelParams kp{};
  std::vector<hm::DevBuf<float>> storage;  // factor / dense chunks
  hm_hmatrix_stats stats{};
  hm::MatvecPlan plan;
  // host mirror of the block list (for export / tests)
  std::vector<hm::LRBlock> h_lr;
  std::vector<hm::DenseBlock> h_dense;
};
