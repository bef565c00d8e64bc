// hm_structure.h -- the block-structure handle.
#pragma once
#include <vector>

#include "hm_internal.h"

struct hm_structure_s {
  hm_kdtree tree = nullptr;             // not owned
  int depth = 0, num_levels = 1, admiss = 0;
  double eta = 1.0;
  std::vector<int> count;               // blocks per level l = 1..depth at [l-1]
  std::vector<long long> start;         // offset of level l's list at [l-1]
  hm::DevBuf<uint32_t> tiles;           // Morton lists, ascending, concatenated
  // row-major layout: level l's row pointers (2^l + 1) at rstart[l-1]; the
  // block indices of each row, by increasing column, at start[l-1] of csr_blk
  std::vector<long long> rstart;
  hm::DevBuf<unsigned int> row_ptr;
  hm::DevBuf<uint32_t> csr_blk;
  // jagged-diagonal layout: rows by decreasing block count at rows_start[l-1];
  // diagonal pointers (max blocks per row + 1) at jds_pstart[l-1]; entries at
  // start[l-1] of jds_blk
  std::vector<long long> rows_start, jds_pstart;
  std::vector<int> jds_maxc;
  hm::DevBuf<uint32_t> jds_rows;
  hm::DevBuf<unsigned int> jds_ptr;
  hm::DevBuf<uint32_t> jds_blk;
};
