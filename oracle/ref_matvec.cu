// ref_matvec.cu -- times the reference's own GPU H-matvec (HMatrixVecMult:
// batched and grouped CUTLASS FP64 GEMMs, src/HMatrixVectorMultiplication.cu)
// against this engine's hm_hmatvec, on the same H-matrix.  Baseline
// measurement only (test infrastructure): oracle/Makefile compiles it with the
// unmodified reference sources into oracle/_ref/ref_matvec.
//
// The reference product needs weak admissibility, N / bucket and nrhs powers
// of two and its own HMatrix layout (src/HMatrix.cuh:9-34): per level, the
// 2^l blocks (row cluster t, column cluster t^1) in row-cluster order, U and
// V of each packed column-major after the previous block's, tileScanRanks
// the inclusive scan of the ranks; diagonal leaf blocks consecutive.  The
// engine builds the H-matrix (weak admissibility, FP32 factors); the driver
// widens it to FP64 in that layout (a block stored dense becomes U = D,
// V = I), runs both products on the same X and reports their times and the
// relative difference of the results.
//
// Usage: ref_matvec N d bucket nrhs tol reps
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <vector>

#include "HMatrix.cuh"
#include "HMatrixVectorMultiplication.cuh"
#include "hm.h"

#define CK(x)                                                                                        \
  do {                                                                                               \
    cudaError_t e_ = (x);                                                                            \
    if (e_ != cudaSuccess) {                                                                         \
      fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__);      \
      return 2;                                                                                      \
    }                                                                                                \
  } while (0)
#define HK(x)                                                                                        \
  do {                                                                                               \
    hm_status s_ = (x);                                                                              \
    if (s_ != HM_OK) {                                                                               \
      fprintf(stderr, "hm error %d: %s at %s:%d\n", (int)s_, hm_last_error(), __FILE__, __LINE__); \
      return 3;                                                                                      \
    }                                                                                                \
  } while (0)

int main(int argc, char** argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: %s N d bucket nrhs tol reps\n", argv[0]);
    return 1;
  }
  const int N = atoi(argv[1]), d = atoi(argv[2]), b = atoi(argv[3]), nrhs = atoi(argv[4]);
  const double tol = atof(argv[5]);
  const int reps = atoi(argv[6]);
  double* d_pts = nullptr;
  CK(cudaMalloc(&d_pts, sizeof(double) * (size_t)N * d));
  HK(hm_generate_dataset(N, d, 1234, d_pts, nullptr));
  hm_kdtree tree;
  HK(hm_kdtree_build(d_pts, N, d, b, nullptr, &tree));
  int depth = 0;
  HK(hm_kdtree_info(tree, nullptr, nullptr, nullptr, &depth));
  hm_structure st;
  HK(hm_structure_build(tree, HM_ADMISS_WEAK, 1.0, nullptr, &st));
  hm_build_opts o;
  hm_build_opts_default(d, &o);  // the reference's kernel exp(-r/l), l = 0.1 (2-D) or 0.2 (3-D)
  o.tol = tol;
  o.max_rank = 64;
  o.diag_from_coords = 0;
  hm_hmatrix H;
  HK(hm_hmatrix_build(tree, st, d_pts, &o, nullptr, &H));

  std::vector<int> lo(((size_t)1 << depth) + 1);
  HK(hm_kdtree_copy_out(tree, nullptr, lo.data(), nullptr, nullptr, nullptr));
  for (int x = 0; x < (1 << depth); ++x)
    if (lo[x + 1] - lo[x] != b) {
      fprintf(stderr, "the reference product needs leaves of exactly %d points\n", b);
      return 1;
    }
  long long nl = 0, nd = 0;
  HK(hm_hmatrix_blocks(H, &nl, &nd, nullptr, nullptr));
  std::vector<int> lr(6 * nl), de(5 * nd);
  HK(hm_hmatrix_blocks(H, nullptr, nullptr, lr.data(), de.data()));
  std::map<std::pair<int, int>, int> lr_at, de_at;  // (r0, c0) -> index
  for (long long i = 0; i < nl; ++i) lr_at[{lr[6 * i], lr[6 * i + 2]}] = (int)i;
  for (long long i = 0; i < nd; ++i) de_at[{de[5 * i], de[5 * i + 2]}] = (int)i;

  // ---- the reference layout (FP64) ----------------------------------------
  HMatrix R{};
  const int numLevels = depth + 1, nseg = 1 << depth;
  R.matrixStructure.numLevels = numLevels;
  std::vector<int> numTiles(numLevels);
  for (int l = 1; l < numLevels; ++l) numTiles[l - 1] = 1 << l;
  R.matrixStructure.numTiles = numTiles.data();
  std::vector<double> diag((size_t)nseg * b * b);
  std::vector<float> buf;
  for (int x = 0; x < nseg; ++x) {
    auto it = de_at.find({lo[x], lo[x]});
    if (it == de_at.end()) {
      fprintf(stderr, "missing diagonal block %d\n", x);
      return 1;
    }
    buf.resize((size_t)b * b);
    HK(hm_hmatrix_dense_block(H, it->second, buf.data()));
    for (size_t e = 0; e < buf.size(); ++e) diag[(size_t)x * b * b + e] = buf[e];
  }
  CK(cudaMalloc(&R.diagonalBlocks, sizeof(double) * diag.size()));
  CK(cudaMemcpy(R.diagonalBlocks, diag.data(), sizeof(double) * diag.size(), cudaMemcpyHostToDevice));
  std::vector<HMatrixLevel> levels(numLevels - 1);
  R.levels = levels.data();
  long long rank_total = 0;
  int dense_offdiag = 0, over_half = 0;  // the reference's V transpose covers ranks up to half a tile
  for (int l = 1; l < numLevels; ++l) {
    const int nt = 1 << l, dim = N >> l;
    std::vector<int> scan(nt);
    std::vector<double> U, V;
    int acc = 0;
    for (int t = 0; t < nt; ++t) {
      const int r0 = t * dim, c0 = (t ^ 1) * dim;
      std::vector<float> fu, fv;
      int k = 0;
      auto il = lr_at.find({r0, c0});
      if (il != lr_at.end()) {
        const int i = il->second;
        k = lr[6 * i + 4];
        fu.resize((size_t)dim * std::max(k, 1));
        fv.resize((size_t)dim * std::max(k, 1));
        HK(hm_hmatrix_block_factors(H, i, fu.data(), fv.data()));
      } else {
        auto id = de_at.find({r0, c0});
        if (id == de_at.end()) {
          fprintf(stderr, "missing block level %d tile %d\n", l, t);
          return 1;
        }
        k = dim;  // dense block D = D * I^T
        ++dense_offdiag;
        fu.resize((size_t)dim * dim);
        HK(hm_hmatrix_dense_block(H, id->second, fu.data()));
        fv.assign((size_t)dim * dim, 0.f);
        for (int j = 0; j < dim; ++j) fv[(size_t)j * dim + j] = 1.f;
      }
      if (2 * k > dim) ++over_half;
      for (size_t e = 0; e < (size_t)dim * k; ++e) U.push_back(fu[e]);
      for (size_t e = 0; e < (size_t)dim * k; ++e) V.push_back(fv[e]);
      acc += k;
      scan[t] = acc;
    }
    rank_total += acc;
    HMatrixLevel& L = levels[l - 1];
    L.level = l;
    CK(cudaMalloc(&L.tileScanRanks, sizeof(int) * nt));
    CK(cudaMemcpy(L.tileScanRanks, scan.data(), sizeof(int) * nt, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&L.U, sizeof(double) * std::max<size_t>(U.size(), 1)));
    CK(cudaMalloc(&L.V, sizeof(double) * std::max<size_t>(V.size(), 1)));
    CK(cudaMemcpy(L.U, U.data(), sizeof(double) * U.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(L.V, V.data(), sizeof(double) * V.size(), cudaMemcpyHostToDevice));
  }

  // ---- the same X for both products ---------------------------------------
  std::vector<double> xh((size_t)N * nrhs);
  unsigned long long st64 = 88172645463325252ull;
  for (auto& v : xh) {
    st64 ^= st64 << 13;
    st64 ^= st64 >> 7;
    st64 ^= st64 << 17;
    v = (double)(st64 >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  }
  std::vector<float> xf(xh.begin(), xh.end());
  double *dX, *dY;
  float *fX, *fY;
  CK(cudaMalloc(&dX, sizeof(double) * xh.size()));
  CK(cudaMalloc(&dY, sizeof(double) * xh.size()));
  CK(cudaMalloc(&fX, sizeof(float) * xh.size()));
  CK(cudaMalloc(&fY, sizeof(float) * xh.size()));
  CK(cudaMemcpy(dX, xh.data(), sizeof(double) * xh.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(fX, xf.data(), sizeof(float) * xf.size(), cudaMemcpyHostToDevice));

  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto time_ms = [&](auto&& fn) {
    std::vector<float> t;
    for (int r = 0; r < reps + 2; ++r) {
      cudaDeviceSynchronize();
      cudaEventRecord(e0);
      fn();
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r >= 2) t.push_back(ms);
    }
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
  };
  const float ref_ms = time_ms([&] { HMatrixVecMult(N, b, nseg, nrhs, R, dX, dY); });
  const float our_ms = time_ms([&] { hm_hmatvec(H, 0, nrhs, fX, N, fY, N, 0, nullptr); });
  CK(cudaDeviceSynchronize());
  std::vector<double> yr(xh.size());
  std::vector<float> yo(xh.size());
  CK(cudaMemcpy(yr.data(), dY, sizeof(double) * yr.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(yo.data(), fY, sizeof(float) * yo.size(), cudaMemcpyDeviceToHost));
  double num = 0, den = 0;
  for (size_t e = 0; e < yr.size(); ++e) {
    num += (yr[e] - yo[e]) * (yr[e] - yo[e]);
    den += yr[e] * yr[e];
  }
  hm_hmatrix_stats hs;
  HK(hm_hmatrix_stats_get(H, &hs));
  printf("ref_matvec: N=%d d=%d b=%d nrhs=%d tol=%g levels=%d rank_sum=%lld dense_offdiag=%d "
         "over_half_tile=%d (valid: %s) reference_ms=%.3f ours_ms=%.3f speedup=%.1f rel_diff=%.3e\n",
         N, d, b, nrhs, tol, numLevels, rank_total, dense_offdiag, over_half, over_half ? "no" : "yes", ref_ms,
         our_ms, ref_ms / our_ms, std::sqrt(num / den));
  return 0;
}
