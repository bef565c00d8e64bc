// ref_pipeline.cu -- drives the reference's own compiled pipeline stages
// (generateDataset -> allocateKDTree/constructKDTree -> constructHMatrixStructure)
// and dumps every output as one binary file.  TEST INFRASTRUCTURE ONLY: it is
// linked against the unmodified reference sources by oracle/Makefile into
// oracle/_ref/ref_pipeline and is used to generate the golden fixtures in
// tests/golden/ that pin the CPU oracle (hm_oracle.c).
//
// Usage: ref_pipeline N d bucket admiss(0 weak,1 boxCenter) out.bin [points.bin]
//   points.bin (optional): N*d doubles, SoA p[dim*N+i]; when absent the points
//   come from the reference's generateDataset (src/generateDataset.cu:15-19).
//
// Output layout (little endian):
//   char magic[8] = "HMREF01\0"; int32 N, d, bucket, admiss, depth, numLevels
//   double pts[N*d]; int32 perm[N]; int32 offsets[2^depth+1]
//   for level in [0, depth): double bmin[2^level*d], bmax[2^level*d]
//   int32 numTiles[numLevels]; for l in [0, numLevels-1): int32 tiles[numTiles[l]]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "config.h"
#include "generateDataset.cuh"
#include "HMatrixStructure.cuh"
#include "kDTree.cuh"
#include "kDTreeConstruction.cuh"
#include "kDTreeHelpers.cuh"

#define CK(x)                                                                     \
  do {                                                                            \
    cudaError_t e_ = (x);                                                         \
    if (e_ != cudaSuccess) {                                                      \
      fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                          \
      return 2;                                                                   \
    }                                                                             \
  } while (0)

int main(int argc, char** argv) {
  if (argc < 6) {
    fprintf(stderr, "usage: %s N d bucket admiss out.bin [points.bin]\n", argv[0]);
    return 1;
  }
  unsigned int N = (unsigned)atoi(argv[1]);
  unsigned int d = (unsigned)atoi(argv[2]);
  unsigned int b = (unsigned)atoi(argv[3]);
  int admiss = atoi(argv[4]);
  const char* out = argv[5];

  double* d_pts = nullptr;
  CK(cudaMalloc((void**)&d_pts, sizeof(double) * N * d));
  std::vector<double> h_pts((size_t)N * d);
  if (argc > 6) {
    FILE* f = fopen(argv[6], "rb");
    if (!f || fread(h_pts.data(), sizeof(double), h_pts.size(), f) != h_pts.size()) {
      fprintf(stderr, "cannot read %s\n", argv[6]);
      return 1;
    }
    fclose(f);
    CK(cudaMemcpy(d_pts, h_pts.data(), sizeof(double) * N * d, cudaMemcpyHostToDevice));
  } else {
    generateDataset((int)N, (int)d, d_pts);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(h_pts.data(), d_pts, sizeof(double) * N * d, cudaMemcpyDeviceToHost));
  }

  // wall time of the reference's own stages (device synchronised), printed
  // with the summary line for baseline measurements
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto t0 = now();
  KDTree tree;
  allocateKDTree(tree, N, d, b, FULL_TREE);
  constructKDTree(N, d, b, tree, d_pts, FULL_TREE);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  auto t1 = now();

  int depth = getMaxSegmentSize((int)N, (int)b).second;
  int nleaf = 1 << depth;
  std::vector<int> perm(N), offs(nleaf + 1);
  CK(cudaMemcpy(perm.data(), tree.segmentIndices, sizeof(int) * N, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(offs.data(), tree.segmentOffsets, sizeof(int) * (nleaf + 1),
                cudaMemcpyDeviceToHost));

  auto t2 = now();
  HMatrixStructure st;
  constructHMatrixStructure(&st, upperPowerOfTwo((int)N), d, b,
                            admiss ? BOX_CENTER_ADMISSIBILITY : WEAK_ADMISSIBILITY,
                            tree.boundingBoxes, tree.boundingBoxes);
  CK(cudaDeviceSynchronize());
  auto t3 = now();

  FILE* f = fopen(out, "wb");
  if (!f) return 1;
  const char magic[8] = {'H', 'M', 'R', 'E', 'F', '0', '1', 0};
  fwrite(magic, 1, 8, f);
  int hdr[6] = {(int)N, (int)d, (int)b, admiss, depth, st.numLevels};
  fwrite(hdr, sizeof(int), 6, f);
  fwrite(h_pts.data(), sizeof(double), h_pts.size(), f);
  fwrite(perm.data(), sizeof(int), N, f);
  fwrite(offs.data(), sizeof(int), nleaf + 1, f);
  for (int l = 0; l < depth; ++l) {
    fwrite(tree.boundingBoxes.levels[l].minBBData, sizeof(double), (size_t)(1 << l) * d, f);
    fwrite(tree.boundingBoxes.levels[l].maxBBData, sizeof(double), (size_t)(1 << l) * d, f);
  }
  fwrite(st.numTiles, sizeof(int), st.numLevels, f);
  for (int l = 0; l < st.numLevels - 1; ++l) fwrite(st.tileIndices[l], sizeof(int), st.numTiles[l], f);
  fclose(f);
  printf("ref_pipeline: N=%u d=%u b=%u admiss=%d depth=%d levels=%d kdtree_ms=%.3f structure_ms=%.3f\n", N,
         d, b, admiss, depth, st.numLevels, std::chrono::duration<double, std::milli>(t1 - t0).count(),
         std::chrono::duration<double, std::milli>(t3 - t2).count());
  freeKDTree(tree);
  cudaFree(d_pts);
  return 0;
}
