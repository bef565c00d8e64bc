// refcompat_main.cpp -- the reference's main pipeline (src/main.cu:52-173),
// written against include/hm_refcompat.h and linked with -lhmb200, as a
// reference maintainer would switch it.  Test program: tests/test_refcompat_gpu.py
// compiles and runs it on a GPU and checks its output file against the CPU
// oracle.
//
// Usage: refcompat_main N d bucket nrhs tol out.bin
// Output (little endian): int32 N, d, nrhs, depth, status_pow2;
//   double points[d*N]; int32 perm[N]; int32 offsets[2^depth + 1];
//   double X[N*nrhs]; double Y[N*nrhs] (tree order, column-major)
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hm_refcompat.h"

using namespace hmref;

#define CHECK(x)                                                                       \
  do {                                                                                 \
    hm_status s_ = (x);                                                                \
    if (s_ != HM_OK) {                                                                 \
      std::fprintf(stderr, "%s failed (%d): %s\n", #x, (int)s_, hm_last_error());      \
      return 2;                                                                        \
    }                                                                                  \
  } while (0)
#define CK(x)                                                                          \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      std::fprintf(stderr, "%s failed: %s\n", #x, cudaGetErrorString(e_));             \
      return 3;                                                                        \
    }                                                                                  \
  } while (0)

int main(int argc, char** argv) {
  if (argc < 7) {
    std::fprintf(stderr, "usage: %s N d bucket nrhs tol out.bin\n", argv[0]);
    return 1;
  }
  const unsigned N = (unsigned)std::atoi(argv[1]), d = (unsigned)std::atoi(argv[2]);
  const unsigned bucket = (unsigned)std::atoi(argv[3]), nrhs = (unsigned)std::atoi(argv[4]);
  const float tol = (float)std::atof(argv[5]);

  double* d_pointCloud = nullptr;
  CK(cudaMalloc((void**)&d_pointCloud, sizeof(double) * N * d));
  CHECK(generateDataset((int)N, (int)d, d_pointCloud));

  KDTree kDTree;
  CHECK(allocateKDTree(kDTree, N, d, bucket, FULL_TREE));
  CHECK(constructKDTree(N, d, bucket, kDTree, d_pointCloud, FULL_TREE));

  // the reference's other division methods: DIVIDE_IN_HALF is the same tree;
  // POWER_OF_TWO_ON_LEFT is refused for a non-power-of-two N
  KDTree other;
  CHECK(constructKDTree(N, d, bucket, other, d_pointCloud, DIVIDE_IN_HALF));
  std::vector<int> a(N), b(N);
  CK(cudaMemcpy(a.data(), kDTree.segmentIndices, 4 * N, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(b.data(), other.segmentIndices, 4 * N, cudaMemcpyDeviceToHost));
  for (unsigned i = 0; i < N; ++i)
    if (a[i] != b[i]) {
      std::fprintf(stderr, "DIVIDE_IN_HALF tree differs at %u\n", i);
      return 4;
    }
  freeKDTree(other);
  KDTree p2;
  const int status_pow2 = (int)constructKDTree(N - 1, d, bucket, p2, d_pointCloud, POWER_OF_TWO_ON_LEFT);
  freeKDTree(p2);

  HMatrix hierarchicalMatrix;
  CHECK(constructHMatrixStructure(&hierarchicalMatrix.matrixStructure, (unsigned)upperPowerOfTwo((int)N), d, bucket,
                                  BOX_CENTER_ADMISSIBILITY, kDTree.boundingBoxes, kDTree.boundingBoxes));
  hm_build_opts opts;
  hm_build_opts_default((int)d, &opts);
  opts.max_rank = 64;
  CHECK(generateHMatrixFromStruct(kDTree, hierarchicalMatrix, d_pointCloud, tol, &opts));

  std::vector<double> hX((size_t)N * nrhs), hY((size_t)N * nrhs, 0.0);
  for (size_t i = 0; i < hX.size(); ++i) hX[i] = std::sin(0.37 * (double)i) + 0.25 * std::cos(1.9 * (double)i);
  double *d_inputVectors = nullptr, *d_resultVectors = nullptr;
  CK(cudaMalloc((void**)&d_inputVectors, sizeof(double) * hX.size()));
  CK(cudaMalloc((void**)&d_resultVectors, sizeof(double) * hX.size()));
  CK(cudaMemcpy(d_inputVectors, hX.data(), sizeof(double) * hX.size(), cudaMemcpyHostToDevice));
  CK(cudaMemset(d_resultVectors, 0, sizeof(double) * hX.size()));
  CHECK(HMatrixVecMult(N, bucket, kDTree.numSegments, nrhs, hierarchicalMatrix, d_inputVectors, d_resultVectors));
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(hY.data(), d_resultVectors, sizeof(double) * hY.size(), cudaMemcpyDeviceToHost));

  std::vector<double> pts((size_t)N * d);
  std::vector<int> offs(kDTree.numSegments + 1);
  CK(cudaMemcpy(pts.data(), d_pointCloud, sizeof(double) * pts.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(offs.data(), kDTree.segmentOffsets, 4 * offs.size(), cudaMemcpyDeviceToHost));
  int depth = 0;
  while ((1u << depth) < kDTree.numSegments) ++depth;

  FILE* f = std::fopen(argv[6], "wb");
  if (!f) return 5;
  const int hdr[5] = {(int)N, (int)d, (int)nrhs, depth, status_pow2};
  std::fwrite(hdr, 4, 5, f);
  std::fwrite(pts.data(), 8, pts.size(), f);
  std::fwrite(a.data(), 4, N, f);
  std::fwrite(offs.data(), 4, offs.size(), f);
  std::fwrite(hX.data(), 8, hX.size(), f);
  std::fwrite(hY.data(), 8, hY.size(), f);
  std::fclose(f);

  freeHMatrix(hierarchicalMatrix);
  freeHMatrixStructure(hierarchicalMatrix.matrixStructure);
  freeKDTree(kDTree);
  cudaFree(d_inputVectors);
  cudaFree(d_resultVectors);
  cudaFree(d_pointCloud);
  std::printf("refcompat_main: N=%u d=%u bucket=%u nrhs=%u levels=%d ok\n", N, d, bucket, nrhs,
              hierarchicalMatrix.matrixStructure.numLevels);
  return 0;
}
