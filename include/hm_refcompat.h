/*
 * hm_refcompat.h -- the reference's operator names and argument lists over the
 * C ABI.
 *
 * A maintainer of the reference (a C++/CUDA program, no FFI) switches its
 * pipeline to libhmb200.so by including this header instead of the reference's
 * kDTree*.cuh / HMatrixStructure.cuh / constructHMatrixFromStruct.cuh /
 * HMatrixVectorMultiplication.cuh, adding `using namespace hmref;`, and
 * linking -lhmb200.  The calls of the reference's main (src/main.cu:52-173)
 * keep their names, argument order and meaning:
 *
 *   reference (file:line)                                        here
 *   generateDataset(N, d, d_points)       src/generateDataset.cu:15    generateDataset
 *   allocateKDTree(tree, N, d, b, div)    src/kDTree.cu:6              allocateKDTree
 *   constructKDTree(N, d, b, tree, p, div) src/kDTreeConstruction.cu:14 constructKDTree
 *   constructHMatrixStructure(&st, N, d, b, cond, boxes, boxes)
 *                                         src/HMatrixStructure.cu:133  constructHMatrixStructure
 *   allocateHMatrix + generateHMatrixFromStruct
 *                                         src/HMatrix.cu:57,
 *                                         src/constructHMatrixFromStruct.cu:13
 *                                                                      generateHMatrixFromStruct
 *   HMatrixVecMult(N, b, ns, nrhs, H, double* X, double* Y)
 *                                         src/HMatrixVectorMultiplication.cu:10
 *                                                                      HMatrixVecMult (FP64 vectors)
 *   freeKDTree / freeHMatrixStructure / freeHMatrix
 *                                         src/kDTree.cu:33, src/HMatrixStructure.cu:162,
 *                                         src/HMatrix.cu:105           same names
 *
 * Differences a caller sees: every function returns hm_status (0 on success,
 * like cudaSuccess) instead of exiting; the tree, structure and matrix are
 * opaque handles (the bounding boxes live in the tree, so KDTreeBoundingBoxes
 * only names its tree); the H-matrix is built straight from the points (there
 * is no leaf-TLR matrix to pass, src/constructTLRMatrix.cu:13); an optional
 * trailing stream argument makes each call stream-ordered.
 */
#ifndef HM_REFCOMPAT_H
#define HM_REFCOMPAT_H

#include "hm.h"

namespace hmref {

enum DIVISION_METHOD {  // src/config.h:48-52
  POWER_OF_TWO_ON_LEFT = HM_DIV_POWER_OF_TWO_ON_LEFT,
  DIVIDE_IN_HALF = HM_DIV_DIVIDE_IN_HALF,
  FULL_TREE = HM_DIV_FULL_TREE
};

enum ADMISSIBILITY_CONDITION {  // src/config.h:88-91
  WEAK_ADMISSIBILITY = HM_ADMISS_WEAK,
  BOX_CENTER_ADMISSIBILITY = HM_ADMISS_BOX_CENTER
};

// The reference's per-level boxes (src/boundingBoxes.h:8-23); here they stay
// in the tree, which this names.
struct KDTreeBoundingBoxes {
  hm_kdtree tree = nullptr;
};

// src/kDTree.cuh:8-14: segmentIndices / segmentOffsets are device pointers
// owned by the tree (valid until freeKDTree).
struct KDTree {
  hm_kdtree h = nullptr;
  unsigned numberOfInputPoints = 0, dimensionOfInputPoints = 0, bucketSize = 0;
  DIVISION_METHOD divMethod = FULL_TREE;
  unsigned numSegments = 0, segmentSize = 0;
  const int* segmentIndices = nullptr;
  const int* segmentOffsets = nullptr;
  KDTreeBoundingBoxes boundingBoxes;
};

struct HMatrixStructure {  // src/HMatrixStructure.cuh:8-13
  hm_structure h = nullptr;
  int numLevels = 0;
};

struct HMatrix {  // src/HMatrix.cuh:28-34
  hm_hmatrix h = nullptr;
  HMatrixStructure matrixStructure;
};

// src/kDTreeHelpers.cu:107-116
inline int upperPowerOfTwo(int v) {
  v--;
  v |= v >> 1;
  v |= v >> 2;
  v |= v >> 4;
  v |= v >> 8;
  v |= v >> 16;
  return v + 1;
}

inline hm_status generateDataset(int numberOfInputPoints, int dimensionOfInputPoints, double* d_pointCloud,
                                 void* stream = nullptr) {
  return hm_generate_dataset(numberOfInputPoints, dimensionOfInputPoints, 1234ull, d_pointCloud, stream);
}

// Records the sizes; the storage is allocated by constructKDTree.
inline hm_status allocateKDTree(KDTree& tree, unsigned numberOfInputPoints, unsigned dimensionOfInputPoints,
                                unsigned bucketSize, DIVISION_METHOD divMethod) {
  tree.numberOfInputPoints = numberOfInputPoints;
  tree.dimensionOfInputPoints = dimensionOfInputPoints;
  tree.bucketSize = bucketSize;
  tree.divMethod = divMethod;
  return HM_OK;
}

inline hm_status constructKDTree(unsigned numberOfInputPoints, unsigned dimensionOfInputPoints, unsigned bucketSize,
                                 KDTree& tree, const double* d_pointCloud, DIVISION_METHOD divMethod,
                                 void* stream = nullptr) {
  if (tree.h) {
    hm_kdtree_free(tree.h);
    tree.h = nullptr;
  }
  allocateKDTree(tree, numberOfInputPoints, dimensionOfInputPoints, bucketSize, divMethod);
  hm_status s = hm_kdtree_build_div(d_pointCloud, (int)numberOfInputPoints, (int)dimensionOfInputPoints,
                                    (int)bucketSize, (int)divMethod, stream, &tree.h);
  if (s != HM_OK) return s;
  int n = 0, depth = 0;
  hm_kdtree_info(tree.h, &n, nullptr, nullptr, &depth);
  tree.numSegments = 1u << depth;
  unsigned seg = (unsigned)n;  // the largest leaf: ceil-halved depth times
  for (int l = 0; l < depth; ++l) seg = (seg + 1) / 2;
  tree.segmentSize = seg;
  tree.segmentIndices = hm_kdtree_device_perm(tree.h);
  tree.segmentOffsets = hm_kdtree_device_offsets(tree.h);
  tree.boundingBoxes.tree = tree.h;
  return HM_OK;
}

// numberOfInputPoints is the reference's upperPowerOfTwo(N) (src/main.cu:91);
// the level count comes from the tree.  Both box arguments must name the same
// tree (the reference passes kDTree.boundingBoxes twice).  eta: the
// box-center parameter the reference fixes to 1.0 (src/HMatrixStructure.cu:7).
inline hm_status constructHMatrixStructure(HMatrixStructure* st, unsigned numberOfInputPoints,
                                           unsigned dimensionOfInputPoints, unsigned bucketSize,
                                           ADMISSIBILITY_CONDITION admissibilityCondition,
                                           KDTreeBoundingBoxes rowBoxes, KDTreeBoundingBoxes columnBoxes,
                                           double eta = 1.0, void* stream = nullptr) {
  (void)numberOfInputPoints;
  (void)dimensionOfInputPoints;
  (void)bucketSize;
  if (!st || !rowBoxes.tree || rowBoxes.tree != columnBoxes.tree) return HM_ERR_INVALID;
  if (st->h) {
    hm_structure_free(st->h);
    st->h = nullptr;
  }
  hm_status s = hm_structure_build(rowBoxes.tree, (int)admissibilityCondition, eta, stream, &st->h);
  if (s != HM_OK) return s;
  return hm_structure_info(st->h, &st->numLevels, nullptr);
}

// Compresses every block of H.matrixStructure from the kernel on the points.
// opts (optional) carries the kernel, length scale, rank caps and precision;
// by default the reference's (hm_build_opts_default).  tol overrides
// opts->tol, as the reference's lowestLevelTolerance argument does.
inline hm_status generateHMatrixFromStruct(const KDTree& tree, HMatrix& H, const double* d_pointCloud,
                                           float tolerance, const hm_build_opts* opts = nullptr,
                                           void* stream = nullptr) {
  hm_build_opts o;
  if (opts) {
    o = *opts;
  } else {
    hm_build_opts_default((int)tree.dimensionOfInputPoints, &o);
  }
  o.tol = tolerance;
  if (H.h) {
    hm_hmatrix_free(H.h);
    H.h = nullptr;
  }
  return hm_hmatrix_build(tree.h, H.matrixStructure.h, d_pointCloud, &o, stream, &H.h);
}

// The reference's product: X and Y device, column-major N x nrhs FP64, tree
// order (src/HMatrixVectorMultiplication.cu:10-27).  b and ns are implied by
// the matrix.  The product runs in the matrix's form (FP32 or mixed).
inline hm_status HMatrixVecMult(unsigned numberOfInputPoints, unsigned bucketSize, unsigned numSegments,
                                unsigned vectorWidth, const HMatrix& H, double* inputVectors,
                                double* resultVectors, void* stream = nullptr) {
  (void)bucketSize;
  (void)numSegments;
  return hm_hmatvec_f64(H.h, 0, (int)vectorWidth, inputVectors, (int)numberOfInputPoints, resultVectors,
                        (int)numberOfInputPoints, 0, stream);
}

// The same product on FP32 vectors (no conversion).
inline hm_status HMatrixVecMult(unsigned numberOfInputPoints, unsigned vectorWidth, const HMatrix& H,
                                const float* inputVectors, float* resultVectors, void* stream = nullptr) {
  return hm_hmatvec(H.h, 0, (int)vectorWidth, inputVectors, (int)numberOfInputPoints, resultVectors,
                    (int)numberOfInputPoints, 0, stream);
}

inline void freeKDTree(KDTree& t) {
  hm_kdtree_free(t.h);
  t.h = nullptr;
  t.segmentIndices = t.segmentOffsets = nullptr;
  t.boundingBoxes.tree = nullptr;
}
inline void freeHMatrixStructure(HMatrixStructure& s) {
  hm_structure_free(s.h);
  s.h = nullptr;
}
// Frees the factors and dense blocks, not H.matrixStructure, as the
// reference's freeHMatrix does (src/HMatrix.cu:104-109).
inline void freeHMatrix(HMatrix& H) {
  hm_hmatrix_free(H.h);
  H.h = nullptr;
}

}  // namespace hmref

#endif /* HM_REFCOMPAT_H */
