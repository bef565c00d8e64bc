/*
 * hm_refcompat.h -- the reference's operator names over the C ABI.
 *
 * A maintainer of the reference (a C++/CUDA program, no FFI) switches its
 * pipeline to libhmb200.so by including this header instead of the reference's
 * kDTree*.cuh / HMatrixStructure.cuh / constructHMatrixFromStruct.cuh /
 * HMatrixVectorMultiplication.cuh and linking -lhmb200.  The functions keep
 * the reference's names and argument meaning; they return hm_status instead of
 * exiting, and the tree / structure / matrix are opaque handles.
 *
 *   reference (file:line)                                     here
 *   generateDataset(N, d, d_points)  src/generateDataset.cu:15  generateDataset
 *   allocateKDTree + constructKDTree src/kDTree.cu:6,
 *                                    src/kDTreeConstruction.cu:14 constructKDTree
 *   constructHMatrixStructure        src/HMatrixStructure.cu:133  constructHMatrixStructure
 *   allocateHMatrix +
 *   generateHMatrixFromStruct        src/HMatrix.cu:57,
 *                                    src/constructHMatrixFromStruct.cu:13 generateHMatrixFromStruct
 *   HMatrixVecMult(..., double* X, double* Y) src/HMatrixVectorMultiplication.cu:10
 *                                                             HMatrixVecMult (FP32 vectors)
 */
#ifndef HM_REFCOMPAT_H
#define HM_REFCOMPAT_H

#include "hm.h"

namespace hmref {

struct KDTree {
  hm_kdtree h = nullptr;
};
struct HMatrixStructure {
  hm_structure h = nullptr;
};
struct HMatrix {
  hm_hmatrix h = nullptr;
};

enum ADMISSIBILITY_CONDITION { WEAK_ADMISSIBILITY = HM_ADMISS_WEAK, BOX_CENTER_ADMISSIBILITY = HM_ADMISS_BOX_CENTER };

inline hm_status generateDataset(int numberOfInputPoints, int dimensionOfInputPoints, double* d_pointCloud,
                                 void* stream = nullptr) {
  return hm_generate_dataset(numberOfInputPoints, dimensionOfInputPoints, 1234ull, d_pointCloud, stream);
}

inline hm_status constructKDTree(unsigned numberOfInputPoints, unsigned dimensionOfInputPoints,
                                 unsigned bucketSize, KDTree& tree, const double* d_pointCloud,
                                 void* stream = nullptr) {
  return hm_kdtree_build(d_pointCloud, (int)numberOfInputPoints, (int)dimensionOfInputPoints, (int)bucketSize,
                         stream, &tree.h);
}

inline hm_status constructHMatrixStructure(HMatrixStructure* st, const KDTree& tree,
                                           ADMISSIBILITY_CONDITION admissibilityCondition, double eta = 1.0,
                                           void* stream = nullptr) {
  return hm_structure_build(tree.h, (int)admissibilityCondition, eta, stream, &st->h);
}

inline hm_status generateHMatrixFromStruct(const KDTree& tree, const HMatrixStructure& st,
                                           const double* d_pointCloud, float tolerance, HMatrix& out,
                                           hm_build_opts* opts = nullptr, void* stream = nullptr) {
  int d = 0;
  hm_status s = hm_kdtree_info(tree.h, nullptr, &d, nullptr, nullptr);
  if (s != HM_OK) return s;
  hm_build_opts o;
  if (opts) {
    o = *opts;
  } else {
    hm_build_opts_default(d, &o);
  }
  o.tol = tolerance;
  return hm_hmatrix_build(tree.h, st.h, d_pointCloud, &o, stream, &out.h);
}

inline hm_status HMatrixVecMult(unsigned numberOfInputPoints, unsigned vectorWidth, const HMatrix& H,
                                const float* inputVectors, float* resultVectors, void* stream = nullptr) {
  return hm_hmatvec(H.h, 0, (int)vectorWidth, inputVectors, (int)numberOfInputPoints, resultVectors,
                    (int)numberOfInputPoints, 0, stream);
}

inline void freeKDTree(KDTree& t) {
  hm_kdtree_free(t.h);
  t.h = nullptr;
}
inline void freeHMatrixStructure(HMatrixStructure& s) {
  hm_structure_free(s.h);
  s.h = nullptr;
}
inline void freeHMatrix(HMatrix& H) {
  hm_hmatrix_free(H.h);
  H.h = nullptr;
}

}  // namespace hmref

#endif /* HM_REFCOMPAT_H */
