/*
 * hm_oracle.c -- CPU restatement of the reference H-matrix pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by
 * tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and
 * by nothing else.  The product path (libhmb200.so) never links or calls it.
 *
 * Parity status: pinned.  The KD tree, bounding boxes and block structure
 * produced here are compared bit for bit against outputs of the reference's
 * own compiled code (oracle/ref_pipeline.cu built from the reference sources,
 * run on a GPU; fixtures in tests/golden/).
 *
 * Every function cites the reference file:line it restates.  Citations are
 * relative to the reference project root.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ENOMEM 2

/* ------------------------------------------------------------------ */
/* tree depth: number of ceil-halvings until the segment fits a bucket */
/* src/kDTreeHelpers.cu:118-128 (getMaxSegmentSize)                    */
/* ------------------------------------------------------------------ */
int orc_tree_depth(int n, int bucket) {
  int it = 0;
  while (n > bucket) {
    n = (n + 1) / 2;
    ++it;
  }
  return it;
}

/* src/kDTreeHelpers.cu:107-116 (upperPowerOfTwo) */
int orc_upper_pow2(int v) {
  v--;
  v |= v >> 1;
  v |= v >> 2;
  v |= v >> 4;
  v |= v >> 8;
  v |= v >> 16;
  v++;
  return v;
}

/* Stable merge sort of (key, payload) by key, ascending.  The reference uses
 * cub::DeviceSegmentedRadixSort::SortPairs (src/kDTreeConstruction.cu:167-174),
 * which is stable and orders doubles by value with -0.0 == +0.0; a stable
 * comparison sort on IEEE `<` gives the same permutation for non-NaN keys. */
static void merge_sort_stable(double* key, int* val, double* tk, int* tv, int n) {
  for (int width = 1; width < n; width *= 2) {
    for (int lo = 0; lo < n; lo += 2 * width) {
      int mid = lo + width < n ? lo + width : n;
      int hi = lo + 2 * width < n ? lo + 2 * width : n;
      int i = lo, j = mid, o = lo;
      while (i < mid && j < hi) {
        if (key[j] < key[i]) { tk[o] = key[j]; tv[o++] = val[j++]; }
        else { tk[o] = key[i]; tv[o++] = val[i++]; }
      }
      while (i < mid) { tk[o] = key[i]; tv[o++] = val[i++]; }
      while (j < hi) { tk[o] = key[j]; tv[o++] = val[j++]; }
    }
    memcpy(key, tk, sizeof(double) * (size_t)n);
    memcpy(val, tv, sizeof(int) * (size_t)n);
  }
}

/*
 * KD tree, FULL_TREE division (src/kDTreeConstruction.cu:14-231):
 *   per level, per segment: min/max of each dimension (cub segmented Min/Max,
 *   :113-127), span = max-min (src/kDTreeHelpers.cu:52-64), split dimension =
 *   first index of the maximum span (cub ArgMax, :145-150), stable sort of the
 *   segment by the coordinate along that dimension (:167-174), children are
 *   [o, o+ceil(len/2)) and [o+ceil(len/2), o+len) (src/kDTreeHelpers.cu:81-94).
 *
 * pts:      SoA, pts[dim*n + i] (src/generateDataset.cu:11)
 * perm:     out, n ints: tree position -> original index (segmentIndices)
 * offsets:  out, 2^depth + 1 ints (segmentOffsets)
 * bmin/bmax:out, per level l in [0, depth] a block of 2^l * d doubles at
 *           offset (2^l - 1) * d, node-major [node*d + dim]
 *           (src/boundingBoxes.cu:23-36,52-72).  Level `depth` (leaves) is
 *           filled here too although the reference never fills it.
 * split_dim:out, per level l in [0, depth) a block of 2^l ints at 2^l - 1.
 */
int orc_kdtree(int n, int d, int bucket, const double* pts, int* perm, int* offsets,
               double* bmin, double* bmax, int* split_dim) {
  if (n <= 0 || d <= 0 || bucket <= 0) return ORC_EINVAL;
  int depth = orc_tree_depth(n, bucket);
  int nleaf = 1 << depth;
  int* off = (int*)malloc(sizeof(int) * (size_t)(nleaf + 1));
  int* off2 = (int*)malloc(sizeof(int) * (size_t)(nleaf + 1));
  double* key = (double*)malloc(sizeof(double) * (size_t)n);
  double* tk = (double*)malloc(sizeof(double) * (size_t)n);
  int* tv = (int*)malloc(sizeof(int) * (size_t)n);
  if (!off || !off2 || !key || !tk || !tv) {
    free(off); free(off2); free(key); free(tk); free(tv);
    return ORC_ENOMEM;
  }
  for (int i = 0; i < n; ++i) perm[i] = i; /* initIndexMap, src/kDTreeHelpers.cu:12-26 */
  off[0] = 0;
  off[1] = n;
  int nseg = 1;
  for (int level = 0; level <= depth; ++level) {
    double* lmin = bmin + (size_t)(nseg - 1) * d;
    double* lmax = bmax + (size_t)(nseg - 1) * d;
    for (int s = 0; s < nseg; ++s) {
      for (int k = 0; k < d; ++k) {
        double mn = INFINITY, mx = -INFINITY;
        for (int p = off[s]; p < off[s + 1]; ++p) {
          double x = pts[(size_t)k * n + perm[p]];
          if (x < mn) mn = x;
          if (x > mx) mx = x;
        }
        lmin[(size_t)s * d + k] = mn;
        lmax[(size_t)s * d + k] = mx;
      }
    }
    if (level == depth) break;
    int* ldim = split_dim + (nseg - 1);
    for (int s = 0; s < nseg; ++s) {
      int best = 0;
      double bspan = lmax[(size_t)s * d] - lmin[(size_t)s * d];
      for (int k = 1; k < d; ++k) {
        double sp = lmax[(size_t)s * d + k] - lmin[(size_t)s * d + k];
        if (sp > bspan) { bspan = sp; best = k; }
      }
      ldim[s] = best;
      int lo = off[s], len = off[s + 1] - off[s];
      for (int p = 0; p < len; ++p) key[p] = pts[(size_t)best * n + perm[lo + p]];
      merge_sort_stable(key, perm + lo, tk, tv, len);
      off2[2 * s] = lo;
      off2[2 * s + 1] = lo + (len + 1) / 2;
    }
    off2[2 * nseg] = n;
    nseg *= 2;
    memcpy(off, off2, sizeof(int) * (size_t)(nseg + 1));
  }
  memcpy(offsets, off, sizeof(int) * (size_t)(nleaf + 1));
  free(off); free(off2); free(key); free(tk); free(tv);
  return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* Admissibility (src/admissibilityCondition.cu:7-68)                  */
/* ------------------------------------------------------------------ */
static double box_center_distance(const double* umin, const double* umax, const double* vmin,
                                  const double* vmax, int d) {
  /* src/admissibilityCondition.cu:7-15 */
  double distance = 0;
  for (int i = 0; i < d; ++i) {
    double c = 0.5 * ((umax[i] + umin[i]) - (vmax[i] + vmin[i]));
    distance += c * c;
  }
  return sqrt(distance);
}

static double box_diameter(const double* mn, const double* mx, int d) {
  /* src/admissibilityCondition.cu:17-25 */
  double diameter = 0;
  for (int i = 0; i < d; ++i) {
    double e = mx[i] - mn[i];
    diameter += e * e;
  }
  return sqrt(diameter);
}

/* admiss: 0 = weak (src/admissibilityCondition.cu:54-68),
 *         1 = box-center (src/admissibilityCondition.cu:27-52) */
int orc_admissible(int admiss, int u, int v, const double* umin, const double* umax,
                   const double* vmin, const double* vmax, int d, double eta) {
  if (u == v) return 0;
  if (admiss == 0) return 1;
  double dist = box_center_distance(umin, umax, vmin, vmax, d);
  double du = box_diameter(umin, umax, d);
  double dv = box_diameter(vmin, vmax, d);
  if (du == 0 || dv == 0) return 0;
  return 0.5 * (du + dv) <= eta * dist;
}

/* Morton index of (column cluster u, row cluster v): src/helperKernels.cuh:87-109 */
uint32_t orc_morton(uint32_t u, uint32_t v) {
  uint32_t z = 0;
  for (int b = 0; b < 16; ++b) {
    z |= ((u >> b) & 1u) << (2 * b);
    z |= ((v >> b) & 1u) << (2 * b + 1);
  }
  return z;
}

typedef struct {
  int admiss;
  double eta;
  int d;
  int max_depth;
  const double* bmin;
  const double* bmax;
  int* counts;         /* per level 1..max_depth at [level-1] */
  int* const* lists;   /* per level buffer */
  const int* caps;     /* capacity of each list */
  int overflow;
} orc_struct_ctx;

/* src/HMatrixStructure.cu:9-90 (constructMatrixStruct_recursive) */
static void struct_rec(orc_struct_ctx* c, int u, int v, int level) {
  int diag = (u == v);
  int leaf = (level == c->max_depth);
  if (diag && leaf) return;
  int adm = 0;
  if (!leaf) {
    size_t base = (size_t)((1 << level) - 1) * c->d;
    adm = orc_admissible(c->admiss, u, v, c->bmin + base + (size_t)u * c->d,
                         c->bmax + base + (size_t)u * c->d, c->bmin + base + (size_t)v * c->d,
                         c->bmax + base + (size_t)v * c->d, c->d, c->eta);
  }
  if (leaf || adm) {
    int li = level - 1;
    if (c->counts[li] >= c->caps[li]) { c->overflow = 1; return; }
    c->lists[li][c->counts[li]++] = (int)orc_morton((uint32_t)u, (uint32_t)v);
    return;
  }
  struct_rec(c, 2 * u, 2 * v, level + 1);
  struct_rec(c, 2 * u + 1, 2 * v, level + 1);
  struct_rec(c, 2 * u, 2 * v + 1, level + 1);
  struct_rec(c, 2 * u + 1, 2 * v + 1, level + 1);
}

/*
 * Block structure (src/HMatrixStructure.cu:92-160).  max_depth = tree depth;
 * counts[l-1], lists[l-1] for l = 1..max_depth hold the Morton indices of the
 * blocks recorded at level l, in the reference's DFS order.
 * Returns ORC_ENOMEM (and sets nothing further) if a list overflows its cap.
 */
int orc_structure(int d, int max_depth, int admiss, double eta, const double* bmin,
                  const double* bmax, int* counts, int* const* lists, const int* caps) {
  orc_struct_ctx c;
  c.admiss = admiss;
  c.eta = eta;
  c.d = d;
  c.max_depth = max_depth;
  c.bmin = bmin;
  c.bmax = bmax;
  c.counts = counts;
  c.lists = lists;
  c.caps = caps;
  c.overflow = 0;
  for (int l = 0; l < max_depth; ++l) counts[l] = 0;
  struct_rec(&c, 0, 0, 0);
  return c.overflow ? ORC_ENOMEM : ORC_OK;
}

/* ------------------------------------------------------------------ */
/* Kernel functions.  The reference evaluates exp(-r/l) with l = 0.2 for */
/* d = 3 else 0.1 (src/TLRMatrixHelpers.cu:40-58); the others extend it  */
/* with the kernels the workloads name.                                  */
/* ------------------------------------------------------------------ */
enum { ORC_K_EXP = 0, ORC_K_MATERN32 = 1, ORC_K_GAUSS = 2 };

double orc_kernel_r2(int kind, int deriv, double r2, double ell) {
  double r = sqrt(r2);
  switch (kind) {
    case ORC_K_EXP: {
      double e = exp(-r / ell);
      return deriv ? (r / (ell * ell)) * e : e;
    }
    case ORC_K_MATERN32: {
      double a = sqrt(3.0) * r / ell;
      double e = exp(-a);
      return deriv ? a * a * e / ell : (1.0 + a) * e;
    }
    case ORC_K_GAUSS: {
      double g = exp(-r2 / (2.0 * ell * ell));
      return deriv ? g * r2 / (ell * ell * ell) : g;
    }
  }
  return NAN;
}

/* entry (i, j) for original point indices pi, pj; src/TLRMatrixHelpers.cu:44-58 */
static double entry(int kind, int deriv, double ell, double nugget, const double* pts, int n,
                    int d, int pi, int pj) {
  double r2 = 0;
  for (int k = 0; k < d; ++k) {
    double t = pts[(size_t)k * n + pj] - pts[(size_t)k * n + pi];
    r2 += t * t;
  }
  double v = orc_kernel_r2(kind, deriv, r2, ell);
  if (pi == pj && !deriv) v += nugget;
  return v;
}

/*
 * Dense FP64 product on selected rows: Y[r, :] = sum_j A(rows[r], j) X[j, :],
 * with A in tree order, A(i, j) = K(p[perm[i]], p[perm[j]]).  X is column-major
 * n x nrhs (ld n), Y is column-major nrows x nrhs (ld nrows).  This is the
 * dense reference product of src/expandMatrix.cu:142-199, restricted to rows.
 */
int orc_dense_rows_matvec(int n, int d, const double* pts, const int* perm, int kind, int deriv,
                          double ell, double nugget, const int* rows, int nrows, int nrhs,
                          const double* X, double* Y) {
  int err = 0;
#pragma omp parallel
  {
    double* arow = (double*)malloc(sizeof(double) * (size_t)n);
    if (!arow) {
#pragma omp atomic write
      err = 1;
    } else {
#pragma omp for schedule(dynamic, 4)
      for (int r = 0; r < nrows; ++r) {
        int pi = perm[rows[r]];
        for (int j = 0; j < n; ++j) arow[j] = entry(kind, deriv, ell, nugget, pts, n, d, pi, perm[j]);
        for (int c = 0; c < nrhs; ++c) {
          double acc = 0;
          const double* x = X + (size_t)c * n;
          for (int j = 0; j < n; ++j) acc += arow[j] * x[j];
          Y[(size_t)c * nrows + r] = acc;
        }
      }
      free(arow);
    }
  }
  return err ? ORC_ENOMEM : ORC_OK;
}

/*
 * Dense block A(r0:r0+m, c0:c0+n) in tree order, column-major (ld m), FP64.
 * src/TLRMatrixHelpers.cu:60-101 (generateDenseBlockColumn) without padding.
 */
int orc_dense_block(int n, int d, const double* pts, const int* perm, int kind, int deriv,
                    double ell, double nugget, int r0, int m, int c0, int ncols, double* out) {
  for (int j = 0; j < ncols; ++j)
    for (int i = 0; i < m; ++i)
      out[(size_t)j * m + i] =
          entry(kind, deriv, ell, nugget, pts, n, d, perm[r0 + i], perm[c0 + j]);
  return ORC_OK;
}

/*
 * Relative Frobenius error ||A - U V^T||_F / ||A||_F of one block, FP64.
 * U is m x k, V is n x k, both column-major.  src/expandMatrix.cu:31-37,66-97.
 */
double orc_block_error(int n, int d, const double* pts, const int* perm, int kind, int deriv,
                       double ell, double nugget, int r0, int m, int c0, int ncols, int k,
                       const double* U, const double* V) {
  double num = 0, den = 0;
  for (int j = 0; j < ncols; ++j) {
    for (int i = 0; i < m; ++i) {
      double a = entry(kind, deriv, ell, nugget, pts, n, d, perm[r0 + i], perm[c0 + j]);
      double s = 0;
      for (int t = 0; t < k; ++t) s += U[(size_t)t * m + i] * V[(size_t)t * ncols + j];
      num += (a - s) * (a - s);
      den += a * a;
    }
  }
  return den > 0 ? sqrt(num / den) : sqrt(num);
}

/*
 * Rows `rows[0..nrows)` (tree-order indices) of the kernel matrix restricted to
 * columns [c0, c0+ncols): out is nrows x ncols, row-major.  Used to check
 * sampled rows of large blocks.
 */
int orc_dense_rows_block(int n, int d, const double* pts, const int* perm, int kind, int deriv,
                         double ell, double nugget, const int* rows, int nrows, int c0, int ncols,
                         double* out) {
#pragma omp parallel for schedule(static)
  for (int r = 0; r < nrows; ++r)
    for (int j = 0; j < ncols; ++j)
      out[(size_t)r * ncols + j] =
          entry(kind, deriv, ell, nugget, pts, n, d, perm[rows[r]], perm[c0 + j]);
  return ORC_OK;
}

/* Relative error ||y - y_ref|| / ||y_ref|| (src/expandMatrix.cu:221-231). */
double orc_rel_error(const double* y, const double* yref, long long len) {
  double num = 0, den = 0;
  for (long long i = 0; i < len; ++i) {
    double t = y[i] - yref[i];
    num += t * t;
    den += yref[i] * yref[i];
  }
  return den > 0 ? sqrt(num / den) : sqrt(num);
}
