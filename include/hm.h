/*
 * hm.h -- C ABI of the B200 hierarchical-matrix engine (libhmb200.so).
 *
 * The entry points replace the reference's pipeline functions one for one
 * (citations are file:line in the reference project):
 *
 *   hm_generate_dataset     generateDataset              src/generateDataset.cu:15-19
 *   hm_kdtree_build         allocateKDTree+constructKDTree src/kDTree.cu:6-31,
 *                                                         src/kDTreeConstruction.cu:14-231
 *   hm_kdtree_copy_out      KDTree / KDTreeBoundingBoxes   src/kDTree.cuh:8-14,
 *                           (perm, offsets, boxes)         src/boundingBoxes.h:8-23
 *   hm_structure_build      constructHMatrixStructure      src/HMatrixStructure.cu:133-160
 *   hm_structure_tiles      HMatrixStructure.tileIndices   src/HMatrixStructure.cuh:8-13
 *   hm_tlr_build            createColumnMajorLRMatrix      src/constructTLRMatrix.cu:13-151
 *   hm_hmatrix_build        allocateHMatrix +              src/HMatrix.cu:57-103,
 *                           generateHMatrixFromStruct      src/constructHMatrixFromStruct.cu:13-103
 *   hm_hmatvec              HMatrixVecMult                 src/HMatrixVectorMultiplication.cu:10-27
 *   hm_*_free               freeKDTree / freeMatrix /      src/kDTree.cu:33-36, src/TLRMatrix.cu:5,
 *                           freeHMatrix / freeHMatrixStructure src/HMatrix.cu:105-110,
 *                                                         src/HMatrixStructure.cu:162-168
 *
 * Conventions.  Every function returns an hm_status and never exits the
 * process; hm_last_error() gives a message for the last failure on the calling
 * thread.  Points are caller-owned device buffers in the reference's SoA
 * layout p[dim*n + i].  Vectors are caller-owned device buffers, column-major
 * n x nrhs.  `stream` is a cudaStream_t passed as void* (NULL = legacy default
 * stream).  Objects are opaque handles owned by the library; one handle may be
 * used by one host thread at a time.
 */
#ifndef HM_H
#define HM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HM_API __attribute__((visibility("default")))
#else
#define HM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  HM_OK = 0,
  HM_ERR_INVALID = 1,       /* bad argument (null pointer, size, enum) */
  HM_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  HM_ERR_NOMEM = 3,         /* device or host allocation failed */
  HM_ERR_UNSUPPORTED = 4,   /* valid request outside what this library supports */
  HM_ERR_TIMEOUT = 5,       /* a bounded device-side wait gave up */
  HM_ERR_NOT_CONVERGED = 6  /* an iterative solve stopped at its iteration limit */
} hm_status;

typedef enum { HM_ADMISS_WEAK = 0, HM_ADMISS_BOX_CENTER = 1 } hm_admissibility;

typedef enum {
  HM_KERNEL_EXP = 0,       /* exp(-r/l)                       src/TLRMatrixHelpers.cu:44-58 */
  HM_KERNEL_MATERN32 = 1,  /* (1 + sqrt3 r/l) exp(-sqrt3 r/l) */
  HM_KERNEL_GAUSS = 2      /* exp(-r^2 / (2 l^2))             */
} hm_kernel;

typedef enum {
  HM_PREC_FP32 = 0,        /* FP32 factors, FP32 arithmetic (TF32 hi + lo tensor-core products) */
  HM_PREC_MIXED = 1        /* BF16 factors with a BF16 low part where the tolerance needs it; the FP32
                              factors are released once the BF16 panels are built */
} hm_precision;

typedef struct hm_kdtree_s* hm_kdtree;
typedef struct hm_structure_s* hm_structure;
typedef struct hm_hmatrix_s* hm_hmatrix;
typedef struct hm_batch_s* hm_batch;

/* Message describing the last failure on this thread ("" if none). */
HM_API const char* hm_last_error(void);

/* Library version string. */
HM_API const char* hm_version(void);

/* --- points ------------------------------------------------------------- */

/* generateDataset (src/generateDataset.cu:15-19): d_points[i] for i < n*d is
 * curand_uniform of a XORWOW state initialised with (seed, subsequence i, 0).
 * seed = 1234 reproduces the reference bit for bit. */
HM_API hm_status hm_generate_dataset(int n, int d, unsigned long long seed, double* d_points,
                              void* stream);

/* Points from an isotropic Gaussian mixture (no counterpart in the reference;
 * the scale-stress workload): ncomp components with centres uniform in
 * [0,1]^d, standard deviations log-uniform in [sigma_min, sigma_max] and
 * weights from Dirichlet(1, ..., 1), all drawn from `seed`; d_points gets the
 * SoA layout of hm_generate_dataset (d * n doubles). */
HM_API hm_status hm_generate_mixture(int n, int d, int ncomp, double sigma_min, double sigma_max,
                                     unsigned long long seed, double* d_points, void* stream);

/* --- KD tree ------------------------------------------------------------ */

/* allocateKDTree + constructKDTree, FULL_TREE division
 * (src/kDTree.cu:6-31, src/kDTreeConstruction.cu:14-231).  The permutation,
 * leaf offsets and per-level boxes equal the reference's bit for bit.
 * d_points is read during the call only.  bucket >= 1; n >= 1; 1 <= d <= 16. */
HM_API hm_status hm_kdtree_build(const double* d_points, int n, int d, int bucket, void* stream,
                          hm_kdtree* out);

/* The reference's DIVISION_METHOD (src/config.h:48-52, same values). */
typedef enum {
  HM_DIV_POWER_OF_TWO_ON_LEFT = 0,
  HM_DIV_DIVIDE_IN_HALF = 1,
  HM_DIV_FULL_TREE = 2
} hm_division;

/* allocateKDTree(tree, N, d, b, divMethod) + constructKDTree(N, d, b, tree,
 * points, divMethod) (src/kDTree.cu:6-31, src/kDTreeConstruction.cu:14-231)
 * with the reference's division argument.  FULL_TREE and DIVIDE_IN_HALF run
 * the same construction in the reference (they differ only in how many
 * segment offsets allocateKDTree reserves, src/kDTree.cu:17-22) and give
 * hm_kdtree_build's tree.  POWER_OF_TWO_ON_LEFT splits segments at
 * power-of-two offsets (src/kDTreeConstruction.cu:77-206); for a power-of-two
 * n every such split is the ceil(len/2) split, so the tree is again
 * hm_kdtree_build's; other n return HM_ERR_UNSUPPORTED.  Any other value is
 * HM_ERR_INVALID. */
HM_API hm_status hm_kdtree_build_div(const double* d_points, int n, int d, int bucket, int division,
                                     void* stream, hm_kdtree* out);

/* depth = number of levels below the root; leaves = 2^depth. */
HM_API hm_status hm_kdtree_info(hm_kdtree t, int* n, int* d, int* bucket, int* depth);

/* Host copies.  Any pointer may be NULL.  perm: n ints (tree position ->
 * original index, segmentIndices); offsets: 2^depth+1 ints (segmentOffsets);
 * bmin/bmax: levels 0..depth, level l at [(2^l - 1)*d], node-major
 * [node*d + dim] (levels 0..depth-1 are the reference's
 * KDTreeBoundingBoxes); split_dim: levels 0..depth-1, level l at [2^l - 1]. */
HM_API hm_status hm_kdtree_copy_out(hm_kdtree t, int* perm, int* offsets, double* bmin, double* bmax,
                             int* split_dim);

/* Device pointers owned by the tree (valid until hm_kdtree_free). */
HM_API const int* hm_kdtree_device_perm(hm_kdtree t);
HM_API const int* hm_kdtree_device_offsets(hm_kdtree t);

HM_API void hm_kdtree_free(hm_kdtree t);

/* --- block structure ----------------------------------------------------- */

/* constructHMatrixStructure (src/HMatrixStructure.cu:133-160): per level
 * l = 1..depth the list of blocks recorded at that level, as Morton indices
 * z = interleave(column cluster) | interleave(row cluster) << 1, in the
 * reference's order.  eta is the box-center parameter (the reference fixes
 * 1.0, src/HMatrixStructure.cu:7). */
HM_API hm_status hm_structure_build(hm_kdtree t, int admissibility, double eta, void* stream,
                             hm_structure* out);

/* num_levels = depth + 1 as in the reference; counts[l-1] for l = 1..depth
 * (counts needs num_levels - 1 entries; may be NULL). */
HM_API hm_status hm_structure_info(hm_structure s, int* num_levels, int* counts);

/* Host copy of the Morton list of level l (1 <= l <= depth). */
HM_API hm_status hm_structure_tiles(hm_structure s, int level, int* tiles);

/* Row-major (CSR) and jagged-diagonal (JDS) layouts of level l, built on the
 * device (the reference's JDS.cuh declares HMatrixLevelJDS, src/JDS.cuh:7-17,
 * but never fills it).  Any pointer may be NULL.  row_ptr: 2^l + 1; csr_blk:
 * counts[l-1] indices into the level's Morton list, grouped by row cluster,
 * increasing column within a row; jds_rows: 2^l row clusters by decreasing
 * block count; jds_ptr: max_row_blocks + 1 diagonal starts; jds_blk:
 * counts[l-1] entries, jds_blk[jds_ptr[j] + r] = j-th block of row jds_rows[r]. */
HM_API hm_status hm_structure_jds(hm_structure s, int level, int* row_ptr, int* csr_blk,
                                  int* jds_rows, int* jds_ptr, int* jds_blk, int* max_row_blocks);

HM_API void hm_structure_free(hm_structure s);

/* --- H-matrix ------------------------------------------------------------ */

typedef struct {
  int kernel;          /* hm_kernel */
  double ell;          /* length scale */
  double nugget;       /* added to the diagonal */
  double tol;          /* per-block relative Frobenius tolerance */
  int max_rank;        /* rank cap for admissible blocks above the leaf level */
  int leaf_max_rank;   /* rank cap for leaf-level blocks (reference: bucket/2); 0 = bucket/2 */
  int sample_block;    /* ARA sample block (reference: 16) */
  int precision;       /* hm_precision */
  int derivative;      /* 0: K, 1: dK/dl */
  unsigned long long seed;  /* seed of the Gaussian test matrices */
  int diag_from_coords;     /* diagonal leaf blocks: 0 stored, 1 recomputed from the coordinates in
                               every product, -1 (default) recomputed for derivative builds only */
  int level_schedule;       /* 0 (default): tol and max_rank at every level above the leaves;
                               1: the reference's schedule -- the tolerance doubles at each level
                               above the leaves (tol 2^(depth - l) at level l,
                               src/constructHMatrixFromStruct.cu:31,54) and the cap at level l is
                               bucket 2^i, / 4 beyond i = 5, i = depth - 1 - l (generateMaxRanks,
                               src/helperFunctions.cu:67-74), at most 256; max_rank is unused */
} hm_build_opts;

/* Fills opts with the reference's settings: exp kernel, l = 0.2 if d == 3
 * else 0.1 (src/TLRMatrixHelpers.cu:40-42), tol 1e-5, sample block 16. */
HM_API void hm_build_opts_default(int d, hm_build_opts* opts);

/* allocateHMatrix + generateHMatrixFromStruct: compresses every block of the
 * structure by adaptive randomized approximation on kernel entries generated
 * from the points, leaf diagonal blocks dense.  d_points: the points the tree
 * was built from. */
HM_API hm_status hm_hmatrix_build(hm_kdtree t, hm_structure s, const double* d_points,
                           const hm_build_opts* opts, void* stream, hm_hmatrix* out);

/* One block-row shard of the H-matrix, for a product spread over several
 * GPUs (no counterpart in the reference, which runs on one GPU).  The shard
 * owns the rows of leaves [leaf_begin, leaf_end) -- for G ranks, a contiguous
 * run of the 2^L subtrees at tree level L = ceil(log2 G) -- and compresses
 * only the blocks whose row or column cluster overlaps those rows (a pair
 * across two shards is compressed by both), plus its own diagonal leaves.
 * Its product (hm_hmatvec, hm_hmatvec_f64) reads all of X and writes only
 * the shard's rows of Y: the other rows are left untouched.  Stacking the
 * shards' rows gives the whole matrix's product.  Same tree, structure and
 * options as hm_hmatrix_build.  A shard saved to a file (hm_hmatrix_save)
 * loads back as the same shard: the pieces of an out-of-core product, built
 * and applied one at a time (hmatrix.PiecewiseHMatrix). */
HM_API hm_status hm_hmatrix_build_rows(hm_kdtree t, hm_structure s, const double* d_points,
                                       const hm_build_opts* opts, int leaf_begin, int leaf_end, void* stream,
                                       hm_hmatrix* out);

typedef struct {
  long long num_lowrank;     /* low-rank blocks (each stored pair counted twice) */
  long long num_dense;       /* dense blocks, diagonal leaves included */
  long long rank_sum;        /* sum of ranks over low-rank blocks */
  int max_rank_seen;
  long long factor_bytes;    /* bytes of stored factors */
  long long dense_bytes;     /* bytes of stored dense blocks */
  long long num_unconverged; /* low-rank blocks stored above the tolerance (none: a block that misses it
                                at its rank cap is split, see num_split) */
  long long mixed_bytes;     /* mixed form: bytes one product reads from the BF16 copies
                                (2 B per high part, 2 B per low part, both orientations) */
  double build_seconds;      /* device time of hm_hmatrix_build */
  long long num_split;       /* admissible blocks that missed the tolerance at their rank cap and were
                                compressed as their four child blocks instead (recursively; at the
                                leaf level such a block is stored dense) */
  long long device_bytes;    /* device memory the matrix holds now (factors, panels, plans, workspaces) */
  double phase_seconds[8];   /* wall time of the build's phases (device work charged to the phase that
                                launched it): [0] set-up of problem lists, batches and workspaces,
                                [1] sketches Y = A Omega, [2] orthogonalisation and stopping tests,
                                [3] projections B = A^T Q, [4] truncation (Gram, Jacobi) and factor
                                packing, [5] diagonal leaf blocks, [6] block lists and factor panels,
                                [7] the product's plan */
} hm_hmatrix_stats;

HM_API hm_status hm_hmatrix_stats_get(hm_hmatrix h, hm_hmatrix_stats* st);

/* Y = H X (trans = 0) or Y = H^T X (trans = 1).  X, Y: device, column-major
 * n x nrhs with leading dimensions ldx, ldy >= n, FP32.  original_order = 0:
 * X and Y are in tree order (the reference's convention); 1: in the points'
 * original order (the permutation is applied inside).  No allocation and no
 * host synchronisation: the call is stream-ordered. */
HM_API hm_status hm_hmatvec(hm_hmatrix h, int trans, int nrhs, const float* X, int ldx, float* Y,
                     int ldy, int original_order, void* stream);

/* HMatrixVecMult with the reference's FP64 vectors
 * (src/HMatrixVectorMultiplication.cu:10, H2Opus_Real = double,
 * src/precision.h:6): Y = H X (trans = 0) or H^T X (trans = 1) for X, Y
 * device, column-major n x nrhs FP64 with leading dimensions ldx, ldy >= n.
 * The library narrows X to FP32 and widens the FP32 result into Y on the
 * device, a pass of right-hand sides at a time, in the matrix's own per-pass
 * buffers: no allocation and no host synchronisation.  The arithmetic is the
 * FP32 or mixed form the matrix was built in, so Y carries that form's error,
 * not FP64's.  original_order as for hm_hmatvec (the permutation is applied
 * by the same conversion kernels). */
HM_API hm_status hm_hmatvec_f64(hm_hmatrix h, int trans, int nrhs, const double* X, int ldx, double* Y, int ldy,
                                int original_order, void* stream);

/* Allocation-free product.  No counterpart in the reference.
 *
 * Same result as hm_hmatvec(h, 0, nrhs, X, ldx, Y, ldy, 0, stream) (tree
 * order), for callers that may not allocate device memory when they apply the
 * operator -- code running under an external allocator that owns all device
 * memory, or a latency-bound loop in which a cudaMalloc (which can synchronise
 * the device) is not acceptable.  It allocates nothing and does not use the
 * matrix's own projection workspace: its scratch is one fixed 16 MiB array
 * (4 Mi floats) in the library's device image, held by every GPU that loads
 * the library until the process exits.  It runs passes of 16 right-hand
 * sides, and a pass must fit in the array:
 *   mixed form: 16 floats per point (X split into BF16 hi + lo fragments,
 *               rows padded to 32 per leaf), plus 128 floats per
 *               (row chunk, 8-column tile) of panels projected in several
 *               row chunks, plus the projections (64 words per 8 factor
 *               columns, 128 for columns with a low part);
 *   FP32 form on panels (its default product): 32 floats per point (X as
 *               TF32 hi + lo fragments), the chunk partials as above, plus
 *               16 floats per factor column (the projections);
 *   FP32 form with the per-block kernels (schedule "fp32 p1_rows=..."):
 *               16 floats per factor column (sum of ranks over both
 *               orientations, padded to 8 per block), plus the chunk partials
 *               of blocks with more than p1_rows rows of V.
 * The floats per point put the limit near 2^18 points (mixed) or 2^17 (FP32
 * on panels) whatever the ranks.  A matrix beyond the array is rejected
 * with HM_ERR_UNSUPPORTED and a message naming its need.
 *
 * The first call on a device resolves the array's device address on that
 * device (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  All calls on a device share the one array, which keeps the last
 * call's contents; every word of it that a product reads is written earlier
 * in the same pass, so nothing needs clearing.  Calls whose work overlaps on
 * the GPU (other streams, other host threads) race and must be serialised by
 * the caller. */
HM_API hm_status hm_hmatvec_noalloc(hm_hmatrix h, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                    void* stream);

/* Conjugate gradients on the H-matrix: solves H X = B (tree order, X and B
 * n x nrhs column-major) for a symmetric positive definite kernel matrix, e.g.
 * a kernel with a nugget on its diagonal (kernel ridge regression, a
 * Gaussian-process solve).  No counterpart in the reference, which has no
 * solver; it is the natural consumer of the product (hm_hmatvec).
 *
 * One CG per column, all columns sharing every product; X starts at zero.
 * Vectors are FP32, dot products FP64 in a fixed order.  A column is done when
 * ||r|| <= tol ||b|| on CG's recurrence; from then on it is frozen on the
 * device (its X and r no longer change) while the other columns go on.  The
 * host checks the stream's work every `check_every` iterations and stops when
 * every column is done.  On a created stream
 * each chunk of check_every iterations is recorded once into a CUDA graph and
 * relaunched; on the legacy stream the iterations are launched directly.
 * Allocates its workspace (4 n x nrhs floats) from the stream-ordered pool
 * and synchronises the stream between chunks.  *iterations receives the
 * iterations run, *rel_residual the worst column's true relative residual
 * ||B - H X|| / ||B||, recomputed with one more product.  The tolerance is
 * tested on CG's recurrence; the mixed form's product is linear only to its
 * BF16 rounding (about 1e-4 relative), so there the true residual levels off
 * near that however small tol is.  Returns
 * HM_ERR_NOT_CONVERGED when max_iter iterations do not meet tol (X holds the
 * last iterate), HM_ERR_UNSUPPORTED when the operator shows itself not
 * positive definite (p.Ap <= 0 on a column that is not done). */
HM_API hm_status hm_cg_solve(hm_hmatrix h, int nrhs, const float* B, int ldb, float* X, int ldx, double tol,
                             int max_iter, int check_every, void* stream, int* iterations, double* rel_residual);

/* hm_hmatvec for one pass (nrhs <= 16; <= 128 for the mixed form, whose
 * passes multiply up to eight parts of 16 right-hand sides per factor read), X and Y
 * in tree order, with CUDA events recorded on `stream`
 * around its two kernels; synchronises and returns each kernel's device time
 * and algorithmic bytes (stored factors and dense blocks read once, X read,
 * Y written).  For measurement; the hot path is hm_hmatvec. */
HM_API hm_status hm_hmatvec_profile(hm_hmatrix h, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                    void* stream, float* ms_project, float* ms_expand,
                                    long long* bytes_project, long long* bytes_expand);

/* Per-kernel device times of one pass (nrhs as for hm_hmatvec_profile, X and
 * Y in tree order):
 * CUDA events on `stream` after each kernel, synchronised before return.
 * Fills up to `cap` entries of names (static strings), ms and algorithmic
 * bytes (what the kernel must read and write at least); *count receives the
 * number of kernels the product launched.  For measurement only; no
 * counterpart in the reference. */
HM_API hm_status hm_hmatvec_kernels(hm_hmatrix h, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                    void* stream, int cap, const char** names, float* ms, long long* bytes,
                                    int* count);

/* Block list as the matvec sees it (both orientations of each stored pair),
 * the counterpart of the reference's HMatrixLevel (src/HMatrix.cuh:9-18).
 * Any pointer may be NULL.  lowrank: *num_lowrank rows of 6 ints
 * [r0, m, c0, n, k, level] (tree-order row / column ranges); dense:
 * *num_dense rows of 5 ints [r0, m, c0, n, transposed]. */
HM_API hm_status hm_hmatrix_blocks(hm_hmatrix h, long long* num_lowrank, long long* num_dense,
                                   int* lowrank, int* dense);

/* Host copy of low-rank block i's factors as FP32: U (m x k), V (n x k),
 * column-major, A_block ~ U V^T. */
HM_API hm_status hm_hmatrix_block_factors(hm_hmatrix h, int i, float* U, float* V);

/* Host copy of stored dense block i (m x n, column-major, FP32; the order of
 * hm_hmatrix_blocks' dense rows).  Diagonal blocks recomputed from the
 * coordinates (diag_from_coords) are not stored and not listed. */
HM_API hm_status hm_hmatrix_dense_block(hm_hmatrix h, int i, float* D);

HM_API void hm_hmatrix_free(hm_hmatrix h);

/* Binary H-matrix files: build once, apply many times.  No counterpart in the
 * reference, which only dumps text (src/helperFunctions.cu:76-169).
 *
 * hm_hmatrix_save writes the options, every stored low-rank pair (FP32
 * factors, rank, low-part columns) and dense block, and a fingerprint of the
 * tree and structure (permutation, leaf offsets, admissibility, block lists);
 * it synchronises the device.  hm_hmatrix_load reads such a file into a new
 * H-matrix on `t` and `s`, which must be the tree and structure it was built
 * on (rebuild them from the same points, bucket and admissibility; a
 * different one is refused with HM_ERR_INVALID), and rebuilds the product's
 * plans (and the mixed form's BF16 panels) exactly as the build does: its
 * products equal the saved matrix's.  A file from another version of the
 * library, or a damaged one, is refused with HM_ERR_INVALID. */
HM_API hm_status hm_hmatrix_save(hm_hmatrix h, const char* path);
HM_API hm_status hm_hmatrix_load(hm_kdtree t, hm_structure s, const char* path, void* stream, hm_hmatrix* out);

/* Waits for the stream, then returns HM_ERR_TIMEOUT if a bounded device-side
 * wait in one of this matrix's product kernels gave up since the last check
 * (the products concerned hold wrong values; the report is cleared), else
 * HM_OK.  Only the tcgen05 phase 1 of the mixed form's 128-column passes
 * waits on the device; the wait ends the kernel instead of hanging it. */
HM_API hm_status hm_hmatrix_check(hm_hmatrix h, void* stream);

/* Schedule autotuner (no counterpart in the reference).  Times the product's
 * schedule candidates on this matrix (nrhs columns, at most one pass of the
 * product: 128 for the mixed form, 16 for the FP32 form) and keeps the
 * fastest: for the mixed form the phase-1 unit shape and kernel, for the
 * FP32 form its two products -- FP32 tiles on the factor panels with a
 * phase-1 unit shape, or the per-block kernels with the rows of V per
 * phase-1 item.  With cache_path set, the choice is appended
 * to that text file under a key of the GPU and the matrix's shape, and a
 * later call whose key is in the file applies the cached choice without
 * timing (*from_cache = 1).  choice receives a description (may be NULL).
 * Products recorded into graphs before the call must be recorded again
 * (hm_batch_matvec does that by itself). */
HM_API hm_status hm_autotune(hm_hmatrix h, int nrhs, const char* cache_path, void* stream, int* from_cache,
                             char* choice, int choice_len);

/* Applies a schedule given as hm_autotune describes it, e.g.
 * "mixed chunk_tiles=64 group_tiles=8 p1_ring=1 wide_tc=1 tc_chunk=32",
 * "fp32 chunk_tiles=32 group_tiles=4" (FP32 panels) or "fp32 p1_rows=256"
 * (FP32 per-block kernels; they read the FP32 factors, which FP32 matrices
 * keep).  For the mixed form, wide_tc and tc_chunk are optional: wide_tc = 1
 * (the default) runs passes of 65-128 right-hand sides on tcgen05 kernels
 * (tensor memory accumulators), whose phase-1 units span tc_chunk row tiles
 * (default 32); wide_tc = 0 runs them on the warp-level MMA kernels. */
HM_API hm_status hm_schedule_set(hm_hmatrix h, const char* choice, void* stream);

/* --- Batches of independent clouds ------------------------------------------
 * No counterpart in the reference (one cloud per run, src/main.cu:33-200).
 * A batch joins C clouds (each with its own KD tree and block structure) as
 * the subtrees of one forest, so that one build compresses the blocks of all
 * clouds in the same batched launches and one product covers all clouds.
 * Rows are the clouds' tree-order rows concatenated: cloud c owns rows
 * [row_offsets[c], row_offsets[c+1]).  The trees and structures must outlive
 * the batch; all clouds share the dimension and the admissibility rule, and
 * the forest may be at most 16 levels deep (ceil(log2 C) + the deepest tree). */
HM_API hm_status hm_batch_create(int nclouds, const hm_kdtree* trees, const hm_structure* structures, void* stream,
                                 hm_batch* out);

/* row_offsets: nclouds + 1 ints; any pointer may be NULL. */
HM_API hm_status hm_batch_info(hm_batch b, int* nclouds, int* n_total, int* depth, int* row_offsets);

/* Builds (or rebuilds) the batch's H-matrix with the given options. */
HM_API hm_status hm_batch_build(hm_batch b, const hm_build_opts* opts, void* stream);

/* The batch's H-matrix (owned by the batch): stats, blocks, hm_hmatvec. */
HM_API hm_hmatrix hm_batch_hmatrix(hm_batch b);

/* Y = H X over all clouds (X, Y: n_total x nrhs, column-major; tree order,
 * or each cloud's original order when original_order != 0).  The first call
 * for a given (X, Y, nrhs, ldx, ldy, original_order, stream) records the
 * product's kernels into a CUDA graph; every call launches that graph, one
 * launch for the whole batch.  `stream` must be a created stream (the legacy
 * default stream cannot be recorded). */
HM_API hm_status hm_batch_matvec(hm_batch b, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                 int original_order, void* stream);

HM_API void hm_batch_free(hm_batch b);

#ifdef __cplusplus
}
#endif
#endif /* HM_H */
