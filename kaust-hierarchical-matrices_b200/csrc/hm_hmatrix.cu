// hm_hmatrix.cu -- H-matrix construction by batched adaptive randomized
// approximation (ARA) on kernel entries generated from the points.
//
// Reference: createColumnMajorLRMatrix (src/constructTLRMatrix.cu:13-151)
// compresses leaf tiles with kblas_ara_batch and generateHMatrixFromStruct
// (src/constructHMatrixFromStruct.cu:13-103) recompresses coarser blocks from
// the leaf factors with lr_kblas_ara_batch, both from the un-vendored KBLAS
// fork.  The ARA they call is the blocked adaptive range finder of Halko,
// Martinsson & Tropp (2011, Alg. 4.2) as batched by Boukaram, Turkiyyah &
// Keyes (2019): draw a Gaussian sample block, project out the basis found so
// far, stop when the sample's norm says the residual is below the tolerance,
// otherwise orthonormalise it and append it; finally B = A^T Q, A ~ Q B^T.
//
// B200 design.  Every block of every level is compressed directly from the
// kernel function (no dense tiles in HBM, no leaf-TLR stage): each ARA pass is
// one batched "kernel block x tall-skinny" launch (k_kmm) whose tiles are
// generated on the fly from the tree-ordered FP32 coordinates, so the O(N^2)
// part never touches memory.  Orthogonalisation runs per block in one CTA
// (k_orth): block classical Gram-Schmidt applied twice against the basis, then
// a pivoted Cholesky-QR of the sample with two Cholesky-QR refinements, Gram
// matrices in FP64.  The kernel matrix is symmetric, so of each block pair
// (u, v) / (v, u) only the one with v > u is compressed; the mirror block uses
// the same factors exchanged.  Leaf blocks that do not reach the tolerance
// within the leaf rank cap (bucket/2 as in src/constructTLRMatrix.cu:14) are
// stored dense, as are the diagonal leaves.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>

#include "hm_hmatrix.h"
#include "hm_structure.h"

namespace hm {

hm_status matvec_plan_build(hm_hmatrix h, int nrhs_cap, cudaStream_t stream);

namespace {

constexpr int kTR = 64;        // rows of a KMM tile
constexpr int kTC = 64;        // columns per KMM chunk
constexpr int kKmmThreads = 256;
constexpr int kOrthThreads = 256;
constexpr int kMaxCols = 128;  // max basis columns of one block (rank cap + sample block)
constexpr int kMaxBs = 32;     // max sample block

struct Prob {
  int r0, m, c0, n;
  int kmax;
  int level;
  int u, v;
  long long qoff, yoff, boff;  // workspace offsets (floats)
};

struct ProbState {
  double normA2;
  double est;
  int k;
  int active;
  int converged;
  int rounds;
};

template <typename W>
struct KmmArgs {
  const Prob* probs;
  ProbState* st;
  const int2* items;  // (problem, tile)
  const float* pts;   // tree-ordered FP32 coordinates [d][npts]
  int npts, d;
  KernelParams kp;
  int mode;           // 0: Y = A Omega (bs columns); 1: B = A^T Q (k columns)
  int bs;
  uint32_t seed;
  int round;
  W* ws;              // workspace (Y, Q, B) in the ARA's working precision
};

// ---------------------------------------------------------------------------
// k_kmm: out(rows x s) = K(rows, cols) W(cols x s) for one 64-row tile.
// Thread t: row r = t % 64, q = t / 64 splits the s output columns into
// `nslab` slabs of 32 and the chunk columns into 4/nslab groups.  Kernel
// entries are FP32; products and sums are in the workspace type W (an FP32 x
// FP32 product is exact in FP64, so W = double gives FP64-accurate samples).
// ---------------------------------------------------------------------------
template <typename W>
__global__ void __launch_bounds__(kKmmThreads) k_kmm(KmmArgs<W> a) {
  extern __shared__ __align__(16) unsigned char kmm_raw[];
  W* Wsm = reinterpret_cast<W*>(kmm_raw);          // [kTC][kMaxCols]
  float* Asm = reinterpret_cast<float*>(Wsm + kTC * kMaxCols);  // [kTC][kTR]
  float* colc = Asm + kTC * kTR;                   // [d][kTC]
  double* red = reinterpret_cast<double*>(colc + kMaxDim * kTC);  // [kKmmThreads/32]

  const int2 it = a.items[blockIdx.x];
  const Prob P = a.probs[it.x];
  const ProbState S = a.st[it.x];
  if (a.mode == 0 && !S.active) return;
  const int s = a.mode == 0 ? a.bs : S.k;
  if (s <= 0) return;
  const int mr = a.mode ? P.n : P.m;        // rows of the operator
  const int nc = a.mode ? P.m : P.n;        // columns of the operator
  const int rbase = a.mode ? P.c0 : P.r0;
  const int cbase = a.mode ? P.r0 : P.c0;
  W* out = a.ws + (a.mode ? P.boff : P.yoff);
  const W* Q = a.ws + P.qoff;               // mode 1: W = Q (m x k, ld m)
  const int nslab = s <= 32 ? 1 : (s <= 64 ? 2 : 4);
  const int ncg = 4 / nslab;
  const int t = threadIdx.x, r = t & 63, q = t >> 6;
  const int slab = q % nslab, cg = q / nslab;
  const int row = it.y * kTR + r;
  const bool row_ok = row < mr;
  float rc[kMaxDim];
#pragma unroll
  for (int k = 0; k < kMaxDim; ++k)
    rc[k] = (k < a.d && row_ok) ? a.pts[(size_t)k * a.npts + rbase + row] : 0.f;
  W acc[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) acc[c] = W(0);
  double nrm = 0.0;
  const bool want_norm = a.mode == 0 && a.round == 0;
  const int wcols = nslab * 32;

  for (int c0 = 0; c0 < nc; c0 += kTC) {
    // column coordinates and the W chunk
    if (t < kTC) {
      int j = c0 + t;
      for (int k = 0; k < a.d; ++k) colc[k * kTC + t] = j < nc ? a.pts[(size_t)k * a.npts + cbase + j] : 0.f;
    }
    for (int e = t; e < kTC * wcols; e += kKmmThreads) {
      int jj = e % kTC, cc = e / kTC;
      int j = c0 + jj;
      W w = W(0);
      if (j < nc && cc < s) {
        if (a.mode == 0)
          w = (W)gauss_at(a.seed, (uint32_t)it.x, (uint32_t)j, (uint32_t)(a.round * kMaxBs + cc));
        else
          w = Q[(size_t)cc * P.m + j];
      }
      Wsm[jj * kMaxCols + cc] = w;
    }
    __syncthreads();
    // kernel entries of this thread's row, columns q, q+4, ...
    for (int jj = q; jj < kTC; jj += 4) {
      float v = 0.f;
      if (row_ok && c0 + jj < nc) {
        float r2 = 0.f;
        for (int k = 0; k < a.d; ++k) {
          float df = rc[k] - colc[k * kTC + jj];
          r2 = fmaf(df, df, r2);
        }
        v = kernel_r2(a.kp, r2);
        if (want_norm) nrm += (double)v * (double)v;
      }
      Asm[jj * kTR + r] = v;
    }
    __syncthreads();
    for (int jj = cg; jj < kTC; jj += ncg) {
      W av = (W)Asm[jj * kTR + r];
      const W* w = Wsm + jj * kMaxCols + slab * 32;
#pragma unroll
      for (int c = 0; c < 32; ++c) acc[c] = fma(av, w[c], acc[c]);
    }
    __syncthreads();
  }
  // reduce over column groups through shared memory (reuses Asm/Wsm)
  if (ncg > 1) {
    W* part = Wsm;  // [4][32][64] (reuses the W chunk)
    for (int c = 0; c < 32; ++c) part[(q * 32 + c) * kTR + r] = acc[c];
    __syncthreads();
    if (cg == 0) {
      for (int g = 1; g < ncg; ++g) {
        int qq = g * nslab + slab;
        for (int c = 0; c < 32; ++c) acc[c] += part[(qq * 32 + c) * kTR + r];
      }
    }
  }
  if (cg == 0 && row_ok) {
    const int ld = mr;
    for (int c = 0; c < 32; ++c) {
      int col = slab * 32 + c;
      if (col < s) out[(size_t)col * ld + row] = acc[c];
    }
  }
  if (want_norm) {
    for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    __syncthreads();
    if ((t & 31) == 0) red[t >> 5] = nrm;
    __syncthreads();
    if (t == 0) {
      double tot = 0;
      for (int w = 0; w < kKmmThreads / 32; ++w) tot += red[w];
      atomicAdd(&a.st[it.x].normA2, tot);
    }
  }
}

// ---------------------------------------------------------------------------
// per-block orthogonalisation of the new sample
// ---------------------------------------------------------------------------
template <typename W>
struct OrthArgs {
  const Prob* probs;
  ProbState* st;
  W* ws;
  int bs;
  double thresh2;  // stop when est <= thresh2 * normA2
  int round;
};

// C[j][c] = sum_i Q[i, j] Y[i, c]  (k x bs), result in shared Csm
template <typename W>
__device__ void block_qty(const W* Q, const W* Y, int m, int k, int bs, W* Csm, W* stage) {
  const int t = threadIdx.x;
  W accv[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) accv[i] = W(0);
  W* Qs = stage;                  // [kMaxCols][33]
  W* Ys = stage + kMaxCols * 33;  // [kMaxBs][33]
  const int nout = k * bs;
  for (int i0 = 0; i0 < m; i0 += 32) {
    for (int e = t; e < 32 * k; e += kOrthThreads) {
      int ii = e & 31, j = e >> 5;
      Qs[j * 33 + ii] = (i0 + ii < m) ? Q[(size_t)j * m + i0 + ii] : W(0);
    }
    for (int e = t; e < 32 * bs; e += kOrthThreads) {
      int ii = e & 31, c = e >> 5;
      Ys[c * 33 + ii] = (i0 + ii < m) ? Y[(size_t)c * m + i0 + ii] : W(0);
    }
    __syncthreads();
#pragma unroll
    for (int x = 0; x < 16; ++x) {
      int o = t + x * kOrthThreads;
      if (o < nout) {
        int j = o / bs, c = o % bs;
        W sacc = accv[x];
        for (int ii = 0; ii < 32; ++ii) sacc = fma(Qs[j * 33 + ii], Ys[c * 33 + ii], sacc);
        accv[x] = sacc;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 16; ++x) {
    int o = t + x * kOrthThreads;
    if (o < nout) Csm[o] = accv[x];  // Csm[j*bs + c]
  }
  __syncthreads();
}

// Y -= Q C
template <typename W>
__device__ void block_update(const W* Q, W* Y, int m, int k, int bs, const W* Csm) {
  for (int i = threadIdx.x; i < m; i += kOrthThreads) {
    W y[kMaxBs];
    for (int c = 0; c < bs; ++c) y[c] = Y[(size_t)c * m + i];
    for (int j = 0; j < k; ++j) {
      W qv = Q[(size_t)j * m + i];
      for (int c = 0; c < bs; ++c) y[c] = fma(-qv, Csm[j * bs + c], y[c]);
    }
    for (int c = 0; c < bs; ++c) Y[(size_t)c * m + i] = y[c];
  }
  __syncthreads();
}

// G = Y^T Y in FP64 (cols x cols), into shared Gs
template <typename W>
__device__ void gram64(const W* Y, int m, int cols, double* Gs, W* stage) {
  const int t = threadIdx.x;
  double accv[4] = {0, 0, 0, 0};
  W* Ys = stage;  // [kMaxBs][33]
  const int nout = cols * cols;
  for (int i0 = 0; i0 < m; i0 += 32) {
    for (int e = t; e < 32 * cols; e += kOrthThreads) {
      int ii = e & 31, c = e >> 5;
      Ys[c * 33 + ii] = (i0 + ii < m) ? Y[(size_t)c * m + i0 + ii] : W(0);
    }
    __syncthreads();
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      int o = t + x * kOrthThreads;
      if (o < nout) {
        int a = o / cols, b = o % cols;
        double sacc = accv[x];
        for (int ii = 0; ii < 32; ++ii) sacc += (double)Ys[a * 33 + ii] * (double)Ys[b * 33 + ii];
        accv[x] = sacc;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 4; ++x) {
    int o = t + x * kOrthThreads;
    if (o < nout) Gs[o] = accv[x];
  }
  __syncthreads();
}

// Cholesky of the leading principal part of G (cols x cols, row-major), in
// place into its lower triangle, with symmetric pivoting when `pivot`; stops at
// the first pivot <= tau.  perm receives the column order.  Returns the rank.
// Runs on thread 0 (cols <= 32).
__device__ int chol_pivoted(double* G, int cols, int* perm, bool pivot, double tau) {
  for (int i = 0; i < cols; ++i) perm[i] = i;
  int rank = 0;
  for (int j = 0; j < cols; ++j) {
    int p = j;
    if (pivot) {
      for (int i = j + 1; i < cols; ++i)
        if (G[i * cols + i] > G[p * cols + p]) p = i;
    }
    if (!(G[p * cols + p] > tau)) break;
    if (p != j) {
      // symmetric swap of rows/cols j and p
      for (int c = 0; c < cols; ++c) {
        double x = G[j * cols + c];
        G[j * cols + c] = G[p * cols + c];
        G[p * cols + c] = x;
      }
      for (int r = 0; r < cols; ++r) {
        double x = G[r * cols + j];
        G[r * cols + j] = G[r * cols + p];
        G[r * cols + p] = x;
      }
      int x = perm[j];
      perm[j] = perm[p];
      perm[p] = x;
    }
    double d = sqrt(G[j * cols + j]);
    G[j * cols + j] = d;
    for (int i = j + 1; i < cols; ++i) G[i * cols + j] /= d;
    for (int i = j + 1; i < cols; ++i)
      for (int c = j + 1; c <= i; ++c) {
        G[i * cols + c] -= G[i * cols + j] * G[c * cols + j];
        G[c * cols + i] = G[i * cols + c];
      }
    rank = j + 1;
  }
  return rank;
}

// Y[:, 0:r] <- Y[:, perm[0:r]] L^{-T}  (row by row, in place)
template <typename W>
__device__ void apply_linv(W* Y, int m, int cols, const double* L, const int* perm, int r) {
  for (int i = threadIdx.x; i < m; i += kOrthThreads) {
    W y[kMaxBs];
    for (int c = 0; c < cols; ++c) y[c] = Y[(size_t)c * m + i];
    double x[kMaxBs];
    for (int a = 0; a < r; ++a) {
      double v = y[perm[a]];
      for (int b = 0; b < a; ++b) v -= L[a * cols + b] * x[b];
      x[a] = v / L[a * cols + a];
    }
    for (int a = 0; a < r; ++a) Y[(size_t)a * m + i] = (W)x[a];
  }
  __syncthreads();
}

template <typename W>
__global__ void __launch_bounds__(kOrthThreads) k_orth(OrthArgs<W> a) {
  extern __shared__ __align__(16) unsigned char osm[];
  double* Gs = reinterpret_cast<double*>(osm);              // [kMaxBs*kMaxBs]
  W* Csm = reinterpret_cast<W*>(Gs + kMaxBs * kMaxBs);      // [kMaxCols*kMaxBs]
  W* stage = Csm + kMaxCols * kMaxBs;                       // (kMaxCols+kMaxBs)*33
  __shared__ int perm[kMaxBs];
  __shared__ int rank_sh;
  __shared__ int decision;  // 0 continue, 1 converged, 2 cap reached

  const int p = blockIdx.x;
  ProbState S = a.st[p];
  if (!S.active) return;
  const Prob P = a.probs[p];
  const int m = P.m, bs = a.bs;
  W* Q = a.ws + P.qoff;
  W* Y = a.ws + P.yoff;
  int k = S.k;
  for (int pass = 0; pass < 2 && k > 0; ++pass) {
    block_qty(Q, Y, m, k, bs, Csm, stage);
    block_update(Q, Y, m, k, bs, Csm);
  }
  gram64(Y, m, bs, Gs, stage);
  if (threadIdx.x == 0) {
    double tr = 0;
    for (int c = 0; c < bs; ++c) tr += Gs[c * bs + c];
    double est = tr / bs;
    S.est = est;
    S.rounds += 1;
    if (est <= a.thresh2 * S.normA2 || S.normA2 == 0.0) decision = 1;
    else if (k + bs > P.kmax) decision = 2;
    else decision = 0;
    if (decision == 0) {
      // columns whose norm is below FP32 resolution of the sample are noise
      double tau = 1e-10 * tr;
      rank_sh = chol_pivoted(Gs, bs, perm, true, tau);
    }
  }
  __syncthreads();
  if (decision != 0) {
    if (threadIdx.x == 0) {
      S.active = 0;
      S.converged = decision == 1;
      a.st[p] = S;
    }
    return;
  }
  int r = rank_sh;
  if (r == 0) {
    if (threadIdx.x == 0) {
      S.active = 0;
      S.converged = 1;
      a.st[p] = S;
    }
    return;
  }
  apply_linv(Y, m, bs, Gs, perm, r);
  // Refinements.  R^{-1} of an ill-conditioned sample magnifies whatever the
  // Gram-Schmidt left along the old basis, so after the first refinement the
  // block is projected against Q once more before the final Cholesky-QR.
  for (int pass = 0; pass < 2 && r > 0; ++pass) {
    if (pass == 1 && k > 0) {
      block_qty(Q, Y, m, k, r, Csm, stage);
      block_update(Q, Y, m, k, r, Csm);
    }
    const int rg = r;  // dimension (and row stride) of this Gram matrix
    gram64(Y, m, rg, Gs, stage);
    if (threadIdx.x == 0) rank_sh = chol_pivoted(Gs, rg, perm, pass == 1, pass == 1 ? 1e-12 * rg : 0.0);
    __syncthreads();
    r = rank_sh;  // a refinement that loses rank keeps the leading columns
    if (r > 0) apply_linv(Y, m, rg, Gs, perm, r);
  }
  // append to Q
  for (int c = 0; c < r; ++c)
    for (int i = threadIdx.x; i < m; i += kOrthThreads) Q[(size_t)(k + c) * m + i] = Y[(size_t)c * m + i];
  __syncthreads();
  if (threadIdx.x == 0) {
    S.k = k + r;
    if (r == 0) {
      S.active = 0;
      S.converged = 1;
    }
    a.st[p] = S;
  }
}

// ---------------------------------------------------------------------------
// packing and dense blocks
// ---------------------------------------------------------------------------
struct PackItem {
  long long src_q, src_b;  // workspace offsets
  long long dst_u, dst_v;  // offsets in the chunk
  int m, n, k;
};

template <typename W>
__global__ void k_pack(const PackItem* items, int nitems, const W* ws, float* dst) {
  const PackItem it = items[blockIdx.x];
  size_t nu = (size_t)it.m * it.k, nv = (size_t)it.n * it.k;
  for (size_t e = threadIdx.x; e < nu; e += blockDim.x) dst[it.dst_u + e] = (float)ws[it.src_q + e];
  for (size_t e = threadIdx.x; e < nv; e += blockDim.x) dst[it.dst_v + e] = (float)ws[it.src_b + e];
}

struct DenseItem {
  int r0, m, c0, n;
  long long off;
};

__global__ void k_dense_gen(const DenseItem* items, const float* pts, int npts, int d,
                            KernelParams kp, float* dst) {
  const DenseItem it = items[blockIdx.x];
  size_t tot = (size_t)it.m * it.n;
  for (size_t e = threadIdx.x; e < tot; e += blockDim.x) {
    int i = (int)(e % it.m), j = (int)(e / it.m);
    int gi = it.r0 + i, gj = it.c0 + j;
    float r2 = 0.f;
    for (int k = 0; k < d; ++k) {
      float df = pts[(size_t)k * npts + gi] - pts[(size_t)k * npts + gj];
      r2 = fmaf(df, df, r2);
    }
    float v = kernel_r2(kp, r2);
    if (gi == gj && !kp.deriv) v += kp.nugget;
    dst[it.off + e] = v;
  }
}

template <typename W>
size_t kmm_smem() {
  return sizeof(W) * (kTC * kMaxCols) + sizeof(float) * (kTC * kTR + kMaxDim * kTC) +
         sizeof(double) * (kKmmThreads / 32);
}

template <typename W>
size_t orth_smem() {
  return sizeof(double) * kMaxBs * kMaxBs + sizeof(W) * kMaxCols * kMaxBs + sizeof(W) * (kMaxCols + kMaxBs) * 33;
}

}  // namespace

hm_status hmatrix_build(hm_kdtree t, hm_structure s, const double* d_points, const hm_build_opts* o,
                        cudaStream_t stream, hm_hmatrix* out) {
  if (!out) return fail(HM_ERR_INVALID, "hm_hmatrix_build: out is NULL");
  *out = nullptr;
  if (!t || !s || !o) return fail(HM_ERR_INVALID, "hm_hmatrix_build: null argument");
  if (s->tree != t) return fail(HM_ERR_INVALID, "hm_hmatrix_build: structure was built on another tree");
  (void)d_points;  // the tree keeps its own tree-ordered copy of the points
  hm_build_opts opt = *o;
  if (opt.kernel < 0 || opt.kernel > 2) return fail(HM_ERR_INVALID, "hm_hmatrix_build: unknown kernel");
  if (!(opt.ell > 0) || !(opt.tol > 0) || opt.tol >= 1)
    return fail(HM_ERR_INVALID, "hm_hmatrix_build: need ell > 0 and 0 < tol < 1");
  if (opt.sample_block <= 0) opt.sample_block = 16;
  if (opt.sample_block > kMaxBs) return fail(HM_ERR_UNSUPPORTED, "hm_hmatrix_build: sample_block > 32");
  if (opt.leaf_max_rank <= 0) opt.leaf_max_rank = std::max(1, t->bucket / 2);
  if (opt.max_rank <= 0) opt.max_rank = 64;
  const int bs = opt.sample_block;
  if (opt.max_rank > kMaxCols || opt.leaf_max_rank > kMaxCols)
    return fail(HM_ERR_UNSUPPORTED, "hm_hmatrix_build: rank caps must be <= 128");

  cudaEvent_t ev0, ev1;
  HM_CUDA(cudaEventCreate(&ev0));
  HM_CUDA(cudaEventCreate(&ev1));
  HM_CUDA(cudaEventRecord(ev0, stream));

  auto* h = new hm_hmatrix_s();
  auto cleanup = [&](hm_status st) {
    delete h;
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    return st;
  };
  h->tree = t;
  h->structure = s;
  h->n = t->n;
  h->d = t->d;
  h->depth = t->depth;
  h->opts = opt;
  h->kp.kind = opt.kernel;
  h->kp.deriv = opt.derivative ? 1 : 0;
  h->kp.ell = (float)opt.ell;
  h->kp.inv_ell = (float)(1.0 / opt.ell);
  h->kp.nugget = (float)opt.nugget;
  const int depth = t->depth;
  const std::vector<int>& lo = t->h_offsets;
  auto coff = [&](int level, int c) { return lo[(size_t)c << (depth - level)]; };

  // ---- the problems: stored pairs (row cluster v > column cluster u) ------
  std::vector<uint32_t> tiles(std::max<long long>(s->start[depth], 1));
  if (s->start[depth] > 0)
    HM_CUDA(cudaMemcpy(tiles.data(), s->tiles.p, 4 * (size_t)s->start[depth], cudaMemcpyDeviceToHost));
  std::vector<Prob> probs;
  for (int l = 1; l <= depth; ++l) {
    for (long long i = s->start[l - 1]; i < s->start[l]; ++i) {
      uint32_t z = tiles[i];
      int u = (int)compact16(z), v = (int)compact16(z >> 1);
      if (v <= u) continue;
      Prob P{};
      P.level = l;
      P.u = u;
      P.v = v;
      P.r0 = coff(l, v);
      P.m = coff(l, v + 1) - P.r0;
      P.c0 = coff(l, u);
      P.n = coff(l, u + 1) - P.c0;
      P.kmax = std::min(l == depth ? opt.leaf_max_rank : opt.max_rank, std::min(P.m, P.n));
      probs.push_back(P);
    }
  }
  const long long nprob = (long long)probs.size();

  // ---- batches bounded by the workspace budget -----------------------------
  size_t freeb = 0, totb = 0;
  HM_CUDA(cudaMemGetInfo(&freeb, &totb));
  const size_t budget_bytes = std::min<size_t>(freeb / 4, (size_t)24 << 30);
  std::vector<int> rank(nprob, 0), conv(nprob, 0);
  std::vector<double> nrm(nprob, 0.0);
  long long pstart = 0;
  const double thresh2 = 0.09 * opt.tol * opt.tol;  // (0.3 tol)^2
  long long lr_count = 0, dense_count = 0, rank_sum = 0;
  int max_rank_seen = 0;
  long long factor_bytes = 0, dense_bytes = 0, unconverged = 0;

  // per-problem results that survive the batch: the factor location
  std::vector<const float*> fu(nprob, nullptr), fv(nprob, nullptr);
  std::vector<const float*> fd(nprob, nullptr);

  // Sketches, bases and projections run in FP64 when the tolerance is below
  // what FP32 sums over a block can resolve (~u*sqrt(m) relative), else FP32.
  const bool fp64 = opt.tol < 5e-6;
  auto batch_loop = [&](auto tag) -> hm_status {
    using W = decltype(tag);
    const size_t budget_elems = budget_bytes / sizeof(W);
    HM_CUDA(cudaFuncSetAttribute(k_kmm<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kmm_smem<W>()));
    HM_CUDA(cudaFuncSetAttribute(k_orth<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)orth_smem<W>()));
    while (pstart < nprob) {
      // greedy batch
      long long pend = pstart;
      size_t wsz = 0;
      while (pend < nprob) {
        const Prob& P = probs[pend];
        size_t need = (size_t)P.m * (P.kmax + bs) + (size_t)P.m * bs + (size_t)P.n * (P.kmax + bs);
        if (pend > pstart && wsz + need > budget_elems) break;
        wsz += need;
        ++pend;
      }
      const int nb = (int)(pend - pstart);
      std::vector<Prob> bp(probs.begin() + pstart, probs.begin() + pend);
      size_t off = 0;
      std::vector<int2> items_rows, items_cols;
      for (int i = 0; i < nb; ++i) {
        Prob& P = bp[i];
        P.qoff = (long long)off;
        off += (size_t)P.m * (P.kmax + bs);
        P.yoff = (long long)off;
        off += (size_t)P.m * bs;
        P.boff = (long long)off;
        off += (size_t)P.n * (P.kmax + bs);
        for (int tt = 0; tt * kTR < P.m; ++tt) items_rows.push_back(make_int2(i, tt));
        for (int tt = 0; tt * kTR < P.n; ++tt) items_cols.push_back(make_int2(i, tt));
      }
      DevBuf<W> ws;
      DevBuf<Prob> dprobs;
      DevBuf<ProbState> dst;
      DevBuf<int2> drows, dcols;
      hm_status st;
      if ((st = ws.alloc(std::max<size_t>(off, 1))) || (st = dprobs.alloc(nb)) || (st = dst.alloc(nb)) ||
          (st = drows.alloc(items_rows.size())) || (st = dcols.alloc(items_cols.size())))
        return st;
      std::vector<ProbState> hst(nb);
      for (auto& x : hst) {
        x = ProbState{};
        x.active = 1;
      }
      HM_CUDA(cudaMemcpyAsync(dprobs.p, bp.data(), sizeof(Prob) * nb, cudaMemcpyHostToDevice, stream));
      HM_CUDA(cudaMemcpyAsync(dst.p, hst.data(), sizeof(ProbState) * nb, cudaMemcpyHostToDevice, stream));
      HM_CUDA(cudaMemcpyAsync(drows.p, items_rows.data(), sizeof(int2) * items_rows.size(),
                              cudaMemcpyHostToDevice, stream));
      HM_CUDA(cudaMemcpyAsync(dcols.p, items_cols.data(), sizeof(int2) * items_cols.size(),
                              cudaMemcpyHostToDevice, stream));

      KmmArgs<W> ka;
      ka.probs = dprobs.p;
      ka.st = dst.p;
      ka.pts = t->pts_tree_f.p;
      ka.npts = t->n;
      ka.d = t->d;
      ka.kp = h->kp;
      ka.bs = bs;
      ka.seed = (uint32_t)(opt.seed ^ (opt.seed >> 32)) ^ 0x5bd1e995u;
      ka.ws = ws.p;
      OrthArgs<W> oa;
      oa.probs = dprobs.p;
      oa.st = dst.p;
      oa.ws = ws.p;
      oa.bs = bs;
      oa.thresh2 = thresh2;
      const int max_rounds = kMaxCols / bs + 2;
      for (int round = 0; round < max_rounds; ++round) {
        ka.mode = 0;
        ka.round = round;
        ka.items = drows.p;
        k_kmm<W><<<(unsigned)items_rows.size(), kKmmThreads, kmm_smem<W>(), stream>>>(ka);
        HM_LAUNCH_CHECK();
        oa.round = round;
        k_orth<W><<<nb, kOrthThreads, orth_smem<W>(), stream>>>(oa);
        HM_LAUNCH_CHECK();
        HM_CUDA(cudaMemcpyAsync(hst.data(), dst.p, sizeof(ProbState) * nb, cudaMemcpyDeviceToHost, stream));
        HM_CUDA(cudaStreamSynchronize(stream));
        bool any = false;
        for (auto& x : hst) any |= x.active != 0;
        if (!any) break;
      }
      // B = A^T Q
      ka.mode = 1;
      ka.items = dcols.p;
      k_kmm<W><<<(unsigned)items_cols.size(), kKmmThreads, kmm_smem<W>(), stream>>>(ka);
      HM_LAUNCH_CHECK();

      // ---- results: low rank where converged, dense otherwise ---------------
      std::vector<PackItem> packs;
      std::vector<DenseItem> dens;
      size_t chunk_floats = 0;
      for (int i = 0; i < nb; ++i) {
        const Prob& P = bp[i];
        const ProbState& S = hst[i];
        long long gi = pstart + i;
        nrm[gi] = S.normA2;
        // a block that missed the tolerance at its rank cap is stored dense when
        // that is affordable (leaf blocks always are); a large one keeps its
        // capped factors and is counted as unconverged
        const bool small = (size_t)P.m * P.n <= 2 * (size_t)(P.m + P.n) * (size_t)std::max(S.k, 1);
        if (!(S.converged || S.active) && !(P.level == depth || small)) ++unconverged;
        if (S.converged || S.active || !(P.level == depth || small)) {
          PackItem pi;
          pi.src_q = P.qoff;
          pi.src_b = P.boff;
          pi.m = P.m;
          pi.n = P.n;
          pi.k = S.k;
          pi.dst_u = (long long)chunk_floats;
          chunk_floats += (size_t)P.m * S.k;
          pi.dst_v = (long long)chunk_floats;
          chunk_floats += (size_t)P.n * S.k;
          packs.push_back(pi);
          rank[gi] = S.k;
          conv[gi] = 1;
        } else {
          DenseItem di;
          di.r0 = P.r0;
          di.m = P.m;
          di.c0 = P.c0;
          di.n = P.n;
          di.off = (long long)chunk_floats;
          chunk_floats += (size_t)P.m * P.n;
          dens.push_back(di);
          rank[gi] = -1;
        }
      }
      DevBuf<float> chunk;
      if ((st = chunk.alloc(std::max<size_t>(chunk_floats, 1)))) return st;
      DevBuf<PackItem> dpk;
      DevBuf<DenseItem> ddi;
      if (!packs.empty()) {
        if ((st = dpk.alloc(packs.size()))) return st;
        HM_CUDA(cudaMemcpyAsync(dpk.p, packs.data(), sizeof(PackItem) * packs.size(), cudaMemcpyHostToDevice,
                                stream));
        k_pack<W><<<(unsigned)packs.size(), 256, 0, stream>>>(dpk.p, (int)packs.size(), ws.p, chunk.p);
        HM_LAUNCH_CHECK();
      }
      if (!dens.empty()) {
        if ((st = ddi.alloc(dens.size()))) return st;
        HM_CUDA(cudaMemcpyAsync(ddi.p, dens.data(), sizeof(DenseItem) * dens.size(), cudaMemcpyHostToDevice,
                                stream));
        k_dense_gen<<<(unsigned)dens.size(), 256, 0, stream>>>(ddi.p, t->pts_tree_f.p, t->n, t->d, h->kp,
                                                               chunk.p);
        HM_LAUNCH_CHECK();
      }
      HM_CUDA(cudaStreamSynchronize(stream));
      size_t pk = 0, dk = 0;
      for (int i = 0; i < nb; ++i) {
        long long gi = pstart + i;
        if (rank[gi] >= 0) {
          fu[gi] = chunk.p + packs[pk].dst_u;
          fv[gi] = chunk.p + packs[pk].dst_v;
          ++pk;
          lr_count += 2;
          rank_sum += 2 * (long long)rank[gi];
          max_rank_seen = std::max(max_rank_seen, rank[gi]);
          factor_bytes += 4ll * (bp[i].m + bp[i].n) * rank[gi];
        } else {
          fd[gi] = chunk.p + dens[dk].off;
          ++dk;
          dense_count += 2;
          dense_bytes += 4ll * bp[i].m * bp[i].n;
        }
      }
      h->storage.push_back(std::move(chunk));
      pstart = pend;
    }
    return HM_OK;
  };
  {
    hm_status bst = fp64 ? batch_loop(double(0)) : batch_loop(float(0));
    if (bst) return cleanup(bst);
  }

  // ---- diagonal leaves ------------------------------------------------------
  const int nleaf = 1 << depth;
  {
    std::vector<DenseItem> dens(nleaf);
    size_t tot = 0;
    for (int l = 0; l < nleaf; ++l) {
      dens[l].r0 = lo[l];
      dens[l].m = lo[l + 1] - lo[l];
      dens[l].c0 = lo[l];
      dens[l].n = dens[l].m;
      dens[l].off = (long long)tot;
      tot += (size_t)dens[l].m * dens[l].m;
    }
    DevBuf<float> chunk;
    DevBuf<DenseItem> ddi;
    hm_status st;
    if ((st = chunk.alloc(std::max<size_t>(tot, 1))) || (st = ddi.alloc(nleaf))) return cleanup(st);
    HM_CUDA(cudaMemcpyAsync(ddi.p, dens.data(), sizeof(DenseItem) * nleaf, cudaMemcpyHostToDevice, stream));
    k_dense_gen<<<nleaf, 256, 0, stream>>>(ddi.p, t->pts_tree_f.p, t->n, t->d, h->kp, chunk.p);
    HM_LAUNCH_CHECK();
    HM_CUDA(cudaStreamSynchronize(stream));
    for (int l = 0; l < nleaf; ++l) {
      DenseBlock db;
      db.r0 = dens[l].r0;
      db.m = dens[l].m;
      db.c0 = dens[l].c0;
      db.n = dens[l].n;
      db.trans = 0;
      db.D = chunk.p + dens[l].off;
      if (db.m > 0) h->h_dense.push_back(db);
    }
    dense_count += nleaf;
    dense_bytes += 4ll * (long long)tot;
    h->storage.push_back(std::move(chunk));
  }

  // ---- block lists (both orientations) --------------------------------------
  for (long long i = 0; i < nprob; ++i) {
    const Prob& P = probs[i];
    if (rank[i] >= 0) {
      LRBlock b{};
      b.level = P.level;
      b.k = rank[i];
      b.r0 = P.r0;
      b.m = P.m;
      b.c0 = P.c0;
      b.n = P.n;
      b.U = fu[i];
      b.V = fv[i];
      h->h_lr.push_back(b);
      LRBlock bt = b;
      bt.r0 = P.c0;
      bt.m = P.n;
      bt.c0 = P.r0;
      bt.n = P.m;
      bt.U = fv[i];
      bt.V = fu[i];
      h->h_lr.push_back(bt);
    } else {
      DenseBlock db{P.r0, P.m, P.c0, P.n, 0, fd[i]};
      h->h_dense.push_back(db);
      DenseBlock dt{P.c0, P.n, P.r0, P.m, 1, fd[i]};
      h->h_dense.push_back(dt);
    }
  }
  h->stats.num_lowrank = lr_count;
  h->stats.num_dense = dense_count;
  h->stats.rank_sum = rank_sum;
  h->stats.max_rank_seen = max_rank_seen;
  h->stats.factor_bytes = factor_bytes;
  h->stats.dense_bytes = dense_bytes;
  h->stats.num_unconverged = unconverged;
  hm_status st = matvec_plan_build(h, 16, stream);
  if (st) return cleanup(st);
  HM_CUDA(cudaEventRecord(ev1, stream));
  HM_CUDA(cudaEventSynchronize(ev1));
  float ms = 0;
  HM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  h->stats.build_seconds = ms * 1e-3;
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  *out = h;
  return HM_OK;
}

}  // namespace hm

extern "C" {

void hm_build_opts_default(int d, hm_build_opts* o) {
  if (!o) return;
  o->kernel = HM_KERNEL_EXP;
  o->ell = d == 3 ? 0.2 : 0.1;  // src/TLRMatrixHelpers.cu:40-42
  o->nugget = 0.0;
  o->tol = 1e-5;                // src/config.h:127
  o->max_rank = 64;
  o->leaf_max_rank = 0;
  o->sample_block = 16;         // src/constructTLRMatrix.cu:73
  o->precision = HM_PREC_FP32;
  o->derivative = 0;
  o->seed = 0;
}

hm_status hm_hmatrix_build(hm_kdtree t, hm_structure s, const double* d_points, const hm_build_opts* opts,
                           void* stream, hm_hmatrix* out) {
  return hm::hmatrix_build(t, s, d_points, opts, hm::as_stream(stream), out);
}

hm_status hm_hmatrix_stats_get(hm_hmatrix h, hm_hmatrix_stats* st) {
  if (!h || !st) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_stats_get: null argument");
  *st = h->stats;
  return HM_OK;
}

hm_status hm_hmatrix_blocks(hm_hmatrix h, long long* num_lowrank, long long* num_dense, int* lowrank,
                            int* dense) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_blocks: null matrix");
  if (num_lowrank) *num_lowrank = (long long)h->h_lr.size();
  if (num_dense) *num_dense = (long long)h->h_dense.size();
  if (lowrank)
    for (size_t i = 0; i < h->h_lr.size(); ++i) {
      const hm::LRBlock& b = h->h_lr[i];
      int* r = lowrank + 6 * i;
      r[0] = b.r0;
      r[1] = b.m;
      r[2] = b.c0;
      r[3] = b.n;
      r[4] = b.k;
      r[5] = b.level;
    }
  if (dense)
    for (size_t i = 0; i < h->h_dense.size(); ++i) {
      const hm::DenseBlock& b = h->h_dense[i];
      int* r = dense + 5 * i;
      r[0] = b.r0;
      r[1] = b.m;
      r[2] = b.c0;
      r[3] = b.n;
      r[4] = b.trans;
    }
  return HM_OK;
}

hm_status hm_hmatrix_block_factors(hm_hmatrix h, int i, float* U, float* V) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_block_factors: null matrix");
  if (i < 0 || (size_t)i >= h->h_lr.size()) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_block_factors: bad index");
  const hm::LRBlock& b = h->h_lr[i];
  if (U && b.k) HM_CUDA(cudaMemcpy(U, b.U, sizeof(float) * (size_t)b.m * b.k, cudaMemcpyDeviceToHost));
  if (V && b.k) HM_CUDA(cudaMemcpy(V, b.V, sizeof(float) * (size_t)b.n * b.k, cudaMemcpyDeviceToHost));
  return HM_OK;
}

void hm_hmatrix_free(hm_hmatrix h) { delete h; }

}  // extern "C"
