// hm_matvec.cu -- H-matrix x multi-vector product, Y = H X.
//
// Reference: HMatrixVecMult (src/HMatrixVectorMultiplication.cu:10-27) runs a
// CUTLASS batched GEMM on the diagonal blocks, then per level a transpose of V,
// a grouped GEMM T = V^T X and a grouped GEMM Y += U T, with a host round trip
// per level (src/cutlassHMatrixXVector.cu:50-398), for weak admissibility only.
//
// Here the product is two launches for any admissibility.  Both are warp-level
// tensor-core kernels whose operands are loaded straight from HBM in MMA
// fragment order (no shared memory, no block-wide barriers); 16 right-hand
// sides form the MMA's M dimension:
//   phase 1 (projection) T_b^T = X[cols(b)]^T V_b: one warp per (block, chunk
//     of <= 256 rows of V_b); the MMA accumulates over the rows; blocks with
//     several chunks write per-chunk partials that a small kernel sums in
//     chunk order (bitwise reproducible);
//   phase 2 (expansion) Y^T = sum_b T_b^T U_b^T + sum_D X^T D^T: one warp per
//     32 rows of a leaf, over every low-rank block covering the leaf (all
//     levels) and the leaf's dense blocks; Y is written once, no atomics.
// FP32 factors use three TF32 passes (hi/lo split of both operands), which
// reproduces FP32 products.
#include <algorithm>
#include <mutex>
#include <numeric>

#include "hm_hmatrix.h"
#include "hm_mma.cuh"
#include "hm_structure.h"

// Scratch of the allocation-free product (hm_hmatvec_noalloc): 4 Mi floats
// (16 MiB) in the library's device image.  Every GPU that loads the library
// holds this array until the process exits.  Host code must not take its
// address directly (on the host the name is only a stand-in); the device
// address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) float hm_noalloc_scratch[size_t(4) << 20];

namespace hm {

// Right-hand sides per pass of the product: the mixed form reads every factor
// tile once for up to eight parts of 16, the FP32 form runs 16 at a time.
int pass_width(hm_hmatrix h) { return h->mx.enabled && h->mx.fmt == 0 ? 128 : 16; }

namespace {

constexpr int kWarpsPerCta = 4;
constexpr int kMaxK = 128;
constexpr int kMaxTiles = kMaxK / 8;

// ---------------------------------------------------------------------------
// phase 1
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// phase 1: T_b^T (16 x kpad) = X^T V_b over a chunk of rows.  NT: tile count
// the code is compiled for (>= the block's), U: k-steps (8 rows each) whose
// loads are issued together before their MMAs.
// ---------------------------------------------------------------------------
template <int NT, int U>
__device__ __forceinline__ void p1_item(const LRBlock& B, int i_lo, int i_hi, const float* __restrict__ X, int ldx,
                                        int nr, float* out, int g, int t) {
  const int k = B.k, kpad = (k + 7) & ~7, ntiles = kpad >> 3;
  const float* __restrict__ V = B.V;
  const float* __restrict__ xg = X + (size_t)g * ldx + B.c0;
  const float* __restrict__ xg8 = X + (size_t)(g + 8) * ldx + B.c0;
  const bool g_ok = g < nr, g8_ok = g + 8 < nr;
  float acc[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
  for (int i0 = i_lo; i0 < i_hi; i0 += 8 * U) {
    float xa[U][4], vb[U][NT][2];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int ra = i0 + 8 * u + t, rb = ra + 4;
      const bool ra_ok = ra < i_hi, rb_ok = rb < i_hi;
      xa[u][0] = g_ok && ra_ok ? __ldg(xg + ra) : 0.f;
      xa[u][1] = g8_ok && ra_ok ? __ldg(xg8 + ra) : 0.f;
      xa[u][2] = g_ok && rb_ok ? __ldg(xg + rb) : 0.f;
      xa[u][3] = g8_ok && rb_ok ? __ldg(xg8 + rb) : 0.f;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int col = nt * 8 + g;
        const bool c_ok = nt < ntiles && col < k;
        const float* vc = V + (size_t)col * B.n;
        vb[u][nt][0] = c_ok && ra_ok ? __ldcs(vc + ra) : 0.f;
        vb[u][nt][1] = c_ok && rb_ok ? __ldcs(vc + rb) : 0.f;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      uint32_t ah[4], al[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) split_tf32(xa[u][q], ah[q], al[q]);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        if (nt < ntiles) {
          uint32_t bh0, bl0, bh1, bl1;
          split_tf32(vb[u][nt][0], bh0, bl0);
          split_tf32(vb[u][nt][1], bh1, bl1);
          mma_3xtf32(acc[nt], ah, al, bh0, bh1, bl0, bl1);
        }
      }
    }
  }
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    if (nt < ntiles) {
      const int j = nt * 8 + 2 * t;
      *reinterpret_cast<float2*>(out + (size_t)g * kpad + j) = make_float2(acc[nt][0], acc[nt][1]);
      *reinterpret_cast<float2*>(out + (size_t)(g + 8) * kpad + j) = make_float2(acc[nt][2], acc[nt][3]);
    }
  }
}

__global__ void __launch_bounds__(32 * kWarpsPerCta, 3) k_p1(const P1Item* items, int nitems, const LRBlock* lr,
                                                          const float* __restrict__ X, int ldx, int nr,
                                                          float* __restrict__ T, float* __restrict__ Tpart,
                                                          int p1_rows) {
  const int w = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
  if (w >= nitems) return;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const P1Item it = items[w];
  const LRBlock B = lr[it.block];
  const int i_lo = it.chunk * p1_rows;
  const int i_hi = min(B.n, i_lo + p1_rows);
  float* out = it.part >= 0 ? Tpart + it.part : T + B.toff;  // [16][kpad]
  if (B.k <= 8)
    p1_item<1, 8>(B, i_lo, i_hi, X, ldx, nr, out, g, t);
  else if (B.k <= 16)
    p1_item<2, 4>(B, i_lo, i_hi, X, ldx, nr, out, g, t);
  else if (B.k <= 32)
    p1_item<4, 4>(B, i_lo, i_hi, X, ldx, nr, out, g, t);
  else
    p1_item<kMaxTiles, 1>(B, i_lo, i_hi, X, ldx, nr, out, g, t);
}

// projections of blocks split into several chunks: sum the chunk partials in
// chunk order (deterministic)
__global__ void k_reduce_multi(const MultiItem* mi, int n, const float* __restrict__ Tpart, float* __restrict__ T) {
  for (int b = blockIdx.x; b < n; b += gridDim.x) {
    const MultiItem M = mi[b];
    const int len = 16 * M.kpad;
    for (int e = threadIdx.x; e < len; e += blockDim.x) {
      float sacc = 0.f;
      for (int c = 0; c < M.nch; ++c) sacc += Tpart[M.poff + (long long)c * len + e];
      T[M.toff + e] = sacc;
    }
  }
}

// ---------------------------------------------------------------------------
// phase 2: Y^T (16 x 32 rows) = sum_b T_b^T U_b^T + sum_D X^T D^T
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * kWarpsPerCta) k_p2(const int2* groups, int ngroups, const int* leaf_off,
                                                          const int* leaf_ptr, const int* leaf_blk,
                                                          const LRBlock* lr, const int* leaf_dptr,
                                                          const int* leaf_dblk, const DenseBlock* dense,
                                                          const float* __restrict__ T,
                                                          const float* __restrict__ X, int ldx, int nr,
                                                          float* __restrict__ Y, int ldy) {
  const int w = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
  if (w >= ngroups) return;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int2 gr = groups[w];  // (leaf, first row of the group within the leaf)
  const int leaf = gr.x;
  const int l0 = leaf_off[leaf];
  const int nrow = min(32, leaf_off[leaf + 1] - l0 - gr.y);
  const int row0 = l0 + gr.y;  // tree-order index of the group's first row
  float acc[4][4];
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
  const int q_lo = leaf_ptr[leaf], q_hi = leaf_ptr[leaf + 1];
  for (int qb = q_lo; qb < q_hi; qb += 32) {
    // descriptors of up to 32 blocks, one per lane, loaded together
    const int nq = min(32, q_hi - qb);
    const float* my_u = nullptr;
    const float* my_t = nullptr;
    int my_m = 0, my_k = 0;
    if (lane < nq) {
      const LRBlock& Bl = lr[leaf_blk[qb + lane]];
      my_u = Bl.U + (row0 - Bl.r0);
      my_t = T + Bl.toff;
      my_m = Bl.m;
      my_k = Bl.k;
    }
    for (int q = 0; q < nq; ++q) {
      const float* __restrict__ ub =
          reinterpret_cast<const float*>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(my_u), q));
      const float* __restrict__ tb =
          reinterpret_cast<const float*>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(my_t), q));
      const int m = __shfl_sync(0xffffffffu, my_m, q);
      const int k = __shfl_sync(0xffffffffu, my_k, q);
      const int kpad = (k + 7) & ~7;
      for (int j0 = 0; j0 < kpad; j0 += 8) {
        uint32_t ah[4], al[4];
        split_tf32(__ldg(tb + (size_t)g * kpad + j0 + t), ah[0], al[0]);
        split_tf32(__ldg(tb + (size_t)(g + 8) * kpad + j0 + t), ah[1], al[1]);
        split_tf32(__ldg(tb + (size_t)g * kpad + j0 + t + 4), ah[2], al[2]);
        split_tf32(__ldg(tb + (size_t)(g + 8) * kpad + j0 + t + 4), ah[3], al[3]);
        const bool c0_ok = j0 + t < k, c1_ok = j0 + t + 4 < k;
        const float* u0 = ub + (size_t)(j0 + t) * m;
        const float* u1 = ub + (size_t)(j0 + t + 4) * m;
        float ubuf[4][2];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int rr = nt * 8 + g;
          const bool r_ok = rr < nrow;
          ubuf[nt][0] = c0_ok && r_ok ? __ldcs(u0 + rr) : 0.f;
          ubuf[nt][1] = c1_ok && r_ok ? __ldcs(u1 + rr) : 0.f;
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          uint32_t bh0, bl0, bh1, bl1;
          split_tf32(ubuf[nt][0], bh0, bl0);
          split_tf32(ubuf[nt][1], bh1, bl1);
          mma_3xtf32(acc[nt], ah, al, bh0, bh1, bl0, bl1);
        }
      }
    }
  }
  const float* __restrict__ xg = X + (size_t)g * ldx;
  const float* __restrict__ xg8 = X + (size_t)(g + 8) * ldx;
  const bool g_ok = g < nr, g8_ok = g + 8 < nr;
  for (int q = leaf_dptr[leaf]; q < leaf_dptr[leaf + 1]; ++q) {
    const DenseBlock D = dense[leaf_dblk[q]];
    const float* __restrict__ db = D.D + (row0 - D.r0);
    for (int j0 = 0; j0 < D.n; j0 += 8) {
      const int ca = j0 + t, cb = j0 + t + 4;
      const bool ca_ok = ca < D.n, cb_ok = cb < D.n;
      uint32_t ah[4], al[4];
      split_tf32(g_ok && ca_ok ? __ldg(xg + D.c0 + ca) : 0.f, ah[0], al[0]);
      split_tf32(g8_ok && ca_ok ? __ldg(xg8 + D.c0 + ca) : 0.f, ah[1], al[1]);
      split_tf32(g_ok && cb_ok ? __ldg(xg + D.c0 + cb) : 0.f, ah[2], al[2]);
      split_tf32(g8_ok && cb_ok ? __ldg(xg8 + D.c0 + cb) : 0.f, ah[3], al[3]);
      const float* d0 = db + (size_t)ca * D.m;
      const float* d1 = db + (size_t)cb * D.m;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int rr = nt * 8 + g;
        const bool r_ok = rr < nrow;
        uint32_t bh0, bl0, bh1, bl1;
        split_tf32(ca_ok && r_ok ? __ldcs(d0 + rr) : 0.f, bh0, bl0);
        split_tf32(cb_ok && r_ok ? __ldcs(d1 + rr) : 0.f, bh1, bl1);
        mma_3xtf32(acc[nt], ah, al, bh0, bh1, bl0, bl1);
      }
    }
  }
  // acc[nt]: rows nt*8 + 2t, +1 of right-hand sides g and g + 8
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) {
    const int rr = nt * 8 + 2 * t;
    if (g_ok) {
      if (rr < nrow) Y[(size_t)g * ldy + row0 + rr] = acc[nt][0];
      if (rr + 1 < nrow) Y[(size_t)g * ldy + row0 + rr + 1] = acc[nt][1];
    }
    if (g8_ok) {
      if (rr < nrow) Y[(size_t)(g + 8) * ldy + row0 + rr] = acc[nt][2];
      if (rr + 1 < nrow) Y[(size_t)(g + 8) * ldy + row0 + rr + 1] = acc[nt][3];
    }
  }
}

__global__ void k_gather_rows(const float* X, int ldx, const int* perm, int n, int nrhs, float* Xp) {
  long long tot = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % n), c = (int)(e / n);
    Xp[(size_t)c * n + i] = X[(size_t)c * ldx + perm[i]];
  }
}

__global__ void k_scatter_rows(const float* Yp, const int* perm, int n, int nrhs, float* Y, int ldy) {
  long long tot = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % n), c = (int)(e / n);
    Y[(size_t)c * ldy + perm[i]] = Yp[(size_t)c * n + i];
  }
}


// FP64 vectors of the reference's interface: X (double, ldx; rows gathered
// through perm when perm != null) narrowed into Xp (float, ld n) ...
__global__ void k_narrow_rows(const double* __restrict__ X, int ldx, const int* __restrict__ perm, int n, int nrhs,
                              float* __restrict__ Xp) {
  long long tot = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % n), c = (int)(e / n);
    Xp[(size_t)c * n + i] = (float)X[(size_t)c * ldx + (perm ? perm[i] : i)];
  }
}

// ... and the FP32 result Yp (ld n) widened into Y (double, ldy; rows
// scattered through perm when perm != null)
__global__ void k_widen_rows(const float* __restrict__ Yp, const int* __restrict__ perm, int n, int nrhs,
                             double* __restrict__ Y, int ldy) {
  long long tot = (long long)n * nrhs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e % n), c = (int)(e / n);
    Y[(size_t)c * ldy + (perm ? perm[i] : i)] = (double)Yp[(size_t)c * n + i];
  }
}

// Y[leaf] += K(leaf, leaf) X[leaf], one CTA per leaf, entries from the
// tree-ordered FP32 coordinates exactly as the stored diagonal blocks are
// generated (kernel_r2, plus the nugget on the diagonal unless dK/dl).
constexpr int kFlyT = 64;
__global__ void __launch_bounds__(kFlyT) k_diag_fly(const int* __restrict__ leaf_off, const float* __restrict__ pts,
                                                    int npts, int d, KernelParams kp, const float* __restrict__ X,
                                                    int ldx, int nr, float* __restrict__ Y, int ldy) {
  __shared__ float cs[kMaxDim][kFlyT];
  __shared__ float xs[16][kFlyT];
  const int r0 = leaf_off[blockIdx.x];
  const int m = leaf_off[blockIdx.x + 1] - r0;
  for (int i0 = 0; i0 < m; i0 += kFlyT) {
    const int i = i0 + threadIdx.x;
    const bool iok = i < m;
    float ci[kMaxDim];
#pragma unroll
    for (int k = 0; k < kMaxDim; ++k) ci[k] = (k < d && iok) ? pts[(size_t)k * npts + r0 + i] : 0.f;
    float acc[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) acc[r] = 0.f;
    for (int j0 = 0; j0 < m; j0 += kFlyT) {
      __syncthreads();
      const int j = j0 + threadIdx.x;
      for (int k = 0; k < d; ++k) cs[k][threadIdx.x] = j < m ? pts[(size_t)k * npts + r0 + j] : 0.f;
#pragma unroll
      for (int r = 0; r < 16; ++r) xs[r][threadIdx.x] = (j < m && r < nr) ? X[(size_t)r * ldx + r0 + j] : 0.f;
      __syncthreads();
      const int jn = min(kFlyT, m - j0);
      for (int jj = 0; jj < jn; ++jj) {
        float r2 = 0.f;
#pragma unroll
        for (int k = 0; k < kMaxDim; ++k) {
          if (k < d) {
            const float df = ci[k] - cs[k][jj];
            r2 = fmaf(df, df, r2);
          }
        }
        float e = kernel_r2(kp, r2);
        if (i == j0 + jj && !kp.deriv) e += kp.nugget;
#pragma unroll
        for (int r = 0; r < 16; ++r) acc[r] = fmaf(e, xs[r][jj], acc[r]);
      }
    }
    if (iok) {
#pragma unroll
      for (int r = 0; r < 16; ++r)
        if (r < nr) Y[(size_t)r * ldy + r0 + i] += acc[r];
    }
  }
}

// One pass of nr <= pass_width(h) right-hand sides (X, Y in tree order); T:
// projection scratch (FP32 form: 16 x kpad per block, then the chunk
// partials; mixed form: see mixed_run_panel).
hm_status run_panel(hm_hmatrix h, int nr, const float* X, int ldx, float* Y, int ldy, float* T, cudaStream_t s,
                    KernelMarks* km) {
  if (h->mx.enabled) return mixed_run_panel(h, nr, X, ldx, Y, ldy, T, s, km);
  MatvecPlan& P = h->plan;
  float* Tpart = T + P.t_floats;
  if (P.num_p1 > 0) {
    k_p1<<<(P.num_p1 + kWarpsPerCta - 1) / kWarpsPerCta, 32 * kWarpsPerCta, 0, s>>>(P.p1.p, P.num_p1, P.lr.p, X,
                                                                                     ldx, nr, T, Tpart, P.p1_rows);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_p1", P.bytes_p1 + 4ll * h->n * nr, s);
  }
  if (P.num_multi > 0) {
    k_reduce_multi<<<std::min(P.num_multi, 8192), 128, 0, s>>>(P.multi.p, P.num_multi, Tpart, T);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_reduce_multi", 4ll * P.part_floats + 4ll * P.multi_t_floats, s);
  }
  k_p2<<<(P.num_groups + kWarpsPerCta - 1) / kWarpsPerCta, 32 * kWarpsPerCta, 0, s>>>(
      P.groups.p, P.num_groups, h->tree->offsets.p, P.leaf_ptr.p, P.leaf_blk.p, P.lr.p, P.leaf_dptr.p,
      P.leaf_dblk.p, P.dense.p, T, X, ldx, nr, Y, ldy);
  HM_LAUNCH_CHECK();
  if (km) km->mark("k_p2", P.bytes_p2 + 8ll * h->n * nr, s);
  if (h->diag_fly) HM_TRY(diag_fly_panel(h, nr, X, ldx, Y, ldy, s, km));
  return HM_OK;
}

}  // namespace

hm_status matvec_plan_build(hm_hmatrix h, int nrhs_cap, cudaStream_t stream) {
  MatvecPlan& P = h->plan;
  ++h->plan_gen;  // recorded graphs of the old plan are stale
  const int depth = h->depth;
  const int nleaf = 1 << depth;
  const std::vector<int>& lo = h->tree->h_offsets;
  nrhs_cap = 16;
  P.nrhs_cap = nrhs_cap;
  P.num_leaves = nleaf;
  // device block list: blocks of rank above 128 become pieces of at most
  // 128 columns (U and V sliced alike), whose products add up
  std::vector<LRBlock> lr;
  lr.reserve(h->h_lr.size());
  // a block-row shard expands only into its own rows [row_lo, row_hi)
  const int row_lo = lo[h->leaf_lo], row_hi = lo[h->leaf_hi];
  auto own_rows = [&](int r0, int m) { return r0 < row_hi && r0 + m > row_lo; };
  for (const LRBlock& b : h->h_lr) {
    if (!own_rows(b.r0, b.m)) continue;
    for (int c0 = 0; c0 == 0 || c0 < b.k; c0 += kMaxK) {
      LRBlock x = b;
      x.k = std::min(kMaxK, b.k - c0);
      x.U = b.U + (size_t)c0 * b.m;
      x.V = b.V + (size_t)c0 * b.n;
      lr.push_back(x);
    }
  }
  long long tk = 0;
  for (auto& b : lr) {
    b.toff = tk;
    tk += 16ll * ((b.k + 7) & ~7);  // T_b^T: 16 right-hand sides x padded rank
  }
  P.t_floats = tk;
  P.t_per_rhs = tk / 16;
  // phase 1 items; a block spanning several chunks writes one partial per
  // chunk, summed in chunk order afterwards
  std::vector<P1Item> items;
  std::vector<MultiItem> multi;
  long long part = 0;
  for (size_t i = 0; i < lr.size(); ++i) {
    const LRBlock& b = lr[i];
    if (b.k <= 0) continue;
    int nch = (b.n + P.p1_rows - 1) / P.p1_rows;
    const int kpad = (b.k + 7) & ~7;
    for (int c = 0; c < nch; ++c)
      items.push_back(P1Item{(int)i, c, nch == 1 ? -1ll : part + (long long)c * 16 * kpad});
    if (nch > 1) {
      multi.push_back(MultiItem{b.toff, part, kpad, nch});
      part += (long long)nch * 16 * kpad;
    }
  }
  P.num_p1 = (int)items.size();
  P.num_multi = (int)multi.size();
  P.part_floats = part;
  P.bytes_p1 = P.bytes_p2 = P.multi_t_floats = 0;
  for (const auto& b : lr) {
    P.bytes_p1 += 4ll * b.n * b.k;
    P.bytes_p2 += 4ll * b.m * b.k;
  }
  for (const auto& d : h->h_dense)
    if (own_rows(d.r0, d.m)) P.bytes_p2 += 4ll * d.m * d.n;
  for (const auto& mi : multi) P.multi_t_floats += 16ll * mi.kpad;
  // phase 2: leaf lists
  auto leaf_range = [&](int r0, int m, int& a, int& b) {
    a = (int)(std::lower_bound(lo.begin(), lo.end() - 1, r0) - lo.begin());
    b = (int)(std::lower_bound(lo.begin(), lo.end() - 1, r0 + m) - lo.begin());
  };
  std::vector<int> cnt(nleaf + 1, 0), dcnt(nleaf + 1, 0);
  std::vector<std::pair<int, int>> ranges(lr.size()), dranges(h->h_dense.size());
  for (size_t i = 0; i < lr.size(); ++i) {
    int a, e;
    leaf_range(lr[i].r0, lr[i].m, a, e);
    ranges[i] = {a, e};
    if (lr[i].k > 0)
      for (int l = a; l < e; ++l) cnt[l]++;
  }
  for (size_t i = 0; i < h->h_dense.size(); ++i) {
    int a, e;
    leaf_range(h->h_dense[i].r0, h->h_dense[i].m, a, e);
    a = std::max(a, h->leaf_lo);
    e = std::max(a, std::min(e, h->leaf_hi));
    dranges[i] = {a, e};
    for (int l = a; l < e; ++l) dcnt[l]++;
  }
  std::vector<int> ptr(nleaf + 1, 0), dptr(nleaf + 1, 0);
  for (int l = 0; l < nleaf; ++l) {
    ptr[l + 1] = ptr[l] + cnt[l];
    dptr[l + 1] = dptr[l] + dcnt[l];
  }
  std::vector<int> blk(std::max(ptr[nleaf], 1)), dblk(std::max(dptr[nleaf], 1));
  std::vector<int> fill(ptr.begin(), ptr.end() - 1), dfill(dptr.begin(), dptr.end() - 1);
  for (size_t i = 0; i < lr.size(); ++i) {
    if (lr[i].k <= 0) continue;
    for (int l = ranges[i].first; l < ranges[i].second; ++l) blk[fill[l]++] = (int)i;
  }
  for (size_t i = 0; i < h->h_dense.size(); ++i)
    for (int l = dranges[i].first; l < dranges[i].second; ++l) dblk[dfill[l]++] = (int)i;
  std::vector<int2> groups;
  for (int l = h->leaf_lo; l < h->leaf_hi; ++l)
    for (int r = 0; r < lo[l + 1] - lo[l]; r += 32) groups.push_back(make_int2(l, r));
  P.num_groups = (int)groups.size();

  HM_TRY(P.lr.alloc(std::max<size_t>(lr.size(), 1)));
  HM_TRY(P.p1.alloc(std::max<size_t>(items.size(), 1)));
  HM_TRY(P.multi.alloc(std::max<size_t>(multi.size(), 1)));
  HM_TRY(P.groups.alloc(std::max<size_t>(groups.size(), 1)));
  HM_TRY(P.leaf_ptr.alloc(nleaf + 1));
  HM_TRY(P.leaf_blk.alloc(blk.size()));
  HM_TRY(P.dense.alloc(std::max<size_t>(h->h_dense.size(), 1)));
  HM_TRY(P.leaf_dptr.alloc(nleaf + 1));
  HM_TRY(P.leaf_dblk.alloc(dblk.size()));
  // projection scratch of one pass, for whichever product runs (the mixed
  // form's panels: passes of up to 128 right-hand sides; the FP32 form's
  // panels or per-block kernels: 16)
  const long long scratch =
      h->mx.enabled ? h->mx.scratch_floats(h->mx.fmt == 0 ? 8 : 1) : tk + part;
  HM_TRY(P.T.alloc(std::max<long long>(scratch, 1)));
  HM_TRY(P.Xp.alloc((size_t)h->n * pass_width(h)));
  HM_TRY(P.Yp.alloc((size_t)h->n * pass_width(h)));
  auto up = [&](void* dst, const void* src, size_t bytes) -> hm_status {
    if (bytes) HM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
    return HM_OK;
  };
  HM_TRY(up(P.lr.p, lr.data(), sizeof(LRBlock) * lr.size()));
  HM_TRY(up(P.p1.p, items.data(), sizeof(P1Item) * items.size()));
  HM_TRY(up(P.multi.p, multi.data(), sizeof(MultiItem) * multi.size()));
  HM_TRY(up(P.groups.p, groups.data(), sizeof(int2) * groups.size()));
  HM_TRY(up(P.leaf_ptr.p, ptr.data(), 4 * ptr.size()));
  HM_TRY(up(P.leaf_blk.p, blk.data(), 4 * blk.size()));
  HM_TRY(up(P.dense.p, h->h_dense.data(), sizeof(DenseBlock) * h->h_dense.size()));
  HM_TRY(up(P.leaf_dptr.p, dptr.data(), 4 * dptr.size()));
  HM_TRY(up(P.leaf_dblk.p, dblk.data(), 4 * dblk.size()));
  HM_CUDA(cudaStreamSynchronize(stream));
  return HM_OK;
}

hm_status hmatvec(hm_hmatrix h, int trans, int nrhs, const float* X, int ldx, float* Y, int ldy,
                  int original_order, cudaStream_t stream) {
  if (!h) return fail(HM_ERR_INVALID, "hm_hmatvec: null matrix");
  if (nrhs < 1 || !X || !Y || ldx < h->n || ldy < h->n)
    return fail(HM_ERR_INVALID, "hm_hmatvec: bad vector arguments");
  if (trans != 0 && trans != 1) return fail(HM_ERR_INVALID, "hm_hmatvec: trans must be 0 or 1");
  // the stored operator is exactly symmetric (mirror blocks share factors,
  // dense blocks are generated from a symmetric kernel), so H^T X = H X
  MatvecPlan& P = h->plan;
  const int n = h->n;
  for (int c0 = 0; c0 < nrhs;) {
    const int nr = std::min(pass_width(h), nrhs - c0);
    const float* Xin = X + (size_t)c0 * ldx;
    float* Yout = Y + (size_t)c0 * ldy;
    const float* Xt = Xin;
    int ldxt = ldx;
    float* Yt = Yout;
    int ldyt = ldy;
    if (original_order) {
      k_gather_rows<<<592, 256, 0, stream>>>(Xin, ldx, h->tree->perm.p, n, nr, P.Xp.p);
      HM_LAUNCH_CHECK();
      Xt = P.Xp.p;
      ldxt = n;
      Yt = P.Yp.p;
      ldyt = n;
    }
    HM_TRY(run_panel(h, nr, Xt, ldxt, Yt, ldyt, P.T.p, stream, nullptr));
    if (original_order) {
      k_scatter_rows<<<592, 256, 0, stream>>>(P.Yp.p, h->tree->perm.p, n, nr, Yout, ldy);
      HM_LAUNCH_CHECK();
    }
    c0 += nr;
  }
  return HM_OK;
}

// The product on FP64 vectors: per pass, X narrowed into the plan's Xp, the
// FP32 product into Yp, Yp widened into Y; the permutation of original-order
// calls is applied by the same two kernels.
hm_status hmatvec_f64(hm_hmatrix h, int trans, int nrhs, const double* X, int ldx, double* Y, int ldy,
                      int original_order, cudaStream_t stream) {
  if (!h) return fail(HM_ERR_INVALID, "hm_hmatvec_f64: null matrix");
  if (nrhs < 1 || !X || !Y || ldx < h->n || ldy < h->n)
    return fail(HM_ERR_INVALID, "hm_hmatvec_f64: bad vector arguments");
  if (trans != 0 && trans != 1) return fail(HM_ERR_INVALID, "hm_hmatvec_f64: trans must be 0 or 1");
  // H^T X = H X: the stored operator is exactly symmetric (see hmatvec)
  MatvecPlan& P = h->plan;
  const int n = h->n;
  const int* perm = original_order ? h->tree->perm.p : nullptr;
  for (int c0 = 0; c0 < nrhs;) {
    const int nr = std::min(pass_width(h), nrhs - c0);
    k_narrow_rows<<<592, 256, 0, stream>>>(X + (size_t)c0 * ldx, ldx, perm, n, nr, P.Xp.p);
    HM_LAUNCH_CHECK();
    HM_TRY(run_panel(h, nr, P.Xp.p, n, P.Yp.p, n, P.T.p, stream, nullptr));
    k_widen_rows<<<592, 256, 0, stream>>>(P.Yp.p, perm, n, nr, Y + (size_t)c0 * ldy, ldy);
    HM_LAUNCH_CHECK();
    c0 += nr;
  }
  return HM_OK;
}

// Algorithmic bytes of one product with nrhs FP32 columns: factors and dense
// blocks read once, X read once and Y written once per phase that touches them.
void matvec_bytes(hm_hmatrix h, int nrhs, long long* b_project, long long* b_expand) {
  long long p1 = 0, p2 = 0;
  if (h->mx.enabled) {
    // BF16 high parts of every factor column plus the low parts of the
    // columns that keep one (unpadded); dense blocks hi + lo
    p1 = h->mx.bytes_p1;
    p2 = h->mx.bytes_p2;
  } else {
    for (const auto& b : h->h_lr) {
      p1 += 4ll * b.n * b.k;
      p2 += 4ll * b.m * b.k;
    }
    for (const auto& d : h->h_dense) p2 += 4ll * d.m * d.n;
  }
  p1 += 4ll * h->n * nrhs;      // X
  p2 += 4ll * h->n * nrhs * 2;  // X (dense blocks) and Y
  *b_project = p1;
  *b_expand = p2;
}

namespace {

constexpr size_t kNoallocScratchFloats = size_t(4) << 20;
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the static scratch on the current device, resolved on the
// first call for that device.
hm_status noalloc_scratch(float** out) {
  int dev = 0;
  HM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(HM_ERR_UNSUPPORTED, "hm_hmatvec_noalloc: device ordinal >= 64");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, hm_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(hm_noalloc_scratch)", __FILE__, __LINE__);
    g_noalloc_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return HM_OK;
}

}  // namespace
}  // namespace hm

namespace hm {
hm_status diag_fly_panel(hm_hmatrix_s* h, int nr, const float* X, int ldx, float* Y, int ldy, cudaStream_t s,
                         KernelMarks* km) {
  const hm_kdtree t = h->tree;
  // the shard's leaves (every leaf of a whole matrix)
  k_diag_fly<<<h->leaf_hi - h->leaf_lo, kFlyT, 0, s>>>(t->offsets.p + h->leaf_lo, t->pts_tree_f.p, t->n, t->d,
                                                       h->kp, X, ldx, nr, Y, ldy);
  HM_LAUNCH_CHECK();
  if (km) km->mark("k_diag_fly", 4ll * h->n * nr * 3 + 4ll * h->n * h->d, s);
  return HM_OK;
}

// One panel with an event after each kernel; synchronises.  The caller
// destroys km->ev.
hm_status timed_panel(hm_hmatrix h, int nr, const float* X, int ldx, float* Y, int ldy, cudaStream_t s,
                      KernelMarks* km) {
  for (auto& x : km->ev) HM_CUDA(cudaEventCreate(&x));
  km->n = 0;
  HM_CUDA(cudaEventRecord(km->ev[0], s));
  HM_TRY(run_panel(h, nr, X, ldx, Y, ldy, h->plan.T.p, s, km));
  HM_CUDA(cudaEventSynchronize(km->ev[km->n]));
  return HM_OK;
}
}  // namespace hm

// The product of hm_hmatvec (tree order) with its projection workspace taken
// from the library's static scratch instead of the matrix's own buffer; no
// allocation of any kind.
extern "C" hm_status hm_hmatvec_noalloc(hm_hmatrix h, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                        void* stream) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatvec_noalloc: null matrix");
  if (nrhs < 1 || !X || !Y || ldx < h->n || ldy < h->n)
    return hm::fail(HM_ERR_INVALID, "hm_hmatvec_noalloc: bad vector arguments");
  hm::MatvecPlan& P = h->plan;
  const size_t need = h->mx.enabled ? (size_t)h->mx.scratch_floats() : (size_t)P.t_floats + (size_t)P.part_floats;
  if (need > hm::kNoallocScratchFloats) {
    const std::string what =
        !h->mx.enabled ? " floats of projection scratch for a 16-column pass of the FP32 form's per-block product "
                         "(16 per factor column, plus chunk partials)"
        : h->mx.fmt == 0 ? " floats of scratch for a 16-column pass of the mixed form (16 per point for the X "
                           "fragments, plus chunk partials and projections)"
                         : " floats of scratch for a 16-column pass of the FP32 form (32 per point for the X "
                           "fragments, plus chunk partials and projections)";
    return hm::fail(HM_ERR_UNSUPPORTED, "hm_hmatvec_noalloc: this matrix needs " + std::to_string(need) + what +
                                            "; the static scratch holds " +
                                            std::to_string(hm::kNoallocScratchFloats) + " (16 MiB)");
  }
  float* T = nullptr;
  HM_TRY(hm::noalloc_scratch(&T));
  cudaStream_t s = hm::as_stream(stream);
  for (int c0 = 0; c0 < nrhs;) {
    const int nr = std::min(16, nrhs - c0);
    // the scratch keeps the previous call's contents, which need no clearing:
    // every scratch word the pass reads (X fragments, chunk partials,
    // projections, padding columns as zeros) is written earlier in the pass
    HM_TRY(hm::run_panel(h, nr, X + (size_t)c0 * ldx, ldx, Y + (size_t)c0 * ldy, ldy, T, s, nullptr));
    c0 += nr;
  }
  return HM_OK;
}

extern "C" hm_status hm_hmatvec(hm_hmatrix h, int trans, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                int original_order, void* stream) {
  return hm::hmatvec(h, trans, nrhs, X, ldx, Y, ldy, original_order, hm::as_stream(stream));
}

extern "C" hm_status hm_hmatvec_f64(hm_hmatrix h, int trans, int nrhs, const double* X, int ldx, double* Y, int ldy,
                                    int original_order, void* stream) {
  return hm::hmatvec_f64(h, trans, nrhs, X, ldx, Y, ldy, original_order, hm::as_stream(stream));
}

extern "C" hm_status hm_hmatvec_profile(hm_hmatrix h, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                        void* stream, float* ms_project, float* ms_expand,
                                        long long* bytes_project, long long* bytes_expand) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatvec_profile: null matrix");
  if (nrhs < 1 || nrhs > hm::pass_width(h) || !X || !Y || ldx < h->n || ldy < h->n)
    return hm::fail(HM_ERR_INVALID, "hm_hmatvec_profile: need 1 <= nrhs <= one pass (16, or 128 for the mixed "
                                    "form) and valid vectors");
  cudaStream_t s = hm::as_stream(stream);
  hm::KernelMarks km;
  HM_TRY(hm::timed_panel(h, nrhs, X, ldx, Y, ldy, s, &km));
  // projection: every kernel but the last; expansion: the last
  float a = 0, b = 0;
  if (km.n > 0) {
    HM_CUDA(cudaEventElapsedTime(&a, km.ev[0], km.ev[km.n - 1]));
    HM_CUDA(cudaEventElapsedTime(&b, km.ev[km.n - 1], km.ev[km.n]));
  }
  for (auto& x : km.ev) cudaEventDestroy(x);
  if (ms_project) *ms_project = a;
  if (ms_expand) *ms_expand = b;
  long long bp = 0, be = 0;
  hm::matvec_bytes(h, nrhs, &bp, &be);
  if (bytes_project) *bytes_project = bp;
  if (bytes_expand) *bytes_expand = be;
  return HM_OK;
}

extern "C" hm_status hm_hmatvec_kernels(hm_hmatrix h, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                        void* stream, int cap, const char** names, float* ms, long long* bytes,
                                        int* count) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatvec_kernels: null matrix");
  if (nrhs < 1 || nrhs > hm::pass_width(h) || !X || !Y || ldx < h->n || ldy < h->n || cap < 0)
    return hm::fail(HM_ERR_INVALID, "hm_hmatvec_kernels: need 1 <= nrhs <= one pass (16, or 128 for the mixed "
                                    "form) and valid vectors");
  hm::KernelMarks km;
  HM_TRY(hm::timed_panel(h, nrhs, X, ldx, Y, ldy, hm::as_stream(stream), &km));
  for (int i = 0; i < km.n && i < cap; ++i) {
    float t = 0;
    cudaEventElapsedTime(&t, km.ev[i], km.ev[i + 1]);
    if (names) names[i] = km.name[i];
    if (ms) ms[i] = t;
    if (bytes) bytes[i] = km.bytes[i];
  }
  if (count) *count = km.n;
  for (auto& x : km.ev) cudaEventDestroy(x);
  return HM_OK;
}
