// hm_matvec.cu -- H-matrix x multi-vector product, Y = H X.
//
// Reference: HMatrixVecMult (src/HMatrixVectorMultiplication.cu:10-27) runs a
// CUTLASS batched GEMM on the diagonal blocks, then per level a transpose of V,
// a grouped GEMM T = V^T X and a grouped GEMM Y += U T, with a host round trip
// per level (src/cutlassHMatrixXVector.cu:50-398), for weak admissibility only.
//
// Here the product is two launches for any admissibility:
//   phase 1 (projection): T_b = V_b^T X[cols(b)] for every low-rank block b,
//     one work item per (block, 1024-row chunk of V_b), reduced in shared
//     memory and added into T_b;
//   phase 2 (expansion): one CTA per leaf row cluster accumulates, in
//     registers, U_b[rows of the leaf] T_b over every low-rank block whose row
//     cluster contains the leaf (all levels) plus the leaf's dense blocks times
//     X, and writes its rows of Y once (no atomics on Y).
// Both launches are stream ordered and allocation free; X/Y in the points'
// original order are gathered / scattered through the tree permutation.
#include <algorithm>
#include <mutex>
#include <numeric>

#include "hm_hmatrix.h"
#include "hm_structure.h"

// Scratch of the allocation-free product (hm_hmatvec_noalloc): 4 Mi floats
// (16 MiB) in the library's device image.  Every GPU that loads the library
// holds this array until the process exits.  Host code must not take its
// address directly (on the host the name is only a stand-in); the device
// address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) float hm_noalloc_scratch[size_t(4) << 20];

namespace hm {
namespace {

constexpr int kP1Rows = 1024;
constexpr int kThreads = 256;
constexpr int kMaxK = 128;
constexpr int kMaxOut = 16;  // outputs per thread

__global__ void __launch_bounds__(kThreads) k_mv_project(const int2* items, const LRBlock* lr,
                                                         const float* X, int ldx, int nrhs, float* T) {
  extern __shared__ __align__(16) float sm[];
  float* Vs = sm;                 // [kMaxK][33]
  float* Xs = Vs + kMaxK * 33;    // [32][33]
  const int2 it = items[blockIdx.x];
  const LRBlock B = lr[it.x];
  const int k = B.k;
  const int i_lo = it.y * kP1Rows;
  const int i_hi = min(B.n, i_lo + kP1Rows);
  const int nout = k * nrhs;
  const int t = threadIdx.x;
  float acc[kMaxOut];
#pragma unroll
  for (int x = 0; x < kMaxOut; ++x) acc[x] = 0.f;
  for (int i0 = i_lo; i0 < i_hi; i0 += 32) {
    for (int e = t; e < 32 * k; e += kThreads) {
      int ii = e & 31, j = e >> 5;
      int i = i0 + ii;
      Vs[j * 33 + ii] = i < i_hi ? B.V[(size_t)j * B.n + i] : 0.f;
    }
    for (int e = t; e < 32 * nrhs; e += kThreads) {
      int ii = e & 31, c = e >> 5;
      int i = i0 + ii;
      Xs[c * 33 + ii] = i < i_hi ? X[(size_t)c * ldx + B.c0 + i] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int x = 0; x < kMaxOut; ++x) {
      int o = t + x * kThreads;
      if (o < nout) {
        int j = o / nrhs, c = o % nrhs;
        float s = acc[x];
#pragma unroll 8
        for (int ii = 0; ii < 32; ++ii) s = fmaf(Vs[j * 33 + ii], Xs[c * 33 + ii], s);
        acc[x] = s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < kMaxOut; ++x) {
    int o = t + x * kThreads;
    if (o < nout) atomicAdd(&T[B.toff + o], acc[x]);  // T_b[j * nrhs + c]
  }
}

__global__ void __launch_bounds__(kThreads) k_mv_expand(const int* leaf_off, const int* leaf_ptr,
                                                        const int* leaf_blk, const LRBlock* lr,
                                                        const int* leaf_dptr, const int* leaf_dblk,
                                                        const DenseBlock* dense, const float* T,
                                                        const float* X, int ldx, float* Y, int ldy,
                                                        int nrhs) {
  extern __shared__ __align__(16) float sm[];
  const int leaf = blockIdx.x;
  const int r_lo = leaf_off[leaf], rows = leaf_off[leaf + 1] - r_lo;
  if (rows <= 0) return;
  float* Us = sm;                     // [kMaxK][rows]
  float* Ts = Us + kMaxK * rows;      // [kMaxK][nrhs]
  float* Ds = Ts + kMaxK * nrhs;      // [32][rows]
  float* Xs = Ds + 32 * rows;         // [32][nrhs]
  const int t = threadIdx.x;
  const int nout = rows * nrhs;
  float acc[kMaxOut];
#pragma unroll
  for (int x = 0; x < kMaxOut; ++x) acc[x] = 0.f;

  for (int q = leaf_ptr[leaf]; q < leaf_ptr[leaf + 1]; ++q) {
    const LRBlock B = lr[leaf_blk[q]];
    const int k = B.k;
    const int off = r_lo - B.r0;
    for (int e = t; e < k * rows; e += kThreads) {
      int i = e % rows, j = e / rows;
      Us[j * rows + i] = B.U[(size_t)j * B.m + off + i];
    }
    for (int e = t; e < k * nrhs; e += kThreads) Ts[e] = T[B.toff + e];
    __syncthreads();
#pragma unroll
    for (int x = 0; x < kMaxOut; ++x) {
      int o = t + x * kThreads;
      if (o < nout) {
        int i = o % rows, c = o / rows;
        float s = acc[x];
        for (int j = 0; j < k; ++j) s = fmaf(Us[j * rows + i], Ts[j * nrhs + c], s);
        acc[x] = s;
      }
    }
    __syncthreads();
  }
  for (int q = leaf_dptr[leaf]; q < leaf_dptr[leaf + 1]; ++q) {
    const DenseBlock D = dense[leaf_dblk[q]];
    const int doff = r_lo - D.r0;  // a dense block may span several leaves
    for (int j0 = 0; j0 < D.n; j0 += 32) {
      for (int e = t; e < 32 * rows; e += kThreads) {
        int i = e % rows, jj = e / rows;
        int j = j0 + jj;
        float v = 0.f;
        if (j < D.n)
          v = D.trans ? D.D[(size_t)(doff + i) * D.n + j] : D.D[(size_t)j * D.m + doff + i];
        Ds[jj * rows + i] = v;
      }
      for (int e = t; e < 32 * nrhs; e += kThreads) {
        int jj = e & 31, c = e >> 5;
        int j = j0 + jj;
        Xs[jj * nrhs + c] = j < D.n ? X[(size_t)c * ldx + D.c0 + j] : 0.f;
      }
      __syncthreads();
#pragma unroll
      for (int x = 0; x < kMaxOut; ++x) {
        int o = t + x * kThreads;
        if (o < nout) {
          int i = o % rows, c = o / rows;
          float s = acc[x];
#pragma unroll 8
          for (int jj = 0; jj < 32; ++jj) s = fmaf(Ds[jj * rows + i], Xs[jj * nrhs + c], s);
          acc[x] = s;
        }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int x = 0; x < kMaxOut; ++x) {
    int o = t + x * kThreads;
    if (o < nout) {
      int i = o % rows, c = o / rows;
      Y[(size_t)c * ldy + r_lo + i] = acc[x];
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

size_t expand_smem(int rows, int nrhs) {
  return sizeof(float) * ((size_t)kMaxK * rows + (size_t)kMaxK * nrhs + 32 * (size_t)rows + 32 * (size_t)nrhs);
}

}  // namespace

hm_status matvec_plan_build(hm_hmatrix h, int nrhs_cap, cudaStream_t stream) {
  MatvecPlan& P = h->plan;
  const int depth = h->depth;
  const int nleaf = 1 << depth;
  const std::vector<int>& lo = h->tree->h_offsets;
  int maxleaf = 1;
  for (int l = 0; l < nleaf; ++l) maxleaf = std::max(maxleaf, lo[l + 1] - lo[l]);
  // rhs panel: at most kMaxOut outputs per thread in phase 2
  int panel = std::min(32, (kThreads * kMaxOut) / maxleaf);
  if (panel < 1) return fail(HM_ERR_UNSUPPORTED, "matvec: leaves too large");
  nrhs_cap = std::min(nrhs_cap, panel);
  P.nrhs_cap = nrhs_cap;
  P.num_leaves = nleaf;
  // T offsets
  long long tk = 0;
  for (auto& b : h->h_lr) {
    b.toff = tk * nrhs_cap;
    tk += b.k;
  }
  P.t_per_rhs = tk;
  // phase 1 items
  std::vector<int2> items;
  for (size_t i = 0; i < h->h_lr.size(); ++i) {
    const LRBlock& b = h->h_lr[i];
    if (b.k <= 0) continue;
    for (int c = 0; c * kP1Rows < b.n; ++c) items.push_back(make_int2((int)i, c));
  }
  P.num_p1 = (int)items.size();
  // leaf lists: a block with row range [r0, r0+m) covers the leaves whose
  // offsets lie in that range (row clusters are unions of consecutive leaves)
  auto leaf_range = [&](int r0, int m, int& a, int& b) {
    a = (int)(std::lower_bound(lo.begin(), lo.end() - 1, r0) - lo.begin());
    b = (int)(std::lower_bound(lo.begin(), lo.end() - 1, r0 + m) - lo.begin());
    // leaves [a, b) have lo[leaf] in [r0, r0+m); empty leaves at the boundary are harmless
  };
  std::vector<int> cnt(nleaf + 1, 0), dcnt(nleaf + 1, 0);
  std::vector<std::pair<int, int>> ranges(h->h_lr.size());
  for (size_t i = 0; i < h->h_lr.size(); ++i) {
    const LRBlock& b = h->h_lr[i];
    int a, e;
    leaf_range(b.r0, b.m, a, e);
    ranges[i] = {a, e};
    if (b.k <= 0) continue;
    for (int l = a; l < e; ++l) cnt[l]++;
  }
  std::vector<std::pair<int, int>> dranges(h->h_dense.size());
  for (size_t i = 0; i < h->h_dense.size(); ++i) {
    int a, e;
    leaf_range(h->h_dense[i].r0, h->h_dense[i].m, a, e);
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
  for (size_t i = 0; i < h->h_lr.size(); ++i) {
    if (h->h_lr[i].k <= 0) continue;
    for (int l = ranges[i].first; l < ranges[i].second; ++l) blk[fill[l]++] = (int)i;
  }
  for (size_t i = 0; i < h->h_dense.size(); ++i)
    for (int l = dranges[i].first; l < dranges[i].second; ++l) dblk[dfill[l]++] = (int)i;

  HM_TRY(P.lr.alloc(std::max<size_t>(h->h_lr.size(), 1)));
  HM_TRY(P.p1_items.alloc(2 * std::max<size_t>(items.size(), 1)));
  HM_TRY(P.leaf_ptr.alloc(nleaf + 1));
  HM_TRY(P.leaf_blk.alloc(blk.size()));
  HM_TRY(P.dense.alloc(std::max<size_t>(h->h_dense.size(), 1)));
  HM_TRY(P.leaf_dptr.alloc(nleaf + 1));
  HM_TRY(P.leaf_dblk.alloc(dblk.size()));
  HM_TRY(P.T.alloc(std::max<long long>(tk * nrhs_cap, 1)));
  HM_TRY(P.Xp.alloc((size_t)h->n * nrhs_cap));
  HM_TRY(P.Yp.alloc((size_t)h->n * nrhs_cap));
  if (!h->h_lr.empty())
    HM_CUDA(cudaMemcpyAsync(P.lr.p, h->h_lr.data(), sizeof(LRBlock) * h->h_lr.size(), cudaMemcpyHostToDevice,
                            stream));
  if (!items.empty())
    HM_CUDA(cudaMemcpyAsync(P.p1_items.p, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice,
                            stream));
  HM_CUDA(cudaMemcpyAsync(P.leaf_ptr.p, ptr.data(), 4 * (nleaf + 1), cudaMemcpyHostToDevice, stream));
  HM_CUDA(cudaMemcpyAsync(P.leaf_blk.p, blk.data(), 4 * blk.size(), cudaMemcpyHostToDevice, stream));
  if (!h->h_dense.empty())
    HM_CUDA(cudaMemcpyAsync(P.dense.p, h->h_dense.data(), sizeof(DenseBlock) * h->h_dense.size(),
                            cudaMemcpyHostToDevice, stream));
  HM_CUDA(cudaMemcpyAsync(P.leaf_dptr.p, dptr.data(), 4 * (nleaf + 1), cudaMemcpyHostToDevice, stream));
  HM_CUDA(cudaMemcpyAsync(P.leaf_dblk.p, dblk.data(), 4 * dblk.size(), cudaMemcpyHostToDevice, stream));
  HM_CUDA(cudaFuncSetAttribute(k_mv_expand, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)expand_smem(maxleaf, nrhs_cap)));
  HM_CUDA(cudaFuncSetAttribute(k_mv_project, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(sizeof(float) * (kMaxK * 33 + 32 * 33))));
  P.maxleaf = maxleaf;
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
  for (int c0 = 0; c0 < nrhs; c0 += P.nrhs_cap) {
    const int nr = std::min(P.nrhs_cap, nrhs - c0);
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
    if (P.t_per_rhs > 0) {
      HM_CUDA(cudaMemsetAsync(P.T.p, 0, sizeof(float) * (size_t)P.t_per_rhs * P.nrhs_cap, stream));
    }
    if (P.num_p1 > 0) {
      // T offsets were laid out for nrhs_cap columns; a narrower panel uses the
      // first nr*k entries of each block's slot
      k_mv_project<<<P.num_p1, kThreads, sizeof(float) * (kMaxK * 33 + 32 * 33), stream>>>(
          reinterpret_cast<const int2*>(P.p1_items.p), P.lr.p, Xt, ldxt, nr, P.T.p);
      HM_LAUNCH_CHECK();
    }
    k_mv_expand<<<P.num_leaves, kThreads, expand_smem(P.maxleaf, nr), stream>>>(
        h->tree->offsets.p, P.leaf_ptr.p, P.leaf_blk.p, P.lr.p, P.leaf_dptr.p, P.leaf_dblk.p, P.dense.p, P.T.p,
        Xt, ldxt, Yt, ldyt, nr);
    HM_LAUNCH_CHECK();
    if (original_order) {
      k_scatter_rows<<<592, 256, 0, stream>>>(P.Yp.p, h->tree->perm.p, n, nr, Yout, ldy);
      HM_LAUNCH_CHECK();
    }
  }
  return HM_OK;
}

// Algorithmic bytes of one product with nrhs FP32 columns: factors and dense
// blocks read once, X read once and Y written once per phase that touches them.
void matvec_bytes(hm_hmatrix h, int nrhs, long long* b_project, long long* b_expand) {
  long long p1 = 0, p2 = 0;
  for (const auto& b : h->h_lr) {
    p1 += 4ll * b.n * b.k;
    p2 += 4ll * b.m * b.k;
  }
  for (const auto& d : h->h_dense) p2 += 4ll * d.m * d.n;
  p1 += 4ll * h->n * nrhs;      // X
  p2 += 4ll * h->n * nrhs * 2;  // X (dense blocks) and Y
  *b_project = p1;
  *b_expand = p2;
}

}  // namespace hm

extern "C" hm_status hm_hmatvec_profile(hm_hmatrix h, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                        void* stream, float* ms_project, float* ms_expand,
                                        long long* bytes_project, long long* bytes_expand) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatvec_profile: null matrix");
  if (nrhs < 1 || nrhs > h->plan.nrhs_cap || !X || !Y || ldx < h->n || ldy < h->n)
    return hm::fail(HM_ERR_INVALID, "hm_hmatvec_profile: bad vector arguments (nrhs <= panel width)");
  cudaStream_t s = hm::as_stream(stream);
  hm::MatvecPlan& P = h->plan;
  cudaEvent_t e[3];
  for (auto& x : e) HM_CUDA(cudaEventCreate(&x));
  if (P.t_per_rhs > 0) HM_CUDA(cudaMemsetAsync(P.T.p, 0, sizeof(float) * (size_t)P.t_per_rhs * P.nrhs_cap, s));
  HM_CUDA(cudaEventRecord(e[0], s));
  if (P.num_p1 > 0)
    hm::k_mv_project<<<P.num_p1, hm::kThreads, sizeof(float) * (hm::kMaxK * 33 + 32 * 33), s>>>(
        reinterpret_cast<const int2*>(P.p1_items.p), P.lr.p, X, ldx, nrhs, P.T.p);
  HM_LAUNCH_CHECK();
  HM_CUDA(cudaEventRecord(e[1], s));
  hm::k_mv_expand<<<P.num_leaves, hm::kThreads, hm::expand_smem(P.maxleaf, nrhs), s>>>(
      h->tree->offsets.p, P.leaf_ptr.p, P.leaf_blk.p, P.lr.p, P.leaf_dptr.p, P.leaf_dblk.p, P.dense.p, P.T.p, X,
      ldx, Y, ldy, nrhs);
  HM_LAUNCH_CHECK();
  HM_CUDA(cudaEventRecord(e[2], s));
  HM_CUDA(cudaEventSynchronize(e[2]));
  float a = 0, b = 0;
  HM_CUDA(cudaEventElapsedTime(&a, e[0], e[1]));
  HM_CUDA(cudaEventElapsedTime(&b, e[1], e[2]));
  for (auto& x : e) cudaEventDestroy(x);
  if (ms_project) *ms_project = a;
  if (ms_expand) *ms_expand = b;
  long long bp = 0, be = 0;
  hm::matvec_bytes(h, nrhs, &bp, &be);
  if (bytes_project) *bytes_project = bp;
  if (bytes_expand) *bytes_expand = be;
  return HM_OK;
}

namespace hm {
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

// The product of hm_hmatvec (tree order) with its projection workspace taken
// from the library's static scratch instead of the matrix's own buffer; no
// allocation of any kind.
extern "C" hm_status hm_hmatvec_noalloc(hm_hmatrix h, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                        void* stream) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatvec_noalloc: null matrix");
  if (nrhs < 1 || !X || !Y || ldx < h->n || ldy < h->n)
    return hm::fail(HM_ERR_INVALID, "hm_hmatvec_noalloc: bad vector arguments");
  hm::MatvecPlan& P = h->plan;
  const size_t need = (size_t)P.t_per_rhs * (size_t)P.nrhs_cap;
  if (need > hm::kNoallocScratchFloats)
    return hm::fail(HM_ERR_UNSUPPORTED,
                    "hm_hmatvec_noalloc: this matrix needs " + std::to_string(need) +
                        " floats of projection scratch (sum of ranks x panel width); the static scratch holds " +
                        std::to_string(hm::kNoallocScratchFloats) + " (16 MiB)");
  float* T = nullptr;
  HM_TRY(hm::noalloc_scratch(&T));
  cudaStream_t s = hm::as_stream(stream);
  for (int c0 = 0; c0 < nrhs; c0 += P.nrhs_cap) {
    const int nr = std::min(P.nrhs_cap, nrhs - c0);
    const float* Xin = X + (size_t)c0 * ldx;
    float* Yout = Y + (size_t)c0 * ldy;
    // the scratch keeps the previous call's contents: the projections must start at zero
    if (need > 0) HM_CUDA(cudaMemsetAsync(T, 0, sizeof(float) * need, s));
    if (P.num_p1 > 0) {
      hm::k_mv_project<<<P.num_p1, hm::kThreads, sizeof(float) * (hm::kMaxK * 33 + 32 * 33), s>>>(
          reinterpret_cast<const int2*>(P.p1_items.p), P.lr.p, Xin, ldx, nr, T);
      HM_LAUNCH_CHECK();
    }
    hm::k_mv_expand<<<P.num_leaves, hm::kThreads, hm::expand_smem(P.maxleaf, nr), s>>>(
        h->tree->offsets.p, P.leaf_ptr.p, P.leaf_blk.p, P.lr.p, P.leaf_dptr.p, P.leaf_dblk.p, P.dense.p, T, Xin,
        ldx, Yout, ldy, nr);
    HM_LAUNCH_CHECK();
  }
  return HM_OK;
}

extern "C" hm_status hm_hmatvec(hm_hmatrix h, int trans, int nrhs, const float* X, int ldx, float* Y, int ldy,
                                int original_order, void* stream) {
  return hm::hmatvec(h, trans, nrhs, X, ldx, Y, ldy, original_order, hm::as_stream(stream));
}
