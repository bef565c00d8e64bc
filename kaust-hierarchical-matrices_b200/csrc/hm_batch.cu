// hm_batch.cu -- many independent point clouds as one H-matrix.
//
// The clouds become the subtrees of one forest: with C clouds and L0 =
// ceil(log2 C), cloud c is the cluster (L0, c) of a combined KD tree whose
// depth is L0 + max_c depth_c.  A cloud shallower than the deepest one keeps
// its leaves, each followed by empty virtual leaves down to the common depth,
// so that every cluster of cloud c at its level l is the combined cluster
// (L0 + l, c 2^l + a) with exactly the same rows.  The combined block
// structure is the union of the clouds' lists, renumbered that way; no block
// couples two clouds.  The ordinary build and product then run once over the
// concatenation: every ARA pass compresses blocks of all clouds in the same
// launches, and one product over all clouds is one set of kernel launches,
// which hm_batch_matvec records once into a CUDA graph and relaunches.
#include <algorithm>
#include <vector>

#include "hm_hmatrix.h"
#include "hm_structure.h"

struct hm_batch_s {
  int nclouds = 0, l0 = 0, depth = 0;
  std::vector<int> row_off;  // nclouds + 1
  hm_kdtree_s tree;          // the forest (owned)
  hm_structure_s st;         // its block structure (owned)
  hm_hmatrix H = nullptr;
  // one recorded product
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void* g_x = nullptr;
  void* g_y = nullptr;
  int g_nrhs = 0, g_ldx = 0, g_ldy = 0, g_orig = 0, g_gen = -1;
  cudaStream_t g_stream = nullptr;
  ~hm_batch_s() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (H) hm_hmatrix_free(H);
  }
};

namespace hm {
namespace {

__global__ void k_offset_perm(const int* src, int n, int off, int* dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i] + off;
}

hm_status batch_create(int nc, const hm_kdtree* trees, const hm_structure* sts, cudaStream_t s, hm_batch* out) {
  if (!out) return fail(HM_ERR_INVALID, "hm_batch_create: out is NULL");
  *out = nullptr;
  if (nc < 1 || !trees || !sts) return fail(HM_ERR_INVALID, "hm_batch_create: need at least one cloud");
  int d = -1, depth = 0, bucket = 0;
  long long ntot = 0;
  for (int c = 0; c < nc; ++c) {
    if (!trees[c] || !sts[c] || sts[c]->tree != trees[c])
      return fail(HM_ERR_INVALID, "hm_batch_create: cloud " + std::to_string(c) + " has no tree or structure");
    if (d >= 0 && trees[c]->d != d) return fail(HM_ERR_INVALID, "hm_batch_create: clouds differ in dimension");
    if (c > 0 && (sts[c]->admiss != sts[0]->admiss || sts[c]->eta != sts[0]->eta))
      return fail(HM_ERR_INVALID, "hm_batch_create: clouds differ in admissibility");
    d = trees[c]->d;
    depth = std::max(depth, trees[c]->depth);
    bucket = std::max(bucket, trees[c]->bucket);
    ntot += trees[c]->n;
  }
  int l0 = 0;
  while ((1 << l0) < nc) ++l0;
  const int D = l0 + depth;
  // Morton codes hold 16 bits per cluster index
  if (D > 16) return fail(HM_ERR_UNSUPPORTED, "hm_batch_create: the forest would be deeper than 16 levels");
  if (ntot > (1ll << 31) - 1) return fail(HM_ERR_UNSUPPORTED, "hm_batch_create: too many points");

  auto* b = new hm_batch_s();
  auto bail = [&](hm_status st) {
    delete b;
    return st;
  };
  b->nclouds = nc;
  b->l0 = l0;
  b->depth = D;
  b->row_off.assign(nc + 1, 0);
  for (int c = 0; c < nc; ++c) b->row_off[c + 1] = b->row_off[c] + trees[c]->n;

  // ---- the forest ----------------------------------------------------------
  hm_kdtree_s& T = b->tree;
  T.n = (int)ntot;
  T.d = d;
  T.bucket = bucket;
  T.depth = D;
  const long long nleaf = 1ll << D;
  T.h_offsets.assign(nleaf + 1, (int)ntot);
  for (long long y = 0; y < nleaf; ++y) {
    const int c = (int)(y >> depth);
    if (c >= nc) break;  // empty subtrees after the last cloud
    const int dc = trees[c]->depth;
    const long long yl = y & ((1ll << depth) - 1);
    const long long x = yl >> (depth - dc), sub = yl & ((1ll << (depth - dc)) - 1);
    const std::vector<int>& lo = trees[c]->h_offsets;
    T.h_offsets[y] = b->row_off[c] + (sub == 0 ? lo[x] : lo[x + 1]);
  }
  hm_status st;
  if ((st = T.offsets.alloc(nleaf + 1)) || (st = T.perm.alloc(std::max<long long>(ntot, 1))) ||
      (st = T.pts_tree_f.alloc(std::max<long long>(ntot * d, 1))) ||
      (st = T.pts_tree.alloc(std::max<long long>(ntot * d, 1))))
    return bail(st);
  HM_CUDA(cudaMemcpyAsync(T.offsets.p, T.h_offsets.data(), sizeof(int) * (nleaf + 1), cudaMemcpyHostToDevice, s));
  for (int c = 0; c < nc; ++c) {
    const hm_kdtree t = trees[c];
    if (t->n == 0) continue;
    for (int k = 0; k < d; ++k) {
      HM_CUDA(cudaMemcpyAsync(T.pts_tree_f.p + (size_t)k * ntot + b->row_off[c], t->pts_tree_f.p + (size_t)k * t->n,
                              sizeof(float) * t->n, cudaMemcpyDeviceToDevice, s));
      HM_CUDA(cudaMemcpyAsync(T.pts_tree.p + (size_t)k * ntot + b->row_off[c], t->pts_tree.p + (size_t)k * t->n,
                              sizeof(double) * t->n, cudaMemcpyDeviceToDevice, s));
    }
    k_offset_perm<<<std::min(1184, (t->n + 255) / 256), 256, 0, s>>>(t->perm.p, t->n, b->row_off[c],
                                                                      T.perm.p + b->row_off[c]);
    HM_LAUNCH_CHECK();
  }

  // ---- the structure: cloud (l, u, v) -> forest (l0 + l, c 2^l + u, c 2^l + v)
  hm_structure_s& S = b->st;
  S.tree = &T;
  S.depth = D;
  S.num_levels = D + 1;
  S.admiss = sts[0]->admiss;
  S.eta = sts[0]->eta;
  std::vector<std::vector<uint32_t>> lists(D + 1);
  for (int c = 0; c < nc; ++c) {
    const hm_structure sc = sts[c];
    const long long tot = sc->start.empty() ? 0 : sc->start[sc->depth];
    std::vector<uint32_t> tl(std::max<long long>(tot, 1));
    if (tot > 0) HM_CUDA(cudaMemcpy(tl.data(), sc->tiles.p, 4 * (size_t)tot, cudaMemcpyDeviceToHost));
    for (int l = 1; l <= sc->depth; ++l) {
      const uint32_t base = (uint32_t)c << l;
      for (long long i = sc->start[l - 1]; i < sc->start[l]; ++i) {
        const uint32_t u = compact16(tl[i]), v = compact16(tl[i] >> 1);
        lists[l0 + l].push_back(morton_encode(base + u, base + v));
      }
    }
  }
  S.count.assign(D, 0);
  S.start.assign(D + 1, 0);
  std::vector<uint32_t> all;
  for (int L = 1; L <= D; ++L) {
    std::sort(lists[L].begin(), lists[L].end());
    S.count[L - 1] = (int)lists[L].size();
    S.start[L] = S.start[L - 1] + (long long)lists[L].size();
    all.insert(all.end(), lists[L].begin(), lists[L].end());
  }
  if ((st = S.tiles.alloc(std::max<size_t>(all.size(), 1)))) return bail(st);
  if (!all.empty())
    HM_CUDA(cudaMemcpyAsync(S.tiles.p, all.data(), 4 * all.size(), cudaMemcpyHostToDevice, s));
  HM_CUDA(cudaStreamSynchronize(s));
  *out = b;
  return HM_OK;
}

}  // namespace
}  // namespace hm

extern "C" {

hm_status hm_batch_create(int nclouds, const hm_kdtree* trees, const hm_structure* structures, void* stream,
                          hm_batch* out) {
  return hm::batch_create(nclouds, trees, structures, hm::as_stream(stream), out);
}

hm_status hm_batch_info(hm_batch b, int* nclouds, int* n_total, int* depth, int* row_offsets) {
  if (!b) return hm::fail(HM_ERR_INVALID, "hm_batch_info: null batch");
  if (nclouds) *nclouds = b->nclouds;
  if (n_total) *n_total = b->tree.n;
  if (depth) *depth = b->depth;
  if (row_offsets) std::copy(b->row_off.begin(), b->row_off.end(), row_offsets);
  return HM_OK;
}

hm_status hm_batch_build(hm_batch b, const hm_build_opts* opts, void* stream) {
  if (!b) return hm::fail(HM_ERR_INVALID, "hm_batch_build: null batch");
  if (b->H) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    hm_hmatrix_free(b->H);
    b->H = nullptr;
  }
  return hm_hmatrix_build(&b->tree, &b->st, nullptr, opts, stream, &b->H);
}

hm_hmatrix hm_batch_hmatrix(hm_batch b) { return b ? b->H : nullptr; }

hm_status hm_batch_matvec(hm_batch b, int nrhs, const float* X, int ldx, float* Y, int ldy, int original_order,
                          void* stream) {
  if (!b || !b->H) return hm::fail(HM_ERR_INVALID, "hm_batch_matvec: batch not built");
  cudaStream_t s = hm::as_stream(stream);
  if (s == nullptr)
    return hm::fail(HM_ERR_INVALID, "hm_batch_matvec: needs a created stream (the legacy stream cannot be captured)");
  const bool same = b->exec && b->g_x == X && b->g_y == Y && b->g_nrhs == nrhs && b->g_ldx == ldx &&
                    b->g_ldy == ldy && b->g_orig == original_order && b->g_stream == s &&
                    b->g_gen == b->H->plan_gen;
  if (!same) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    // validate outside the capture so that a bad call fails before recording
    if (nrhs < 1 || !X || !Y || ldx < b->tree.n || ldy < b->tree.n)
      return hm::fail(HM_ERR_INVALID, "hm_batch_matvec: bad vector arguments");
    HM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    hm_status st = hm_hmatvec(b->H, 0, nrhs, X, ldx, Y, ldy, original_order, stream);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (st) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (ce != cudaSuccess) return hm::cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
    b->graph = g;
    HM_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    b->g_x = X;
    b->g_y = Y;
    b->g_nrhs = nrhs;
    b->g_ldx = ldx;
    b->g_ldy = ldy;
    b->g_orig = original_order;
    b->g_stream = s;
    b->g_gen = b->H->plan_gen;
  }
  HM_CUDA(cudaGraphLaunch(b->exec, s));
  return HM_OK;
}

void hm_batch_free(hm_batch b) { delete b; }

}  // extern "C"
