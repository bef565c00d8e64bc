// hm_structure.cu -- admissibility test and H-matrix block structure, built on
// the device.
//
// Reference: constructMatrixStruct_recursive (src/HMatrixStructure.cu:9-90)
// walks (column cluster u, row cluster v) pairs depth first from the root; a
// diagonal leaf pair stops, a leaf pair or an admissible pair is appended to
// its level's list as the Morton index interleave(u) | interleave(v) << 1,
// anything else recurses into (u0,v0),(u1,v0),(u0,v1),(u1,v1).  Those four
// children are the four values of the next Morton digit in increasing order,
// so each level's list is in ascending Morton order.
//
// Here the walk is level synchronous: a frontier of pairs (ascending Morton)
// is classified in parallel and compacted stably, so both the recorded list
// and the next frontier stay in ascending Morton order and the lists equal the
// reference's bit for bit.  The admissibility arithmetic uses explicitly
// rounded double operations in the reference's evaluation order
// (src/admissibilityCondition.cu:7-52) so no FMA contraction changes a
// decision.  On top of the lists the builder derives, on the device, a
// row-major (CSR) and a jagged-diagonal (JDS) layout of every level.
#include <algorithm>
#include <numeric>

#include "hm_internal.h"
#include "hm_sort.h"
#include "hm_structure.h"

namespace hm {
namespace {

constexpr int kThreads = 256;

// box-center admissibility, src/admissibilityCondition.cu:7-52
__device__ bool box_center_admissible(const double* umin, const double* umax, const double* vmin,
                                      const double* vmax, int d, double eta) {
  double distance = 0.0;
  for (int i = 0; i < d; ++i) {
    double cu = __dadd_rn(umax[i], umin[i]);
    double cv = __dadd_rn(vmax[i], vmin[i]);
    double c = __dmul_rn(0.5, __dsub_rn(cu, cv));
    distance = __dadd_rn(distance, __dmul_rn(c, c));
  }
  distance = __dsqrt_rn(distance);
  double du = 0.0, dv = 0.0;
  for (int i = 0; i < d; ++i) {
    double e = __dsub_rn(umax[i], umin[i]);
    du = __dadd_rn(du, __dmul_rn(e, e));
  }
  for (int i = 0; i < d; ++i) {
    double e = __dsub_rn(vmax[i], vmin[i]);
    dv = __dadd_rn(dv, __dmul_rn(e, e));
  }
  du = __dsqrt_rn(du);
  dv = __dsqrt_rn(dv);
  if (du == 0.0 || dv == 0.0) return false;
  return __dmul_rn(0.5, __dadd_rn(du, dv)) <= __dmul_rn(eta, distance);
}

struct ClassArgs {
  const uint32_t* frontier;
  int nf;
  int level, depth, d, admiss;
  double eta;
  const double* bmin;
  const double* bmax;
};

// 0 = drop (diagonal leaf), 1 = record, 2 = refine
__device__ int classify(const ClassArgs& a, uint32_t z) {
  uint32_t u = compact16(z), v = compact16(z >> 1);
  bool diag = u == v;
  bool leaf = a.level == a.depth;
  if (diag && leaf) return 0;
  if (leaf) return 1;
  if (diag) return 2;
  if (a.admiss == HM_ADMISS_WEAK) return 1;
  size_t base = (size_t)((1u << a.level) - 1u) * a.d;
  bool adm = box_center_admissible(a.bmin + base + (size_t)u * a.d, a.bmax + base + (size_t)u * a.d,
                                   a.bmin + base + (size_t)v * a.d, a.bmax + base + (size_t)v * a.d,
                                   a.d, a.eta);
  return adm ? 1 : 2;
}

__global__ void __launch_bounds__(kThreads) k_classify_count(ClassArgs a, unsigned int* cnt_rec,
                                                             unsigned int* cnt_ref) {
  __shared__ unsigned int sr, sf;
  if (threadIdx.x == 0) sr = sf = 0;
  __syncthreads();
  int i = blockIdx.x * kThreads + threadIdx.x;
  int c = i < a.nf ? classify(a, a.frontier[i]) : 0;
  unsigned int br = __ballot_sync(0xffffffffu, c == 1);
  unsigned int bf = __ballot_sync(0xffffffffu, c == 2);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&sr, __popc(br));
    atomicAdd(&sf, __popc(bf));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cnt_rec[blockIdx.x] = sr;
    cnt_ref[blockIdx.x] = sf;
  }
}

__global__ void __launch_bounds__(kThreads) k_classify_scatter(ClassArgs a, const unsigned int* off_rec,
                                                               const unsigned int* off_ref,
                                                               uint32_t* rec_out, uint32_t* next_out) {
  __shared__ unsigned int wr[kThreads / 32], wf[kThreads / 32];
  int i = blockIdx.x * kThreads + threadIdx.x;
  uint32_t z = i < a.nf ? a.frontier[i] : 0u;
  int c = i < a.nf ? classify(a, z) : 0;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned int br = __ballot_sync(0xffffffffu, c == 1);
  unsigned int bf = __ballot_sync(0xffffffffu, c == 2);
  if (lane == 0) {
    wr[warp] = __popc(br);
    wf[warp] = __popc(bf);
  }
  __syncthreads();
  unsigned int pr = 0, pf = 0;
  for (int w = 0; w < warp; ++w) {
    pr += wr[w];
    pf += wf[w];
  }
  unsigned int lt = (1u << lane) - 1u;
  if (c == 1) rec_out[off_rec[blockIdx.x] + pr + __popc(br & lt)] = z;
  if (c == 2) {
    unsigned int o = 4u * (off_ref[blockIdx.x] + pf + __popc(bf & lt));
    for (uint32_t q = 0; q < 4; ++q) next_out[o + q] = 4u * z + q;
  }
}

__global__ void k_row_keys(const uint32_t* tiles, int n, uint32_t* keys, uint32_t* vals,
                           unsigned int* row_cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t v = compact16(tiles[i] >> 1);
  keys[i] = v;
  vals[i] = (uint32_t)i;
  atomicAdd(&row_cnt[v], 1u);
}

// JDS row order key: rows with more blocks first, ties by row index (stable sort)
__global__ void k_jds_keys(const unsigned int* row_cnt, int nrows, unsigned int maxc,
                           uint32_t* keys, uint32_t* vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  keys[i] = maxc - row_cnt[i];
  vals[i] = (uint32_t)i;
}

__global__ void k_diag_count(const unsigned int* row_cnt, int nrows, unsigned int* diag_len) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  for (unsigned int j = 0; j < row_cnt[i]; ++j) atomicAdd(&diag_len[j], 1u);
}

// jds_blk[jds_ptr[j] + r] = j-th block (column order) of the r-th row in JDS order
__global__ void k_jds_fill(const uint32_t* jds_rows, int nrows, const unsigned int* row_ptr,
                           const uint32_t* csr_blk, const unsigned int* jds_ptr, uint32_t* jds_blk) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  uint32_t row = jds_rows[r];
  unsigned int b0 = row_ptr[row], b1 = row_ptr[row + 1];
  for (unsigned int j = 0; j < b1 - b0; ++j) jds_blk[jds_ptr[j] + r] = csr_blk[b0 + j];
}

int ceil_log2(unsigned int x) {
  int b = 0;
  while ((1u << b) < x) ++b;
  return b;
}

}  // namespace

hm_status structure_build(hm_kdtree t, int admiss, double eta, cudaStream_t stream,
                          hm_structure* out) {
  if (!out) return fail(HM_ERR_INVALID, "hm_structure_build: out is NULL");
  *out = nullptr;
  if (!t) return fail(HM_ERR_INVALID, "hm_structure_build: null tree");
  if (admiss != HM_ADMISS_WEAK && admiss != HM_ADMISS_BOX_CENTER)
    return fail(HM_ERR_INVALID, "hm_structure_build: unknown admissibility");
  if (t->depth > 16)
    return fail(HM_ERR_UNSUPPORTED, "hm_structure_build: Morton indices hold 16 levels");
  auto* s = new hm_structure_s();
  auto cleanup = [&](hm_status st) {
    delete s;
    return st;
  };
  s->tree = t;
  s->depth = t->depth;
  s->num_levels = t->depth + 1;
  s->admiss = admiss;
  // the reference passes eta as float (src/admissibilityCondition.cuh:7-12)
  s->eta = (double)(float)eta;
  const int depth = t->depth;
  s->count.assign(depth, 0);
  s->start.assign(depth + 1, 0);

  std::vector<DevBuf<uint32_t>> lists(depth);
  DevBuf<uint32_t> front, next;
  DevBuf<unsigned int> crec, cref;
  hm_status st;
  if ((st = front.alloc_async(1, stream))) return cleanup(st);
  uint32_t zero = 0;
  HM_CUDA(cudaMemcpyAsync(front.p, &zero, 4, cudaMemcpyHostToDevice, stream));
  long long nf = 1;
  for (int level = 0; level <= depth && nf > 0; ++level) {
    ClassArgs a;
    a.frontier = front.p;
    a.nf = (int)nf;
    a.level = level;
    a.depth = depth;
    a.d = t->d;
    a.admiss = admiss;
    a.eta = s->eta;
    a.bmin = t->bmin.p;
    a.bmax = t->bmax.p;
    int nb = (int)((nf + kThreads - 1) / kThreads);
    if ((st = crec.alloc_async(nb, stream)) || (st = cref.alloc_async(nb, stream))) return cleanup(st);
    k_classify_count<<<nb, kThreads, 0, stream>>>(a, crec.p, cref.p);
    HM_LAUNCH_CHECK();
    std::vector<unsigned int> hr(nb), hf(nb);
    HM_CUDA(cudaMemcpyAsync(hr.data(), crec.p, 4 * nb, cudaMemcpyDeviceToHost, stream));
    HM_CUDA(cudaMemcpyAsync(hf.data(), cref.p, 4 * nb, cudaMemcpyDeviceToHost, stream));
    HM_CUDA(cudaStreamSynchronize(stream));
    unsigned long long trec = 0, tref = 0;
    for (int b = 0; b < nb; ++b) {
      unsigned int x = hr[b], y = hf[b];
      hr[b] = (unsigned int)trec;
      hf[b] = (unsigned int)tref;
      trec += x;
      tref += y;
    }
    if (4ull * tref > 0x7fffffffull) return cleanup(fail(HM_ERR_UNSUPPORTED, "structure too large"));
    HM_CUDA(cudaMemcpyAsync(crec.p, hr.data(), 4 * nb, cudaMemcpyHostToDevice, stream));
    HM_CUDA(cudaMemcpyAsync(cref.p, hf.data(), 4 * nb, cudaMemcpyHostToDevice, stream));
    DevBuf<uint32_t> rec;
    if (level >= 1 && trec > 0) {
      if ((st = rec.alloc_async(trec, stream))) return cleanup(st);
    }
    if ((st = next.alloc_async(std::max<unsigned long long>(4 * tref, 1), stream))) return cleanup(st);
    k_classify_scatter<<<nb, kThreads, 0, stream>>>(a, crec.p, cref.p, rec.p, next.p);
    HM_LAUNCH_CHECK();
    HM_CUDA(cudaStreamSynchronize(stream));
    if (level >= 1) {
      s->count[level - 1] = (int)trec;
      lists[level - 1] = std::move(rec);
    }
    std::swap(front, next);
    nf = 4 * (long long)tref;
  }
  long long total = 0;
  for (int l = 0; l < depth; ++l) {
    s->start[l] = total;
    total += s->count[l];
  }
  s->start[depth] = total;
  if ((st = s->tiles.alloc(std::max<long long>(total, 1)))) return cleanup(st);
  for (int l = 0; l < depth; ++l)
    if (s->count[l])
      HM_CUDA(cudaMemcpyAsync(s->tiles.p + s->start[l], lists[l].p, 4 * (size_t)s->count[l],
                              cudaMemcpyDeviceToDevice, stream));

  // ---- row-major (CSR) and jagged-diagonal (JDS) layouts per level --------
  // row_ptr: level l occupies 2^l + 1 entries at rstart[l]; csr_blk / jds_blk:
  // block indices (into the level's Morton list) at start[l]; jds_rows: 2^l at
  // rows_start[l]; jds_ptr: per level (max blocks per row + 1) entries.
  s->rstart.assign(depth + 1, 0);
  s->rows_start.assign(depth + 1, 0);
  long long rtot = 0, rowtot = 0;
  for (int l = 1; l <= depth; ++l) {
    s->rstart[l - 1] = rtot;
    rtot += (1ll << l) + 1;
    s->rows_start[l - 1] = rowtot;
    rowtot += 1ll << l;
  }
  s->rstart[depth] = rtot;
  s->rows_start[depth] = rowtot;
  if ((st = s->row_ptr.alloc(std::max<long long>(rtot, 1))) ||
      (st = s->csr_blk.alloc(std::max<long long>(total, 1))) ||
      (st = s->jds_blk.alloc(std::max<long long>(total, 1))) ||
      (st = s->jds_rows.alloc(std::max<long long>(rowtot, 1))))
    return cleanup(st);
  HM_CUDA(cudaMemsetAsync(s->row_ptr.p, 0, 4 * s->row_ptr.n, stream));
  s->jds_maxc.assign(depth, 0);
  std::vector<std::vector<unsigned int>> hptr(depth);
  for (int l = 1; l <= depth; ++l) {
    const int nrows = 1 << l;
    const int nb = s->count[l - 1];
    unsigned int* rp = s->row_ptr.p + s->rstart[l - 1];
    uint32_t* rows = s->jds_rows.p + s->rows_start[l - 1];
    if (nb == 0) {
      k_jds_keys<<<(nrows + 255) / 256, 256, 0, stream>>>(rp, nrows, 0, rows, rows);
      continue;
    }
    DevBuf<uint32_t> keys, vals;
    if ((st = keys.alloc_async(std::max(nb, nrows), stream)) || (st = vals.alloc_async(std::max(nb, nrows), stream)))
      return cleanup(st);
    k_row_keys<<<(nb + 255) / 256, 256, 0, stream>>>(s->tiles.p + s->start[l - 1], nb, keys.p, vals.p,
                                                     rp);
    HM_LAUNCH_CHECK();
    if ((st = sort_pairs_u32(keys.p, vals.p, nb, l, stream))) return cleanup(st);
    HM_CUDA(cudaMemcpyAsync(s->csr_blk.p + s->start[l - 1], vals.p, 4 * (size_t)nb,
                            cudaMemcpyDeviceToDevice, stream));
    // rows sorted by block count (descending), then JDS diagonal lengths
    std::vector<unsigned int> hcnt(nrows);
    HM_CUDA(cudaMemcpyAsync(hcnt.data(), rp, 4 * (size_t)nrows, cudaMemcpyDeviceToHost, stream));
    HM_CUDA(cudaStreamSynchronize(stream));
    unsigned int maxc = *std::max_element(hcnt.begin(), hcnt.end());
    s->jds_maxc[l - 1] = (int)maxc;
    k_jds_keys<<<(nrows + 255) / 256, 256, 0, stream>>>(rp, nrows, maxc, keys.p, vals.p);
    HM_LAUNCH_CHECK();
    if ((st = sort_pairs_u32(keys.p, vals.p, nrows, ceil_log2(maxc + 1), stream))) return cleanup(st);
    HM_CUDA(cudaMemcpyAsync(rows, vals.p, 4 * (size_t)nrows, cudaMemcpyDeviceToDevice, stream));
    DevBuf<unsigned int> dlen;
    if ((st = dlen.alloc_async(maxc + 1, stream))) return cleanup(st);
    HM_CUDA(cudaMemsetAsync(dlen.p, 0, 4 * (size_t)(maxc + 1), stream));
    k_diag_count<<<(nrows + 255) / 256, 256, 0, stream>>>(rp, nrows, dlen.p);
    HM_LAUNCH_CHECK();
    // row counts -> row pointers (exclusive scan; the last entry is the total)
    if ((st = scan_exclusive(rp, nrows + 1, nullptr, stream))) return cleanup(st);
    if ((st = scan_exclusive(dlen.p, maxc + 1, nullptr, stream))) return cleanup(st);
    k_jds_fill<<<(nrows + 255) / 256, 256, 0, stream>>>(rows, nrows, rp, s->csr_blk.p + s->start[l - 1],
                                                        dlen.p, s->jds_blk.p + s->start[l - 1]);
    HM_LAUNCH_CHECK();
    hptr[l - 1].resize(maxc + 1);
    HM_CUDA(cudaMemcpyAsync(hptr[l - 1].data(), dlen.p, 4 * (size_t)(maxc + 1), cudaMemcpyDeviceToHost,
                            stream));
    HM_CUDA(cudaStreamSynchronize(stream));
  }
  // concatenate the JDS diagonal pointers
  s->jds_pstart.assign(depth + 1, 0);
  long long ptot = 0;
  for (int l = 0; l < depth; ++l) {
    s->jds_pstart[l] = ptot;
    ptot += (long long)hptr[l].size();
  }
  s->jds_pstart[depth] = ptot;
  if ((st = s->jds_ptr.alloc(std::max<long long>(ptot, 1)))) return cleanup(st);
  for (int l = 0; l < depth; ++l)
    if (!hptr[l].empty())
      HM_CUDA(cudaMemcpyAsync(s->jds_ptr.p + s->jds_pstart[l], hptr[l].data(), 4 * hptr[l].size(),
                              cudaMemcpyHostToDevice, stream));
  HM_CUDA(cudaStreamSynchronize(stream));
  *out = s;
  return HM_OK;
}

}  // namespace hm

extern "C" {

hm_status hm_structure_build(hm_kdtree t, int admissibility, double eta, void* stream,
                             hm_structure* out) {
  return hm::structure_build(t, admissibility, eta, hm::as_stream(stream), out);
}

hm_status hm_structure_info(hm_structure s, int* num_levels, int* counts) {
  if (!s) return hm::fail(HM_ERR_INVALID, "hm_structure_info: null structure");
  if (num_levels) *num_levels = s->num_levels;
  if (counts)
    for (int l = 0; l < s->depth; ++l) counts[l] = s->count[l];
  return HM_OK;
}

hm_status hm_structure_tiles(hm_structure s, int level, int* tiles) {
  if (!s) return hm::fail(HM_ERR_INVALID, "hm_structure_tiles: null structure");
  if (level < 1 || level > s->depth) return hm::fail(HM_ERR_INVALID, "hm_structure_tiles: bad level");
  if (!tiles) return hm::fail(HM_ERR_INVALID, "hm_structure_tiles: tiles is NULL");
  int n = s->count[level - 1];
  if (n) HM_CUDA(cudaMemcpy(tiles, s->tiles.p + s->start[level - 1], 4 * (size_t)n, cudaMemcpyDeviceToHost));
  return HM_OK;
}

hm_status hm_structure_jds(hm_structure s, int level, int* row_ptr, int* csr_blk, int* jds_rows,
                           int* jds_ptr, int* jds_blk, int* max_row_blocks) {
  if (!s) return hm::fail(HM_ERR_INVALID, "hm_structure_jds: null structure");
  if (level < 1 || level > s->depth) return hm::fail(HM_ERR_INVALID, "hm_structure_jds: bad level");
  int l = level - 1;
  int nrows = 1 << level;
  int nb = s->count[l];
  if (max_row_blocks) *max_row_blocks = s->jds_maxc[l];
  if (row_ptr)
    HM_CUDA(cudaMemcpy(row_ptr, s->row_ptr.p + s->rstart[l], 4 * (size_t)(nrows + 1), cudaMemcpyDeviceToHost));
  if (csr_blk && nb)
    HM_CUDA(cudaMemcpy(csr_blk, s->csr_blk.p + s->start[l], 4 * (size_t)nb, cudaMemcpyDeviceToHost));
  if (jds_rows)
    HM_CUDA(cudaMemcpy(jds_rows, s->jds_rows.p + s->rows_start[l], 4 * (size_t)nrows, cudaMemcpyDeviceToHost));
  if (jds_ptr && nb)
    HM_CUDA(cudaMemcpy(jds_ptr, s->jds_ptr.p + s->jds_pstart[l], 4 * (size_t)(s->jds_maxc[l] + 1),
                       cudaMemcpyDeviceToHost));
  if (jds_blk && nb)
    HM_CUDA(cudaMemcpy(jds_blk, s->jds_blk.p + s->start[l], 4 * (size_t)nb, cudaMemcpyDeviceToHost));
  return HM_OK;
}

void hm_structure_free(hm_structure s) { delete s; }

}  // extern "C"
