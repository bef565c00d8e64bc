// hm_io.cu -- binary H-matrix files: build once, apply many times.
//
// The reference only dumps text (src/helperFunctions.cu:76-169).  A file here
// holds what the product needs and the build cannot cheaply redo: the
// options, every stored low-rank pair (FP32 U, V) with its rank and the number
// of leading columns that keep a BF16 low part, and every dense block.  The
// factor data are the matrix's FP32 storage chunks, written raw; each block
// refers to its data by (chunk, offset).  The tree and the structure are not
// stored: they are rebuilt from the points in milliseconds, and the file
// carries a fingerprint of both (the permutation, the leaf offsets, the
// admissibility and the block lists) that loading checks.  Loading rebuilds
// the product's plans, and the BF16 panels for the mixed form, from the FP32
// factors exactly as the build does.
//
// Layout (host byte order):
//   char[8] "HMB200H1"; u32 version, sizeof(hm_build_opts), sizeof(hm_hmatrix_stats)
//   i32 n, d, depth, diag_fly; hm_build_opts; hm_hmatrix_stats; u64 fingerprint
//   i64 chunks; u64 floats[chunks]
//   i64 pairs;  {i32 level, r0, m, c0, n, k, khi, cu; i64 ou; i32 cv; i64 ov}[pairs]
//   i64 dense;  {i32 r0, m, c0, n, c; i64 o}[dense]
//   the chunks' floats, in order
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <vector>

#include "hm_hmatrix.h"
#include "hm_structure.h"

namespace hm {

hm_status matvec_plan_build(hm_hmatrix h, int nrhs_cap, cudaStream_t stream);

namespace {

constexpr char kMagic[8] = {'H', 'M', 'B', '2', '0', '0', 'H', '1'};
constexpr uint32_t kVersion = 2;  // 2: the block-row range (leaves) after the dimensions

uint64_t fnv(uint64_t hsh, const void* p, size_t bytes) {
  const unsigned char* c = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < bytes; ++i) {
    hsh ^= c[i];
    hsh *= 1099511628211ull;
  }
  return hsh;
}

// the tree (permutation, leaf offsets) and the structure (admissibility, eta,
// per-level block lists) the matrix was built on
hm_status fingerprint(hm_kdtree t, hm_structure s, uint64_t* out) {
  uint64_t hsh = 1469598103934665603ull;
  const int dims[4] = {t->n, t->d, t->bucket, t->depth};
  hsh = fnv(hsh, dims, sizeof dims);
  std::vector<int> perm((size_t)t->n);
  if (t->n > 0) HM_CUDA(cudaMemcpy(perm.data(), t->perm.p, sizeof(int) * perm.size(), cudaMemcpyDeviceToHost));
  hsh = fnv(hsh, perm.data(), sizeof(int) * perm.size());
  hsh = fnv(hsh, t->h_offsets.data(), sizeof(int) * t->h_offsets.size());
  hsh = fnv(hsh, &s->admiss, sizeof s->admiss);
  hsh = fnv(hsh, &s->eta, sizeof s->eta);
  const long long tot = s->start.empty() ? 0 : s->start.back();
  std::vector<uint32_t> tiles((size_t)tot);
  if (tot > 0) HM_CUDA(cudaMemcpy(tiles.data(), s->tiles.p, 4 * (size_t)tot, cudaMemcpyDeviceToHost));
  hsh = fnv(hsh, tiles.data(), 4 * tiles.size());
  hsh = fnv(hsh, s->count.data(), sizeof(int) * s->count.size());
  *out = hsh;
  return HM_OK;
}

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

#pragma pack(push, 1)
struct PairRec {
  int32_t level, r0, m, c0, n, k, khi, cu;
  int64_t ou;
  int32_t cv;
  int64_t ov;
};
struct DenseRec {
  int32_t r0, m, c0, n, c;
  int64_t o;
};
#pragma pack(pop)

}  // namespace
}  // namespace hm

extern "C" hm_status hm_hmatrix_save(hm_hmatrix h, const char* path) {
  using namespace hm;
  if (!h || !path) return fail(HM_ERR_INVALID, "hm_hmatrix_save: null argument");
  // every stored pair sits in h_lr as (block, mirror) at 2i, 2i + 1
  if (h->h_lr.size() % 2) return fail(HM_ERR_UNSUPPORTED, "hm_hmatrix_save: unpaired block list");
  // the storage chunks, or, once the mixed form released them, their ranges
  std::vector<std::pair<const float*, size_t>> chunks = h->chunk_meta;
  if (!h->fp32_released) {
    chunks.clear();
    for (const DevBuf<float>& b : h->storage) chunks.push_back({b.p, b.n});
  }
  auto locate = [&](const float* p, int32_t* c, int64_t* o) {
    for (size_t i = 0; i < chunks.size(); ++i) {
      const float* base = chunks[i].first;
      if (std::less_equal<const float*>()(base, p) && std::less<const float*>()(p, base + chunks[i].second)) {
        *c = (int32_t)i;
        *o = (int64_t)(p - base);
        return true;
      }
    }
    return false;
  };
  std::vector<PairRec> pairs;
  pairs.reserve(h->h_lr.size() / 2);
  for (size_t i = 0; i < h->h_lr.size(); i += 2) {
    const LRBlock& b = h->h_lr[i];
    const LRBlock& t = h->h_lr[i + 1];
    if (t.r0 != b.c0 || t.c0 != b.r0 || t.U != b.V || t.V != b.U)
      return fail(HM_ERR_UNSUPPORTED, "hm_hmatrix_save: block list not in (block, mirror) pairs");
    PairRec r{b.level, b.r0, b.m, b.c0, b.n, b.k, b.khi, 0, 0, 0, 0};
    if (!locate(b.U, &r.cu, &r.ou) || !locate(b.V, &r.cv, &r.ov))
      return fail(HM_ERR_UNSUPPORTED, "hm_hmatrix_save: a factor outside the matrix's storage");
    pairs.push_back(r);
  }
  std::vector<DenseRec> dense;
  for (const DenseBlock& d : h->h_dense) {
    DenseRec r{d.r0, d.m, d.c0, d.n, 0, 0};
    if (!locate(d.D, &r.c, &r.o)) return fail(HM_ERR_UNSUPPORTED, "hm_hmatrix_save: a dense block outside storage");
    dense.push_back(r);
  }
  uint64_t fp = 0;
  HM_TRY(fingerprint(h->tree, h->structure, &fp));

  File out;
  out.f = std::fopen(path, "wb");
  if (!out.f) return fail(HM_ERR_INVALID, std::string("hm_hmatrix_save: cannot open ") + path);
  bool ok = true;
  auto put = [&](const void* p, size_t bytes) {
    if (ok && bytes) ok = std::fwrite(p, 1, bytes, out.f) == bytes;
  };
  const uint32_t vers[3] = {kVersion, (uint32_t)sizeof(hm_build_opts), (uint32_t)sizeof(hm_hmatrix_stats)};
  const int32_t dims[4] = {h->n, h->d, h->depth, h->diag_fly ? 1 : 0};
  const int32_t leaves[2] = {h->leaf_lo, h->leaf_hi};  // the whole matrix, or a block-row shard
  put(kMagic, 8);
  put(vers, sizeof vers);
  put(dims, sizeof dims);
  put(leaves, sizeof leaves);
  put(&h->opts, sizeof h->opts);
  put(&h->stats, sizeof h->stats);
  put(&fp, sizeof fp);
  const int64_t nch = (int64_t)chunks.size();
  put(&nch, sizeof nch);
  for (const auto& c : chunks) {
    const uint64_t nf = c.second;
    put(&nf, sizeof nf);
  }
  const int64_t np = (int64_t)pairs.size(), nd = (int64_t)dense.size();
  put(&np, sizeof np);
  put(pairs.data(), sizeof(PairRec) * pairs.size());
  put(&nd, sizeof nd);
  put(dense.data(), sizeof(DenseRec) * dense.size());
  std::vector<float> stage((size_t)1 << 24);  // 64 MiB at a time
  // released chunks: every factor and dense block of a chunk rebuilt from the
  // panels into a device copy of the chunk (values that convert back to the
  // same tiles), then written like a stored chunk
  std::vector<std::vector<std::pair<int, int64_t>>> per_chunk(chunks.size());  // (h_locs index, offset)
  if (h->fp32_released)
    for (size_t i = 0; i < h->mx.h_locs.size(); ++i) {
      int32_t c = 0;
      int64_t o = 0;
      if (!locate(h->mx.h_locs[i].key, &c, &o))
        return fail(HM_ERR_UNSUPPORTED, "hm_hmatrix_save: a panel block outside the matrix's storage");
      per_chunk[c].push_back({(int)i, o});
    }
  for (size_t ci = 0; ci < chunks.size() && ok; ++ci) {
    const float* src = chunks[ci].first;
    DevBuf<float> rebuilt;
    if (h->fp32_released) {
      HM_TRY(rebuilt.alloc(std::max<size_t>(chunks[ci].second, 1)));
      HM_CUDA(cudaMemset(rebuilt.p, 0, sizeof(float) * chunks[ci].second));
      std::vector<std::pair<int, float*>> jobs;
      for (const auto& lo : per_chunk[ci]) jobs.push_back({lo.first, rebuilt.p + lo.second});
      HM_TRY(mixed_unpack(h, jobs, nullptr));
      src = rebuilt.p;
    }
    for (size_t o = 0; ok && o < chunks[ci].second; o += stage.size()) {
      const size_t c = std::min(stage.size(), chunks[ci].second - o);
      HM_CUDA(cudaMemcpy(stage.data(), src + o, sizeof(float) * c, cudaMemcpyDeviceToHost));
      put(stage.data(), sizeof(float) * c);
    }
  }
  if (!ok) return fail(HM_ERR_INVALID, std::string("hm_hmatrix_save: write to ") + path + " failed");
  if (std::fclose(out.f) != 0) {
    out.f = nullptr;
    return fail(HM_ERR_INVALID, std::string("hm_hmatrix_save: closing ") + path + " failed");
  }
  out.f = nullptr;
  return HM_OK;
}

namespace hm {
namespace {

// The body of hm_hmatrix_load.  Every count read from the file is checked
// against the bytes the file has left before anything is sized by it, and
// every block's extent is checked in 64-bit arithmetic, so a damaged or
// foreign file is refused with HM_ERR_INVALID.
hm_status load_impl(hm_kdtree t, hm_structure s, const char* path, void* stream, hm_hmatrix* result) {
  if (!t || !s || !path) return fail(HM_ERR_INVALID, "hm_hmatrix_load: null argument");
  if (s->tree != t) return fail(HM_ERR_INVALID, "hm_hmatrix_load: structure was built on another tree");
  cudaStream_t st = as_stream(stream);
  File in;
  in.f = std::fopen(path, "rb");
  if (!in.f) return fail(HM_ERR_INVALID, std::string("hm_hmatrix_load: cannot open ") + path);
  long long fsize = -1;
  if (std::fseek(in.f, 0, SEEK_END) == 0) fsize = std::ftell(in.f);
  if (fsize < 0 || std::fseek(in.f, 0, SEEK_SET) != 0)
    return fail(HM_ERR_INVALID, std::string("hm_hmatrix_load: cannot size ") + path);
  long long pos = 0;
  bool ok = true;
  auto get = [&](void* p, size_t bytes) {
    if (ok && bytes) {
      ok = std::fread(p, 1, bytes, in.f) == bytes;
      pos += (long long)bytes;
    }
    return ok;
  };
  // at most `count` records of `size` bytes fit in what is left of the file
  auto fits = [&](long long count, size_t size) { return count >= 0 && count <= (fsize - pos) / (long long)size; };
  auto bad = [&](const std::string& why) { return fail(HM_ERR_INVALID, "hm_hmatrix_load: " + why + ": " + path); };
  char magic[8];
  uint32_t vers[3];
  int32_t dims[4], leaves[2];
  if (!get(magic, 8) || std::memcmp(magic, kMagic, 8) != 0) return bad("not an H-matrix file");
  if (!get(vers, sizeof vers) || vers[0] != kVersion || vers[1] != sizeof(hm_build_opts) ||
      vers[2] != sizeof(hm_hmatrix_stats))
    return bad("written by another version of the library");
  std::unique_ptr<hm_hmatrix_s> h(new hm_hmatrix_s());
  uint64_t fp = 0, mine = 0;
  if (!get(dims, sizeof dims) || !get(leaves, sizeof leaves) || !get(&h->opts, sizeof h->opts) ||
      !get(&h->stats, sizeof h->stats) || !get(&fp, sizeof fp))
    return bad("truncated header");
  if (dims[0] != t->n || dims[1] != t->d || dims[2] != t->depth)
    return bad("the tree's size or depth differs from the one the matrix was built on");
  if (leaves[0] < 0 || leaves[0] >= leaves[1] || leaves[1] > (1 << t->depth)) return bad("bad block-row range");
  HM_TRY(fingerprint(t, s, &mine));
  if (mine != fp) return bad("the tree or structure differs from the one the matrix was built on");
  int64_t nch = 0;
  if (!get(&nch, sizeof nch) || nch < 0 || nch > (1 << 20) || !fits(nch, sizeof(uint64_t)))
    return bad("bad chunk count");
  std::vector<uint64_t> nf((size_t)nch);
  if (!get(nf.data(), sizeof(uint64_t) * nf.size())) return bad("truncated chunk table");
  int64_t np = 0, nd = 0;
  if (!get(&np, sizeof np) || !fits(np, sizeof(PairRec))) return bad("bad pair count");
  std::vector<PairRec> pairs((size_t)np);
  if (!get(pairs.data(), sizeof(PairRec) * pairs.size()) || !get(&nd, sizeof nd) || !fits(nd, sizeof(DenseRec)))
    return bad("truncated pair list");
  std::vector<DenseRec> dense((size_t)nd);
  if (!get(dense.data(), sizeof(DenseRec) * dense.size())) return bad("truncated dense list");
  // the factor data: what the chunk table claims must be what the file holds
  long long data_floats = 0;
  for (uint64_t c : nf) {
    if (c > (uint64_t)(fsize / 4)) return bad("bad chunk size");
    data_floats += (long long)c;
  }
  if (data_floats != (fsize - pos) / 4 || (fsize - pos) % 4 != 0) return bad("factor data of the wrong length");
  // every reference must lie inside its chunk
  auto inside = [&](int32_t c, int64_t o, long long len) {
    return c >= 0 && c < nch && o >= 0 && len >= 0 && (uint64_t)o + (uint64_t)len <= nf[c];
  };
  const long long n64 = t->n;
  for (const PairRec& r : pairs)
    if (r.m <= 0 || r.n <= 0 || r.k <= 0 || r.k > 256 || r.khi < 0 || r.khi > r.k || r.level < 1 ||
        r.level > t->depth || r.r0 < 0 || r.c0 < 0 || (long long)r.r0 + r.m > n64 || (long long)r.c0 + r.n > n64 ||
        !inside(r.cu, r.ou, (long long)r.m * r.k) || !inside(r.cv, r.ov, (long long)r.n * r.k))
      return bad("a low-rank pair outside the matrix or its data");
  for (const DenseRec& r : dense)
    if (r.m < 0 || r.n < 0 || r.r0 < 0 || r.c0 < 0 || (long long)r.r0 + r.m > n64 || (long long)r.c0 + r.n > n64 ||
        !inside(r.c, r.o, (long long)r.m * r.n))
      return bad("a dense block outside the matrix or its data");

  h->tree = t;
  h->structure = s;
  h->n = t->n;
  h->d = t->d;
  h->depth = t->depth;
  h->leaf_lo = leaves[0];
  h->leaf_hi = leaves[1];
  h->diag_fly = dims[3] != 0;
  h->kp.kind = h->opts.kernel;
  h->kp.deriv = h->opts.derivative ? 1 : 0;
  h->kp.ell = (float)h->opts.ell;
  h->kp.inv_ell = (float)(1.0 / h->opts.ell);
  h->kp.nugget = (float)h->opts.nugget;
  std::vector<float> stage((size_t)1 << 24);
  for (int64_t c = 0; c < nch; ++c) {
    DevBuf<float> b;
    HM_TRY(b.alloc(nf[c]));
    for (size_t o = 0; o < nf[c]; o += stage.size()) {
      const size_t k = std::min<size_t>(stage.size(), nf[c] - o);
      if (!get(stage.data(), sizeof(float) * k)) return bad("truncated factor data");
      HM_CUDA(cudaMemcpy(b.p + o, stage.data(), sizeof(float) * k, cudaMemcpyHostToDevice));
    }
    h->storage.push_back(std::move(b));
  }
  auto at = [&](int32_t c, int64_t o) -> const float* { return h->storage[c].p + o; };
  std::vector<MxPair> mp;
  for (const PairRec& r : pairs) {
    LRBlock b{};
    b.level = r.level;
    b.k = r.k;
    b.khi = r.khi;
    b.r0 = r.r0;
    b.m = r.m;
    b.c0 = r.c0;
    b.n = r.n;
    b.U = at(r.cu, r.ou);
    b.V = at(r.cv, r.ov);
    h->h_lr.push_back(b);
    LRBlock m = b;
    m.r0 = b.c0;
    m.m = b.n;
    m.c0 = b.r0;
    m.n = b.m;
    m.U = b.V;
    m.V = b.U;
    h->h_lr.push_back(m);
    mp.push_back(MxPair{r.level, r.r0, r.m, r.c0, r.n, r.k, r.khi, b.U, b.V});
  }
  for (const DenseRec& r : dense) h->h_dense.push_back(DenseBlock{r.r0, r.m, r.c0, r.n, 0, at(r.c, r.o)});
  {
    std::vector<MxDenseIn> md;
    for (const DenseBlock& db : h->h_dense) md.push_back(MxDenseIn{db.r0, db.m, db.c0, db.n, db.D});
    h->mx.fmt = h->opts.precision == HM_PREC_MIXED ? 0 : 1;
    HM_TRY(mixed_build(h.get(), mp, md, st));
    if (h->opts.precision == HM_PREC_MIXED) release_fp32(h.get());  // as the build does
  }
  HM_TRY(matvec_plan_build(h.get(), 16, st));
  HM_CUDA(cudaStreamSynchronize(st));
  *result = h.release();
  return HM_OK;
}

}  // namespace
}  // namespace hm

extern "C" hm_status hm_hmatrix_load(hm_kdtree t, hm_structure s, const char* path, void* stream,
                                     hm_hmatrix* result) {
  if (!result) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_load: out is NULL");
  *result = nullptr;
  try {
    return hm::load_impl(t, s, path, stream, result);
  } catch (const std::bad_alloc&) {
    return hm::fail(HM_ERR_NOMEM, "hm_hmatrix_load: out of host memory");
  }
}
