// hm_autotune.cu -- schedule autotuner for the H-matvec, with a file cache.
//
// The product's schedule has a few free parameters that change its speed but
// not what it computes (up to the order of FP32 sums): for the mixed form the
// phase-1 unit shape (row tiles x column tiles) and the phase-1 kernel; for the
// FP32 form the kernels themselves -- panels with a phase-1 unit shape, or
// the per-block kernels with the rows of V per phase-1 item.  hm_autotune times every candidate on the matrix at
// hand with CUDA events, keeps the fastest, and appends it to a cache file
// under a key made of the GPU and the matrix's shape; a later call with the
// same key (the same workload on the same GPU) applies the cached choice
// without timing anything.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "hm_hmatrix.h"

namespace hm {

hm_status matvec_plan_build(hm_hmatrix h, int nrhs_cap, cudaStream_t stream);
int pass_width(hm_hmatrix h);

namespace {

// mixed: (chunk tiles, group tiles, ring phase 1); FP32 panels: (chunk tiles,
// group tiles >= 1, 0); FP32 per-block kernels: (p1 rows, 0, 0)
struct Choice {
  int a = 0, b = 0, c = 0;
  int d = -1;  // mixed: tcgen05 phase 1 for 128-column passes (1 on, 0 off, -1 unchanged)
};

bool is_mixed(hm_hmatrix h) { return h->opts.precision == HM_PREC_MIXED; }

std::string describe(hm_hmatrix h, const Choice& c) {
  char buf[96];
  if (is_mixed(h))
    std::snprintf(buf, sizeof buf, "mixed chunk_tiles=%d group_tiles=%d p1_ring=%d wide_tc=%d tc_chunk=%d", c.a, c.b,
                  c.c, c.d >= 0 ? c.d : (h->mx.wide_tc ? 1 : 0), h->mx.tc_chunk_tiles);
  else if (c.b > 0)
    std::snprintf(buf, sizeof buf, "fp32 chunk_tiles=%d group_tiles=%d", c.a, c.b);
  else
    std::snprintf(buf, sizeof buf, "fp32 p1_rows=%d", c.a);
  return buf;
}

hm_status apply(hm_hmatrix h, const Choice& c, cudaStream_t s) {
  if (is_mixed(h) || c.b > 0) {
    h->mx.enabled = true;
    if (c.d >= 0) h->mx.wide_tc = c.d != 0;
    HM_TRY(mixed_schedule(h, c.a, c.b, c.c, s));
  } else {
    h->mx.enabled = false;  // the FP32 per-block kernels
    h->plan.p1_rows = c.a;
  }
  return matvec_plan_build(h, 16, s);
}

std::string shape_key(hm_hmatrix h, int nrhs) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp pr{};
  cudaGetDeviceProperties(&pr, dev);
  std::ostringstream k;
  std::string name = pr.name;
  for (char& ch : name)
    if (ch == ' ' || ch == '\t') ch = '_';
  k << name << "/sm" << pr.multiProcessorCount << "/" << (is_mixed(h) ? "mixed" : "fp32") << "/n" << h->n
    << "/d" << h->d << "/depth" << h->depth << "/lr" << h->stats.num_lowrank << "/ranks" << h->stats.rank_sum
    << "/dense" << h->stats.num_dense << "/nrhs" << nrhs;
  return k.str();
}

bool lookup(const char* path, const std::string& key, Choice* c) {
  std::ifstream f(path);
  std::string line;
  bool found = false;
  while (std::getline(f, line)) {  // the last entry of a key wins
    std::istringstream ls(line);
    std::string k;
    Choice x;
    if ((ls >> k >> x.a >> x.b >> x.c) && k == key) {
      *c = x;
      found = true;
    }
  }
  return found;
}

}  // namespace
}  // namespace hm

extern "C" hm_status hm_autotune(hm_hmatrix h, int nrhs, const char* cache_path, void* stream, int* from_cache,
                                 char* choice, int choice_len) {
  using namespace hm;
  if (!h) return fail(HM_ERR_INVALID, "hm_autotune: null matrix");
  if (nrhs < 1 || nrhs > pass_width(h))
    return fail(HM_ERR_INVALID, "hm_autotune: need 1 <= nrhs <= one pass of the product (16, or 128 for the mixed form)");
  cudaStream_t s = as_stream(stream);
  const std::string key = shape_key(h, nrhs);
  Choice best;
  bool cached = cache_path && lookup(cache_path, key, &best);
  if (!cached) {
    std::vector<Choice> cand;
    if (is_mixed(h)) {
      for (int ring : {1, 0})
        for (int ch : {16, 32, 64, 128})
          for (int g : {4, 8}) cand.push_back(Choice{ch, g, ring});
    } else {
      for (int ch : {16, 32, 64, 128})
        for (int g : {2, 4}) cand.push_back(Choice{ch, g, 0});
      for (int r : {256, 1024}) cand.push_back(Choice{r, 0, 0});
    }
    DevBuf<float> X, Y;
    HM_TRY(X.alloc((size_t)h->n * nrhs));
    HM_TRY(Y.alloc((size_t)h->n * nrhs));
    HM_CUDA(cudaMemsetAsync(X.p, 0, sizeof(float) * (size_t)h->n * nrhs, s));
    cudaEvent_t e0, e1;
    HM_CUDA(cudaEventCreate(&e0));
    HM_CUDA(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    for (const Choice& c : cand) {
      hm_status st = apply(h, c, s);
      if (st) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return st;
      }
      for (int w = 0; w < 2; ++w) HM_TRY(hm_hmatvec(h, 0, nrhs, X.p, h->n, Y.p, h->n, 0, s));
      HM_CUDA(cudaEventRecord(e0, s));
      const int reps = 5;
      for (int r = 0; r < reps; ++r) HM_TRY(hm_hmatvec(h, 0, nrhs, X.p, h->n, Y.p, h->n, 0, s));
      HM_CUDA(cudaEventRecord(e1, s));
      HM_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      HM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      ms /= reps;
      if (ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cache_path) {
      std::ofstream f(cache_path, std::ios::app);
      if (!f) return fail(HM_ERR_INVALID, std::string("hm_autotune: cannot write the cache ") + cache_path);
      f << key << " " << best.a << " " << best.b << " " << best.c << " " << best_ms << "\n";
    }
  }
  HM_TRY(apply(h, best, s));
  if (from_cache) *from_cache = cached ? 1 : 0;
  if (choice && choice_len > 0) {
    const std::string d = describe(h, best);
    std::strncpy(choice, d.c_str(), (size_t)choice_len - 1);
    choice[choice_len - 1] = '\0';
  }
  return HM_OK;
}

extern "C" hm_status hm_schedule_set(hm_hmatrix h, const char* choice, void* stream) {
  using namespace hm;
  if (!h || !choice) return fail(HM_ERR_INVALID, "hm_schedule_set: null argument");
  Choice c;
  if (is_mixed(h)) {
    int tcc = 0;
    const int got = std::sscanf(choice, "mixed chunk_tiles=%d group_tiles=%d p1_ring=%d wide_tc=%d tc_chunk=%d", &c.a,
                                &c.b, &c.c, &c.d, &tcc);
    if (got == 5) {
      if (tcc < 1) return fail(HM_ERR_INVALID, std::string("hm_schedule_set: tc_chunk must be >= 1: ") + choice);
      h->mx.tc_chunk_tiles = tcc;
    }
    if (got < 3 || (got >= 4 && c.d != 0 && c.d != 1))
      return fail(HM_ERR_INVALID, std::string("hm_schedule_set: not a mixed-form schedule: ") + choice);
  } else if (std::sscanf(choice, "fp32 chunk_tiles=%d group_tiles=%d", &c.a, &c.b) == 2) {
    if (c.b < 1 || c.b > 8)
      return fail(HM_ERR_INVALID, std::string("hm_schedule_set: group_tiles must be 1..8: ") + choice);
  } else {
    c = Choice{};
    if (std::sscanf(choice, "fp32 p1_rows=%d", &c.a) != 1 || c.a < 16)
      return fail(HM_ERR_INVALID, std::string("hm_schedule_set: not an FP32-form schedule: ") + choice);
  }
  return apply(h, c, as_stream(stream));
}
