// hm_capi.cu -- the extern "C" surface of libhmb200.so, error reporting and
// point generation.
#include <curand_kernel.h>

#include <cmath>
#include <vector>

#include <cstdio>
#include <string>

#include "hm_internal.h"
#include "hm_kernels.cuh"

namespace hm {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

hm_status fail(hm_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

hm_status cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  g_last_error = buf;
  if (e == cudaErrorMemoryAllocation) return HM_ERR_NOMEM;
  return HM_ERR_CUDA;
}

// Point generation of the reference (src/generateDataset.cu:5-13): entry i of
// the SoA array is the first curand_uniform draw of a XORWOW state initialised
// with (seed, subsequence i, offset 0).
__global__ void k_generate_dataset(long long count, unsigned long long seed, double* out) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= count) return;
  curandState s;
  curand_init(seed, (unsigned long long)i, 0, &s);
  out[i] = curand_uniform(&s);
}

// Gaussian mixture point i, coordinate k: component by inverse CDF of the
// weights at a uniform draw, then centre + sigma * N(0,1); both draws from the
// counter-based hash generator (seed, point, coordinate).
__global__ void k_generate_mixture(int n, int d, int ncomp, uint32_t seed, const double* cum, const double* ctr,
                                   const double* sig, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double u = (mix32(seed ^ mix32((uint32_t)i * 0x9e3779b9u + 0x632be5abu)) >> 8) * (1.0 / 16777216.0);
  int c = 0;
  while (c + 1 < ncomp && u >= cum[c]) ++c;
  for (int k = 0; k < d; ++k)
    out[(size_t)k * n + i] = ctr[c * d + k] + sig[c] * (double)gauss_at(seed, 0x7f4a7c15u, (uint32_t)i, (uint32_t)k);
}

hm_status kdtree_build(const double* d_points, int n, int d, int bucket, cudaStream_t stream,
                       hm_kdtree* out);
hm_status structure_build(hm_kdtree t, int admiss, double eta, cudaStream_t stream,
                          hm_structure* out);

}  // namespace hm

extern "C" {

const char* hm_last_error(void) { return hm::g_last_error.c_str(); }

const char* hm_version(void) { return "hmb200 0.1.0 (sm_100a)"; }

hm_status hm_generate_dataset(int n, int d, unsigned long long seed, double* d_points,
                              void* stream) {
  if (!d_points) return hm::fail(HM_ERR_INVALID, "hm_generate_dataset: d_points is NULL");
  if (n < 1 || d < 1) return hm::fail(HM_ERR_INVALID, "hm_generate_dataset: n, d must be >= 1");
  long long count = (long long)n * d;
  int threads = 256;
  long long blocks = (count + threads - 1) / threads;
  hm::k_generate_dataset<<<(unsigned)blocks, threads, 0, hm::as_stream(stream)>>>(count, seed,
                                                                                d_points);
  HM_LAUNCH_CHECK();
  return HM_OK;
}

hm_status hm_generate_mixture(int n, int d, int ncomp, double sigma_min, double sigma_max,
                              unsigned long long seed, double* d_points, void* stream) {
  if (!d_points) return hm::fail(HM_ERR_INVALID, "hm_generate_mixture: d_points is NULL");
  if (n < 1 || d < 1 || ncomp < 1 || !(sigma_min > 0) || !(sigma_max >= sigma_min))
    return hm::fail(HM_ERR_INVALID, "hm_generate_mixture: need n, d, ncomp >= 1 and 0 < sigma_min <= sigma_max");
  // component parameters on the host from a splitmix64 stream of the seed
  uint64_t state = seed ^ 0x2545f4914f6cdd1dull;
  auto next = [&]() {
    uint64_t z = (state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
  };
  std::vector<double> ctr((size_t)ncomp * d), sig(ncomp), w(ncomp), cum(ncomp);
  for (auto& x : ctr) x = next();
  const double a = std::log(sigma_min), b = std::log(sigma_max);
  for (auto& x : sig) x = std::exp(a + (b - a) * next());
  double tot = 0;  // Dirichlet(1, ..., 1): normalised Exp(1) draws
  for (auto& x : w) {
    x = -std::log(1.0 - next());
    tot += x;
  }
  double run = 0;
  for (int c = 0; c < ncomp; ++c) {
    run += w[c] / tot;
    cum[c] = run;
  }
  cum[ncomp - 1] = 1.0;
  cudaStream_t s = hm::as_stream(stream);
  hm::DevBuf<double> dcum, dctr, dsig;
  HM_TRY(dcum.alloc_async(ncomp, s));
  HM_TRY(dctr.alloc_async(ctr.size(), s));
  HM_TRY(dsig.alloc_async(ncomp, s));
  HM_CUDA(cudaMemcpyAsync(dcum.p, cum.data(), 8 * cum.size(), cudaMemcpyHostToDevice, s));
  HM_CUDA(cudaMemcpyAsync(dctr.p, ctr.data(), 8 * ctr.size(), cudaMemcpyHostToDevice, s));
  HM_CUDA(cudaMemcpyAsync(dsig.p, sig.data(), 8 * sig.size(), cudaMemcpyHostToDevice, s));
  hm::k_generate_mixture<<<(n + 255) / 256, 256, 0, s>>>(n, d, ncomp, (uint32_t)(seed ^ (seed >> 32)), dcum.p,
                                                        dctr.p, dsig.p, d_points);
  HM_LAUNCH_CHECK();
  HM_CUDA(cudaStreamSynchronize(s));
  return HM_OK;
}

hm_status hm_kdtree_build(const double* d_points, int n, int d, int bucket, void* stream,
                          hm_kdtree* out) {
  return hm::kdtree_build(d_points, n, d, bucket, hm::as_stream(stream), out);
}

// The reference's division methods (src/kDTreeConstruction.cu:14-231):
// DIVIDE_IN_HALF takes the same code path as FULL_TREE; POWER_OF_TWO_ON_LEFT
// starts from upperPowerOfTwo(N) (:77-82) and halves that size per level, which
// equals the ceil(len/2) split at every level exactly when N is a power of two.
hm_status hm_kdtree_build_div(const double* d_points, int n, int d, int bucket, int division, void* stream,
                              hm_kdtree* out) {
  if (out) *out = nullptr;
  if (division != HM_DIV_POWER_OF_TWO_ON_LEFT && division != HM_DIV_DIVIDE_IN_HALF &&
      division != HM_DIV_FULL_TREE)
    return hm::fail(HM_ERR_INVALID, "hm_kdtree_build_div: unknown division method " + std::to_string(division));
  if (division == HM_DIV_POWER_OF_TWO_ON_LEFT && n > 0 && (n & (n - 1)) != 0)
    return hm::fail(HM_ERR_UNSUPPORTED,
                    "hm_kdtree_build_div: POWER_OF_TWO_ON_LEFT is supported for a power-of-two n only (where it "
                    "equals FULL_TREE); n = " + std::to_string(n));
  return hm::kdtree_build(d_points, n, d, bucket, hm::as_stream(stream), out);
}

hm_status hm_kdtree_info(hm_kdtree t, int* n, int* d, int* bucket, int* depth) {
  if (!t) return hm::fail(HM_ERR_INVALID, "hm_kdtree_info: null tree");
  if (n) *n = t->n;
  if (d) *d = t->d;
  if (bucket) *bucket = t->bucket;
  if (depth) *depth = t->depth;
  return HM_OK;
}

hm_status hm_kdtree_copy_out(hm_kdtree t, int* perm, int* offsets, double* bmin, double* bmax,
                             int* split_dim) {
  if (!t) return hm::fail(HM_ERR_INVALID, "hm_kdtree_copy_out: null tree");
  const size_t nleaf = (size_t)1 << t->depth;
  const size_t nodes = 2 * nleaf - 1;
  if (perm) HM_CUDA(cudaMemcpy(perm, t->perm.p, sizeof(int) * t->n, cudaMemcpyDeviceToHost));
  if (offsets)
    HM_CUDA(cudaMemcpy(offsets, t->offsets.p, sizeof(int) * (nleaf + 1), cudaMemcpyDeviceToHost));
  if (bmin)
    HM_CUDA(cudaMemcpy(bmin, t->bmin.p, sizeof(double) * nodes * t->d, cudaMemcpyDeviceToHost));
  if (bmax)
    HM_CUDA(cudaMemcpy(bmax, t->bmax.p, sizeof(double) * nodes * t->d, cudaMemcpyDeviceToHost));
  if (split_dim && nleaf > 1)
    HM_CUDA(cudaMemcpy(split_dim, t->split_dim.p, sizeof(int) * (nleaf - 1),
                       cudaMemcpyDeviceToHost));
  return HM_OK;
}

const int* hm_kdtree_device_perm(hm_kdtree t) { return t ? t->perm.p : nullptr; }
const int* hm_kdtree_device_offsets(hm_kdtree t) { return t ? t->offsets.p : nullptr; }

void hm_kdtree_free(hm_kdtree t) { delete t; }

}  // extern "C"
