// hm_capi.cu -- the extern "C" surface of libhmb200.so, error reporting and
// point generation.
#include <curand_kernel.h>

#include <cstdio>
#include <string>

#include "hm_internal.h"

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

hm_status hm_kdtree_build(const double* d_points, int n, int d, int bucket, void* stream,
                          hm_kdtree* out) {
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
