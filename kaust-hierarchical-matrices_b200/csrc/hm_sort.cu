// hm_sort.cu -- deterministic device primitives used by the structure and
// schedule builders: a stable LSD radix sort of (uint32 key, uint32 value)
// pairs and an exclusive scan.  Stability comes from ranking keys in thread
// order inside each tile (warp match + per-warp digit counts), so results are
// identical run to run.
#include <algorithm>

#include "hm_internal.h"
#include "hm_sort.h"

namespace hm {
namespace {

constexpr int kSortThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kSortThreads * kItems;
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kSortThreads) k_digit_hist(const uint32_t* keys, int n, int shift,
                                                            int ntiles, unsigned int* hist) {
  __shared__ unsigned int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int base = blockIdx.x * kTile;
  for (int i = threadIdx.x; i < kTile; i += kSortThreads) {
    int e = base + i;
    if (e < n) atomicAdd(&h[(keys[e] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// exclusive scan of `count` unsigned ints in place, one CTA; returns total in *total
__global__ void __launch_bounds__(kScanThreads) k_scan_excl(unsigned int* a, long long count,
                                                           unsigned int* total) {
  __shared__ unsigned int part[kScanThreads];
  long long per = (count + kScanThreads - 1) / kScanThreads;
  long long lo = threadIdx.x * per;
  long long hi = lo + per < count ? lo + per : count;
  unsigned int s = 0;
  for (long long i = lo; i < hi; ++i) s += a[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < kScanThreads; o <<= 1) {
    unsigned int t = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += t;
    __syncthreads();
  }
  unsigned int run = part[threadIdx.x] - s;
  for (long long i = lo; i < hi; ++i) {
    unsigned int v = a[i];
    a[i] = run;
    run += v;
  }
  if (threadIdx.x == kScanThreads - 1 && total) *total = part[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) k_digit_scatter(const uint32_t* kin, const uint32_t* vin,
                                                               uint32_t* kout, uint32_t* vout, int n,
                                                               int shift, int ntiles,
                                                               const unsigned int* offs) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ unsigned int run[256];
  __shared__ unsigned int wcnt[kWarps][256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  run[threadIdx.x] = offs[(size_t)threadIdx.x * ntiles + blockIdx.x];
  int base = blockIdx.x * kTile;
  for (int r = 0; r < kItems; ++r) {
    for (int w = 0; w < kWarps; ++w) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    int e = base + r * kSortThreads + threadIdx.x;
    bool valid = e < n;
    uint32_t key = valid ? kin[e] : 0u;
    uint32_t dig = (key >> shift) & 255u;
    unsigned int peers = __match_any_sync(0xffffffffu, valid ? dig : 0x100u + lane);
    int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) wcnt[warp][dig] = __popc(peers);
    __syncthreads();
    // per digit: exclusive prefix over warps, then advance the running base
    {
      unsigned int acc = 0;
      for (int w = 0; w < kWarps; ++w) {
        unsigned int c = wcnt[w][threadIdx.x];
        wcnt[w][threadIdx.x] = acc;
        acc += c;
      }
      __syncthreads();
      if (valid) {
        unsigned int dst = run[dig] + wcnt[warp][dig] + rank;
        kout[dst] = key;
        vout[dst] = vin[e];
      }
      __syncthreads();
      run[threadIdx.x] += acc;
    }
    __syncthreads();
  }
}

}  // namespace

hm_status scan_exclusive(unsigned int* d_a, long long count, unsigned int* d_total,
                         cudaStream_t stream) {
  if (count <= 0) return HM_OK;
  k_scan_excl<<<1, kScanThreads, 0, stream>>>(d_a, count, d_total);
  HM_LAUNCH_CHECK();
  return HM_OK;
}

hm_status sort_pairs_u32(uint32_t* keys, uint32_t* vals, int n, int key_bits, cudaStream_t stream) {
  if (n <= 1) return HM_OK;
  int ntiles = (n + kTile - 1) / kTile;
  DevBuf<uint32_t> k2, v2;
  DevBuf<unsigned int> hist;
  HM_TRY(k2.alloc_async(n, stream));
  HM_TRY(v2.alloc_async(n, stream));
  HM_TRY(hist.alloc_async((size_t)256 * ntiles, stream));
  uint32_t *ka = keys, *va = vals, *kb = k2.p, *vb = v2.p;
  int passes = 0;
  for (int shift = 0; shift < key_bits; shift += 8) {
    k_digit_hist<<<ntiles, kSortThreads, 0, stream>>>(ka, n, shift, ntiles, hist.p);
    HM_LAUNCH_CHECK();
    HM_TRY(scan_exclusive(hist.p, (long long)256 * ntiles, nullptr, stream));
    k_digit_scatter<<<ntiles, kSortThreads, 0, stream>>>(ka, va, kb, vb, n, shift, ntiles, hist.p);
    HM_LAUNCH_CHECK();
    std::swap(ka, kb);
    std::swap(va, vb);
    ++passes;
  }
  if (passes & 1) {
    HM_CUDA(cudaMemcpyAsync(keys, ka, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, stream));
    HM_CUDA(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, stream));
  }
  return HM_OK;  // temporaries are released in stream order
}

}  // namespace hm
