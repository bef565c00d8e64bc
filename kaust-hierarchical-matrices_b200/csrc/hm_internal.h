// hm_internal.h -- shared host/device definitions of the B200 H-matrix engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/hm.h"

namespace hm {

// ---- error reporting (host) ----------------------------------------------
void set_error(const std::string& msg);
hm_status fail(hm_status st, const std::string& msg);
hm_status cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define HM_CUDA(call)                                                  \
  do {                                                                 \
    cudaError_t e__ = (call);                                          \
    if (e__ != cudaSuccess) return ::hm::cuda_fail(e__, #call, __FILE__, __LINE__); \
  } while (0)

#define HM_LAUNCH_CHECK() HM_CUDA(cudaGetLastError())

#define HM_TRY(expr)                   \
  do {                                 \
    hm_status s__ = (expr);            \
    if (s__ != HM_OK) return s__;      \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---- phase trace --------------------------------------------------------------
// A build marks the end of each phase: the stream is synchronised at the
// mark, so device work is charged to the phase that launched it, and the
// wall-clock time since the previous mark is added to the phase's slot (the
// marks sit where the build waits for the device anyway, so this costs a few
// milliseconds per build).  With HM_TRACE=1 in the environment every mark is
// also printed to stderr.
struct PhaseTrace {
  static constexpr int kSlots = 8;
  bool on = false;
  const char* what = "";
  double sec[kSlots] = {};
  std::chrono::steady_clock::time_point last;
  explicit PhaseTrace(const char* w) : what(w) {
    const char* e = std::getenv("HM_TRACE");
    on = e != nullptr && e[0] != '\0' && e[0] != '0';
    last = std::chrono::steady_clock::now();
  }
  void mark(const char* phase, cudaStream_t s, long long arg = -1, int slot = 0) {
    cudaStreamSynchronize(s);
    const auto now = std::chrono::steady_clock::now();
    const double ms = std::chrono::duration<double, std::milli>(now - last).count();
    if (slot >= 0 && slot < kSlots) sec[slot] += ms * 1e-3;
    last = now;
    if (!on) return;
    if (arg >= 0)
      std::fprintf(stderr, "[hm trace] %s %-24s %5lld %10.3f ms\n", what, phase, arg, ms);
    else
      std::fprintf(stderr, "[hm trace] %s %-24s       %10.3f ms\n", what, phase, ms);
  }
};

// ---- device buffer RAII -----------------------------------------------------
// Long-lived buffers use cudaMalloc; temporaries of a build step pass a stream
// and come from the stream-ordered pool (cudaMallocAsync / cudaFreeAsync), so
// freeing them neither synchronises the device nor returns memory to the OS.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  bool async = false;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s), async(o.async) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; s = o.s; async = o.async;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  hm_status alloc(size_t count) {
    release();
    async = false;
    if (count == 0) return HM_OK;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      return fail(HM_ERR_NOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) +
                                    " bytes failed: " + cudaGetErrorString(e));
    }
    n = count;
    return HM_OK;
  }
  hm_status alloc_async(size_t count, cudaStream_t stream) {
    release();
    async = true;
    s = stream;
    if (count == 0) return HM_OK;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), stream);
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      return fail(HM_ERR_NOMEM, "cudaMallocAsync of " + std::to_string(count * sizeof(T)) +
                                    " bytes failed: " + cudaGetErrorString(e));
    }
    n = count;
    return HM_OK;
  }
  void release() {
    if (p) {
      if (async) cudaFreeAsync(p, s);
      else cudaFree(p);
    }
    p = nullptr;
    n = 0;
  }
};

// ---- twiddled (order-preserving) 64-bit keys for doubles --------------------
// Maps a double to an unsigned integer whose unsigned order equals the IEEE
// order of the doubles, with -0.0 and +0.0 mapped to the same key (so they
// compare equal, as IEEE `<` does).  NaN inputs are outside the contract.
__host__ __device__ inline uint64_t twiddle(double x) {
  uint64_t b;
#ifdef __CUDA_ARCH__
  b = static_cast<uint64_t>(__double_as_longlong(x));
#else
  __builtin_memcpy(&b, &x, 8);
#endif
  if (b == 0x8000000000000000ull) b = 0;  // -0.0 -> +0.0
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__host__ __device__ inline double untwiddle(uint64_t k) {
  uint64_t b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  double x;
#ifdef __CUDA_ARCH__
  x = __longlong_as_double(static_cast<long long>(b));
#else
  __builtin_memcpy(&x, &b, 8);
#endif
  return x;
}

// Morton index of (column cluster u, row cluster v): bits of u in the even
// positions, bits of v in the odd positions.
__host__ __device__ inline uint32_t spread16(uint32_t x) {
  x &= 0x0000ffffu;
  x = (x | (x << 8)) & 0x00ff00ffu;
  x = (x | (x << 4)) & 0x0f0f0f0fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}
__host__ __device__ inline uint32_t compact16(uint32_t x) {
  x &= 0x55555555u;
  x = (x | (x >> 1)) & 0x33333333u;
  x = (x | (x >> 2)) & 0x0f0f0f0fu;
  x = (x | (x >> 4)) & 0x00ff00ffu;
  x = (x | (x >> 8)) & 0x0000ffffu;
  return x;
}
__host__ __device__ inline uint32_t morton_encode(uint32_t u, uint32_t v) {
  return spread16(u) | (spread16(v) << 1);
}

constexpr int kMaxDim = 16;
constexpr int kMaxDepth = 28;

}  // namespace hm

// ---- opaque handle types ----------------------------------------------------
struct hm_kdtree_s {
  int n = 0, d = 0, bucket = 0, depth = 0;
  std::vector<int> h_offsets;          // leaf offsets (data independent)
  hm::DevBuf<int> perm;                // n
  hm::DevBuf<int> offsets;             // 2^depth + 1
  hm::DevBuf<double> bmin, bmax;       // (2^(depth+1) - 1) * d
  hm::DevBuf<int> split_dim;           // 2^depth - 1 (at least 1)
  hm::DevBuf<double> pts_tree;         // d * n, SoA, tree order
  hm::DevBuf<float> pts_tree_f;        // d * n, SoA, tree order, FP32
};
