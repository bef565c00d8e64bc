// hm_kernels.cuh -- kernel functions evaluated on the device, and the
// counter-based Gaussian generator of the randomized sketches.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hm {

struct KernelParams {
  int kind;        // hm_kernel
  int deriv;       // 0: K, 1: dK/dl
  float ell;
  float inv_ell;
  float nugget;
};

// K(r) from r^2, FP32.  exp(-r/l) restates `interaction`
// (src/TLRMatrixHelpers.cu:44-58); the others extend it.
__device__ __forceinline__ float kernel_r2(const KernelParams& kp, float r2) {
  if (kp.kind == 2) {  // Gaussian
    float q = r2 * kp.inv_ell * kp.inv_ell;
    float g = __expf(-0.5f * q);
    return kp.deriv ? g * q * kp.inv_ell : g;
  }
  float r = sqrtf(r2);
  if (kp.kind == 1) {  // Matern 3/2
    float a = 1.7320508075688772f * r * kp.inv_ell;
    float e = __expf(-a);
    return kp.deriv ? a * a * e * kp.inv_ell : (1.0f + a) * e;
  }
  float a = r * kp.inv_ell;  // exponential
  float e = __expf(-a);
  return kp.deriv ? a * e * kp.inv_ell : e;
}

// 32-bit mix (a variant of the lowbias32 finaliser)
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Standard normal for the (stream, row, col) counter, Box-Muller.
__device__ __forceinline__ float gauss_at(uint32_t seed, uint32_t stream, uint32_t row, uint32_t col) {
  uint32_t h1 = mix32(seed ^ mix32(stream * 0x9e3779b9u ^ mix32(row * 0x85ebca6bu + col)));
  uint32_t h2 = mix32(h1 ^ 0x68e31da4u);
  float u1 = ((h1 >> 8) + 1u) * (1.0f / 16777217.0f);  // (0, 1]
  float u2 = (h2 >> 8) * (1.0f / 16777216.0f);         // [0, 1)
  float rad = sqrtf(-2.0f * __logf(u1));
  return rad * __cosf(6.283185307179586f * u2);
}

}  // namespace hm
