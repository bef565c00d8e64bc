// hm_mma.cuh -- warp-level tensor-core helpers (mma.sync) used by the matvec.
//
// The H-matvec streams each factor once and performs 16-48 MACs per element,
// far below the tensor pipe's rate, so the legacy warp-synchronous MMA is
// enough to keep it bound by HBM; its fragments are loaded straight from the
// column-major factors with full 32-byte-sector efficiency, no shared memory.
//
// m16n8k8 TF32 fragment layout (lane = 4*g + t):
//   A (16x8, row major): a0 = A[g][t], a1 = A[g+8][t], a2 = A[g][t+4], a3 = A[g+8][t+4]
//   B (8x8, col major):  b0 = B[t][g], b1 = B[t+4][g]
//   C (16x8):            c0 = C[g][2t], c1 = C[g][2t+1], c2 = C[g+8][2t], c3 = C[g+8][2t+1]
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hm {

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// x ~ hi + lo, both TF32; hi*B + lo*B + hi*Blo reproduces an FP32 product
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// The tensor core's internal accumulation does not round to nearest, so a
// long chain of MMAs into one accumulator drifts (the error grows linearly
// with the chain).  Every helper below therefore multiplies into a zeroed
// temporary and adds it to the caller's FP32 sum with an ordinary
// round-to-nearest FADD.
__device__ __forceinline__ void add4(float (&c)[4], const float (&d)[4]) {
  c[0] += d[0];
  c[1] += d[1];
  c[2] += d[2];
  c[3] += d[3];
}

// C += A B in three TF32 passes (A = ah + al, B = bh + bl; the al*bl term is
// below FP32 rounding)
__device__ __forceinline__ void mma_3xtf32(float (&c)[4], const uint32_t (&ah)[4], const uint32_t (&al)[4],
                                           uint32_t bh0, uint32_t bh1, uint32_t bl0, uint32_t bl1) {
  float d[4] = {0.f, 0.f, 0.f, 0.f};
  mma_tf32(d, al[0], al[1], al[2], al[3], bh0, bh1);
  mma_tf32(d, ah[0], ah[1], ah[2], ah[3], bl0, bl1);
  mma_tf32(d, ah[0], ah[1], ah[2], ah[3], bh0, bh1);
  add4(c, d);
}

// ---- BF16 m16n8k16 (lane = 4*g + t) ---------------------------------------
//   A (16x16): a0 = {A[g][2t],A[g][2t+1]}, a1 = {A[g+8][2t],A[g+8][2t+1]},
//              a2 = {A[g][2t+8],A[g][2t+9]}, a3 = {A[g+8][2t+8],A[g+8][2t+9]}
//   B (16x8):  b0 = {B[2t][g],B[2t+1][g]}, b1 = {B[2t+8][g],B[2t+9][g]}
//   C (16x8):  as for TF32
// (the lower-indexed element sits in the low 16 bits)
__device__ __forceinline__ uint32_t pack_bf16(float lo_idx, float hi_idx) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi_idx), "f"(lo_idx));
  return r;
}

__device__ __forceinline__ float bf16_lo_as_float(uint32_t p) { return __uint_as_float(p << 16); }
__device__ __forceinline__ float bf16_hi_as_float(uint32_t p) { return __uint_as_float(p & 0xffff0000u); }

// x0, x1 -> hi = bf16x2(x0, x1), lo = bf16x2(x0 - hi0, x1 - hi1)
__device__ __forceinline__ void split_bf16x2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  hi = pack_bf16(x0, x1);
  lo = pack_bf16(x0 - bf16_lo_as_float(hi), x1 - bf16_hi_as_float(hi));
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

}  // namespace hm
