// hm_mixed.cu -- mixed-precision H-matvec: BF16 hi + lo factor panels on the
// tensor cores (mma.sync m16n8k16, FP32 accumulation).
//
// One product of <= 16 right-hand sides runs three or four kernels:
//   k_mx_split_x  X (FP32, tree order) -> BF16 hi + lo fragments per 32-row tile
//   k_mx_p1       P = panel^T X per (panel, column group, row chunk); a panel
//                 projected in one row chunk stores P as T, else each chunk's
//                 partial
//   k_mx_reduce   (panels of several row chunks only) the partials summed in
//                 chunk order, stored as T
//   k_mx_p2       Y = sum over the ancestors' panels of U T, plus dense blocks
// (Passes of 65-128 right-hand sides run on the tcgen05 kernels of
// hm_mixed_tc.cu unless the schedule says wide_tc=0; k_mx_split_x then writes
// X's image for them instead of the fragments.)
// "Stored as T": the projection on a factor column is the coefficient of the
// mirror block's factor column (block (s,t) = U V^T: V^T X_t multiplies U,
// U^T X_s multiplies V), so each column of P is written, split into BF16
// hi + lo, to the column that it multiplies.  T keeps each column's hi and lo
// in one 32-bit word per right-hand side, so that any column lands on its own
// (8 bytes per lane: right-hand sides g and g + 8) and no permutation pass is
// needed.  Phase 2 rebuilds its B operand pairs {T[c], T[c+1]} (hi, and lo)
// from two such words with one byte permute each.  A factor column without a
// low part (its block's small singular directions, where the factor's own
// BF16 rounding is within the budget) gets T's hi only: one word holds
// right-hand sides g and g + 8, and phase 2 multiplies U_hi T_hi alone.
// Each product of a BF16 pair uses three MMAs (hi*lo, lo*hi, hi*hi; lo*lo is
// below FP32 rounding).  A factor column without a low part is itself only
// BF16-accurate, so it meets X's and T's high parts alone: one MMA per tile
// pair (phase 1 loads no X low part for units of such columns).  The tensor core's internal sums do not round to nearest, so
// each short chain of MMAs goes into a zeroed temporary that is added to the
// running FP32 sum with an ordinary FADD.
#include <algorithm>
#include <vector>

#include "hm_hmatrix.h"
#include "hm_mixed.h"
#include "hm_mma.cuh"

namespace hm {
namespace {


// A P1 tile (32 rows x 8 columns of a factor) keeps lane (g,t)'s 16 bytes
// -- column g at rows rho(t, 0..7) -- at word 4 g + (t ^ ((g >> 1) & 3)): the
// K-major core-matrix layout with the 64-byte swizzle (column g's 64-byte row
// at 64 g, its K block t at 16-byte chunk t ^ ((g >> 1) & 3)), so that a run
// of tiles is a tcgen05 operand image as stored.  The 4 lanes of a column
// only trade places: each quarter-warp still reads one 128-byte line.
__host__ __device__ __forceinline__ int p1_slot(int lane) {
  const int g = lane >> 2, t = lane & 3;
  return 4 * g + (t ^ ((g >> 1) & 3));
}

__device__ __forceinline__ void mma_a4(float (&d)[4], const uint4& a, uint32_t b0, uint32_t b1) {
  mma_bf16(d, a.x, a.y, a.z, a.w, b0, b1);
}

// An L2 policy that keeps lines over streamed ones: the X fragments are read
// once per tree level by phase 1 (and again by phase 2's dense blocks), while
// the panels stream past them with evict-first loads.
__device__ __forceinline__ uint64_t l2_keep_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint4 ld_keep(const uint4* ptr, uint64_t pol) {
  uint4 v;
  asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;\n"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(ptr), "l"(pol));
  return v;
}

// A factor tile: streamed past the caches (evict-first) when one warp reads
// it; through L1 when the warps of a CTA all read it (each for its own
// right-hand sides), so that the siblings of the first reader hit in L1.
template <bool SHARED>
__device__ __forceinline__ uint4 ld_tile(const uint4* p) {
  if (SHARED) return __ldg(p);
  return __ldcs(p);
}

// T layout, per panel: its nctl tiles with low parts, then the others.
//   with low parts (128 words): lane (g,t) x {column 2t at right-hand sides g,
//     g + 8; column 2t + 1 at g, g + 8}, each word bf16x2 {hi, lo}
//   without (64 words): lane (g,t) x {column 2t, column 2t + 1}, each word
//     bf16x2 {hi at g, hi at g + 8}
// Word of (column c of the panel, lane row 0); row g adds 16 g, resp. 8 g.
__host__ __device__ __forceinline__ long long t_word(long long tw0, int nctl, int c) {
  const int tile = c >> 3, t = (c & 7) >> 1, odd = c & 1;
  return tile < nctl ? tw0 + (long long)tile * 128 + 4 * t + 2 * odd
                     : tw0 + (long long)nctl * 128 + (long long)(tile - nctl) * 64 + 2 * t + odd;
}

// One lane's C fragment of a projection tile (columns 2t and 2t+1 at
// right-hand sides g and g + 8), stored as T: each column to its mirror's
// words (m: the tslot entries of columns 2t, 2t+1), split hi + lo or hi only;
// a padding column (no mirror) writes zeros to its own words, which are the
// padding of the same panel in T, so that every T word is written once per
// product.  Both columns of a pair are of the same kind (a panel's tiles with
// low parts come first), so the branch is uniform over the warp.
__device__ __forceinline__ void mx_store_t(uint32_t* __restrict__ T, int2 m, int lane, float a0, float a1, float a2,
                                           float a3) {
  const int g = lane >> 2;
  const int e0 = m.x >= 0 ? m.x : -1 - m.x, e1 = m.y >= 0 ? m.y : -1 - m.y;
  const int o0 = e0 >> 1, o1 = e1 >> 1;
  if ((e0 & 1) == 0) {  // with low parts: 8 bytes per column
    uint32_t h, l, h8, l8;
    split_bf16x2(a0, a1, h, l);    // right-hand side g:     columns 2t, 2t+1
    split_bf16x2(a2, a3, h8, l8);  // right-hand side g + 8
    const uint2 z = make_uint2(0u, 0u);
    const uint2 w0 = m.x >= 0 ? make_uint2(__byte_perm(h, l, 0x5410), __byte_perm(h8, l8, 0x5410)) : z;
    const uint2 w1 = m.y >= 0 ? make_uint2(__byte_perm(h, l, 0x7632), __byte_perm(h8, l8, 0x7632)) : z;
    const int s0 = o0 + 16 * g, s1 = o1 + 16 * g;
    if (s1 == s0 + 2 && (s0 & 3) == 0) {  // a whole 16-byte word of the destination tile
      *reinterpret_cast<uint4*>(T + s0) = make_uint4(w0.x, w0.y, w1.x, w1.y);
    } else {
      *reinterpret_cast<uint2*>(T + s0) = w0;
      *reinterpret_cast<uint2*>(T + s1) = w1;
    }
  } else {  // hi only: 4 bytes per column
    const uint32_t w0 = m.x >= 0 ? pack_bf16(a0, a2) : 0u, w1 = m.y >= 0 ? pack_bf16(a1, a3) : 0u;
    const int s0 = o0 + 8 * g, s1 = o1 + 8 * g;
    if (s1 == s0 + 1 && (s0 & 1) == 0) {
      *reinterpret_cast<uint2*>(T + s0) = make_uint2(w0, w1);
    } else {
      T[s0] = w0;
      T[s1] = w1;
    }
  }
}
__device__ __forceinline__ int2 tslot_pair(const int* __restrict__ tslot, long long col_tile, int lane) {
  return __ldg(reinterpret_cast<const int2*>(tslot + col_tile * 8 + 2 * (lane & 3)));
}

// ---- X -> fragments ---------------------------------------------------------
// Xf[tile][part][lane], part 0/1 = hi of rows 0-15 / 16-31, part 2/3 = lo:
// the m16n8k16 A fragment of X^T (16 right-hand sides x 16 rows):
//   {X[2t,2t+1][g], X[2t,2t+1][g+8], X[2t+8,2t+9][g], X[2t+8,2t+9][g+8]}
// Xtc (a 128-column pass on tcgen05, else null): per tile a 16 KB image,
// hi then lo, of B = X in the K-major core-matrix layout, right-hand side n
// and K block c (8 rows, in the order rho(c, e) = 8 (e / 2) + 2 c + e % 2 of
// the factors' P1 lanes) at 16 bytes (n % 8) + 128 (n / 8) + 2048 c.
__global__ void __launch_bounds__(128) k_mx_split_x(const float* __restrict__ X, int ldx, int nr, int num_tiles,
                                                    const int* __restrict__ tile_leaf,
                                                    const int* __restrict__ leaf_tile0,
                                                    const int* __restrict__ leaf_off, uint4* __restrict__ Xf,
                                                    uint4* __restrict__ Xtc) {
  __shared__ float xs[4][16][33];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int G = blockIdx.x * 4 + w;
  if (G >= num_tiles) return;  // whole warp; only warp-level syncs below
  // half y of a pass of up to 32 right-hand sides: columns 16 y .. 16 y + 15
  X += (size_t)16 * blockIdx.y * ldx;
  nr -= 16 * blockIdx.y;
  Xf += (size_t)blockIdx.y * num_tiles * 128;
  const int x = tile_leaf[G];
  const int row = leaf_off[x] + 32 * (G - leaf_tile0[x]) + lane;
  const bool ok = row < leaf_off[x + 1];
#pragma unroll
  for (int r = 0; r < 16; ++r) xs[w][r][lane] = (ok && r < nr) ? __ldg(X + (size_t)r * ldx + row) : 0.f;
  __syncwarp();
  if (Xtc) {  // this part's 16 right-hand sides x 4 K blocks (no fragments)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int idx = lane + 32 * q, nl = idx >> 2, c = idx & 3;
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int e = 0; e < 4; ++e)  // rows rho(c, 2e), rho(c, 2e + 1) = 8 e + 2 c + {0, 1}
        split_bf16x2(xs[w][nl][8 * e + 2 * c], xs[w][nl][8 * e + 2 * c + 1], hi[e], lo[e]);
      const int n = 16 * blockIdx.y + nl;
      uint4* dst = Xtc + (size_t)G * 1024 + (n & 7) + (n >> 3) * 8 + c * 128;
      dst[0] = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      dst[512] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
    return;
  }
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int i0 = 16 * s + 2 * t;
    uint4 hi, lo;
    split_bf16x2(xs[w][g][i0], xs[w][g][i0 + 1], hi.x, lo.x);
    split_bf16x2(xs[w][g + 8][i0], xs[w][g + 8][i0 + 1], hi.y, lo.y);
    split_bf16x2(xs[w][g][i0 + 8], xs[w][g][i0 + 9], hi.z, lo.z);
    split_bf16x2(xs[w][g + 8][i0 + 8], xs[w][g + 8][i0 + 9], hi.w, lo.w);
    Xf[((size_t)G * 4 + s) * 32 + lane] = hi;
    Xf[((size_t)G * 4 + 2 + s) * 32 + lane] = lo;
  }
}

// ---- phase 1 ----------------------------------------------------------------
// C (16 right-hand sides x 8 columns) per column tile and half = X^T V over
// the unit's row tiles.  NCT: column tiles compiled for, RU: row tiles loaded
// per step, NH: halves of 16 right-hand sides (each V tile is loaded once for
// both); a half's X fragments, S and T sit xh, sh and th elements after the
// previous half's.
template <int NCT, int RU, int NH, bool SH = false>
__device__ __forceinline__ void mx_p1_unit(const MxUnit& u, const MxPanel& P, const uint4* __restrict__ store,
                                           const uint4* __restrict__ Xf, const int* __restrict__ tslot,
                                           float4* __restrict__ S, uint32_t* __restrict__ T, long long xh,
                                           long long sh, long long th, int lane) {
  float acc[NH][NCT][4];
#pragma unroll
  for (int h = 0; h < NH; ++h)
#pragma unroll
    for (int j = 0; j < NCT; ++j) acc[h][j][0] = acc[h][j][1] = acc[h][j][2] = acc[h][j][3] = 0.f;
  const uint4 z = make_uint4(0u, 0u, 0u, 0u);
  const uint64_t keep = l2_keep_policy();
  // the mirrors of the unit's columns, fetched now so that the stores after
  // the loop wait for nothing: lane 4j + t holds tile j's pair t
  int2 mm = make_int2(-1, -1);
  if (P.nchunk == 1 && lane < 4 * NCT && (lane >> 2) < u.nct) mm = tslot_pair(tslot, P.t0 + u.ct0 + (lane >> 2), lane);
  const bool xlo = u.ct0 < P.nctl;  // the unit holds columns with low parts
  for (int r = 0; r < u.nrt; r += RU) {
    uint4 xf[RU][NH][4], vh[RU][NCT], vl[RU][NCT];
#pragma unroll
    for (int q = 0; q < RU; ++q) {
      const bool ok = r + q < u.nrt;
      const long long rt = u.rt0 + r + q;
      const uint4* xp = Xf + (size_t)(P.tile0 + rt) * 128 + lane;
#pragma unroll
      for (int h = 0; h < NH; ++h)
#pragma unroll
        for (int p = 0; p < 4; ++p)  // X's low part only for units with low-part columns
          xf[q][h][p] = ok && (p < 2 || xlo) ? ld_keep(xp + h * xh + p * 32, keep) : z;
      const uint4* hp = store + (P.hi1 + rt * P.nct + u.ct0) * 32 + p1_slot(lane);
      const uint4* lp = store + (P.lo1 + rt * P.nctl + u.ct0) * 32 + p1_slot(lane);
#pragma unroll
      for (int j = 0; j < NCT; ++j) {
        vh[q][j] = ok && j < u.nct ? ld_tile<SH>(hp + j * 32) : z;
        vl[q][j] = ok && j < u.nct && u.ct0 + j < P.nctl ? ld_tile<SH>(lp + j * 32) : z;
      }
    }
#pragma unroll
    for (int q = 0; q < RU; ++q) {
      if (r + q < u.nrt) {
#pragma unroll
        for (int j = 0; j < NCT; ++j) {
          if (j < u.nct) {
#pragma unroll
            for (int h = 0; h < NH; ++h) {
              float d[4] = {0.f, 0.f, 0.f, 0.f};
              if (u.ct0 + j < P.nctl) {  // a column with a low part: X_lo V_hi, X_hi V_lo
                mma_a4(d, xf[q][h][2], vh[q][j].x, vh[q][j].y);
                mma_a4(d, xf[q][h][3], vh[q][j].z, vh[q][j].w);
                mma_a4(d, xf[q][h][0], vl[q][j].x, vl[q][j].y);
                mma_a4(d, xf[q][h][1], vl[q][j].z, vl[q][j].w);
              }
              mma_a4(d, xf[q][h][0], vh[q][j].x, vh[q][j].y);  // X_hi V_hi
              mma_a4(d, xf[q][h][1], vh[q][j].z, vh[q][j].w);
              add4(acc[h][j], d);
            }
          }
        }
      }
    }
  }
  // the whole projection, stored as T, or one chunk's partial
  if (P.nchunk == 1) {
#pragma unroll
    for (int j = 0; j < NCT; ++j)
      if (j < u.nct) {
        const int src = 4 * j + (lane & 3);
        const int2 m = make_int2(__shfl_sync(0xffffffffu, mm.x, src), __shfl_sync(0xffffffffu, mm.y, src));
#pragma unroll
        for (int h = 0; h < NH; ++h)
          mx_store_t(T + h * th, m, lane, acc[h][j][0], acc[h][j][1], acc[h][j][2], acc[h][j][3]);
      }
  } else {
    float4* out = S + (P.s0 + (long long)u.chunk * P.nct + u.ct0) * 32 + lane;
#pragma unroll
    for (int h = 0; h < NH; ++h)
#pragma unroll
      for (int j = 0; j < NCT; ++j)
        if (j < u.nct) out[h * sh + j * 32] = make_float4(acc[h][j][0], acc[h][j][1], acc[h][j][2], acc[h][j][3]);
  }
}

// A unit whose columns have no low parts: X's and V's high parts only, one
// MMA per tile pair.  Without the low parts' registers a warp keeps RU row
// tiles of loads in flight instead of two.
template <int NCT, int RU>
__device__ __forceinline__ void mx_p1_unit_hi(const MxUnit& u, const MxPanel& P, const uint4* __restrict__ store,
                                              const uint4* __restrict__ Xf, const int* __restrict__ tslot,
                                              float4* __restrict__ S, uint32_t* __restrict__ T, int lane) {
  float acc[NCT][4];
#pragma unroll
  for (int j = 0; j < NCT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  const uint4 z = make_uint4(0u, 0u, 0u, 0u);
  const uint64_t keep = l2_keep_policy();
  int2 mm = make_int2(-1, -1);
  if (P.nchunk == 1 && lane < 4 * NCT && (lane >> 2) < u.nct) mm = tslot_pair(tslot, P.t0 + u.ct0 + (lane >> 2), lane);
  for (int r = 0; r < u.nrt; r += RU) {
    uint4 xf[RU][2], vh[RU][NCT];
#pragma unroll
    for (int q = 0; q < RU; ++q) {
      const bool ok = r + q < u.nrt;
      const long long rt = u.rt0 + r + q;
      const uint4* xp = Xf + (size_t)(P.tile0 + rt) * 128 + lane;
      xf[q][0] = ok ? ld_keep(xp, keep) : z;
      xf[q][1] = ok ? ld_keep(xp + 32, keep) : z;
      const uint4* hp = store + (P.hi1 + rt * P.nct + u.ct0) * 32 + p1_slot(lane);
#pragma unroll
      for (int j = 0; j < NCT; ++j) vh[q][j] = ok && j < u.nct ? __ldcs(hp + j * 32) : z;
    }
    // one chain over the step's row tiles per column tile (BF16-accurate
    // products: the chain's drift is far below their rounding)
#pragma unroll
    for (int j = 0; j < NCT; ++j) {
      if (j < u.nct) {
        float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int q = 0; q < RU; ++q) {
          mma_a4(d, xf[q][0], vh[q][j].x, vh[q][j].y);  // X_hi V_hi (zero tiles past the unit's end)
          mma_a4(d, xf[q][1], vh[q][j].z, vh[q][j].w);
        }
        add4(acc[j], d);
      }
    }
  }
  if (P.nchunk == 1) {
#pragma unroll
    for (int j = 0; j < NCT; ++j)
      if (j < u.nct) {
        const int src = 4 * j + (lane & 3);
        const int2 m = make_int2(__shfl_sync(0xffffffffu, mm.x, src), __shfl_sync(0xffffffffu, mm.y, src));
        mx_store_t(T, m, lane, acc[j][0], acc[j][1], acc[j][2], acc[j][3]);
      }
  } else {
    float4* out = S + (P.s0 + (long long)u.chunk * P.nct + u.ct0) * 32 + lane;
#pragma unroll
    for (int j = 0; j < NCT; ++j)
      if (j < u.nct) out[j * 32] = make_float4(acc[j][0], acc[j][1], acc[j][2], acc[j][3]);
  }
}

// One unit per CTA.  WPC = 1: one warp per CTA, 16 per SM (measured): a warp
// runs one unit and retires at once, instead of holding its CTA's slot until
// sibling warps with other units finish; 16 warps keep enough loads in flight
// at 128 registers.  WPC > 1 (passes of more than 64 right-hand sides): the
// CTA's warps take the same unit, warp w parts w NH .. w NH + NH - 1, and
// share its factor tiles through L1.
constexpr int kP1PerSm = 16;
template <int NH, int WPC>
__global__ void __launch_bounds__(32 * WPC, kP1PerSm / WPC) k_mx_p1(const MxUnit* __restrict__ units, int nunits,
                                               const MxPanel* __restrict__ panels, const uint4* __restrict__ store,
                                               const uint4* __restrict__ Xf, const int* __restrict__ tslot,
                                               float4* __restrict__ S, uint32_t* __restrict__ T, long long xh,
                                               long long sh, long long th) {
  const int w = blockIdx.x;
  if (w >= nunits) return;
  const int lane = threadIdx.x & 31;
  constexpr bool SH = WPC > 1;
  if (SH) {  // this warp's parts
    const int h0 = (threadIdx.x >> 5) * NH;
    Xf += h0 * xh;
    S += h0 * sh;
    T += h0 * th;
  }
  const MxUnit u = units[w];
  const MxPanel P = panels[u.panel];
  if (NH == 1 && u.ct0 >= P.nctl) {  // no low parts in this unit
    if (u.nct > 4)
      mx_p1_unit_hi<8, 2>(u, P, store, Xf, tslot, S, T, lane);
    else if (u.nct > 2)
      mx_p1_unit_hi<4, 4>(u, P, store, Xf, tslot, S, T, lane);
    else
      mx_p1_unit_hi<2, 6>(u, P, store, Xf, tslot, S, T, lane);
  } else if (NH == 1) {
    if (u.nct > 4)
      mx_p1_unit<8, 1, 1>(u, P, store, Xf, tslot, S, T, xh, sh, th, lane);
    else if (u.nct > 2)
      mx_p1_unit<4, 2, 1>(u, P, store, Xf, tslot, S, T, xh, sh, th, lane);
    else
      mx_p1_unit<2, 4, 1>(u, P, store, Xf, tslot, S, T, xh, sh, th, lane);
  } else if (NH == 4) {  // four halves: two column tiles at a time
    for (int c = 0; c < u.nct; c += 2) {
      MxUnit a = u;
      a.ct0 = u.ct0 + c;
      a.nct = min(2, u.nct - c);
      mx_p1_unit<2, 1, NH, SH>(a, P, store, Xf, tslot, S, T, xh, sh, th, lane);
    }
  } else if (u.nct > 2) {  // two halves: at most four column tiles at a time
    MxUnit a = u;
    a.nct = min(u.nct, 4);
    mx_p1_unit<4, 1, NH>(a, P, store, Xf, tslot, S, T, xh, sh, th, lane);
    if (u.nct > 4) {
      a.ct0 = u.ct0 + 4;
      a.nct = u.nct - 4;
      mx_p1_unit<4, 1, NH>(a, P, store, Xf, tslot, S, T, xh, sh, th, lane);
    }
  } else {
    mx_p1_unit<2, 2, NH>(u, P, store, Xf, tslot, S, T, xh, sh, th, lane);
  }
}

// ---- phase 1, persistent warps with a cp.async ring --------------------------
// The same product as k_mx_p1.  Each warp walks its units (w, w + W, ...) one
// row tile at a time; a step's tiles (X hi/lo fragments, the V tiles and their
// low parts) are copied into a per-warp shared-memory ring RING - 1 steps
// ahead of the MMAs.  In the fragment order each lane needs exactly the 16
// bytes it copied, so every lane copies and reads its own slots: completion
// is cp.async.wait_group on the lane's own groups, with no barrier.
__device__ __forceinline__ void cp16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// WARPS per CTA, RING stages per warp, VT column tiles per unit at most
// (slots per stage: 4 X fragments + VT high + VT low tiles).
template <int WARPS, int RING, int VT>
constexpr size_t ring_smem() {
  return (size_t)WARPS * RING * (4 + 2 * VT) * 512;
}

template <int WARPS, int RING, int VT>
__global__ void __launch_bounds__(32 * WARPS, 1) k_mx_p1r(const MxUnit* __restrict__ units, int nunits,
                                                          const MxPanel* __restrict__ panels,
                                                          const uint4* __restrict__ store,
                                                          const uint4* __restrict__ Xf, const int* __restrict__ tslot,
                                                          float4* __restrict__ S, uint32_t* __restrict__ T) {
  constexpr int SLOTS = 4 + 2 * VT;
  extern __shared__ __align__(16) uint4 ring[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int W = gridDim.x * WARPS;
  int pu = blockIdx.x * WARPS + warp;  // producer's unit
  if (pu >= nunits) return;            // the whole warp
  uint4* my = ring + (size_t)warp * RING * SLOTS * 32 + lane;  // slot s of stage q: my[(q * SLOTS + s) * 32]
  const uint32_t my_s = (uint32_t)__cvta_generic_to_shared(my);
  MxUnit U = units[pu];
  MxPanel PP = panels[U.panel];
  int prt = 0;
  auto produce = [&](int stage) {
    if (pu < nunits) {
      const long long rt = U.rt0 + prt;
      const uint32_t base = my_s + (uint32_t)(stage * SLOTS * 32) * 16u;
      const uint4* xp = Xf + (size_t)(PP.tile0 + rt) * 128 + lane;
#pragma unroll
      for (int p = 0; p < 4; ++p) cp16(base + (uint32_t)(p * 32) * 16u, xp + p * 32);
      const uint4* hp = store + (PP.hi1 + rt * PP.nct + U.ct0) * 32 + p1_slot(lane);
      for (int j = 0; j < U.nct; ++j) cp16(base + (uint32_t)((4 + j) * 32) * 16u, hp + j * 32);
      const int nl = min(U.nct, max(0, PP.nctl - U.ct0));
      const uint4* lp = store + (PP.lo1 + rt * PP.nctl + U.ct0) * 32 + p1_slot(lane);
      for (int j = 0; j < nl; ++j) cp16(base + (uint32_t)((4 + VT + j) * 32) * 16u, lp + j * 32);
      if (++prt == U.nrt) {
        prt = 0;
        pu += W;
        if (pu < nunits) {
          U = units[pu];
          PP = panels[U.panel];
        }
      }
    }
    cp_commit();  // an empty group past the end keeps the group count uniform
  };
  int cu = blockIdx.x * WARPS + warp;  // consumer's unit
  MxUnit CU = U;
  MxPanel CP = PP;
  int crt = 0;
#pragma unroll
  for (int q = 0; q < RING - 1; ++q) produce(q);
  float acc[VT][4];
#pragma unroll
  for (int j = 0; j < VT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  int stage = 0;
  while (cu < nunits) {
    produce(stage == 0 ? RING - 1 : stage - 1);
    cp_wait<RING - 1>();  // this lane's copies of `stage` have landed
    const uint4* sl = my + (size_t)stage * SLOTS * 32;
    const uint4 x0 = sl[0], x1 = sl[32], x2 = sl[64], x3 = sl[96];
    float d[VT][4];
#pragma unroll
    for (int j = 0; j < VT; ++j) d[j][0] = d[j][1] = d[j][2] = d[j][3] = 0.f;
    // the column tiles' MMA chains interleaved, so that consecutive MMAs are independent
#pragma unroll
    for (int j = 0; j < VT; ++j)
      if (j < CU.nct && CU.ct0 + j < CP.nctl) {  // X_lo V_hi, for columns with low parts
        const uint4 vh = sl[(4 + j) * 32];
        mma_a4(d[j], x2, vh.x, vh.y);
      }
#pragma unroll
    for (int j = 0; j < VT; ++j)
      if (j < CU.nct && CU.ct0 + j < CP.nctl) {
        const uint4 vh = sl[(4 + j) * 32];
        mma_a4(d[j], x3, vh.z, vh.w);
      }
#pragma unroll
    for (int j = 0; j < VT; ++j)
      if (j < CU.nct && CU.ct0 + j < CP.nctl) {  // X_hi V_lo
        const uint4 vl = sl[(4 + VT + j) * 32];
        mma_a4(d[j], x0, vl.x, vl.y);
        mma_a4(d[j], x1, vl.z, vl.w);
      }
#pragma unroll
    for (int j = 0; j < VT; ++j)
      if (j < CU.nct) {
        const uint4 vh = sl[(4 + j) * 32];
        mma_a4(d[j], x0, vh.x, vh.y);  // X_hi V_hi
      }
#pragma unroll
    for (int j = 0; j < VT; ++j)
      if (j < CU.nct) {
        const uint4 vh = sl[(4 + j) * 32];
        mma_a4(d[j], x1, vh.z, vh.w);
        add4(acc[j], d[j]);
      }
    if (++crt == CU.nrt) {
      float4* out = S + (CP.s0 + (long long)CU.chunk * CP.nct + CU.ct0) * 32 + lane;
#pragma unroll
      for (int j = 0; j < VT; ++j) {
        if (j < CU.nct) {
          if (CP.nchunk == 1)
            mx_store_t(T, tslot_pair(tslot, CP.t0 + CU.ct0 + j, lane), lane, acc[j][0], acc[j][1], acc[j][2],
                       acc[j][3]);
          else
            out[j * 32] = make_float4(acc[j][0], acc[j][1], acc[j][2], acc[j][3]);
        }
        acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
      }
      crt = 0;
      cu += W;
      if (cu < nunits) {
        CU = units[cu];
        CP = panels[CU.panel];
      }
    }
    stage = stage + 1 == RING ? 0 : stage + 1;
  }
  cp_wait<0>();
}

// ---- row-chunk reduction ------------------------------------------------------
// For panels projected in several row chunks: the chunk partials of each
// column tile summed in chunk order (deterministic), stored as T.
__global__ void k_mx_reduce(const int2* __restrict__ mtiles, long long nmt, const MxPanel* __restrict__ panels,
                            const float4* __restrict__ S, const int* __restrict__ tslot, uint32_t* __restrict__ T,
                            long long sh, long long th) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nmt * 32) return;
  S += blockIdx.y * sh;  // half y of the pass
  T += blockIdx.y * th;
  const int2 mt = mtiles[i >> 5];  // (panel, column tile)
  const int lane = (int)(i & 31);
  const MxPanel P = panels[mt.x];
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int ch = 0; ch < P.nchunk; ++ch) {
    const float4 a = S[(P.s0 + (long long)ch * P.nct + mt.y) * 32 + lane];
    v.x += a.x;
    v.y += a.y;
    v.z += a.z;
    v.w += a.w;
  }
  mx_store_t(T, tslot_pair(tslot, P.t0 + mt.y, lane), lane, v.x, v.y, v.z, v.w);
}

// ---- phase 2 ----------------------------------------------------------------
// acc[mt][nb] += A (16 rows x 16 columns, tiles h0|h1 + l0|l1) B (16 x 8)
__device__ __forceinline__ void mx_p2_step(float (&acc)[2][2][4], const uint4& h0, const uint4& h1,
                                           const uint4& l0, const uint4& l1, const uint32_t (&bh)[2][2],
                                           const uint32_t (&bl)[2][2], bool lo) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const uint32_t a0 = mt ? h0.z : h0.x, a1 = mt ? h0.w : h0.y, a2 = mt ? h1.z : h1.x, a3 = mt ? h1.w : h1.y;
    const uint32_t c0 = mt ? l0.z : l0.x, c1 = mt ? l0.w : l0.y, c2 = mt ? l1.z : l1.x, c3 = mt ? l1.w : l1.y;
#pragma unroll
    for (int nb = 0; nb < 2; ++nb) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      mma_bf16(d, a0, a1, a2, a3, bl[nb][0], bl[nb][1]);
      if (lo) mma_bf16(d, c0, c1, c2, c3, bh[nb][0], bh[nb][1]);
      mma_bf16(d, a0, a1, a2, a3, bh[nb][0], bh[nb][1]);
      add4(acc[mt][nb], d);
    }
  }
}

// acc[mt][nb] += A_hi (16 rows x 16 columns, tiles h0|h1) B_hi (16 x 8)
__device__ __forceinline__ void mx_p2_step_hi(float (&acc)[2][2][4], const uint4& h0, const uint4& h1,
                                              const uint32_t (&bh)[2][2]) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const uint32_t a0 = mt ? h0.z : h0.x, a1 = mt ? h0.w : h0.y, a2 = mt ? h1.z : h1.x, a3 = mt ? h1.w : h1.y;
#pragma unroll
    for (int nb = 0; nb < 2; ++nb) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      mma_bf16(d, a0, a1, a2, a3, bh[nb][0], bh[nb][1]);
      add4(acc[mt][nb], d);
    }
  }
}

// One warp per global row tile (32 rows of one leaf): every ancestor cluster's
// panel rows times its T, then the dense blocks of the leaf row.
// (one warp per CTA, 28 per SM, measured: the kernel is bound by loads in
// flight, and a warp that finishes its row tile frees its slot at once)
// With two halves of 16 right-hand sides every U tile is loaded once for both,
// and the warp holds twice the accumulators (16 warps per SM, 128 registers).
// WPC > 1 (passes of more than 32 right-hand sides): the CTA's warps take the
// same row tile, warp w parts w NH .., and share its factor tiles through L1.
constexpr int kP2PerSm = 28, kP2PerSm2 = 16;
template <int NH, int WPC>
__global__ void __launch_bounds__(32 * WPC, (NH == 1 ? kP2PerSm : kP2PerSm2) / WPC)
    k_mx_p2(int tile0, int tile_end, int depth, const int* __restrict__ tile_leaf,
                                               const int* __restrict__ leaf_tile0, const int* __restrict__ leaf_off,
                                               const int* __restrict__ pan_of, const MxPanel* __restrict__ panels,
                                               const uint4* __restrict__ store, const uint32_t* __restrict__ T,
                                               const int* __restrict__ leaf_dptr, const int* __restrict__ leaf_dblk,
                                               const MxDense* __restrict__ dense, const uint4* __restrict__ Xf,
                                               float* __restrict__ Y, int ldy, int nr, long long xh_, long long th) {
  // global row tiles [tile0, tile_end): every tile, or a block-row shard's
  const int G = tile0 + blockIdx.x;
  if (G >= tile_end) return;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  constexpr bool SH = WPC > 1;
  if (SH) {  // this warp's parts
    const int h0 = (threadIdx.x >> 5) * NH;
    T += h0 * th;
    Xf += h0 * xh_;
    Y += (size_t)16 * h0 * ldy;
    nr -= 16 * h0;
  }
  const int x = tile_leaf[G];
  float acc[NH][2][2][4];
#pragma unroll
  for (int h = 0; h < NH; ++h)
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nb = 0; nb < 2; ++nb)
        acc[h][mt][nb][0] = acc[h][mt][nb][1] = acc[h][mt][nb][2] = acc[h][mt][nb][3] = 0.f;
  const uint4 z = make_uint4(0u, 0u, 0u, 0u);
  // every ancestor's panel descriptor at once (lane l - 1 holds level l's),
  // instead of a chain of dependent loads per level
  int my_p = -1;
  long long my_u = 0, my_l = 0, my_t = 0;
  int my_nct = 0, my_nctl = 0;
  if (lane < depth) {
    const int l = lane + 1;
    my_p = __ldg(pan_of + (1 << l) - 1 + (x >> (depth - l)));
    if (my_p >= 0) {
      const MxPanel P = panels[my_p];
      const long long rt = G - P.tile0;
      my_u = P.hi2 + rt * P.nct;
      my_l = P.lo2 + rt * P.nctl;
      my_t = P.tw0;
      my_nct = P.nct;
      my_nctl = P.nctl;
    }
  }
  for (int l = 1; l <= depth; ++l) {
    const int p = __shfl_sync(0xffffffffu, my_p, l - 1);
    if (p < 0) continue;
    const long long ou = __shfl_sync(0xffffffffu, my_u, l - 1);
    const long long ol = __shfl_sync(0xffffffffu, my_l, l - 1);
    const long long ot = __shfl_sync(0xffffffffu, my_t, l - 1);
    const int nct = __shfl_sync(0xffffffffu, my_nct, l - 1);
    const int nctl = __shfl_sync(0xffffffffu, my_nctl, l - 1);
    const uint4* uh = store + ou * 32 + lane;
    const uint4* ul = store + ol * 32 + lane;
    // tiles with low parts: U (hi + lo) T (hi + lo)
    const uint4* tl = reinterpret_cast<const uint4*>(T + ot) + lane;
#pragma unroll 2
    for (int ct = 0; ct < nctl; ct += 2) {
      const bool two = ct + 1 < nctl;
      const uint4 h0 = ld_tile<SH>(uh + ct * 32);
      const uint4 h1 = two ? ld_tile<SH>(uh + (ct + 1) * 32) : z;
      const uint4 l0 = ld_tile<SH>(ul + ct * 32);
      const uint4 l1 = two ? ld_tile<SH>(ul + (ct + 1) * 32) : z;
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const uint4 t0 = __ldg(tl + h * (th >> 2) + ct * 32);
        const uint4 t1 = two ? __ldg(tl + h * (th >> 2) + (ct + 1) * 32) : z;
        // B pairs {T[2t], T[2t+1]} per tile from the per-column {hi, lo} words
        const uint32_t bh[2][2] = {{__byte_perm(t0.x, t0.z, 0x5410), __byte_perm(t1.x, t1.z, 0x5410)},
                                   {__byte_perm(t0.y, t0.w, 0x5410), __byte_perm(t1.y, t1.w, 0x5410)}};
        const uint32_t bl[2][2] = {{__byte_perm(t0.x, t0.z, 0x7632), __byte_perm(t1.x, t1.z, 0x7632)},
                                   {__byte_perm(t0.y, t0.w, 0x7632), __byte_perm(t1.y, t1.w, 0x7632)}};
        mx_p2_step(acc[h], h0, h1, l0, l1, bh, bl, true);
      }
    }
    // tiles without: U_hi T_hi
    const uint2* tw = reinterpret_cast<const uint2*>(T + ot + (long long)nctl * 128) + lane;
#pragma unroll 2
    for (int ct = nctl; ct < nct; ct += 2) {
      const bool two = ct + 1 < nct;
      const uint4 h0 = ld_tile<SH>(uh + ct * 32);
      const uint4 h1 = two ? ld_tile<SH>(uh + (ct + 1) * 32) : z;
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const uint2 w0 = __ldg(tw + h * (th >> 1) + (ct - nctl) * 32);
        const uint2 w1 = two ? __ldg(tw + h * (th >> 1) + (ct - nctl + 1) * 32) : make_uint2(0u, 0u);
        const uint32_t bh[2][2] = {{__byte_perm(w0.x, w0.y, 0x5410), __byte_perm(w1.x, w1.y, 0x5410)},
                                   {__byte_perm(w0.x, w0.y, 0x7632), __byte_perm(w1.x, w1.y, 0x7632)}};
        mx_p2_step_hi(acc[h], h0, h1, bh);
      }
    }
  }
  for (int q = leaf_dptr[x]; q < leaf_dptr[x + 1]; ++q) {
    const MxDense D = dense[leaf_dblk[q]];
    const long long rt = G - D.row_tile0;
    const uint4* dh = store + (D.hi + rt * D.nct) * 32 + lane;
    const uint4* dl = store + (D.lo + rt * D.nct) * 32 + lane;
    for (int ct = 0; ct < D.nct; ct += 2) {
      const uint4 h0 = ld_tile<SH>(dh + ct * 32), h1 = ld_tile<SH>(dh + (ct + 1) * 32);
      const uint4 l0 = ld_tile<SH>(dl + ct * 32), l1 = ld_tile<SH>(dl + (ct + 1) * 32);
      const size_t xt = (size_t)(D.col_tile0 + (ct >> 2)) * 128 + (size_t)((ct >> 1) & 1) * 32 + lane;
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const uint4 xh = __ldg(Xf + h * xh_ + xt), xl = __ldg(Xf + h * xh_ + xt + 64);
        const uint32_t bh[2][2] = {{xh.x, xh.z}, {xh.y, xh.w}};
        const uint32_t bl[2][2] = {{xl.x, xl.z}, {xl.y, xl.w}};
        mx_p2_step(acc[h], h0, h1, l0, l1, bh, bl, true);
      }
    }
  }
  const int base = leaf_off[x] + 32 * (G - leaf_tile0[x]);
  const int lim = leaf_off[x + 1];
#pragma unroll
  for (int h = 0; h < NH; ++h)
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nb = 0; nb < 2; ++nb) {
        const int ra = base + 16 * mt + g, rb = ra + 8, c = 16 * h + 8 * nb + 2 * t;
        if (c < nr) {
          if (ra < lim) Y[(size_t)c * ldy + ra] = acc[h][mt][nb][0];
          if (rb < lim) Y[(size_t)c * ldy + rb] = acc[h][mt][nb][2];
        }
        if (c + 1 < nr) {
          if (ra < lim) Y[(size_t)(c + 1) * ldy + ra] = acc[h][mt][nb][1];
          if (rb < lim) Y[(size_t)(c + 1) * ldy + rb] = acc[h][mt][nb][3];
        }
      }
}

// ---- conversion (build time) ------------------------------------------------
__device__ __forceinline__ int find_item(const long long* start, int n, long long w) {
  int lo = 0, hi = n - 1;  // largest i with start[i] <= w
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= w)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// One warp per 32 x 8 panel tile: both fragment orders, hi and (for the
// leading tiles) lo.  colsrc: per panel column, the FP32 factor column over
// the cluster's rows, or null for a padding column.
__global__ void k_mx_conv_panels(const MxPanel* __restrict__ panels, const long long* __restrict__ unit_start,
                                 int npanels, long long nunits, const float* const* __restrict__ colsrc,
                                 const int* __restrict__ tile_leaf, const int* __restrict__ leaf_tile0,
                                 const int* __restrict__ leaf_off, uint4* __restrict__ store) {
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nunits) return;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int pi = find_item(unit_start, npanels, w);
  const MxPanel P = panels[pi];
  const long long local = w - unit_start[pi];
  const int rt = (int)(local / P.nct), ct = (int)(local % P.nct);
  const int G = P.tile0 + rt;
  const int x = tile_leaf[G];
  const int rbase = leaf_off[x] + 32 * (G - leaf_tile0[x]) - P.r0;
  const int rlim = leaf_off[x + 1] - P.r0;
  const float* const* cs = colsrc + P.t0 * 8;
  auto val = [&](int r, int c) -> float {
    const float* col = cs[c];
    const int lr = rbase + r;
    return (col != nullptr && lr < rlim) ? col[lr] : 0.f;
  };
  uint4 h1, l1, h2, l2;
  const int cp1 = 8 * ct + g;
  split_bf16x2(val(2 * t, cp1), val(2 * t + 1, cp1), h1.x, l1.x);
  split_bf16x2(val(2 * t + 8, cp1), val(2 * t + 9, cp1), h1.y, l1.y);
  split_bf16x2(val(2 * t + 16, cp1), val(2 * t + 17, cp1), h1.z, l1.z);
  split_bf16x2(val(2 * t + 24, cp1), val(2 * t + 25, cp1), h1.w, l1.w);
  const int cp2 = 8 * ct + 2 * t;
  split_bf16x2(val(g, cp2), val(g, cp2 + 1), h2.x, l2.x);
  split_bf16x2(val(g + 8, cp2), val(g + 8, cp2 + 1), h2.y, l2.y);
  split_bf16x2(val(g + 16, cp2), val(g + 16, cp2 + 1), h2.z, l2.z);
  split_bf16x2(val(g + 24, cp2), val(g + 24, cp2 + 1), h2.w, l2.w);
  store[(P.hi1 + (long long)rt * P.nct + ct) * 32 + p1_slot(lane)] = h1;
  store[(P.hi2 + (long long)rt * P.nct + ct) * 32 + lane] = h2;
  if (ct < P.nctl) {
    store[(P.lo1 + (long long)rt * P.nctl + ct) * 32 + p1_slot(lane)] = l1;
    store[(P.lo2 + (long long)rt * P.nctl + ct) * 32 + lane] = l2;
  }
}

// One warp per 32 x 8 tile of a dense block (P2 order, hi + lo)
__global__ void k_mx_conv_dense(const MxDense* __restrict__ dense, const long long* __restrict__ unit_start,
                                int ndense, long long nunits, const int* __restrict__ tile_leaf,
                                const int* __restrict__ leaf_tile0, const int* __restrict__ leaf_off,
                                uint4* __restrict__ store) {
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nunits) return;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int di = find_item(unit_start, ndense, w);
  const MxDense D = dense[di];
  const long long local = w - unit_start[di];
  const int rt = (int)(local / D.nct), ct = (int)(local % D.nct);
  const int G = D.row_tile0 + rt;
  const int x = tile_leaf[G];
  const int rbase = leaf_off[x] + 32 * (G - leaf_tile0[x]) - D.r0;
  const int rlim = leaf_off[x + 1] - D.r0;
  const int pc = 8 * ct + 2 * t;  // padded column (even; pc and pc + 1 share a 32-column tile)
  const int GC = D.col_tile0 + (pc >> 5);
  const int y = tile_leaf[GC];
  const int cbase = leaf_off[y] + 32 * (GC - leaf_tile0[y]) - D.c0 + (pc & 31);
  const int clim = leaf_off[y + 1] - D.c0;
  auto val = [&](int r, int c) -> float {
    const int lr = rbase + r;
    return (lr < rlim && c < clim) ? D.src[(size_t)c * D.m + lr] : 0.f;
  };
  uint4 h, l;
  split_bf16x2(val(g, cbase), val(g, cbase + 1), h.x, l.x);
  split_bf16x2(val(g + 8, cbase), val(g + 8, cbase + 1), h.y, l.y);
  split_bf16x2(val(g + 16, cbase), val(g + 16, cbase + 1), h.z, l.z);
  split_bf16x2(val(g + 24, cbase), val(g + 24, cbase + 1), h.w, l.w);
  store[(D.hi + (long long)rt * D.nct + ct) * 32 + lane] = h;
  store[(D.lo + (long long)rt * D.nct + ct) * 32 + lane] = l;
}

template <class T>
hm_status upload(DevBuf<T>& b, const std::vector<T>& v, cudaStream_t s) {
  HM_TRY(b.alloc(std::max<size_t>(v.size(), 1)));
  if (!v.empty()) HM_CUDA(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  return HM_OK;
}

}  // namespace

hm_status mixed_build(hm_hmatrix_s* h, const std::vector<MxPair>& pairs, const std::vector<MxDenseIn>& dense_in,
                      cudaStream_t s) {
  MxPlan& M = h->mx;
  // FP32 format: no low parts, 1 KB tiles (two 512-byte units), T indexed by
  // global column (128 words per 8-column tile)
  const bool f32 = M.fmt == 1;
  const int tu = f32 ? 2 : 1;  // 512-byte units per tile
  const int depth = h->depth;
  const std::vector<int>& lo = h->tree->h_offsets;
  const int nleaf = 1 << depth;

  // global 32-row tiles, padded per leaf
  std::vector<int> leaf_tile0(nleaf + 1), tile_leaf;
  for (int x = 0; x < nleaf; ++x) {
    leaf_tile0[x] = (int)tile_leaf.size();
    const int nt = (lo[x + 1] - lo[x] + 31) / 32;
    for (int i = 0; i < nt; ++i) tile_leaf.push_back(x);
  }
  leaf_tile0[nleaf] = (int)tile_leaf.size();
  M.num_tiles = (int)tile_leaf.size();
  // phase 2 runs over the row tiles of the matrix's rows (a block-row shard's own leaves)
  M.p2_tile0 = leaf_tile0[h->leaf_lo];
  M.p2_tiles = leaf_tile0[h->leaf_hi] - M.p2_tile0;

  // leaf range [first, end) of the cluster whose rows are [r0, r0 + m)
  auto leaf_range = [&](int r0, int m, int* first, int* end) {
    *first = (int)(std::lower_bound(lo.begin(), lo.end() - 1, r0) - lo.begin());
    *end = (int)(std::lower_bound(lo.begin(), lo.end() - 1, r0 + m) - lo.begin());
  };
  // the level-l cluster with rows [r0, r0 + m) (m > 0)
  auto cluster_of = [&](int level, int r0, int m) -> int {
    const int sh = depth - level;
    int a = 0, b = (1 << level) - 1;  // first a with lo[a << sh] >= r0
    while (a < b) {
      const int mid = (a + b) >> 1;
      if (lo[(size_t)mid << sh] < r0)
        a = mid + 1;
      else
        b = mid;
    }
    while (a + 1 < (1 << level) && lo[(size_t)(a + 1) << sh] - r0 < m) ++a;  // skip empty clusters
    return a;
  };

  // ---- panels ----------------------------------------------------------------
  std::vector<int> pan_of(((size_t)2 << depth) - 1, -1);
  struct Side {
    int pair, side;  // side 0: fu (row cluster), 1: fv (column cluster)
  };
  std::vector<std::vector<Side>> members;
  std::vector<int> plevel, pcl;
  std::vector<int> panel_u(pairs.size(), -1), panel_v(pairs.size(), -1);
  for (size_t i = 0; i < pairs.size(); ++i) {
    const MxPair& q = pairs[i];
    if (q.k <= 0) continue;
    for (int side = 0; side < 2; ++side) {
      const int a = side ? cluster_of(q.level, q.c0, q.n) : cluster_of(q.level, q.r0, q.m);
      const size_t id = ((size_t)1 << q.level) - 1 + a;
      if (pan_of[id] < 0) {
        pan_of[id] = (int)members.size();
        members.emplace_back();
        plevel.push_back(q.level);
        pcl.push_back(a);
      }
      members[pan_of[id]].push_back(Side{(int)i, side});
      (side ? panel_v : panel_u)[i] = pan_of[id];
    }
  }
  const int np = (int)members.size();
  std::vector<MxPanel> panels(np);
  std::vector<int> colL_u(pairs.size()), colH_u(pairs.size()), colL_v(pairs.size()), colH_v(pairs.size());
  long long tiles = 0, t_tiles = 0, t_words = 0, t_blocks = 0;
  for (int p = 0; p < np; ++p) {
    long long sl = 0, sh_ = 0;
    for (const Side& m : members[p]) {
      const int kl = f32 ? 0 : pairs[m.pair].khi;
      sl += kl;
      sh_ += pairs[m.pair].k - kl;
    }
    const int KL = (int)((sl + 7) / 8 * 8), KH = (int)((sh_ + 7) / 8 * 8);
    long long al = 0, ah = KL;
    for (const Side& m : members[p]) {
      const MxPair& q = pairs[m.pair];
      const int kl = f32 ? 0 : q.khi;
      (m.side ? colL_v : colL_u)[m.pair] = (int)al;
      (m.side ? colH_v : colH_u)[m.pair] = (int)ah;
      al += kl;
      ah += q.k - kl;
    }
    MxPanel& P = panels[p];
    const int sh = depth - plevel[p];
    const int x0 = pcl[p] << sh, x1 = (pcl[p] + 1) << sh;
    P.nct = (KL + KH) / 8;
    P.nctl = KL / 8;
    P.tile0 = leaf_tile0[x0];
    P.nrt = leaf_tile0[x1] - P.tile0;
    P.r0 = lo[x0];
    P.hi1 = tiles;
    tiles += (long long)P.nrt * P.nct * tu;
    P.lo1 = tiles;
    tiles += (long long)P.nrt * P.nctl;
    P.hi2 = tiles;
    tiles += (long long)P.nrt * P.nct * tu;
    P.lo2 = tiles;
    tiles += (long long)P.nrt * P.nctl;
    P.t0 = t_tiles;
    t_tiles += P.nct;
    P.tw0 = t_words;
    t_words += f32 ? (long long)P.nct * 128 : (long long)P.nctl * 128 + (long long)(P.nct - P.nctl) * 64;
    P.tb0 = t_blocks;
    t_blocks += P.nct + P.nctl;
  }

  // column sources and the projection's column map
  if ((long long)t_tiles * 8 > 0x7fffffffll || (!f32 && t_words >= (1ll << 30)))
    return fail(HM_ERR_UNSUPPORTED, "panel form: too many factor columns");
  std::vector<const float*> colsrc((size_t)t_tiles * 8, nullptr);
  std::vector<int> mirror((size_t)t_tiles * 8, -1);  // partner column (an involution)
  long long bytes_lr = 0;
  for (size_t i = 0; i < pairs.size(); ++i) {
    const MxPair& q = pairs[i];
    if (q.k <= 0) continue;
    const int pu = panel_u[i], pv = panel_v[i];
    const long long bu = panels[pu].t0 * 8, bv = panels[pv].t0 * 8;
    const int kl = f32 ? 0 : q.khi;
    for (int c = 0; c < q.k; ++c) {
      const int cu = c < kl ? colL_u[i] + c : colH_u[i] + c - kl;
      const int cv = c < kl ? colL_v[i] + c : colH_v[i] + c - kl;
      colsrc[bu + cu] = q.fu + (size_t)c * q.m;
      colsrc[bv + cv] = q.fv + (size_t)c * q.n;
      mirror[bv + cv] = (int)(bu + cu);  // Y_u += fu (fv^T X_v)
      mirror[bu + cu] = (int)(bv + cv);  // Y_v += fv (fu^T X_u)
    }
    bytes_lr += f32 ? 4ll * (q.m + q.n) * q.k : 2ll * (q.m + q.n) * (q.k + q.khi);
  }
  std::vector<MxLoc> locs;
  locs.reserve(2 * pairs.size() + dense_in.size());
  for (size_t i = 0; i < pairs.size(); ++i) {
    const MxPair& q = pairs[i];
    if (q.k <= 0) continue;
    const int kl = f32 ? 0 : q.khi;
    locs.push_back(MxLoc{q.fu, 0, panel_u[i], q.m, q.k, kl, colL_u[i], colH_u[i]});
    locs.push_back(MxLoc{q.fv, 0, panel_v[i], q.n, q.k, kl, colL_v[i], colH_v[i]});
  }


  // ---- dense blocks ----------------------------------------------------------
  std::vector<MxDense> dense;
  std::vector<std::vector<int>> leaf_d(nleaf);
  long long bytes_dense = 0;
  for (const MxDenseIn& di : dense_in) {
    if (di.m <= 0 || di.n <= 0) continue;
    int xs, xe, ys, ye;
    leaf_range(di.r0, di.m, &xs, &xe);
    leaf_range(di.c0, di.n, &ys, &ye);
    MxDense D{};
    D.row_tile0 = leaf_tile0[xs];
    D.nrt = leaf_tile0[xe] - D.row_tile0;
    D.col_tile0 = leaf_tile0[ys];
    D.nct = 4 * (leaf_tile0[ye] - D.col_tile0);
    D.r0 = di.r0;
    D.c0 = di.c0;
    D.m = di.m;
    D.n = di.n;
    D.src = di.D;
    D.hi = tiles;
    tiles += (long long)D.nrt * D.nct * tu;
    D.lo = tiles;
    if (!f32) tiles += (long long)D.nrt * D.nct;
    for (int x = xs; x < xe; ++x) leaf_d[x].push_back((int)dense.size());
    locs.push_back(MxLoc{di.D, 1, (int)dense.size(), di.m, di.n, 0, 0, 0});
    dense.push_back(D);
    bytes_dense += 4ll * di.m * di.n;
  }
  std::vector<int> dptr(nleaf + 1, 0), dblk;
  for (int x = 0; x < nleaf; ++x) {
    dptr[x] = (int)dblk.size();
    dblk.insert(dblk.end(), leaf_d[x].begin(), leaf_d[x].end());
  }
  dptr[nleaf] = (int)dblk.size();

  // ---- upload and convert ----------------------------------------------------
  M.store_tiles = tiles;
  HM_TRY(M.store.alloc((size_t)std::max<long long>(tiles, 1) * 32));
  M.h_panels = panels;
  HM_TRY(mixed_schedule(h, M.chunk_tiles, M.group_tiles, M.p1_ring ? 1 : 0, s));
  HM_TRY(upload(M.pan_of, pan_of, s));
  HM_TRY(upload(M.tile_leaf, tile_leaf, s));
  HM_TRY(upload(M.leaf_tile0, leaf_tile0, s));
  // BF16 format: (word << 1) | no-low-part of the destination; FP32 format:
  // the destination's global column (its T words follow from it)
  std::vector<int> own(mirror.size()), tslot(mirror.size());
  for (const MxPanel& P : panels)
    for (int c = 0; c < P.nct * 8; ++c)
      own[P.t0 * 8 + c] = f32 ? (int)(P.t0 * 8 + c)
                              : (int)(t_word(P.tw0, P.nctl, c) << 1) | ((c >> 3) >= P.nctl ? 1 : 0);
  for (size_t c = 0; c < mirror.size(); ++c) tslot[c] = mirror[c] >= 0 ? own[mirror[c]] : -1 - own[c];
  HM_TRY(upload(M.tslot, tslot, s));
  if (!f32) {
    // 128-column passes on tcgen05: the T blocks' column map, and phase 2's
    // blocks of 4 row tiles with their sources
    std::vector<int2> own_tc(mirror.size()), tslot_tc(mirror.size());
    for (const MxPanel& P : panels)
      for (int c = 0; c < P.nct * 8; ++c) {
        const int j = c >> 3, cc = c & 7;
        own_tc[P.t0 * 8 + c] = make_int2((int)((P.tb0 + j) * 8 + cc),
                                         j < P.nctl ? (int)((P.tb0 + P.nct + j) * 8 + cc) : -1);
      }
    for (size_t c = 0; c < mirror.size(); ++c)
      tslot_tc[c] = mirror[c] >= 0 ? own_tc[mirror[c]] : make_int2(-1 - own_tc[c].x, own_tc[c].y);
    HM_TRY(upload(M.tslot_tc, tslot_tc, s));
    std::vector<P2Step> steps;
    std::vector<int> step_ptr(1, 0);
    const int tend = M.p2_tile0 + M.p2_tiles;
    auto mask_of = [](int k, int k2) { return ((1 << k2) - 1) & ~((1 << k) - 1); };
    auto add_panel = [&](int p, int mask, int G0) {
      const MxPanel& P = panels[p];
      const long long rb = G0 - P.tile0;  // the panel's row tile of the block's tile 0
      for (int j0 = 0; j0 < P.nctl; j0 += 4)
        steps.push_back(P2Step{P.hi2 + rb * P.nct + j0, P.lo2 + rb * P.nctl + j0, (P.tb0 + j0) * 128,
                               (P.tb0 + P.nct + j0) * 128, P.nct, P.nctl,
                               0 | (std::min(4, P.nctl - j0) << 2) | (mask << 8), 0});
      for (int j0 = P.nctl; j0 < P.nct; j0 += 8)
        steps.push_back(P2Step{P.hi2 + rb * P.nct + j0, -1, (P.tb0 + j0) * 128, -1, P.nct, 0,
                               1 | (std::min(8, P.nct - j0) << 2) | (mask << 8), 0});
    };
    for (int G0 = M.p2_tile0; G0 < tend; G0 += 4) {
      const int nk = std::min(4, tend - G0);
      for (int l = 1; l <= depth; ++l)
        for (int k = 0; k < nk;) {
          const int p = pan_of[((size_t)1 << l) - 1 + (tile_leaf[G0 + k] >> (depth - l))];
          int k2 = k + 1;
          while (k2 < nk && pan_of[((size_t)1 << l) - 1 + (tile_leaf[G0 + k2] >> (depth - l))] == p) ++k2;
          if (p >= 0) add_panel(p, mask_of(k, k2), G0);
          k = k2;
        }
      for (int k = 0; k < nk;) {
        const int x = tile_leaf[G0 + k];
        int k2 = k + 1;
        while (k2 < nk && tile_leaf[G0 + k2] == x) ++k2;
        for (int q = dptr[x]; q < dptr[x + 1]; ++q) {
          const MxDense& D = dense[dblk[q]];
          const long long rb = G0 - D.row_tile0;
          for (int j0 = 0; j0 < D.nct; j0 += 4)
            steps.push_back(P2Step{D.hi + rb * D.nct + j0, D.lo + rb * D.nct + j0,
                                   (long long)(D.col_tile0 + j0 / 4) * 1024, (long long)(D.col_tile0 + j0 / 4) * 1024 + 512,
                                   D.nct, D.nct, 2 | (4 << 2) | (mask_of(k, k2) << 8), 0});
        }
        k = k2;
      }
      if ((int)steps.size() == step_ptr.back()) steps.push_back(P2Step{0, -1, 0, -1, 0, 0, 3, 0});
      step_ptr.push_back((int)steps.size());
    }
    HM_TRY(upload(M.p2_steps, steps, s));
    HM_TRY(upload(M.p2_step_ptr, step_ptr, s));
    M.p2_blocks = (int)step_ptr.size() - 1;
  }
  HM_TRY(upload(M.dense, dense, s));
  HM_TRY(upload(M.leaf_dptr, dptr, s));
  HM_TRY(upload(M.leaf_dblk, dblk, s));
  M.num_panels = np;
  M.num_dense = (int)dense.size();
  M.h_dense = dense;
  M.h_locs = std::move(locs);
  M.loc_index.clear();
  M.t_tiles = t_tiles;
  M.t_words = t_words;
  // each factor is read once per phase (as V of one orientation in phase 1,
  // as U of the other in phase 2)
  M.bytes_p1 = bytes_lr;
  M.bytes_p2 = bytes_lr + bytes_dense;

  if (f32) {
    HM_TRY(fp32_convert(h, colsrc, dense, s));
    HM_CUDA(cudaStreamSynchronize(s));
    M.enabled = true;
    return HM_OK;
  }
  DevBuf<const float*> dcol;
  DevBuf<long long> dstart;
  if (np > 0) {
    std::vector<long long> start(np);
    long long tot = 0;
    for (int p = 0; p < np; ++p) {
      start[p] = tot;
      tot += (long long)panels[p].nrt * panels[p].nct;
    }
    HM_TRY(upload(dcol, colsrc, s));
    HM_TRY(upload(dstart, start, s));
    if (tot > 0) {
      k_mx_conv_panels<<<(unsigned)((tot * 32 + 255) / 256), 256, 0, s>>>(
          M.panels.p, dstart.p, np, tot, dcol.p, M.tile_leaf.p, M.leaf_tile0.p, h->tree->offsets.p, M.store.p);
      HM_LAUNCH_CHECK();
    }
    HM_CUDA(cudaStreamSynchronize(s));
  }
  if (!dense.empty()) {
    std::vector<long long> start(dense.size());
    long long tot = 0;
    for (size_t i = 0; i < dense.size(); ++i) {
      start[i] = tot;
      tot += (long long)dense[i].nrt * dense[i].nct;
    }
    DevBuf<long long> ds;
    HM_TRY(upload(ds, start, s));
    if (tot > 0) {
      k_mx_conv_dense<<<(unsigned)((tot * 32 + 255) / 256), 256, 0, s>>>(
          M.dense.p, ds.p, (int)dense.size(), tot, M.tile_leaf.p, M.leaf_tile0.p, h->tree->offsets.p, M.store.p);
      HM_LAUNCH_CHECK();
    }
    HM_CUDA(cudaStreamSynchronize(s));
  }
  HM_CUDA(cudaStreamSynchronize(s));
  M.enabled = true;
  return HM_OK;
}

namespace {

struct UnpackJob {
  int kind, idx, rows, cols, khi, colL, colH;
  float* dst;
};

// row R (tree order) -> its global 32-row tile and the row within it
__device__ __forceinline__ void row_tile(const int* __restrict__ leaf_off, const int* __restrict__ leaf_tile0,
                                         int nleaf, int R, int* G, int* rr) {
  int lo = 0, hi = nleaf - 1;  // the leaf x with leaf_off[x] <= R < leaf_off[x + 1]
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (leaf_off[mid] <= R)
      lo = mid;
    else
      hi = mid - 1;
  }
  *G = leaf_tile0[lo] + (R - leaf_off[lo]) / 32;
  *rr = (R - leaf_off[lo]) % 32;
}

// element (rr, cc) of a P2-order BF16 tile at unit `tile`, as a float
__device__ __forceinline__ float p2_elem(const uint4* __restrict__ store, long long tile, int rr, int cc) {
  const int lane = 4 * (rr & 7) + (cc >> 1), comp = rr >> 3;
  const uint32_t w = reinterpret_cast<const uint32_t*>(store + tile * 32 + lane)[comp];
  return (cc & 1) ? bf16_hi_as_float(w) : bf16_lo_as_float(w);
}

__global__ void k_mx_unpack(const UnpackJob* __restrict__ jobs, const long long* __restrict__ start, int njobs,
                            long long total, const MxPanel* __restrict__ panels, const MxDense* __restrict__ dense,
                            const uint4* __restrict__ store, const int* __restrict__ leaf_off,
                            const int* __restrict__ leaf_tile0, int nleaf) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  const int j = find_item(start, njobs, e);
  const UnpackJob J = jobs[j];
  const long long local = e - start[j];
  const int r = (int)(local % J.rows), c = (int)(local / J.rows);
  int G, rr, ct, cc;
  long long thi, tlo = -1;
  if (J.kind == 0) {
    const MxPanel P = panels[J.idx];
    row_tile(leaf_off, leaf_tile0, nleaf, P.r0 + r, &G, &rr);
    const int pc = c < J.khi ? J.colL + c : J.colH + c - J.khi;
    ct = pc >> 3;
    cc = pc & 7;
    thi = P.hi2 + (long long)(G - P.tile0) * P.nct + ct;
    if (ct < P.nctl) tlo = P.lo2 + (long long)(G - P.tile0) * P.nctl + ct;
  } else {
    const MxDense D = dense[J.idx];
    row_tile(leaf_off, leaf_tile0, nleaf, D.r0 + r, &G, &rr);
    int GC, cr;
    row_tile(leaf_off, leaf_tile0, nleaf, D.c0 + c, &GC, &cr);
    const int pc = (GC - D.col_tile0) * 32 + cr;
    ct = pc >> 3;
    cc = pc & 7;
    thi = D.hi + (long long)(G - D.row_tile0) * D.nct + ct;
    tlo = D.lo + (long long)(G - D.row_tile0) * D.nct + ct;
  }
  const float hi = p2_elem(store, thi, rr, cc);
  float y = hi;
  if (tlo >= 0) {
    const float lo = p2_elem(store, tlo, rr, cc);
    y = hi + lo;  // exact: hi + lo has at most 24 significant bits
    // a tie (|lo| half a BF16 ulp of hi) would round to the other neighbour
    if (bf16_lo_as_float(pack_bf16(y, 0.f)) != hi) y = nextafterf(y, hi);
  }
  J.dst[(size_t)c * J.rows + r] = y;
}

}  // namespace

int mixed_find_loc(hm_hmatrix_s* h, const float* key) {
  MxPlan& M = h->mx;
  if (M.loc_index.size() != M.h_locs.size()) {
    M.loc_index.resize(M.h_locs.size());
    for (size_t i = 0; i < M.h_locs.size(); ++i) M.loc_index[i] = {M.h_locs[i].key, (int)i};
    std::sort(M.loc_index.begin(), M.loc_index.end(),
              [](const std::pair<const float*, int>& a, const std::pair<const float*, int>& b) {
                return std::less<const float*>()(a.first, b.first);
              });
  }
  auto it = std::lower_bound(M.loc_index.begin(), M.loc_index.end(), std::make_pair(key, -1),
                             [](const std::pair<const float*, int>& a, const std::pair<const float*, int>& b) {
                               return std::less<const float*>()(a.first, b.first);
                             });
  return (it != M.loc_index.end() && it->first == key) ? it->second : -1;
}

hm_status mixed_unpack(hm_hmatrix_s* h, const std::vector<std::pair<int, float*>>& jobs, cudaStream_t s) {
  MxPlan& M = h->mx;
  if (jobs.empty()) return HM_OK;
  if (M.fmt != 0) return fail(HM_ERR_UNSUPPORTED, "panel unpack: FP32 panels keep their FP32 factors");
  std::vector<UnpackJob> uj;
  std::vector<long long> start;
  long long tot = 0;
  for (const auto& jb : jobs) {
    if (jb.first < 0 || (size_t)jb.first >= M.h_locs.size())
      return fail(HM_ERR_INVALID, "panel unpack: unknown factor");
    const MxLoc& L = M.h_locs[jb.first];
    if ((long long)L.rows * L.cols == 0) continue;
    uj.push_back(UnpackJob{L.kind, L.idx, L.rows, L.cols, L.khi, L.colL, L.colH, jb.second});
    start.push_back(tot);
    tot += (long long)L.rows * L.cols;
  }
  if (tot == 0) return HM_OK;
  DevBuf<UnpackJob> dj;
  DevBuf<long long> ds;
  HM_TRY(upload(dj, uj, s));
  HM_TRY(upload(ds, start, s));
  k_mx_unpack<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(dj.p, ds.p, (int)uj.size(), tot, M.panels.p, M.dense.p,
                                                            M.store.p, h->tree->offsets.p, M.leaf_tile0.p,
                                                            1 << h->depth);
  HM_LAUNCH_CHECK();
  HM_CUDA(cudaStreamSynchronize(s));
  return HM_OK;
}

hm_status mixed_schedule(hm_hmatrix_s* h, int chunk_tiles, int group_tiles, int p1_ring, cudaStream_t s) {
  MxPlan& M = h->mx;
  if (M.fmt == 1) p1_ring = 0;  // the ring variant exists for the BF16 format only
  if (p1_ring) {
    int dev = 0;
    HM_CUDA(cudaGetDevice(&dev));
    HM_CUDA(cudaDeviceGetAttribute(&M.num_sms, cudaDevAttrMultiProcessorCount, dev));
    HM_CUDA(cudaFuncSetAttribute(k_mx_p1r<8, 3, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ring_smem<8, 3, 4>()));
    HM_CUDA(cudaFuncSetAttribute(k_mx_p1r<4, 4, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ring_smem<4, 4, 8>()));
  }
  M.p1_ring = p1_ring != 0;
  if (chunk_tiles < 1 || group_tiles < 1 || group_tiles > 8)
    return fail(HM_ERR_INVALID, "mixed schedule: need chunk >= 1 and 1 <= group <= 8 column tiles");
  std::vector<MxPanel>& panels = M.h_panels;
  long long s_tiles = 0;
  std::vector<MxUnit> units;
  std::vector<int2> mtiles;  // column tiles of panels projected in several row chunks
  for (int p = 0; p < (int)panels.size(); ++p) {
    MxPanel& P = panels[p];
    P.nchunk = std::max(1, (P.nrt + chunk_tiles - 1) / chunk_tiles);
    P.s0 = s_tiles;
    if (P.nchunk > 1) {
      s_tiles += (long long)P.nchunk * P.nct;
      for (int c = 0; c < P.nct; ++c) mtiles.push_back(make_int2(p, c));
    }
    for (int c = 0; c < P.nct; c += group_tiles)
      for (int ch = 0; ch < P.nchunk; ++ch)
        units.push_back(MxUnit{p, c, std::min(group_tiles, P.nct - c), ch * chunk_tiles,
                               std::min(chunk_tiles, P.nrt - ch * chunk_tiles), ch});
  }
  // the largest units first, so that the small ones fill the tail
  auto larger = [](const MxUnit& a, const MxUnit& b) { return a.nrt * a.nct > b.nrt * b.nct; };
  std::stable_sort(units.begin(), units.end(), larger);
  // tcgen05 units (128-column passes): 16 column tiles, low-part tiles apart,
  // over row chunks of their own size, with their own partials
  std::vector<TcUnit> tcu;
  std::vector<int2> mtiles_tc;
  long long s_tiles_tc = 0;
  if (M.fmt == 0) {
    const int tch = std::max(1, M.tc_chunk_tiles);
    for (int p = 0; p < (int)panels.size(); ++p) {
      MxPanel& P = panels[p];
      P.nchunkt = std::max(1, (P.nrt + tch - 1) / tch);
      P.s0t = s_tiles_tc;
      if (P.nchunkt > 1) {
        s_tiles_tc += (long long)P.nchunkt * P.nct;
        for (int c = 0; c < P.nct; ++c) mtiles_tc.push_back(make_int2(p, c));
      }
      for (int part = 0; part < 2; ++part) {
        const int c0 = part ? P.nctl : 0, c1 = part ? P.nct : P.nctl;
        for (int c = c0; c < c1; c += 16)
          for (int ch = 0; ch < P.nchunkt; ++ch) {
            TcUnit t{};
            const int rt0 = ch * tch;
            t.nct = std::min(16, c1 - c);
            t.nrt = std::min(tch, P.nrt - rt0);
            t.shi = P.nct;
            t.slo = P.nctl;
            t.vhi = P.hi1 + (long long)rt0 * P.nct + c;
            t.vlo = part ? -1 : P.lo1 + (long long)rt0 * P.nctl + c;
            t.xtile = P.tile0 + rt0;
            t.flags = (part ? 0 : 1) | (P.nchunkt == 1 ? 2 : 0);
            t.out = P.nchunkt == 1 ? P.t0 + c : P.s0t + (long long)ch * P.nct + c;
            tcu.push_back(t);
          }
      }
    }
    // in row order (the larger unit first among those that start on the same
    // row tile): the CTAs, each walking every gridDim-th unit, then work on
    // nearby rows at every level at once, and X's image of those rows is
    // read from HBM about once for all levels (it stays in L2 between them)
    std::stable_sort(tcu.begin(), tcu.end(), [](const TcUnit& a, const TcUnit& b) {
      return a.xtile != b.xtile ? a.xtile < b.xtile : a.nrt > b.nrt;
    });
    int dev = 0;
    HM_CUDA(cudaGetDevice(&dev));
    HM_CUDA(cudaDeviceGetAttribute(&M.num_sms, cudaDevAttrMultiProcessorCount, dev));
    if (!M.tc_err.p) {
      HM_TRY(M.tc_err.alloc(1));
      HM_CUDA(cudaMemsetAsync(M.tc_err.p, 0, sizeof(int), s));
    }
  }
  HM_TRY(upload(M.tc_units, tcu, s));
  HM_TRY(upload(M.mtiles_tc, mtiles_tc, s));
  M.num_tc_units = (int)tcu.size();
  M.nmt_tc = (long long)mtiles_tc.size();
  M.s_tiles_tc = s_tiles_tc;
  HM_TRY(upload(M.panels, panels, s));
  HM_TRY(upload(M.units, units, s));
  HM_TRY(upload(M.mtiles, mtiles, s));
  HM_CUDA(cudaStreamSynchronize(s));
  M.nmt = (long long)mtiles.size();
  M.num_units = (int)units.size();
  M.s_tiles = s_tiles;
  M.chunk_tiles = chunk_tiles;
  M.group_tiles = group_tiles;
  return HM_OK;
}

hm_status mixed_warp_pass(hm_hmatrix_s* h, int nh, int nr, uint4* Xf, float4* S, uint32_t* T, long long xh,
                          long long sh, long long th, float* Y, int ldy, cudaStream_t s, KernelMarks* km);

hm_status mixed_run_panel(hm_hmatrix_s* h, int nr, const float* X, int ldx, float* Y, int ldy, float* scratch,
                          cudaStream_t s, KernelMarks* km) {
  MxPlan& M = h->mx;
  if (M.fmt == 1) return fp32_run_panel(h, nr, X, ldx, Y, ldy, scratch, s, km);
  if (nr < 1 || nr > 128) return fail(HM_ERR_INVALID, "mixed product: a pass holds 1 to 128 right-hand sides");
  // 16-column parts of this pass: 1, 2, 4 or 8 (the parts past nr are zero)
  const int nh = nr > 64 ? 8 : (nr > 32 ? 4 : (nr > 16 ? 2 : 1));
  // scratch: the parts' X fragments, then their chunk partials, then their T
  const long long xh = (long long)M.num_tiles * 128, sh = M.s_tiles * 32, th = M.t_words;
  // (a 128-column pass on tcgen05: X's image where the fragments would be,
  // T in blocks where the parts' T would be)
  const bool tc = M.tc_pass(nh);
  uint4* Xf = reinterpret_cast<uint4*>(scratch);
  float4* S = reinterpret_cast<float4*>(Xf + nh * xh);
  // (the tcgen05 pass's partials, 4 KB per tile of its own chunking, may take more room)
  const long long s_room = tc ? std::max(M.s_tiles, M.s_tiles_tc) * 32 : sh;
  uint32_t* T = reinterpret_cast<uint32_t*>(S + nh * s_room);
  const int* leaf_off = h->tree->offsets.p;
  const long long xbytes = 4ll * h->n * 16 * nh;  // the X fragments, hi + lo
  if (M.num_tiles > 0) {
    k_mx_split_x<<<dim3((M.num_tiles + 3) / 4, nh), 128, 0, s>>>(X, ldx, nr, M.num_tiles, M.tile_leaf.p,
                                                                 M.leaf_tile0.p, leaf_off, Xf, tc ? Xf : nullptr);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_mx_split_x", 4ll * h->n * nr + xbytes, s);
  }
  if (tc) {
    HM_TRY(mixed_tc_pass(h, nr, Xf, reinterpret_cast<float*>(S), reinterpret_cast<uint4*>(T), Y, ldy, s, km));
  } else {
    HM_TRY(mixed_warp_pass(h, nh, nr, Xf, S, T, xh, sh, th, Y, ldy, s, km));
  }
  if (h->diag_fly)  // the diagonal from coordinates, 16 columns at a time
    for (int c0 = 0; c0 < nr; c0 += 16)
      HM_TRY(diag_fly_panel(h, std::min(16, nr - c0), X + (size_t)c0 * ldx, ldx, Y + (size_t)c0 * ldy, ldy, s, km));
  return HM_OK;
}

// Phases 1 and 2 of a pass on the warp-level MMA kernels (nh parts of 16).
hm_status mixed_warp_pass(hm_hmatrix_s* h, int nh, int nr, uint4* Xf, float4* S, uint32_t* T, long long xh,
                          long long sh, long long th, float* Y, int ldy, cudaStream_t s, KernelMarks* km) {
  MxPlan& M = h->mx;
  const int* leaf_off = h->tree->offsets.p;
  const long long xbytes = 4ll * h->n * 16 * nh;
  if (M.num_units > 0) {
    const unsigned nu = (unsigned)M.num_units;
    if (M.p1_ring && nh == 1 && M.group_tiles <= 4) {
      k_mx_p1r<8, 3, 4><<<M.num_sms, 256, ring_smem<8, 3, 4>(), s>>>(M.units.p, M.num_units, M.panels.p, M.store.p,
                                                                      Xf, M.tslot.p, S, T);
    } else if (M.p1_ring && nh == 1) {
      k_mx_p1r<4, 4, 8><<<M.num_sms, 128, ring_smem<4, 4, 8>(), s>>>(M.units.p, M.num_units, M.panels.p, M.store.p,
                                                                      Xf, M.tslot.p, S, T);
    } else if (nh == 1) {
      k_mx_p1<1, 1><<<nu, 32, 0, s>>>(M.units.p, M.num_units, M.panels.p, M.store.p, Xf, M.tslot.p, S, T, xh, sh, th);
    } else if (nh == 2) {
      k_mx_p1<2, 1><<<nu, 32, 0, s>>>(M.units.p, M.num_units, M.panels.p, M.store.p, Xf, M.tslot.p, S, T, xh, sh, th);
    } else if (nh == 4) {
      k_mx_p1<4, 1><<<nu, 32, 0, s>>>(M.units.p, M.num_units, M.panels.p, M.store.p, Xf, M.tslot.p, S, T, xh, sh, th);
    } else {  // eight parts: two warps of four parts share each unit's tiles
      k_mx_p1<4, 2><<<nu, 64, 0, s>>>(M.units.p, M.num_units, M.panels.p, M.store.p, Xf, M.tslot.p, S, T, xh, sh, th);
    }
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_mx_p1", M.bytes_p1 + xbytes, s);
  }
  if (M.nmt > 0) {
    k_mx_reduce<<<dim3((unsigned)((M.nmt * 32 + 255) / 256), nh), 256, 0, s>>>(M.mtiles.p, M.nmt, M.panels.p, S,
                                                                               M.tslot.p, T, sh, th);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_mx_reduce", (512ll * M.s_tiles + 512ll * M.nmt) * nh, s);
  }
  if (M.p2_tiles > 0) {
    const unsigned grid = (unsigned)M.p2_tiles;
    const int te = M.p2_tile0 + M.p2_tiles;
#define HM_P2_ARGS                                                                                            \
  M.p2_tile0, te, h->depth, M.tile_leaf.p, M.leaf_tile0.p, leaf_off, M.pan_of.p, M.panels.p, M.store.p, T,      \
      M.leaf_dptr.p, M.leaf_dblk.p, M.dense.p, Xf, Y, ldy, nr, xh, th
    if (nh == 1)
      k_mx_p2<1, 1><<<grid, 32, 0, s>>>(HM_P2_ARGS);
    else if (nh == 2)
      k_mx_p2<2, 1><<<grid, 32, 0, s>>>(HM_P2_ARGS);
    else if (nh == 4)  // two warps of two parts share each row tile's factor tiles
      k_mx_p2<2, 2><<<grid, 64, 0, s>>>(HM_P2_ARGS);
    else  // four warps of two parts
      k_mx_p2<2, 4><<<grid, 128, 0, s>>>(HM_P2_ARGS);
#undef HM_P2_ARGS
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_mx_p2", M.bytes_p2 + xbytes + 4ll * h->n * nr, s);
  }
  return HM_OK;
}

}  // namespace hm
