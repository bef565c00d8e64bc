// hm_fp32.cu -- the FP32 form of the H-matvec on factor panels.
//
// The same panels, phase-1 units, chunk partials and projection column map as
// the mixed form (hm_mixed.h), with the factors stored as FP32 in the
// fragment order of the TF32 tensor-core MMA (mma.sync m16n8k8) and split
// into TF32 hi + lo in registers: three MMAs per operand pair (hi*lo, lo*hi,
// hi*hi; lo*lo is below FP32 rounding) reproduce FP32 products.  Each chain
// of three MMAs goes into a zeroed temporary added to the FP32 sum with an
// ordinary FADD, as in the per-block FP32 kernels.
//
// Tile orders (32 rows x 8 columns, 1 KB, two 512-byte warp loads; lane
// L = 4 g + t; V[r][c], U[r][c] with r the row in the tile, c the column):
//   P1 (phase 1, V is the B operand of X^T V, k = rows):
//     part 0 = {V[t][g], V[t+4][g], V[8+t][g], V[12+t][g]}
//     part 1 = {V[16+t][g], V[20+t][g], V[24+t][g], V[28+t][g]}
//   P2 (phase 2, U is the A operand of U T, k = columns), part m (rows 16 m..):
//     {U[16m+g][t], U[16m+g+8][t], U[16m+g][t+4], U[16m+g+8][t+4]}
// X fragments (A operand of X^T V) per 32-row tile and 16 right-hand sides:
//   Xf[tile][p][lane], p = 0..3 the TF32 hi of k-step p, 4..7 the lo:
//     {X[8p+t][g], X[8p+t][g+8], X[8p+t+4][g], X[8p+t+4][g+8]}
//   and, read as B operands, the X columns of a dense block.
// T (FP32), per global 8-column tile 128 words, lane L's 16 bytes
//   {T[c=t][r=g], T[t+4][g], T[t][g+8], T[t+4][g+8]} (c column, r right-hand
//   side): phase 2's two B fragments in one 16-byte load.
#include <algorithm>
#include <vector>

#include "hm_hmatrix.h"
#include "hm_mixed.h"
#include "hm_mma.cuh"

namespace hm {
namespace {

__device__ __forceinline__ uint64_t fp_keep_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint4 fp_ld_keep(const uint4* ptr, uint64_t pol) {
  uint4 v;
  asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;\n"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(ptr), "l"(pol));
  return v;
}

__device__ __forceinline__ void split4(const uint4& v, uint32_t (&h)[4], uint32_t (&l)[4]) {
  split_tf32(__uint_as_float(v.x), h[0], l[0]);
  split_tf32(__uint_as_float(v.y), h[1], l[1]);
  split_tf32(__uint_as_float(v.z), h[2], l[2]);
  split_tf32(__uint_as_float(v.w), h[3], l[3]);
}

// word of T for (global factor column e, right-hand side g of the lower
// eight); right-hand side g + 8 is two words further
__device__ __forceinline__ long long fp_t_word(int e, int g) {
  return (long long)(e >> 3) * 128 + 4 * (4 * g + (e & 3)) + ((e & 7) >> 2);
}

// One lane's C fragment of a projection tile (columns 2t, 2t+1 at right-hand
// sides g, g + 8), each column stored to its mirror's words (m: the tslot
// entries of columns 2t, 2t+1); a padding column (no mirror) writes zeros to
// its own words, so every T word is written once per product.
__device__ __forceinline__ void fp_store_t(float* __restrict__ T, int2 m, int lane, float a0, float a1, float a2,
                                           float a3) {
  const int g = lane >> 2;
  const int e0 = m.x >= 0 ? m.x : -1 - m.x, e1 = m.y >= 0 ? m.y : -1 - m.y;
  const long long w0 = fp_t_word(e0, g), w1 = fp_t_word(e1, g);
  T[w0] = m.x >= 0 ? a0 : 0.f;
  T[w0 + 2] = m.x >= 0 ? a2 : 0.f;
  T[w1] = m.y >= 0 ? a1 : 0.f;
  T[w1 + 2] = m.y >= 0 ? a3 : 0.f;
}

__device__ __forceinline__ int2 fp_tslot_pair(const int* __restrict__ tslot, long long col_tile, int lane) {
  return __ldg(reinterpret_cast<const int2*>(tslot + col_tile * 8 + 2 * (lane & 3)));
}

// ---- X -> TF32 hi / lo fragments ------------------------------------------
__global__ void __launch_bounds__(128) k_fp_split_x(const float* __restrict__ X, int ldx, int nr, int num_tiles,
                                                    const int* __restrict__ tile_leaf,
                                                    const int* __restrict__ leaf_tile0,
                                                    const int* __restrict__ leaf_off, uint4* __restrict__ Xf) {
  __shared__ float xs[4][16][33];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int G = blockIdx.x * 4 + w;
  if (G >= num_tiles) return;  // whole warp; only warp-level syncs below
  const int x = tile_leaf[G];
  const int row = leaf_off[x] + 32 * (G - leaf_tile0[x]) + lane;
  const bool ok = row < leaf_off[x + 1];
#pragma unroll
  for (int r = 0; r < 16; ++r) xs[w][r][lane] = (ok && r < nr) ? __ldg(X + (size_t)r * ldx + row) : 0.f;
  __syncwarp();
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int r0 = 8 * p + t;
    uint4 hi, lo;
    split_tf32(xs[w][g][r0], hi.x, lo.x);
    split_tf32(xs[w][g + 8][r0], hi.y, lo.y);
    split_tf32(xs[w][g][r0 + 4], hi.z, lo.z);
    split_tf32(xs[w][g + 8][r0 + 4], hi.w, lo.w);
    Xf[((size_t)G * 8 + p) * 32 + lane] = hi;
    Xf[((size_t)G * 8 + 4 + p) * 32 + lane] = lo;
  }
}

// ---- phase 1 ----------------------------------------------------------------
// C (16 right-hand sides x 8 columns) per column tile = X^T V over the unit's
// row tiles; NCT: column tiles compiled for.
template <int NCT>
__device__ __forceinline__ void fp_p1_unit(const MxUnit& u, const MxPanel& P, const uint4* __restrict__ store,
                                           const uint4* __restrict__ Xf, const int* __restrict__ tslot,
                                           float4* __restrict__ S, float* __restrict__ T, int lane) {
  float acc[NCT][4];
#pragma unroll
  for (int j = 0; j < NCT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  const uint4 z = make_uint4(0u, 0u, 0u, 0u);
  const uint64_t keep = fp_keep_policy();
  int2 mm = make_int2(-1, -1);
  if (P.nchunk == 1 && lane < 4 * NCT && (lane >> 2) < u.nct) mm = fp_tslot_pair(tslot, P.t0 + u.ct0 + (lane >> 2), lane);
  for (int r = 0; r < u.nrt; ++r) {
    const long long rt = u.rt0 + r;
    const uint4* xp = Xf + (size_t)(P.tile0 + rt) * 256 + lane;
    uint4 xh[4], xl[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      xh[p] = fp_ld_keep(xp + p * 32, keep);
      xl[p] = fp_ld_keep(xp + (4 + p) * 32, keep);
    }
    const uint4* vp = store + (P.hi1 + (rt * P.nct + u.ct0) * 2) * 32 + lane;
    uint4 v0[NCT], v1[NCT];
#pragma unroll
    for (int j = 0; j < NCT; ++j) {
      v0[j] = j < u.nct ? __ldcs(vp + (2 * j) * 32) : z;
      v1[j] = j < u.nct ? __ldcs(vp + (2 * j + 1) * 32) : z;
    }
    // k-step by k-step, the column tiles' three-MMA chains interleaved so
    // that consecutive MMAs are independent
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      uint32_t bh[NCT][2], bl[NCT][2];
#pragma unroll
      for (int j = 0; j < NCT; ++j) {
        const uint4& v = p < 2 ? v0[j] : v1[j];
        const float b0 = __uint_as_float((p & 1) ? v.z : v.x), b1 = __uint_as_float((p & 1) ? v.w : v.y);
        split_tf32(b0, bh[j][0], bl[j][0]);
        split_tf32(b1, bh[j][1], bl[j][1]);
      }
      float d[NCT][4];
#pragma unroll
      for (int j = 0; j < NCT; ++j) d[j][0] = d[j][1] = d[j][2] = d[j][3] = 0.f;
#pragma unroll
      for (int j = 0; j < NCT; ++j)
        if (j < u.nct) mma_tf32(d[j], xl[p].x, xl[p].y, xl[p].z, xl[p].w, bh[j][0], bh[j][1]);  // X_lo V_hi
#pragma unroll
      for (int j = 0; j < NCT; ++j)
        if (j < u.nct) mma_tf32(d[j], xh[p].x, xh[p].y, xh[p].z, xh[p].w, bl[j][0], bl[j][1]);  // X_hi V_lo
#pragma unroll
      for (int j = 0; j < NCT; ++j)
        if (j < u.nct) mma_tf32(d[j], xh[p].x, xh[p].y, xh[p].z, xh[p].w, bh[j][0], bh[j][1]);  // X_hi V_hi
#pragma unroll
      for (int j = 0; j < NCT; ++j) add4(acc[j], d[j]);
    }
  }
  if (P.nchunk == 1) {
#pragma unroll
    for (int j = 0; j < NCT; ++j)
      if (j < u.nct) {
        const int src = 4 * j + (lane & 3);
        const int2 m = make_int2(__shfl_sync(0xffffffffu, mm.x, src), __shfl_sync(0xffffffffu, mm.y, src));
        fp_store_t(T, m, lane, acc[j][0], acc[j][1], acc[j][2], acc[j][3]);
      }
  } else {
    float4* out = S + (P.s0 + (long long)u.chunk * P.nct + u.ct0) * 32 + lane;
#pragma unroll
    for (int j = 0; j < NCT; ++j)
      if (j < u.nct) out[j * 32] = make_float4(acc[j][0], acc[j][1], acc[j][2], acc[j][3]);
  }
}

// one warp per CTA, 16 per SM (as the mixed form's phase 1)
__global__ void __launch_bounds__(32, 16) k_fp_p1(const MxUnit* __restrict__ units, int nunits,
                                                  const MxPanel* __restrict__ panels, const uint4* __restrict__ store,
                                                  const uint4* __restrict__ Xf, const int* __restrict__ tslot,
                                                  float4* __restrict__ S, float* __restrict__ T) {
  const int w = blockIdx.x;
  if (w >= nunits) return;
  const int lane = threadIdx.x & 31;
  const MxUnit u = units[w];
  const MxPanel P = panels[u.panel];
  for (int c = 0; c < u.nct; c += 4) {  // at most four column tiles at a time
    MxUnit a = u;
    a.ct0 = u.ct0 + c;
    a.nct = min(4, u.nct - c);
    if (a.nct > 2)
      fp_p1_unit<4>(a, P, store, Xf, tslot, S, T, lane);
    else
      fp_p1_unit<2>(a, P, store, Xf, tslot, S, T, lane);
  }
}

// ---- row-chunk reduction ------------------------------------------------------
__global__ void k_fp_reduce(const int2* __restrict__ mtiles, long long nmt, const MxPanel* __restrict__ panels,
                            const float4* __restrict__ S, const int* __restrict__ tslot, float* __restrict__ T) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nmt * 32) return;
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
  fp_store_t(T, fp_tslot_pair(tslot, P.t0 + mt.y, lane), lane, v.x, v.y, v.z, v.w);
}

// ---- phase 2 ----------------------------------------------------------------
// acc[mt][nb] += A (rows 16 mt.., 8 columns; hi / lo) B (8 columns x right-hand
// sides 8 nb..; hi / lo)
__device__ __forceinline__ void fp_p2_step(float (&acc)[2][2][4], const uint32_t (&ah)[2][4],
                                           const uint32_t (&al)[2][4], const uint32_t (&bh)[2][2],
                                           const uint32_t (&bl)[2][2]) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nb = 0; nb < 2; ++nb) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
      mma_tf32(d, al[mt][0], al[mt][1], al[mt][2], al[mt][3], bh[nb][0], bh[nb][1]);
      mma_tf32(d, ah[mt][0], ah[mt][1], ah[mt][2], ah[mt][3], bl[nb][0], bl[nb][1]);
      mma_tf32(d, ah[mt][0], ah[mt][1], ah[mt][2], ah[mt][3], bh[nb][0], bh[nb][1]);
      add4(acc[mt][nb], d);
    }
}

// One warp per global row tile (32 rows of one leaf), as the mixed form's
// phase 2: every ancestor cluster's panel rows times its T, then the dense
// blocks of the leaf row.
__global__ void __launch_bounds__(32, 24) k_fp_p2(int tile0, int tile_end, int depth,
                                                  const int* __restrict__ tile_leaf,
                                                  const int* __restrict__ leaf_tile0,
                                                  const int* __restrict__ leaf_off, const int* __restrict__ pan_of,
                                                  const MxPanel* __restrict__ panels,
                                                  const uint4* __restrict__ store, const float* __restrict__ T,
                                                  const int* __restrict__ leaf_dptr,
                                                  const int* __restrict__ leaf_dblk, const MxDense* __restrict__ dense,
                                                  const uint4* __restrict__ Xf, float* __restrict__ Y, int ldy,
                                                  int nr) {
  const int G = tile0 + blockIdx.x;
  if (G >= tile_end) return;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int x = tile_leaf[G];
  float acc[2][2][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nb = 0; nb < 2; ++nb) acc[mt][nb][0] = acc[mt][nb][1] = acc[mt][nb][2] = acc[mt][nb][3] = 0.f;
  // every ancestor's panel descriptor at once (lane l - 1 holds level l's)
  int my_p = -1, my_nct = 0;
  long long my_u = 0, my_t = 0;
  if (lane < depth) {
    const int l = lane + 1;
    my_p = __ldg(pan_of + (1 << l) - 1 + (x >> (depth - l)));
    if (my_p >= 0) {
      const MxPanel P = panels[my_p];
      my_u = P.hi2 + (long long)(G - P.tile0) * P.nct * 2;
      my_t = P.t0;
      my_nct = P.nct;
    }
  }
  for (int l = 1; l <= depth; ++l) {
    const int p = __shfl_sync(0xffffffffu, my_p, l - 1);
    if (p < 0) continue;
    const long long ou = __shfl_sync(0xffffffffu, my_u, l - 1);
    const long long ot = __shfl_sync(0xffffffffu, my_t, l - 1);
    const int nct = __shfl_sync(0xffffffffu, my_nct, l - 1);
    const uint4* up = store + ou * 32 + lane;
    const uint4* tp = reinterpret_cast<const uint4*>(T + ot * 128) + lane;
#pragma unroll 2
    for (int ct = 0; ct < nct; ++ct) {
      const uint4 a0 = __ldcs(up + (2 * ct) * 32), a1 = __ldcs(up + (2 * ct + 1) * 32);
      const uint4 tq = __ldg(tp + ct * 32);
      uint32_t ah[2][4], al[2][4], th[4], tl[4];
      split4(a0, ah[0], al[0]);
      split4(a1, ah[1], al[1]);
      split4(tq, th, tl);
      const uint32_t bh[2][2] = {{th[0], th[1]}, {th[2], th[3]}};
      const uint32_t bl[2][2] = {{tl[0], tl[1]}, {tl[2], tl[3]}};
      fp_p2_step(acc, ah, al, bh, bl);
    }
  }
  for (int q = leaf_dptr[x]; q < leaf_dptr[x + 1]; ++q) {
    const MxDense D = dense[leaf_dblk[q]];
    const long long rt = G - D.row_tile0;
    const uint4* dp = store + (D.hi + rt * D.nct * 2) * 32 + lane;
    for (int ct = 0; ct < D.nct; ++ct) {
      const uint4 a0 = __ldcs(dp + (2 * ct) * 32), a1 = __ldcs(dp + (2 * ct + 1) * 32);
      const size_t xt = ((size_t)(D.col_tile0 + (ct >> 2)) * 8 + (ct & 3)) * 32 + lane;
      const uint4 xh = __ldg(Xf + xt), xl = __ldg(Xf + xt + 128);
      uint32_t ah[2][4], al[2][4];
      split4(a0, ah[0], al[0]);
      split4(a1, ah[1], al[1]);
      const uint32_t bh[2][2] = {{xh.x, xh.z}, {xh.y, xh.w}};
      const uint32_t bl[2][2] = {{xl.x, xl.z}, {xl.y, xl.w}};
      fp_p2_step(acc, ah, al, bh, bl);
    }
  }
  const int base = leaf_off[x] + 32 * (G - leaf_tile0[x]);
  const int lim = leaf_off[x + 1];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nb = 0; nb < 2; ++nb) {
      const int ra = base + 16 * mt + g, rb = ra + 8, c = 8 * nb + 2 * t;
      if (c < nr) {
        if (ra < lim) Y[(size_t)c * ldy + ra] = acc[mt][nb][0];
        if (rb < lim) Y[(size_t)c * ldy + rb] = acc[mt][nb][2];
      }
      if (c + 1 < nr) {
        if (ra < lim) Y[(size_t)(c + 1) * ldy + ra] = acc[mt][nb][1];
        if (rb < lim) Y[(size_t)(c + 1) * ldy + rb] = acc[mt][nb][3];
      }
    }
}

// ---- conversion (build time) ------------------------------------------------
__device__ __forceinline__ int fp_find_item(const long long* start, int n, long long w) {
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

__device__ __forceinline__ uint4 f4(float a, float b, float c, float d) {
  return make_uint4(__float_as_uint(a), __float_as_uint(b), __float_as_uint(c), __float_as_uint(d));
}

// One warp per 32 x 8 panel tile: both orders.  colsrc: per panel column, the
// FP32 factor column over the cluster's rows, or null for a padding column.
__global__ void k_fp_conv_panels(const MxPanel* __restrict__ panels, const long long* __restrict__ unit_start,
                                 int npanels, long long nunits, const float* const* __restrict__ colsrc,
                                 const int* __restrict__ tile_leaf, const int* __restrict__ leaf_tile0,
                                 const int* __restrict__ leaf_off, uint4* __restrict__ store) {
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nunits) return;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int pi = fp_find_item(unit_start, npanels, w);
  const MxPanel P = panels[pi];
  const long long local = w - unit_start[pi];
  const int rt = (int)(local / P.nct), ct = (int)(local % P.nct);
  const int G = P.tile0 + rt;
  const int x = tile_leaf[G];
  const int rbase = leaf_off[x] + 32 * (G - leaf_tile0[x]) - P.r0;
  const int rlim = leaf_off[x + 1] - P.r0;
  const float* const* cs = colsrc + P.t0 * 8 + 8 * ct;
  auto val = [&](int r, int c) -> float {
    const float* col = cs[c];
    const int lr = rbase + r;
    return (col != nullptr && lr < rlim) ? col[lr] : 0.f;
  };
  const long long tile = (long long)rt * P.nct + ct;
  uint4* p1 = store + (P.hi1 + tile * 2) * 32 + lane;
  uint4* p2 = store + (P.hi2 + tile * 2) * 32 + lane;
  p1[0] = f4(val(t, g), val(t + 4, g), val(8 + t, g), val(12 + t, g));
  p1[32] = f4(val(16 + t, g), val(20 + t, g), val(24 + t, g), val(28 + t, g));
  p2[0] = f4(val(g, t), val(g + 8, t), val(g, t + 4), val(g + 8, t + 4));
  p2[32] = f4(val(16 + g, t), val(24 + g, t), val(16 + g, t + 4), val(24 + g, t + 4));
}

// One warp per 32 x 8 tile of a dense block (P2 order)
__global__ void k_fp_conv_dense(const MxDense* __restrict__ dense, const long long* __restrict__ unit_start,
                                int ndense, long long nunits, const int* __restrict__ tile_leaf,
                                const int* __restrict__ leaf_tile0, const int* __restrict__ leaf_off,
                                uint4* __restrict__ store) {
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nunits) return;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int di = fp_find_item(unit_start, ndense, w);
  const MxDense D = dense[di];
  const long long local = w - unit_start[di];
  const int rt = (int)(local / D.nct), ct = (int)(local % D.nct);
  const int G = D.row_tile0 + rt;
  const int x = tile_leaf[G];
  const int rbase = leaf_off[x] + 32 * (G - leaf_tile0[x]) - D.r0;
  const int rlim = leaf_off[x + 1] - D.r0;
  // padded columns 8 ct + t and 8 ct + t + 4 lie in one 32-column tile
  const int GC = D.col_tile0 + ((8 * ct) >> 5);
  const int y = tile_leaf[GC];
  const int cbase = leaf_off[y] + 32 * (GC - leaf_tile0[y]) - D.c0 + ((8 * ct) & 31);
  const int clim = leaf_off[y + 1] - D.c0;
  auto val = [&](int r, int c) -> float {
    const int lr = rbase + r;
    return (lr < rlim && c < clim) ? D.src[(size_t)c * D.m + lr] : 0.f;
  };
  uint4* p2 = store + (D.hi + ((long long)rt * D.nct + ct) * 2) * 32 + lane;
  const int ca = cbase + t, cb = cbase + t + 4;
  p2[0] = f4(val(g, ca), val(g + 8, ca), val(g, cb), val(g + 8, cb));
  p2[32] = f4(val(16 + g, ca), val(24 + g, ca), val(16 + g, cb), val(24 + g, cb));
}

}  // namespace

hm_status fp32_convert(hm_hmatrix_s* h, const std::vector<const float*>& colsrc, const std::vector<MxDense>& dense,
                       cudaStream_t s) {
  MxPlan& M = h->mx;
  const std::vector<MxPanel>& panels = M.h_panels;
  const int np = (int)panels.size();
  if (np > 0) {
    std::vector<long long> start(np);
    long long tot = 0;
    for (int p = 0; p < np; ++p) {
      start[p] = tot;
      tot += (long long)panels[p].nrt * panels[p].nct;
    }
    DevBuf<const float*> dcol;
    DevBuf<long long> dstart;
    HM_TRY(dcol.alloc(std::max<size_t>(colsrc.size(), 1)));
    HM_TRY(dstart.alloc(np));
    if (!colsrc.empty())
      HM_CUDA(cudaMemcpyAsync(dcol.p, colsrc.data(), sizeof(const float*) * colsrc.size(), cudaMemcpyHostToDevice, s));
    HM_CUDA(cudaMemcpyAsync(dstart.p, start.data(), sizeof(long long) * np, cudaMemcpyHostToDevice, s));
    if (tot > 0) {
      k_fp_conv_panels<<<(unsigned)((tot * 32 + 255) / 256), 256, 0, s>>>(
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
    HM_TRY(ds.alloc(dense.size()));
    HM_CUDA(cudaMemcpyAsync(ds.p, start.data(), sizeof(long long) * start.size(), cudaMemcpyHostToDevice, s));
    if (tot > 0) {
      k_fp_conv_dense<<<(unsigned)((tot * 32 + 255) / 256), 256, 0, s>>>(
          M.dense.p, ds.p, M.num_dense, tot, M.tile_leaf.p, M.leaf_tile0.p, h->tree->offsets.p, M.store.p);
      HM_LAUNCH_CHECK();
    }
    HM_CUDA(cudaStreamSynchronize(s));
  }
  return HM_OK;
}

// One pass of nr <= 16 right-hand sides in tree order; scratch holds
// scratch_floats(1) floats: X fragments, chunk partials, T.
hm_status fp32_run_panel(hm_hmatrix_s* h, int nr, const float* X, int ldx, float* Y, int ldy, float* scratch,
                         cudaStream_t s, KernelMarks* km) {
  MxPlan& M = h->mx;
  if (nr < 1 || nr > 16) return fail(HM_ERR_INVALID, "FP32 panel product: a pass holds 1 to 16 right-hand sides");
  uint4* Xf = reinterpret_cast<uint4*>(scratch);
  float4* S = reinterpret_cast<float4*>(Xf + (size_t)M.num_tiles * 256);
  float* T = reinterpret_cast<float*>(S + (size_t)M.s_tiles * 32);
  const int* leaf_off = h->tree->offsets.p;
  const long long xbytes = 4ll * h->n * 16 * 2;  // the X fragments, hi + lo
  if (M.num_tiles > 0) {
    k_fp_split_x<<<(M.num_tiles + 3) / 4, 128, 0, s>>>(X, ldx, nr, M.num_tiles, M.tile_leaf.p, M.leaf_tile0.p,
                                                       leaf_off, Xf);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_fp_split_x", 4ll * h->n * nr + xbytes, s);
  }
  if (M.num_units > 0) {
    k_fp_p1<<<M.num_units, 32, 0, s>>>(M.units.p, M.num_units, M.panels.p, M.store.p, Xf, M.tslot.p, S, T);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_fp_p1", M.bytes_p1 + xbytes, s);
  }
  if (M.nmt > 0) {
    k_fp_reduce<<<(unsigned)((M.nmt * 32 + 255) / 256), 256, 0, s>>>(M.mtiles.p, M.nmt, M.panels.p, S, M.tslot.p,
                                                                       T);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_fp_reduce", 512ll * M.s_tiles + 512ll * M.nmt, s);
  }
  if (M.p2_tiles > 0) {
    k_fp_p2<<<(unsigned)M.p2_tiles, 32, 0, s>>>(M.p2_tile0, M.p2_tile0 + M.p2_tiles, h->depth, M.tile_leaf.p,
                                                M.leaf_tile0.p, leaf_off, M.pan_of.p, M.panels.p, M.store.p, T,
                                                M.leaf_dptr.p, M.leaf_dblk.p, M.dense.p, Xf, Y, ldy, nr);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_fp_p2", M.bytes_p2 + xbytes + 4ll * h->n * nr, s);
  }
  if (h->diag_fly) HM_TRY(diag_fly_panel(h, nr, X, ldx, Y, ldy, s, km));
  return HM_OK;
}

}  // namespace hm
