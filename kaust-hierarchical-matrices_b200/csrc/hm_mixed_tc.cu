// hm_mixed_tc.cu -- phase 1 of the mixed form's 128-column passes on the
// Blackwell tensor cores (tcgen05.mma, accumulator in tensor memory).
//
// A pass of 128 right-hand sides multiplies every factor element 128 times
// (hi and lo: up to 3 BF16 products each), more than the warp-level MMA
// keeps up with at HBM speed.  Here one CTA per SM walks its units -- a
// panel's 128 columns (16 column tiles) over a chunk of row tiles -- and per
// 32-row tile issues D (128 columns x 128 right-hand sides, FP32 in TMEM) +=
// V^T X as tcgen05.mma of M = 128, N = 128, K = 16:
//   A = V^T: the factor tiles as stored (P1 fragment order, lane (g,t) holds
//     column g at rows rho(t, 0..7)), each lane's 16 bytes copied by cp.async
//     to its core-matrix row: column 8 j + g, K block t.  The K order inside
//     a 32-row tile is therefore rho(c, e) = 8 (e / 2) + 2 c + (e % 2) for
//     K index 8 c + e -- a permutation of the rows, harmless in a sum as long
//     as B uses the same one.
//   B = X: the pass's right-hand sides, written by k_mx_split_x as one
//     16 KB image per 32-row tile (hi 8 KB, then lo), already in the K-major
//     core-matrix layout with the same row order, so that it is copied as is.
// Columns with low parts take three products per tile (V_hi X_hi, V_hi X_lo,
// V_lo X_hi); the others one (V_hi X_hi), two row tiles per step.
//
// Pipeline: six 32 KB shared-memory stages; every thread copies its share of
// a stage four steps ahead (cp.async), waits for its own copies, fences them
// to the async proxy and meets the others at a CTA barrier; thread 0 then
// issues the step's MMAs and commits them to the stage's mbarrier, which
// tells the copies when the stage may be refilled.  The accumulator has two
// TMEM buffers: a chain of MMAs (one step for columns with low parts, two for
// the others) goes into one while the previous chain is read out (tcgen05.ld:
// 256 threads, warps w and w + 4 share TMEM lanes 32 (w % 4) .. and take 64
// of the 128 right-hand sides each) and added to the thread's FP32 sums
// with ordinary round-to-nearest adds, as the warp-level path does for its
// short MMA chains.  At a unit's end each thread stores its column: as T
// (into the mirror column's slots, split hi + lo or hi only) when the panel
// is projected in one row chunk, else as the chunk's partial S.
//
// T of such a pass is kept in 2 KB blocks, one per 8 columns and part (hi,
// lo): the K-major core-matrix image of B = T (128 right-hand sides x 8
// columns), so that phase 2 copies it as is.
//
// Phase 2 (k_mx_p2_tc): one CTA per SM walks blocks of 4 row tiles (128
// rows), D (128 rows x 128 right-hand sides) += U T per ancestor panel and
// D X per dense block, M = 128, N = 128.  A = the factor tiles as stored (P2
// order: lane (g,t) holds rows g + 8 w, w = 0..3, at columns 2t, 2t+1), each
// 4-byte word copied by cp.async to its row of the core-matrix image; rows of
// the block's tiles that a source does not cover are zero.  Dense blocks take
// their columns in X's row order rho so that B is X's image of the column
// cluster's tile.  Panels' columns with low parts take three products per 16
// columns; the others one per 16 columns, 32 columns per step; dense blocks
// three per 16 columns, 32 per step.
#include "hm_hmatrix.h"
#include "hm_mixed.h"
#include "hm_mma.cuh"
#include "hm_tc.cuh"

namespace hm {
namespace {

constexpr int kTcStages = 6;
constexpr int kTcAhead = kTcStages - 2;  // steps copied ahead of the MMAs
constexpr int kTcStage = 32768;          // bytes per stage
constexpr int kTcBars = kTcStages + 3;   // per-stage "MMAs done", two "chain done", one "end"
constexpr size_t kTcSmem = (size_t)kTcStages * kTcStage + 8 * kTcBars + 16;
constexpr uint32_t kTcCols = 256;  // two accumulators of 128 FP32 columns
constexpr uint32_t kIdesc = tc_idesc_bf16(128, 128);
constexpr int kTcThreads = 256;
constexpr int kChainHi = 2;  // steps per MMA chain for columns without low parts

// Stage layout (bytes): columns with low parts: A_hi 0, A_lo 8192, B_hi
// 16384, B_lo 24576 (one row tile); without: A_hi of two row tiles at 0 and
// 8192, B_hi of the same at 16384 and 24576.  LBO = 2048 (K blocks), SBO =
// 128 (8-row groups) everywhere.

// A position in the CTA's step sequence: unit index (>= nunits: done) and
// the first row tile of the next step.  Unit and panel fields are read from
// the (cached) lists where they are needed.
struct TcCursor {
  int u, r;
};

__device__ __forceinline__ bool unit_lo(const MxUnit& U, const MxPanel& P) { return U.ct0 < P.nctl; }
__device__ __forceinline__ int step_tiles(const MxUnit& U, bool lo, int r) { return lo ? 1 : min(2, U.nrt - r); }

// This thread's copies of the step at c into the stage at `base`.
__device__ __forceinline__ void tc_produce(const TcCursor& c, const MxUnit& U, const MxPanel& P, uint32_t base,
                                           const uint4* __restrict__ store, const uint4* __restrict__ Xtc, int tid) {
  const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const uint32_t arow = (uint32_t)(g * 16 + t * 2048);  // the lane's core-matrix row in a tile's A image
  const bool lo = unit_lo(U, P);
  const int nt = step_tiles(U, lo, c.r);
  for (int k = 0; k < nt; ++k) {
    const long long rt = U.rt0 + c.r + k;
    const uint32_t a_hi = base + (uint32_t)(k * 8192);
    const uint4* hp = store + (P.hi1 + rt * P.nct + U.ct0) * 32 + lane;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int j = warp + 8 * q;
      if (j < U.nct) cpa16(a_hi + (uint32_t)(j * 128) + arow, hp + j * 32);
    }
    if (lo) {  // low parts; a tile past the panel's low-part tiles would be zero
      const uint4* lp = store + (P.lo1 + rt * P.nctl + U.ct0) * 32 + lane;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int j = warp + 8 * q;
        if (j < U.nct) {
          const uint32_t dst = base + 8192u + (uint32_t)(j * 128) + arow;
          if (U.ct0 + j < P.nctl)
            cpa16(dst, lp + j * 32);
          else
            cpa16_zero(dst, store);
        }
      }
    }
    // X's image of this row tile: hi, and lo for columns with low parts
    const uint4* xp = Xtc + (size_t)(P.tile0 + rt) * 1024 + tid;
    const uint32_t b_hi = base + 16384u + (uint32_t)(k * 8192) + (uint32_t)(tid * 16);
#pragma unroll
    for (int q = 0; q < 2; ++q) cpa16(b_hi + (uint32_t)(q * 4096), xp + q * 256);
    if (lo) {
      const uint32_t b_lo = base + 24576u + (uint32_t)(tid * 16);
#pragma unroll
      for (int q = 0; q < 2; ++q) cpa16(b_lo + (uint32_t)(q * 4096), xp + 512 + q * 256);
    }
  }
}

// Thread 0: the step's MMAs into accumulator d (first: the chain's first step
// overwrites it).
__device__ __forceinline__ void tc_issue(bool lo, int nt, uint32_t base, uint32_t d, bool first) {
  uint32_t acc = first ? 0u : 1u;
  if (lo) {
#pragma unroll
    for (int p = 0; p < 3; ++p) {  // V_hi X_hi, V_hi X_lo, V_lo X_hi
      const uint32_t pa = p == 2 ? 8192u : 0u, pb = p == 1 ? 24576u : 16384u;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        tc_mma_bf16(d, tc_sdesc(base + pa + (uint32_t)(q * 4096), 2048, 128),
                    tc_sdesc(base + pb + (uint32_t)(q * 4096), 2048, 128), kIdesc, acc);
        acc = 1u;
      }
    }
  } else {
    for (int q = 0; q < 2 * nt; ++q) {  // K blocks of 16 rows
      tc_mma_bf16(d, tc_sdesc(base + (uint32_t)(q * 4096), 2048, 128),
                  tc_sdesc(base + 16384u + (uint32_t)(q * 4096), 2048, 128), kIdesc, acc);
      acc = 1u;
    }
  }
}

// BF16 element (right-hand side n, column pos % 8) of T's block pos / 8
__device__ __forceinline__ long long tb_elem(long long pos, int n) {
  return (pos >> 3) * 1024 + (n & 7) * 8 + (n >> 3) * 64 + (pos & 7);
}
__device__ __forceinline__ unsigned short bf16_bits(float v) {
  return (unsigned short)(pack_bf16(v, 0.f) & 0xffffu);
}
// The thread's column m (its TMEM lane) of a finished unit, right-hand sides
// 64 hf .. 64 hf + 63: T or the chunk's partial S.
__device__ __forceinline__ void tc_store(const MxUnit& U, const MxPanel& P, const float (&acc)[64],
                                         const int2* __restrict__ tslot_tc, float* __restrict__ S,
                                         unsigned short* __restrict__ Tb, long long sh, int m, int hf) {
  const int jt = m >> 3, c = m & 7;
  if (jt >= U.nct) return;
  const long long ctile = P.t0 + U.ct0 + jt;
  if (P.nchunk == 1) {
    const int2 e = __ldg(tslot_tc + ctile * 8 + c);
    const bool pad = e.x < 0;
    const long long hp = pad ? -1 - (long long)e.x : e.x;
#pragma unroll
    for (int i = 0; i < 64; ++i) {
      const int n = 64 * hf + i;
      const unsigned short hi = pad ? 0 : bf16_bits(acc[i]);
      Tb[tb_elem(hp, n)] = hi;
      if (e.y >= 0) Tb[tb_elem(e.y, n)] = pad ? 0 : bf16_bits(acc[i] - __uint_as_float((uint32_t)hi << 16));
    }
  } else {  // the chunk's partial: float4 (g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1) per lane (g, t)
    float* out = S + ((P.s0 + (long long)U.chunk * P.nct + U.ct0 + jt) * 32 + (c >> 1)) * 4 + (c & 1);
#pragma unroll
    for (int h = 0; h < 4; ++h)
#pragma unroll
      for (int r = 0; r < 16; ++r) out[(4 * hf + h) * sh * 4 + (r & 7) * 16 + (r >> 3) * 2] = acc[16 * h + r];
  }
}

__global__ void __launch_bounds__(kTcThreads, 1)
    k_mx_p1_tc(const MxUnit* __restrict__ units, int nunits, const MxPanel* __restrict__ panels,
               const uint4* __restrict__ store, const uint4* __restrict__ Xtc, const int2* __restrict__ tslot_tc,
               float* __restrict__ S, unsigned short* __restrict__ Tb, long long sh, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t sbase = smem_u32(smem);
  // mbarriers: "MMAs of stage s done" at bars + 8 s, "chain done" per
  // accumulator after them, then one for the end; then the TMEM address
  const uint32_t bars = sbase + (uint32_t)(kTcStages * kTcStage);
  const uint32_t chain_bar = bars + 8u * kTcStages, final_bar = chain_bar + 16u;
  const uint32_t slot = bars + 8u * kTcBars;
  if (tid == 0) {
    for (int i = 0; i < kTcBars; ++i) mbar_init(bars + 8u * i, 1);
    mbar_init_fence();
  }
  if (warp == 0) {
    tmem_alloc(slot, kTcCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + kTcStages * kTcStage + 8 * kTcBars);
  // this thread's TMEM lane (= the unit's column) and half of the right-hand sides
  const int m = (warp & 3) * 32 + (tid & 31), hf = warp >> 2;
  const uint32_t my_lanes = (uint32_t)((warp & 3) * 32) << 16;
  const int stride = gridDim.x;

  // the producer's cursor runs kTcAhead steps ahead of the consumer's over the
  // same sequence: units blockIdx.x, + gridDim.x, ..., each in row steps
  TcCursor pc{(int)blockIdx.x, 0}, cc{(int)blockIdx.x, 0};
  auto advance = [&](TcCursor& c, const MxUnit& U, bool lo) {
    c.r += step_tiles(U, lo, c.r);
    if (c.r >= U.nrt) {
      c.r = 0;
      c.u += stride;
    }
  };
  bool failed = false;
  auto produce = [&](int stage) {
    if (pc.u < nunits) {
      const MxUnit U = units[pc.u];
      const MxPanel P = panels[U.panel];
      if (!failed) tc_produce(pc, U, P, sbase + (uint32_t)(stage * kTcStage), store, Xtc, tid);
      advance(pc, U, unit_lo(U, P));
    }
    cpa_commit();  // an empty group past the end keeps the group count uniform
  };
  for (int i = 0; i < kTcAhead; ++i) produce(i);

  float acc[64];
#pragma unroll
  for (int i = 0; i < 64; ++i) acc[i] = 0.f;
  long long step = 0;
  int chain = -1, chain_len = 0;
  bool pend = false, pend_end = false;  // a finished chain to read out, and whether it ends its unit
  int pend_chain = 0, pend_u = 0;
  auto drain = [&]() {
    const int b = pend_chain & 1;
    if (!mbar_wait(chain_bar + 8u * b, (uint32_t)((pend_chain >> 1) & 1))) failed = true;
    tc_fence_after();
    if (!failed) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        uint32_t v[32];
        tc_ld32(tmem + my_lanes + (uint32_t)(b * 128 + hf * 64 + q * 32), v);
        tc_wait_ld();
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[q * 32 + i] += __uint_as_float(v[i]);
      }
    }
    if (pend_end) {
      if (!failed) {
        const MxUnit U = units[pend_u];
        tc_store(U, panels[U.panel], acc, tslot_tc, S, Tb, sh, m, hf);
      }
#pragma unroll
      for (int i = 0; i < 64; ++i) acc[i] = 0.f;
    }
    pend = false;
  };
  while (cc.u < nunits) {
    // refill the stage of step - 2 with step + kTcAhead once its MMAs are done
    const long long ps = step + kTcAhead;
    const int pst = (int)(ps % kTcStages);
    if (pc.u < nunits && ps >= kTcStages &&
        !mbar_wait(bars + 8u * pst, (uint32_t)(((ps - kTcStages) / kTcStages) & 1)))
      failed = true;
    produce(pst);
    cpa_wait<kTcAhead>();  // this thread's copies of `step` have landed
    fence_proxy_async_smem();
    if (__syncthreads_or(failed ? 1 : 0)) break;
    const MxUnit U = units[cc.u];
    const bool lo = unit_lo(U, panels[U.panel]);
    const int nt = step_tiles(U, lo, cc.r);
    const int st = (int)(step % kTcStages);
    const bool first = chain_len == 0;
    if (first) ++chain;
    ++chain_len;
    const bool unit_end = cc.r + nt >= U.nrt;
    const bool chain_end = unit_end || lo || chain_len == kChainHi;
    if (tid == 0) {
      tc_fence_after();
      tc_issue(lo, nt, sbase + (uint32_t)(st * kTcStage), tmem + (uint32_t)((chain & 1) * 128), first);
      tc_commit(bars + 8u * st);
      if (chain_end) tc_commit(chain_bar + 8u * (chain & 1));
    }
    if (pend) drain();  // the previous chain, while this one runs
    if (chain_end) {
      pend = true;
      pend_end = unit_end;
      pend_chain = chain;
      pend_u = cc.u;
      chain_len = 0;
    }
    tc_fence_before();
    advance(cc, U, lo);
    ++step;
  }
  if (pend && !failed) drain();
  cpa_wait<0>();
  // every MMA issued has completed before the tensor memory is released (the
  // commit arrives once all of thread 0's MMAs are done; bounded wait)
  if (tid == 0) tc_commit(final_bar);
  if (!mbar_wait(final_bar, 0)) failed = true;
  if (failed) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTcCols);
  }
}

// ---- chunk reduction (panels projected in several row chunks) -----------------
// The chunk partials of each column tile summed in chunk order, as T blocks.
__global__ void k_mx_reduce_tc(const int2* __restrict__ mtiles, long long nmt, const MxPanel* __restrict__ panels,
                               const float4* __restrict__ S, const int2* __restrict__ tslot_tc,
                               unsigned short* __restrict__ Tb, long long sh) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nmt * 32) return;
  const int h = blockIdx.y;  // part: right-hand sides 16 h .. 16 h + 15
  S += h * sh;
  const int2 mt = mtiles[i >> 5];
  const int lane = (int)(i & 31), g = lane >> 2, t = lane & 3;
  const MxPanel P = panels[mt.x];
  float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int ch = 0; ch < P.nchunk; ++ch) {
    const float4 a = S[(P.s0 + (long long)ch * P.nct + mt.y) * 32 + lane];
    v.x += a.x;
    v.y += a.y;
    v.z += a.z;
    v.w += a.w;
  }
  const float val[2][2] = {{v.x, v.z}, {v.y, v.w}};  // [column 2t + odd][right-hand side g, g + 8]
#pragma unroll
  for (int odd = 0; odd < 2; ++odd) {
    const int2 e = __ldg(tslot_tc + (P.t0 + mt.y) * 8 + 2 * t + odd);
    const bool pad = e.x < 0;
    const long long hp = pad ? -1 - (long long)e.x : e.x;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int n = 16 * h + g + 8 * r;
      const unsigned short hi = pad ? 0 : bf16_bits(val[odd][r]);
      Tb[tb_elem(hp, n)] = hi;
      if (e.y >= 0) Tb[tb_elem(e.y, n)] = pad ? 0 : bf16_bits(val[odd][r] - __uint_as_float((uint32_t)hi << 16));
    }
  }
}

// ---- phase 2 ------------------------------------------------------------------
// Step kinds: panel columns with low parts (16 per step: A_hi 0, A_lo 8192,
// B_hi 16384, B_lo 24576; three MMAs), panel columns without (32 per step:
// A_hi 0, B_hi 16384; two MMAs), dense block (32 columns: A_hi 0, A_lo 8192,
// X's image hi 16384, lo 24576; six MMAs), zero (a block without sources).
enum { kStLo = 0, kStHi = 1, kStDense = 2, kStZero = 3 };
struct P2Step {
  int kind, j0, cnt;  // column tiles j0 .. j0 + cnt - 1 of the source
};
__device__ __forceinline__ int seg_steps(const MxSeg& sg, const MxPanel* __restrict__ panels,
                                         const MxDense* __restrict__ dense) {
  if (sg.kind == kSegZero) return 1;
  if (sg.kind >= 0) {
    const int nct = panels[sg.kind].nct, nctl = panels[sg.kind].nctl;
    return (nctl + 1) / 2 + (nct - nctl + 3) / 4;
  }
  return dense[-1 - sg.kind].nct / 4;
}
__device__ __forceinline__ P2Step seg_step(const MxSeg& sg, int i, const MxPanel* __restrict__ panels) {
  if (sg.kind == kSegZero) return P2Step{kStZero, 0, 0};
  if (sg.kind < 0) return P2Step{kStDense, 4 * i, 4};
  const int nct = panels[sg.kind].nct, nctl = panels[sg.kind].nctl;
  const int nlo = (nctl + 1) / 2;
  if (i < nlo) return P2Step{kStLo, 2 * i, min(2, nctl - 2 * i)};
  const int j0 = nctl + 4 * (i - nlo);
  return P2Step{kStHi, j0, min(4, nct - j0)};
}

__device__ __forceinline__ void cpa4(uint32_t saddr, const void* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa4_zero(uint32_t saddr, const void* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, 0;\n" ::"r"(saddr), "l"(g) : "memory");
}

// A's image of NRT x NCT tiles (rows: the block's tile k; K blocks jj), each
// tile's 128 words copied to their rows: word w of lane (g, t) = rows g + 8 w
// of tile k at columns 2t, 2t+1 -> byte g 16 + (4 k + w) 128 + col_byte(t, jj).
// DENSE: the columns in X's row order (K block t, bytes 4 jj); else natural
// (K block jj, bytes 4 t).
template <int NCT, bool DENSE>
__device__ __forceinline__ void p2_copy_a(uint32_t base, const uint4* __restrict__ store, long long tile_of_k0,
                                          long long row_stride, int mask, int cnt, int tid) {
#pragma unroll
  for (int it = 0; it < 2 * NCT; ++it) {
    const int W = tid + kTcThreads * it, ti = W >> 7, k = ti / NCT, jj = ti % NCT, wi = W & 127;
    const int lane = wi >> 2, w = wi & 3, g = lane >> 2, t = lane & 3;
    const uint32_t dst = base + (uint32_t)(g * 16 + (4 * k + w) * 128) +
                         (DENSE ? (uint32_t)(4 * jj + t * 2048) : (uint32_t)(4 * t + jj * 2048));
    if (((mask >> k) & 1) && jj < cnt)
      cpa4(dst, reinterpret_cast<const uint32_t*>(store + (tile_of_k0 + k * row_stride + jj) * 32) + wi);
    else
      cpa4_zero(dst, store);
  }
}
// NB 2 KB blocks (16-byte copies) to base; blocks >= cnt are zero.
template <int NB>
__device__ __forceinline__ void p2_copy_b(uint32_t base, const uint4* __restrict__ src, int cnt, int tid) {
#pragma unroll
  for (int it = 0; it < NB / 2; ++it) {
    const int u = tid + kTcThreads * it, jj = u >> 7;
    if (jj < cnt)
      cpa16(base + (uint32_t)(u * 16), src + u);
    else
      cpa16_zero(base + (uint32_t)(u * 16), src);
  }
}

struct P2Cur {
  int b, s, i;  // block, segment (absolute), step within the segment
};

__global__ void __launch_bounds__(kTcThreads, 1)
    k_mx_p2_tc(int nblocks, int tile0, int tile_end, const int* __restrict__ seg_ptr, const MxSeg* __restrict__ segs,
               const MxPanel* __restrict__ panels, const MxDense* __restrict__ dense,
               const uint4* __restrict__ store, const uint4* __restrict__ Tb, const uint4* __restrict__ Xtc,
               const int* __restrict__ tile_leaf, const int* __restrict__ leaf_tile0,
               const int* __restrict__ leaf_off, float* __restrict__ Y, int ldy, int nr, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bars = sbase + (uint32_t)(kTcStages * kTcStage);
  const uint32_t chain_bar = bars + 8u * kTcStages, final_bar = chain_bar + 16u;
  const uint32_t slot = bars + 8u * kTcBars;
  if (tid == 0) {
    for (int i = 0; i < kTcBars; ++i) mbar_init(bars + 8u * i, 1);
    mbar_init_fence();
  }
  if (warp == 0) {
    tmem_alloc(slot, kTcCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + kTcStages * kTcStage + 8 * kTcBars);
  // this thread's TMEM lane (= row of the block) and half of the right-hand sides
  const int m = (warp & 3) * 32 + (tid & 31), hf = warp >> 2;
  const uint32_t my_lanes = (uint32_t)((warp & 3) * 32) << 16;
  const int stride = gridDim.x;

  P2Cur pc{(int)blockIdx.x, 0, 0}, cc{(int)blockIdx.x, 0, 0};
  if (pc.b < nblocks) pc.s = cc.s = seg_ptr[pc.b];
  auto advance = [&](P2Cur& c) {
    if (++c.i < seg_steps(segs[c.s], panels, dense)) return;
    c.i = 0;
    if (++c.s < seg_ptr[c.b + 1]) return;
    c.b += stride;
    if (c.b < nblocks) c.s = seg_ptr[c.b];
  };
  bool failed = false;
  auto produce = [&](int stage) {
    if (pc.b < nblocks && !failed) {
      const uint32_t base = sbase + (uint32_t)(stage * kTcStage);
      const MxSeg sg = segs[pc.s];
      const P2Step st = seg_step(sg, pc.i, panels);
      const int G0 = tile0 + 4 * pc.b;
      if (st.kind == kStLo) {
        const MxPanel& P = panels[sg.kind];
        p2_copy_a<2, false>(base, store, P.hi2 + (long long)sg.rt_base * P.nct + st.j0, P.nct, sg.mask, st.cnt, tid);
        p2_copy_a<2, false>(base + 8192u, store, P.lo2 + (long long)sg.rt_base * P.nctl + st.j0, P.nctl, sg.mask,
                            st.cnt, tid);
        p2_copy_b<2>(base + 16384u, Tb + (P.tb0 + st.j0) * 128, st.cnt, tid);
        p2_copy_b<2>(base + 24576u, Tb + (P.tb0 + P.nct + st.j0) * 128, st.cnt, tid);
      } else if (st.kind == kStHi) {
        const MxPanel& P = panels[sg.kind];
        p2_copy_a<4, false>(base, store, P.hi2 + (long long)sg.rt_base * P.nct + st.j0, P.nct, sg.mask, st.cnt, tid);
        p2_copy_b<4>(base + 16384u, Tb + (P.tb0 + st.j0) * 128, st.cnt, tid);
      } else if (st.kind == kStDense) {
        const MxDense& D = dense[-1 - sg.kind];
        p2_copy_a<4, true>(base, store, D.hi + (long long)sg.rt_base * D.nct + st.j0, D.nct, sg.mask, 4, tid);
        p2_copy_a<4, true>(base + 8192u, store, D.lo + (long long)sg.rt_base * D.nct + st.j0, D.nct, sg.mask, 4,
                           tid);
        const uint4* xb = Xtc + (size_t)(D.col_tile0 + st.j0 / 4) * 1024;
        p2_copy_b<4>(base + 16384u, xb, 4, tid);
        p2_copy_b<4>(base + 24576u, xb + 512, 4, tid);
      } else {  // zero: A and B of one MMA
        p2_copy_b<2>(base, store, 0, tid);
        p2_copy_b<2>(base + 16384u, store, 0, tid);
      }
      (void)G0;
    }
    if (pc.b < nblocks) advance(pc);
    cpa_commit();
  };
  for (int i = 0; i < kTcAhead; ++i) produce(i);

  float acc[64];
#pragma unroll
  for (int i = 0; i < 64; ++i) acc[i] = 0.f;
  long long step = 0;
  int chain = -1, chain_len = 0;
  bool pend = false, pend_end = false;
  int pend_chain = 0, pend_b = 0;
  auto drain = [&]() {
    const int b = pend_chain & 1;
    if (!mbar_wait(chain_bar + 8u * b, (uint32_t)((pend_chain >> 1) & 1))) failed = true;
    tc_fence_after();
    if (!failed) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        uint32_t v[32];
        tc_ld32(tmem + my_lanes + (uint32_t)(b * 128 + hf * 64 + q * 32), v);
        tc_wait_ld();
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[q * 32 + i] += __uint_as_float(v[i]);
      }
    }
    if (pend_end) {  // row m of the block, right-hand sides 64 hf .. 64 hf + 63
      const int G = tile0 + 4 * pend_b + (m >> 5);
      if (!failed && G < tile_end) {
        const int x = tile_leaf[G];
        const int row = leaf_off[x] + 32 * (G - leaf_tile0[x]) + (m & 31);
        if (row < leaf_off[x + 1]) {
#pragma unroll
          for (int i = 0; i < 64; ++i)
            if (64 * hf + i < nr) Y[(size_t)(64 * hf + i) * ldy + row] = acc[i];
        }
      }
#pragma unroll
      for (int i = 0; i < 64; ++i) acc[i] = 0.f;
    }
    pend = false;
  };
  while (cc.b < nblocks) {
    const long long ps = step + kTcAhead;
    const int pst = (int)(ps % kTcStages);
    if (pc.b < nblocks && ps >= kTcStages &&
        !mbar_wait(bars + 8u * pst, (uint32_t)(((ps - kTcStages) / kTcStages) & 1)))
      failed = true;
    produce(pst);
    cpa_wait<kTcAhead>();
    fence_proxy_async_smem();
    if (__syncthreads_or(failed ? 1 : 0)) break;
    const MxSeg sg = segs[cc.s];
    const P2Step stp = seg_step(sg, cc.i, panels);
    const int st = (int)(step % kTcStages);
    const bool first = chain_len == 0;
    if (first) ++chain;
    ++chain_len;
    const bool block_end = cc.i + 1 == seg_steps(sg, panels, dense) && cc.s + 1 == seg_ptr[cc.b + 1];
    const bool chain_end = block_end || stp.kind != kStHi || chain_len == kChainHi;
    if (tid == 0) {
      tc_fence_after();
      const uint32_t base = sbase + (uint32_t)(st * kTcStage);
      const uint32_t d = tmem + (uint32_t)((chain & 1) * 128);
      uint32_t accf = first ? 0u : 1u;
      auto mma = [&](uint32_t a, uint32_t b) {
        tc_mma_bf16(d, tc_sdesc(base + a, 2048, 128), tc_sdesc(base + b, 2048, 128), kIdesc, accf);
        accf = 1u;
      };
      if (stp.kind == kStLo) {
        mma(0u, 16384u);
        mma(0u, 24576u);
        mma(8192u, 16384u);
      } else if (stp.kind == kStHi) {
        mma(0u, 16384u);
        if (stp.cnt > 2) mma(4096u, 20480u);
      } else if (stp.kind == kStDense) {
        for (int q = 0; q < 2; ++q) {
          const uint32_t o = (uint32_t)(q * 4096);
          mma(o, 16384u + o);
          mma(o, 24576u + o);
          mma(8192u + o, 16384u + o);
        }
      } else {
        mma(0u, 16384u);
      }
      tc_commit(bars + 8u * st);
      if (chain_end) tc_commit(chain_bar + 8u * (chain & 1));
    }
    if (pend) drain();
    if (chain_end) {
      pend = true;
      pend_end = block_end;
      pend_chain = chain;
      pend_b = cc.b;
      chain_len = 0;
    }
    tc_fence_before();
    advance(cc);
    ++step;
  }
  if (pend && !failed) drain();
  cpa_wait<0>();
  if (tid == 0) tc_commit(final_bar);
  if (!mbar_wait(final_bar, 0)) failed = true;
  if (failed) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTcCols);
  }
}

}  // namespace

hm_status mixed_tc_pass(hm_hmatrix_s* h, int nr, const uint4* Xtc, float4* S, long long sh, uint4* Tb, float* Y,
                        int ldy, cudaStream_t s, KernelMarks* km) {
  MxPlan& M = h->mx;
  static bool attr = false;
  if (!attr) {
    HM_CUDA(cudaFuncSetAttribute(k_mx_p1_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    HM_CUDA(cudaFuncSetAttribute(k_mx_p2_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    attr = true;
  }
  const long long xbytes = 4ll * h->n * 128;  // X's image: hi + lo of 128 right-hand sides
  unsigned short* Tb16 = reinterpret_cast<unsigned short*>(Tb);
  if (M.num_tc_units > 0) {
    const int grid = std::min(M.num_sms, M.num_tc_units);
    k_mx_p1_tc<<<grid, kTcThreads, kTcSmem, s>>>(M.tc_units.p, M.num_tc_units, M.panels.p, M.store.p, Xtc, M.tslot_tc.p,
                                          reinterpret_cast<float*>(S), Tb16, sh, M.tc_err.p);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_mx_p1_tc", M.bytes_p1 + xbytes, s);
  }
  if (M.nmt > 0) {
    k_mx_reduce_tc<<<dim3((unsigned)((M.nmt * 32 + 255) / 256), 8), 256, 0, s>>>(M.mtiles.p, M.nmt, M.panels.p, S,
                                                                                 M.tslot_tc.p, Tb16, sh);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_mx_reduce_tc", (512ll * M.s_tiles + 512ll * M.nmt) * 8, s);
  }
  if (M.p2_blocks > 0) {
    const int grid = std::min(M.num_sms, M.p2_blocks);
    k_mx_p2_tc<<<grid, kTcThreads, kTcSmem, s>>>(M.p2_blocks, M.p2_tile0, M.p2_tile0 + M.p2_tiles, M.p2_seg_ptr.p,
                                          M.p2_segs.p, M.panels.p, M.dense.p, M.store.p, Tb, Xtc, M.tile_leaf.p,
                                          M.leaf_tile0.p, h->tree->offsets.p, Y, ldy, nr, M.tc_err.p);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_mx_p2_tc", M.bytes_p2 + xbytes + 4ll * h->n * nr, s);
  }
  return HM_OK;
}

}  // namespace hm

extern "C" hm_status hm_hmatrix_check(hm_hmatrix h, void* stream) {
  using namespace hm;
  if (!h) return fail(HM_ERR_INVALID, "hm_hmatrix_check: null matrix");
  HM_CUDA(cudaStreamSynchronize(as_stream(stream)));
  if (!h->mx.tc_err.p) return HM_OK;
  int v = 0;
  HM_CUDA(cudaMemcpy(&v, h->mx.tc_err.p, sizeof v, cudaMemcpyDeviceToHost));
  if (v == 0) return HM_OK;
  HM_CUDA(cudaMemset(h->mx.tc_err.p, 0, sizeof v));
  return fail(HM_ERR_TIMEOUT, "a bounded wait of the tcgen05 phase-1 kernel gave up: products since the last check are wrong");
}
