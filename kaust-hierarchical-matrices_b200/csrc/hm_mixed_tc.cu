// hm_mixed_tc.cu -- the mixed form's 128-column passes on the Blackwell
// tensor cores (tcgen05.mma, accumulator in tensor memory).
//
// A pass of 128 right-hand sides multiplies every factor element 128 times
// (hi and lo: up to 3 BF16 products each), more than the warp-level MMA
// keeps up with at HBM speed.
//
// Phase 1 (k_mx_p1_tc): one CTA per SM walks its units -- up to 16 column
// tiles of a panel, all with low parts or none, over a chunk of row tiles --
// and per 32-row tile issues D (128 columns x 128 right-hand sides, FP32 in
// TMEM) += V^T X as tcgen05.mma of M = 128, N = 128, K = 16:
//   A = V^T: the unit's P1 tiles of one row tile, one bulk copy (TMA
//     engine): the tiles are stored in the K-major core-matrix layout with the
//     64-byte swizzle (column 8 j + g's 64-byte row at 512 j + 64 g; SBO 512).
//     A K block t holds rows rho(t, e) = 8 (e / 2) + 2 t + e % 2, a
//     permutation of the tile's rows, harmless in a sum as B uses the same.
//   B = X: the pass's image per 32-row tile written by k_mx_split_x (hi 8 KB,
//     then lo; right-hand side n at 16 (n % 8) + 128 (n / 8), K block c at
//     2048 c: SBO 128, LBO 2048), one bulk copy each.
// Columns with low parts take three products per tile (V_hi X_hi, V_hi X_lo,
// V_lo X_hi), one row tile per step; the others one, two row tiles per step.
//
// Warp roles, no CTA-wide barrier in the loop: warp 0 lane 0 copies each
// step into one of six 32 KB stages (bulk copies, counted in bytes on the
// stage's "full" mbarrier); warp 1 lane 0 waits for it, issues the step's
// MMAs and commits them to the stage's "empty" mbarrier; chains of four steps
// go into one of four TMEM accumulators (128 columns each), committed to its
// "ready" mbarrier; warps 2-5 (TMEM lanes 32 (w % 4) ..) read a ready accumulator
// out (tcgen05.ld), add it to their FP32 sums with round-to-nearest adds,
// and release it.  The tensor core's own sums do not round to nearest, so the
// chains are kept short: 24 MMAs for columns with low parts, a drift far
// below the BF16 hi + lo rounding of T.  At a unit's end each drain thread
// stores its column (its TMEM lane): as T (into the mirror column's slots,
// split hi + lo or hi only) when the panel is projected in one row chunk,
// else as the chunk's partial S (per column its 128 FP32 sums, contiguous).
// Every wait is bounded; a wait that gives up raises an abort flag that the
// other roles see, sets the error word, and the kernel ends after every
// issued copy and MMA has completed.
//
// T of such a pass is kept in 2 KB blocks, one per 8 columns and part (hi,
// lo): the MN-major core-matrix image of B = T for phase 2 (right-hand sides
// n, columns c: 2 (n % 8) + 128 (n / 8) + 16 c bytes; SBO 128, LBO 2048),
// in which a column's 8 consecutive right-hand sides are 16 contiguous bytes:
// a drain thread writes its column with 16-byte stores.
//
// Phase 2 (k_mx_p2_tc): one CTA per SM walks blocks of 4 row tiles (128
// rows), D (128 rows x 128 right-hand sides) += U T per ancestor panel and
// D X per dense block, M = 128, N = 128.  A = the factor tiles as stored (P2
// order: lane (g,t) holds rows g + 8 w, w = 0..3, at columns 2t, 2t+1), each
// 4-byte word copied by cp.async to its row of the core-matrix image; rows of
// the block's tiles that a source does not cover are zero.  Dense blocks take
// their columns in X's row order rho so that B is X's image of the column
// cluster's tile.  Panels' columns with low parts take three products per 16
// columns, 32 columns per step; the others one per 16 columns, 64 per step;
// dense blocks three per 16 columns, 32 per step.
#include "hm_hmatrix.h"
#include "hm_mixed.h"
#include "hm_mma.cuh"
#include "hm_tc.cuh"

namespace hm {
namespace {

constexpr int kTcStage = 32768;          // bytes per stage
constexpr uint32_t kIdesc = tc_idesc_bf16(128, 128);
constexpr uint32_t kIdescBmn = tc_idesc_bf16(128, 128) | (1u << 16);  // B MN-major

// ---- phase 1 ------------------------------------------------------------------
constexpr int kP1Stages = 6;
constexpr int kP1Bufs = 4;       // TMEM accumulators of 128 columns (all 512)
constexpr int kP1Chain = 4;      // steps per MMA chain
constexpr int kP1Threads = 192;  // copy warp 0, MMA warp 1, drain warps 2-5
// shared memory: stages, then mbarriers full[S], empty[S], ready[B], free[B],
// done; then the TMEM address and the abort flag
constexpr int kP1BarBytes = 8 * (2 * kP1Stages + 2 * kP1Bufs + 1);
constexpr size_t kP1Smem = (size_t)kP1Stages * kTcStage + kP1BarBytes + 16;

// Stage layout (bytes): columns with low parts: A_hi 0, A_lo 8192, B_hi
// 16384, B_lo 24576 (one row tile); without: A_hi of row tile k at 8192 k,
// B_hi at 16384 + 8192 k (two row tiles).  A: 64-byte swizzle, SBO 512, K
// chunk q (16 rows) at +32 q bytes; B: no swizzle, SBO 128, LBO 2048, K chunk
// q at +4096 q.

// 16-byte word (right-hand sides 8 q .. 8 q + 7, column pos % 8) of T's block pos / 8
__device__ __forceinline__ long long tb_word(long long pos, int q) { return (pos >> 3) * 128 + q * 8 + (pos & 7); }
// 8 values as BF16 hi, and their BF16 lo (value - hi)
__device__ __forceinline__ void split8(const float* v, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) split_bf16x2(v[2 * i], v[2 * i + 1], h[i], l[i]);
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// Drain thread m (the unit's column m, its TMEM lane) of a finished unit: T
// or the chunk's partial S (column c of S tile i at floats 128 (8 i + c)),
// all 128 right-hand sides.
__device__ __forceinline__ void p1_store(const TcUnit& U, const float (&acc)[128], const int2* __restrict__ tslot_tc,
                                         float* __restrict__ S, uint4* __restrict__ Tb, int m) {
  const int jt = m >> 3, c = m & 7;
  if (jt >= U.nct) return;
  if (U.flags & 2) {
    const int2 e = __ldg(tslot_tc + (U.out + jt) * 8 + c);
    const bool pad = e.x < 0;  // a padding column: zeros into its own slots
    const long long hp = pad ? -1 - (long long)e.x : e.x;
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      uint4 hi, lo;
      split8(acc + 8 * q, hi, lo);
      Tb[tb_word(hp, q)] = pad ? z : hi;
      if (e.y >= 0) Tb[tb_word(e.y, q)] = pad ? z : lo;
    }
  } else {
    float4* out = reinterpret_cast<float4*>(S + ((U.out + jt) * 8 + c) * 128);
#pragma unroll
    for (int q = 0; q < 32; ++q) out[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
  }
}

__device__ __forceinline__ int p1_step_tiles(const TcUnit& U, int r) { return (U.flags & 1) ? 1 : min(2, U.nrt - r); }

__global__ void __launch_bounds__(kP1Threads, 1)
    k_mx_p1_tc(const TcUnit* __restrict__ units, int nunits, const uint4* __restrict__ store,
               const uint4* __restrict__ Xtc, const int2* __restrict__ tslot_tc, float* __restrict__ S,
               uint4* __restrict__ Tb, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t full = sbase + (uint32_t)(kP1Stages * kTcStage), empty = full + 8u * kP1Stages;
  const uint32_t ready = empty + 8u * kP1Stages, freeb = ready + 8u * kP1Bufs, done = freeb + 8u * kP1Bufs;
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kP1Stages * kTcStage + kP1BarBytes);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(slot + 1);
  if (tid == 0) {
    for (int i = 0; i < kP1Stages; ++i) {
      mbar_init(full + 8u * i, 1);  // thread 0's expect_tx (bulk copies)
      mbar_init(empty + 8u * i, 1);
    }
    for (int i = 0; i < kP1Bufs; ++i) {
      mbar_init(ready + 8u * i, 1);
      mbar_init(freeb + 8u * i, 128);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    mbar_init_fence();
  }
  if (warp == 0) {
    tmem_alloc(smem_u32(slot), 128 * kP1Bufs);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(slot);
  const int stride = gridDim.x;
  bool failed = false;
  auto give_up = [&]() {
    failed = true;
    *abort_flag = 1;
  };

  if (warp == 0) {
    if (lane == 0) {  // ---- producer: bulk copies of each step
      long long j = 0;
      int u = blockIdx.x;
      TcUnit U;
      if (u < nunits) U = units[u];
      while (u < nunits && !failed) {
        TcUnit nxt;
        if (u + stride < nunits) nxt = units[u + stride];
        const bool lo = U.flags & 1;
        const uint32_t abytes = (uint32_t)U.nct * 512u;
        for (int r = 0; r < U.nrt;) {
          const int nt = p1_step_tiles(U, r), s = (int)(j % kP1Stages);
          if (j >= kP1Stages &&
              !mbar_wait_or(empty + 8u * s, (uint32_t)(((j - kP1Stages) / kP1Stages) & 1), abort_flag)) {
            give_up();
            break;
          }
          const uint32_t base = sbase + (uint32_t)(s * kTcStage), bar = full + 8u * s;
          mbar_arrive_expect_tx(bar, (uint32_t)nt * (abytes + 8192u) + (lo ? abytes + 8192u : 0u));
          for (int k = 0; k < nt; ++k) {
            bulk_g2s(base + (uint32_t)(k * 8192), store + (U.vhi + (long long)(r + k) * U.shi) * 32, abytes, bar);
            bulk_g2s(base + 16384u + (uint32_t)(k * 8192), Xtc + (size_t)(U.xtile + r + k) * 1024, 8192u, bar);
          }
          if (lo) {
            bulk_g2s(base + 8192u, store + (U.vlo + (long long)r * U.slo) * 32, abytes, bar);
            bulk_g2s(base + 24576u, Xtc + (size_t)(U.xtile + r) * 1024 + 512, 8192u, bar);
          }
          r += nt;
          ++j;
        }
        u += stride;
        U = nxt;
      }
      // every copy issued has landed before the CTA ends (bounded)
      for (long long jj = j > kP1Stages ? j - kP1Stages : 0; jj < j; ++jj)
        mbar_wait(full + 8u * (uint32_t)(jj % kP1Stages), (uint32_t)((jj / kP1Stages) & 1), 1000000000ull);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer
      const uint64_t adesc0 = tc_sdesc_sw64(sbase, 512), bdesc0 = tc_sdesc(sbase, 2048, 128);
      long long j = 0;
      int chain = -1;
      int u = blockIdx.x;
      TcUnit U;
      if (u < nunits) U = units[u];
      while (u < nunits && !failed) {
        TcUnit nxt;
        if (u + stride < nunits) nxt = units[u + stride];
        const bool lo = U.flags & 1;
        int in_chain = 0;
        for (int r = 0; r < U.nrt && !failed;) {
          const int nt = p1_step_tiles(U, r), s = (int)(j % kP1Stages);
          if (in_chain == 0) {
            ++chain;
            if (chain >= kP1Bufs && !mbar_wait_or(freeb + 8u * (uint32_t)(chain % kP1Bufs),
                                                  (uint32_t)((chain / kP1Bufs - 1) & 1), abort_flag)) {
              give_up();
              break;
            }
          }
          if (!mbar_wait_or(full + 8u * s, (uint32_t)((j / kP1Stages) & 1), abort_flag)) {
            give_up();
            break;
          }
          tc_fence_after();
          // descriptors of this stage; an offset of o bytes adds o >> 4 to the start address field
          const uint64_t da = adesc0 + (uint64_t)((s * kTcStage) >> 4), db = bdesc0 + (uint64_t)((s * kTcStage) >> 4);
          const uint32_t d = tmem + (uint32_t)((chain % kP1Bufs) * 128);
          uint32_t acc = in_chain == 0 ? 0u : 1u;
          if (lo) {
#pragma unroll
            for (int p = 0; p < 3; ++p) {  // V_hi X_hi, V_hi X_lo, V_lo X_hi
              const uint32_t pa = p == 2 ? 8192u : 0u, pb = p == 1 ? 24576u : 16384u;
#pragma unroll
              for (int q = 0; q < 2; ++q) {
                tc_mma_bf16(d, da + ((pa + (uint32_t)(q * 32)) >> 4), db + ((pb + (uint32_t)(q * 4096)) >> 4), kIdesc,
                            acc);
                acc = 1u;
              }
            }
          } else {
            for (int k = 0; k < nt; ++k)
#pragma unroll
              for (int q = 0; q < 2; ++q) {
                tc_mma_bf16(d, da + ((uint32_t)(k * 8192 + q * 32) >> 4),
                            db + ((16384u + (uint32_t)(k * 8192 + q * 4096)) >> 4), kIdesc, acc);
                acc = 1u;
              }
          }
          tc_commit(empty + 8u * s);
          r += nt;
          ++j;
          if (r >= U.nrt || ++in_chain == kP1Chain) {
            tc_commit(ready + 8u * (uint32_t)(chain % kP1Bufs));
            in_chain = 0;
          }
        }
        u += stride;
        U = nxt;
      }
    }
    if (lane == 0) tc_commit(done);  // arrives once every MMA issued above is done
  } else {  // ---- drain warps 2-5: TMEM lanes 32 (warp % 4) ..
    const int m = (warp & 3) * 32 + lane;
    const uint32_t my_lanes = (uint32_t)((warp & 3) * 32) << 16;
    float acc[128];
#pragma unroll
    for (int i = 0; i < 128; ++i) acc[i] = 0.f;
    int chain = -1;
    int u = blockIdx.x;
    TcUnit U;
    if (u < nunits) U = units[u];
    while (u < nunits && !failed) {
      TcUnit nxt;
      if (u + stride < nunits) nxt = units[u + stride];
      const int nsteps = (U.flags & 1) ? U.nrt : (U.nrt + 1) / 2;
      const int nchains = (nsteps + kP1Chain - 1) / kP1Chain;
      for (int c = 0; c < nchains; ++c) {
        ++chain;
        const uint32_t b = (uint32_t)(chain % kP1Bufs);
        if (!mbar_wait_or(ready + 8u * b, (uint32_t)((chain / kP1Bufs) & 1), abort_flag)) {
          give_up();
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          uint32_t v[32];
          tc_ld32(tmem + my_lanes + b * 128u + (uint32_t)(q * 32), v);
          tc_wait_ld();
#pragma unroll
          for (int i = 0; i < 32; ++i) acc[q * 32 + i] += __uint_as_float(v[i]);
        }
        tc_fence_before();
        mbar_arrive(freeb + 8u * b);
      }
      if (failed) break;
      p1_store(U, acc, tslot_tc, S, Tb, m);
#pragma unroll
      for (int i = 0; i < 128; ++i) acc[i] = 0.f;
      u += stride;
      U = nxt;
    }
  }
  if (failed) atomicExch(err, 1);
  // the tensor memory is released once every MMA is done (thread 0 waits,
  // bounded; the others wait at the barrier)
  if (tid == 0 && !mbar_wait(done, 0, 10000000000ull)) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 128 * kP1Bufs);
  }
}

// ---- chunk reduction (panels projected in several row chunks) -----------------
// The chunk partials of each column summed in chunk order, as T blocks: one
// thread per column tile, column c and 8 right-hand sides q.
__global__ void k_mx_reduce_tc(const int2* __restrict__ mtiles, long long nmt, const MxPanel* __restrict__ panels,
                               const float* __restrict__ S, const int2* __restrict__ tslot_tc,
                               uint4* __restrict__ Tb) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nmt * 128) return;
  const int2 mt = mtiles[i >> 7];
  const int c = (int)((i >> 4) & 7), q = (int)(i & 15);
  const MxPanel P = panels[mt.x];
  float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int ch = 0; ch < P.nchunkt; ++ch) {
    const float4* a = reinterpret_cast<const float4*>(S + ((P.s0t + (long long)ch * P.nct + mt.y) * 8 + c) * 128 + 8 * q);
    const float4 a0 = a[0], a1 = a[1];
    v[0] += a0.x;
    v[1] += a0.y;
    v[2] += a0.z;
    v[3] += a0.w;
    v[4] += a1.x;
    v[5] += a1.y;
    v[6] += a1.z;
    v[7] += a1.w;
  }
  const int2 e = __ldg(tslot_tc + (P.t0 + mt.y) * 8 + c);
  const bool pad = e.x < 0;
  const long long hp = pad ? -1 - (long long)e.x : e.x;
  uint4 hi, lo;
  split8(v, hi, lo);
  const uint4 z = make_uint4(0u, 0u, 0u, 0u);
  Tb[tb_word(hp, q)] = pad ? z : hi;
  if (e.y >= 0) Tb[tb_word(e.y, q)] = pad ? z : lo;
}

// ---- phase 2 ------------------------------------------------------------------
// Warp roles as in phase 1, with 27 copy warps and four drain warps that keep
// the running sums in tensor memory: A (the factor tiles in
// P2 order) is rearranged word by word into its core-matrix image by
// cp.async (4 bytes, any destination); B (T blocks, X's image) comes by bulk
// copies from producer thread 0.  A producer thread's copies of step j are
// fenced to the async proxy and announced on the stage's "full" mbarrier
// kP2Delay steps later, once they have landed (cp.async.wait_group), so that
// producers do not wait on their own copies.
// Stage layout (bytes): kind 0: A_hi 0, A_lo 8192, B_hi 16384, B_lo 24576
// (K blocks of 8 columns 2048 apart); kind 1: A_hi 0, B_hi 16384 (8 K
// blocks); kind 2: as kind 0, with X's image as B; kind 3: zero A at 0 and B
// at 16384 (one K chunk).  A: row m = 32 k + g + 8 w at 16 g + 128 (4 k + w)
// (K-major, SBO 128, LBO 2048); B: T blocks MN-major (right-hand side n at
// 2 (n % 8) + 128 (n / 8), column c at 16 c; SBO 128, LBO 2048), X's image
// K-major (n at 16 (n % 8) + 128 (n / 8); SBO 128, LBO 2048).
constexpr int kP2Stages = 6;
constexpr int kP2Bufs = 2;        // TMEM chain accumulators (columns 0-255); running sums at 256-383
constexpr int kP2Chain = 4;      // steps per MMA chain
constexpr int kP2Delay = 3;      // steps between a producer's copies and its arrival
constexpr int kP2CopyWarps = 27;
constexpr int kP2Producers = 32 * kP2CopyWarps;  // threads of the copy warps 0-26
constexpr int kP2Threads = 1024;                 // copy warps 0-26, MMA warp 27, drain warps 28-31
constexpr int kP2BarBytes = 8 * (2 * kP2Stages + 2 * kP2Bufs + 1);
constexpr size_t kP2Smem = (size_t)kP2Stages * kTcStage + kP2BarBytes + 16;

__device__ __forceinline__ void cpa4(uint32_t saddr, const void* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cpa4_zero(uint32_t saddr, const void* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, 0;\n" ::"r"(saddr), "l"(g) : "memory");
}

// A's image of the block's 4 row tiles x nk K blocks (column tiles j0 + jj),
// word W of the tiles per copy thread (tile W / 128, jj-major; word W % 128):
// word w of lane (g, t) of tile (k, jj) = rows g + 8 w of row tile k at
// columns 2t, 2t+1 -> 16 g + 128 (4 k + w) + (DENSE ? 4 jj + 2048 t : 4 t +
// 2048 jj).  Rows of tiles outside the mask, and K blocks cnt .. nk - 1, are
// zero.  (Measured: more copy warps raise the rate; fewer instructions per
// copy with fewer warps, or 16-byte zeroing of whole masked row tiles, did not.)
template <bool DENSE>
__device__ __forceinline__ void p2_copy_a(uint32_t base, const uint4* __restrict__ store, long long a0, int stride,
                                          int mask, int cnt, int nk, int pt) {
  for (int W = pt; W < 512 * nk; W += kP2Producers) {
    const int it = W >> 7, wi = W & 127, jj = it >> 2, k = it & 3;
    const int lane = wi >> 2, w = wi & 3, g = lane >> 2, t = lane & 3;
    const uint32_t dst = base + (uint32_t)(g * 16 + (4 * k + w) * 128) +
                         (DENSE ? (uint32_t)(4 * jj + t * 2048) : (uint32_t)(4 * t + jj * 2048));
    if (((mask >> k) & 1) && jj < cnt)
      cpa4(dst, reinterpret_cast<const uint32_t*>(store + (a0 + (long long)k * stride + jj) * 32) + wi);
    else
      cpa4_zero(dst, store);
  }
}
// zero 2 KB blocks [from, to) of a B image at base (16 bytes per copy)
__device__ __forceinline__ void p2_zero_blocks(uint32_t base, int from, int to, const void* any, int pt) {
  for (int u = pt + 128 * from; u < 128 * to; u += kP2Producers) cpa16_zero(base + (uint32_t)(u * 16), any);
}

__global__ void __launch_bounds__(kP2Threads, 1)
    k_mx_p2_tc(int nblocks, int tile0, int tile_end, const int* __restrict__ step_ptr,
               const P2Step* __restrict__ steps, const uint4* __restrict__ store, const uint4* __restrict__ Tb,
               const uint4* __restrict__ Xtc, const int* __restrict__ tile_leaf,
               const int* __restrict__ leaf_tile0, const int* __restrict__ leaf_off, float* __restrict__ Y, int ldy,
               int nr, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t full = sbase + (uint32_t)(kP2Stages * kTcStage), empty = full + 8u * kP2Stages;
  const uint32_t ready = empty + 8u * kP2Stages, freeb = ready + 8u * kP2Bufs, done = freeb + 8u * kP2Bufs;
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kP2Stages * kTcStage + kP2BarBytes);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(slot + 1);
  if (tid == 0) {
    for (int i = 0; i < kP2Stages; ++i) {
      mbar_init(full + 8u * i, kP2Producers + 1);  // copy threads, plus thread 0's expect_tx (bulk copies)
      mbar_init(empty + 8u * i, 1);
    }
    for (int i = 0; i < kP2Bufs; ++i) {
      mbar_init(ready + 8u * i, 1);
      mbar_init(freeb + 8u * i, 128);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    mbar_init_fence();
  }
  if (warp == 0) {
    tmem_alloc(smem_u32(slot), 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(slot);
  const int stride = gridDim.x;
  bool failed = false;
  auto give_up = [&]() {
    failed = true;
    *abort_flag = 1;
  };

  if (warp < kP2CopyWarps) {  // ---- producers
    const int pt = tid;
    long long j = 0, arrived = 0;  // steps issued; steps announced
    for (int b = blockIdx.x; b < nblocks && !failed; b += stride) {
      const int e = step_ptr[b + 1];
      P2Step st_next = steps[step_ptr[b]];  // the next step's descriptor, loaded a step ahead
      for (int i = step_ptr[b]; i < e; ++i) {
        const P2Step st = st_next;
        if (i + 1 < e) st_next = steps[i + 1];
        const int s = (int)(j % kP2Stages);
        if (j >= kP2Stages &&
            !mbar_wait_or(empty + 8u * s, (uint32_t)(((j - kP2Stages) / kP2Stages) & 1), abort_flag)) {
          give_up();
          break;
        }
        const int kind = st.info & 3, cnt = (st.info >> 2) & 15, mask = st.info >> 8;
        const int nk = (cnt + 1) & ~1;
        const uint32_t base = sbase + (uint32_t)(s * kTcStage), bar = full + 8u * s;
        if (pt == 0) {  // B by bulk copies
          if (kind == 0) {
            mbar_arrive_expect_tx(bar, (uint32_t)(2 * cnt * 2048));
            bulk_g2s(base + 16384u, Tb + st.b_hi, (uint32_t)(cnt * 2048), bar);
            bulk_g2s(base + 24576u, Tb + st.b_lo, (uint32_t)(cnt * 2048), bar);
          } else if (kind == 1) {
            mbar_arrive_expect_tx(bar, (uint32_t)(cnt * 2048));
            bulk_g2s(base + 16384u, Tb + st.b_hi, (uint32_t)(cnt * 2048), bar);
          } else if (kind == 2) {
            mbar_arrive_expect_tx(bar, 16384u);
            bulk_g2s(base + 16384u, Xtc + st.b_hi, 8192u, bar);
            bulk_g2s(base + 24576u, Xtc + st.b_lo, 8192u, bar);
          } else {
            mbar_arrive(bar);
          }
        }
        if (kind == 0) {
          p2_copy_a<false>(base, store, st.a_hi, st.a_stride, mask, cnt, nk, pt);
          p2_copy_a<false>(base + 8192u, store, st.a_lo, st.a_stride_lo, mask, cnt, nk, pt);
          p2_zero_blocks(base + 16384u, cnt, nk, store, pt);
          p2_zero_blocks(base + 24576u, cnt, nk, store, pt);
        } else if (kind == 1) {
          p2_copy_a<false>(base, store, st.a_hi, st.a_stride, mask, cnt, nk, pt);
          p2_zero_blocks(base + 16384u, cnt, nk, store, pt);
        } else if (kind == 2) {
          p2_copy_a<true>(base, store, st.a_hi, st.a_stride, mask, 4, 4, pt);
          p2_copy_a<true>(base + 8192u, store, st.a_lo, st.a_stride_lo, mask, 4, 4, pt);
        } else {
          p2_zero_blocks(base, 0, 2, store, pt);
          p2_zero_blocks(base + 16384u, 0, 2, store, pt);
        }
        cpa_commit();
        ++j;
        if (j - 1 >= kP2Delay) {  // announce step j - 1 - kP2Delay: its copies have landed
          cpa_wait<kP2Delay>();
          fence_proxy_async_smem();
          mbar_arrive(full + 8u * (uint32_t)(arrived % kP2Stages));
          ++arrived;
        }
      }
    }
    cpa_wait<0>();
    fence_proxy_async_smem();
    for (; arrived < j; ++arrived) mbar_arrive(full + 8u * (uint32_t)(arrived % kP2Stages));
    // the bulk copies issued have landed before the CTA ends (bounded)
    if (pt == 0)
      for (long long jj = j > kP2Stages ? j - kP2Stages : 0; jj < j; ++jj)
        mbar_wait(full + 8u * (uint32_t)(jj % kP2Stages), (uint32_t)((jj / kP2Stages) & 1), 1000000000ull);
  } else if (warp == kP2CopyWarps) {  // ---- MMA issuer
    if (lane == 0) {
      const uint64_t desc0 = tc_sdesc(sbase, 2048, 128);  // A, T blocks and X's image: SBO 128, LBO 2048
      long long j = 0;
      int chain = -1;
      for (int b = blockIdx.x; b < nblocks && !failed; b += stride) {
        const int e = step_ptr[b + 1];
        int in_chain = 0;
        int info_next = steps[step_ptr[b]].info;
        for (int i = step_ptr[b]; i < e; ++i) {
          const int info = info_next;
          if (i + 1 < e) info_next = steps[i + 1].info;
          const int s = (int)(j % kP2Stages);
          if (in_chain == 0) {
            ++chain;
            if (chain >= kP2Bufs && !mbar_wait_or(freeb + 8u * (uint32_t)(chain % kP2Bufs),
                                                  (uint32_t)((chain / kP2Bufs - 1) & 1), abort_flag)) {
              give_up();
              break;
            }
          }
          if (!mbar_wait_or(full + 8u * s, (uint32_t)((j / kP2Stages) & 1), abort_flag)) {
            give_up();
            break;
          }
          tc_fence_after();
          const uint64_t ds = desc0 + (uint64_t)((s * kTcStage) >> 4);  // this stage's start
          const uint32_t d = tmem + (uint32_t)((chain % kP2Bufs) * 128);
          uint32_t acc = in_chain == 0 ? 0u : 1u;
          const int kind = info & 3, cnt = (info >> 2) & 15, nq = (cnt + 1) >> 1;
          const uint32_t idesc = kind == 2 ? kIdesc : kIdescBmn;  // T blocks are MN-major, X's image K-major
          auto mma = [&](uint32_t a, uint32_t bb) {
            tc_mma_bf16(d, ds + (a >> 4), ds + (bb >> 4), idesc, acc);
            acc = 1u;
          };
          if (kind == 0) {
            for (int q = 0; q < nq; ++q) {
              const uint32_t o = (uint32_t)(q * 4096);
              mma(o, 16384u + o);
              mma(o, 24576u + o);
              mma(8192u + o, 16384u + o);
            }
          } else if (kind == 1) {
            for (int q = 0; q < nq; ++q) mma((uint32_t)(q * 4096), 16384u + (uint32_t)(q * 4096));
          } else if (kind == 2) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const uint32_t o = (uint32_t)(q * 4096);
              mma(o, 16384u + o);
              mma(o, 24576u + o);
              mma(8192u + o, 16384u + o);
            }
          } else {
            mma(0u, 16384u);
          }
          tc_commit(empty + 8u * s);
          ++j;
          if (i + 1 == e || ++in_chain == kP2Chain) {
            tc_commit(ready + 8u * (uint32_t)(chain % kP2Bufs));
            in_chain = 0;
          }
        }
      }
      tc_commit(done);  // arrives once every MMA issued above is done
    }
  } else {  // ---- drain warps 28-31: TMEM lanes 32 (warp % 4) .., row m of the block
    // Each chain is added to the block's running sums kept in tensor memory
    // (columns 256-383: read, FP32 round-to-nearest add, write back); the last
    // chain's sums go to Y.  Few registers per thread (at most 64 in a CTA of
    // 32 warps), so that 27 warps can copy.
    const int m = (warp & 3) * 32 + lane;
    const uint32_t my_lanes = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t tsum = tmem + my_lanes + 256u;
    int chain = -1;
    for (int b = blockIdx.x; b < nblocks && !failed; b += stride) {
      const int nsteps = step_ptr[b + 1] - step_ptr[b];
      const int nchains = (nsteps + kP2Chain - 1) / kP2Chain;
      const int G = tile0 + 4 * b + (m >> 5);
      int row = -1;
      if (G < tile_end) {
        const int x = tile_leaf[G];
        const int r = leaf_off[x] + 32 * (G - leaf_tile0[x]) + (m & 31);
        if (r < leaf_off[x + 1]) row = r;
      }
      for (int c = 0; c < nchains; ++c) {
        ++chain;
        const uint32_t bb = (uint32_t)(chain % kP2Bufs);
        if (!mbar_wait_or(ready + 8u * bb, (uint32_t)((chain / kP2Bufs) & 1), abort_flag)) {
          give_up();
          break;
        }
        tc_fence_after();
        const bool first = c == 0, last = c + 1 == nchains;
        float* yq = Y + (row >= 0 ? row : 0);
#pragma unroll 1
        for (int q = 0; q < 8; ++q, yq += (size_t)16 * ldy) {
          uint32_t v[16];
          tc_ld16(tmem + my_lanes + bb * 128u + (uint32_t)(q * 16), v);
          if (!first) {
            uint32_t sm[16];
            tc_ld16(tsum + (uint32_t)(q * 16), sm);
            tc_wait_ld();
#pragma unroll
            for (int e = 0; e < 16; ++e) v[e] = __float_as_uint(__uint_as_float(v[e]) + __uint_as_float(sm[e]));
          } else {
            tc_wait_ld();
          }
          if (!last) {
            tc_st16(tsum + (uint32_t)(q * 16), v);
          } else if (row >= 0) {
            float* y = yq;
#pragma unroll
            for (int e = 0; e < 16; ++e, y += ldy)
              if (q * 16 + e < nr) *y = __uint_as_float(v[e]);
          }
        }
        if (!last) tc_wait_st();
        tc_fence_before();
        mbar_arrive(freeb + 8u * bb);
      }
    }
  }
  if (failed) atomicExch(err, 1);
  if (tid == 0 && !mbar_wait(done, 0, 10000000000ull)) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

}  // namespace

hm_status mixed_tc_pass(hm_hmatrix_s* h, int nr, const uint4* Xtc, float* S, uint4* Tb, float* Y, int ldy,
                        cudaStream_t s, KernelMarks* km) {
  MxPlan& M = h->mx;
  // the kernels' shared-memory limit, once per device of this process
  static unsigned long long attr_done = 0;
  int dev = 0;
  HM_CUDA(cudaGetDevice(&dev));
  if (dev >= 64 || !((attr_done >> dev) & 1ull)) {
    HM_CUDA(cudaFuncSetAttribute(k_mx_p1_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP1Smem));
    HM_CUDA(cudaFuncSetAttribute(k_mx_p2_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2Smem));
    if (dev < 64) attr_done |= 1ull << dev;
  }
  const long long xbytes = 4ll * h->n * 128;  // X's image: hi + lo of 128 right-hand sides
  if (M.num_tc_units > 0) {
    const int grid = std::min(M.num_sms, M.num_tc_units);
    k_mx_p1_tc<<<grid, kP1Threads, kP1Smem, s>>>(M.tc_units.p, M.num_tc_units, M.store.p, Xtc, M.tslot_tc.p, S, Tb,
                                                M.tc_err.p);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_mx_p1_tc", M.bytes_p1 + xbytes, s);
  }
  if (M.nmt_tc > 0) {
    k_mx_reduce_tc<<<(unsigned)((M.nmt_tc * 128 + 255) / 256), 256, 0, s>>>(M.mtiles_tc.p, M.nmt_tc, M.panels.p, S,
                                                                            M.tslot_tc.p, Tb);
    HM_LAUNCH_CHECK();
    if (km) km->mark("k_mx_reduce_tc", 4096ll * M.s_tiles_tc + 4096ll * M.nmt_tc, s);
  }
  if (M.p2_blocks > 0) {
    const int grid = std::min(M.num_sms, M.p2_blocks);
    k_mx_p2_tc<<<grid, kP2Threads, kP2Smem, s>>>(M.p2_blocks, M.p2_tile0, M.p2_tile0 + M.p2_tiles, M.p2_step_ptr.p,
                                                M.p2_steps.p, M.store.p, Tb, Xtc, M.tile_leaf.p, M.leaf_tile0.p,
                                                h->tree->offsets.p, Y, ldy, nr, M.tc_err.p);
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
