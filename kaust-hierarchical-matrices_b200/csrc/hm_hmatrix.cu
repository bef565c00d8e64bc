// hm_hmatrix.cu -- H-matrix construction by batched adaptive randomized
// approximation (ARA) on kernel entries generated from the points.
//
// Reference: createColumnMajorLRMatrix (src/constructTLRMatrix.cu:13-151)
// compresses leaf tiles with kblas_ara_batch and generateHMatrixFromStruct
// (src/constructHMatrixFromStruct.cu:13-103) recompresses coarser blocks from
// the leaf factors with lr_kblas_ara_batch, both from the un-vendored KBLAS
// fork.  The ARA they call is the blocked adaptive range finder of Halko,
// Martinsson & Tropp (2011, Alg. 4.2) as batched by Boukaram, Turkiyyah &
// Keyes (2019): draw a Gaussian sample block, project out the basis found so
// far, stop when the sample's norm says the residual is below the tolerance,
// otherwise orthonormalise it and append it; finally B = A^T Q, A ~ Q B^T.
//
// B200 design.  Every block of every level is compressed directly from the
// kernel function (no dense tiles in HBM, no leaf-TLR stage): each ARA pass is
// one batched "kernel block x tall-skinny" launch (k_kmm) whose tiles are
// generated on the fly from the tree-ordered FP32 coordinates, so the O(N^2)
// part never touches memory.  Orthogonalisation runs per block in one CTA
// (k_orth): block classical Gram-Schmidt applied twice against the basis, then
// a pivoted Cholesky-QR of the sample with two Cholesky-QR refinements, Gram
// matrices in FP64.  The kernel matrix is symmetric, so of each block pair
// (u, v) / (v, u) only the one with v > u is compressed; the mirror block uses
// the same factors exchanged.  Leaf blocks that do not reach the tolerance
// within the leaf rank cap (bucket/2 as in src/constructTLRMatrix.cu:14) are
// stored dense, as are the diagonal leaves.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <array>
#include <numeric>
#include <type_traits>

#include "hm_hmatrix.h"
#include "hm_mma.cuh"
#include "hm_structure.h"

namespace hm {

hm_status matvec_plan_build(hm_hmatrix h, int nrhs_cap, cudaStream_t stream);

namespace {

constexpr int kTR = 64;        // rows of a KMM tile
constexpr int kTC = 64;        // columns per KMM chunk
constexpr int kKmmThreads = 256;
constexpr int kOrthThreads = 256;
constexpr int kMaxCols = 256;  // max basis columns of one block (rank cap)
constexpr int kTruncMax = 128; // widest basis the SVD truncation handles (wider: kept as sampled)
constexpr int kColGroup = 128; // projection columns per sketch launch
constexpr int kMaxBs = 32;     // max sample block (the option)
// widest sample (basis + test columns) one orthogonalisation handles; the
// shared memory and per-thread arrays of k_orth scale with it (64 halves the
// CTAs per SM, measured slower while the sample stays at 32 columns)
template <typename W>
constexpr int max_bs() {
  return 32;
}

struct Prob {
  int r0, m, c0, n;
  int kmax;
  int level;
  int u, v;
  long long qoff, yoff, boff;  // workspace offsets (floats)
  double tscale2;              // (this block's tolerance / the build's)^2: 1, or the level schedule's
};

struct ProbState {
  double normA2;
  double est;
  int k;
  int active;
  int converged;
  int rounds;
  int r;      // rank after truncation (<= k)
  int rhi;    // mixed precision: columns [0, rhi) keep a BF16 low part
};

template <typename W>
struct KmmArgs {
  const Prob* probs;
  ProbState* st;
  const int2* items;  // (problem, tile)
  const float* pts;   // tree-ordered FP32 coordinates [d][npts]
  int npts, d;
  KernelParams kp;
  int mode;           // 0: Y = A Omega (bs columns); 1: B = A^T Q (k columns)
  int col0;           // projection: first basis column of this launch (128 per launch)
  int bs;
  uint32_t seed;
  int round;
  W* ws;              // workspace (Y, Q, B) in the ARA's working precision
};

// ---------------------------------------------------------------------------
// k_kmm: out(rows x s) = K(rows, cols) W(cols x s) for one 64-row tile.
// Thread t: row r = t % 64, q = t / 64 splits the s output columns into
// `nslab` slabs of 32 and the chunk columns into 4/nslab groups.  Kernel
// entries are FP32; products and sums are in the workspace type W (an FP32 x
// FP32 product is exact in FP64, so W = double gives FP64-accurate samples).
// ---------------------------------------------------------------------------
template <typename W>
__global__ void __launch_bounds__(kKmmThreads) k_kmm(KmmArgs<W> a) {
  extern __shared__ __align__(16) unsigned char kmm_raw[];
  W* Wsm = reinterpret_cast<W*>(kmm_raw);          // [kTC][kColGroup]
  float* Asm = reinterpret_cast<float*>(Wsm + kTC * kColGroup);  // [kTC][kTR]
  float* colc = Asm + kTC * kTR;                   // [d][kTC]
  double* red = reinterpret_cast<double*>(colc + kMaxDim * kTC);  // [kKmmThreads/32]

  const int2 it = a.items[blockIdx.x];
  const Prob P = a.probs[it.x];
  const ProbState S = a.st[it.x];
  if (a.mode == 0 && !S.active) return;
  const int col0 = a.mode ? a.col0 : 0;
  const int s = min(kColGroup, (a.mode == 0 ? a.bs : S.k) - col0);
  if (s <= 0) return;
  const int mr = a.mode ? P.n : P.m;        // rows of the operator
  const int nc = a.mode ? P.m : P.n;        // columns of the operator
  const int rbase = a.mode ? P.c0 : P.r0;
  const int cbase = a.mode ? P.r0 : P.c0;
  W* out = a.ws + (a.mode ? P.boff : P.yoff) + (size_t)col0 * mr;
  const W* Q = a.ws + P.qoff + (size_t)col0 * P.m;  // mode 1: W = Q (m x k, ld m)
  const int nslab = s <= 32 ? 1 : (s <= 64 ? 2 : 4);
  const int ncg = 4 / nslab;
  const int t = threadIdx.x, r = t & 63, q = t >> 6;
  const int slab = q % nslab, cg = q / nslab;
  const int row = it.y * kTR + r;
  const bool row_ok = row < mr;
  float rc[kMaxDim];
#pragma unroll
  for (int k = 0; k < kMaxDim; ++k)
    rc[k] = (k < a.d && row_ok) ? a.pts[(size_t)k * a.npts + rbase + row] : 0.f;
  W acc[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) acc[c] = W(0);
  double nrm = 0.0;
  const bool want_norm = a.mode == 0 && a.round == 0;
  const int wcols = nslab * 32;

  for (int c0 = 0; c0 < nc; c0 += kTC) {
    // column coordinates and the W chunk
    if (t < kTC) {
      int j = c0 + t;
      for (int k = 0; k < a.d; ++k) colc[k * kTC + t] = j < nc ? a.pts[(size_t)k * a.npts + cbase + j] : 0.f;
    }
    for (int e = t; e < kTC * wcols; e += kKmmThreads) {
      int jj = e % kTC, cc = e / kTC;
      int j = c0 + jj;
      W w = W(0);
      if (j < nc && cc < s) {
        if (a.mode == 0)
          w = (W)gauss_at(a.seed, (uint32_t)it.x, (uint32_t)j, (uint32_t)(a.round * kMaxBs + cc));
        else
          w = Q[(size_t)cc * P.m + j];
      }
      Wsm[jj * kColGroup + cc] = w;
    }
    __syncthreads();
    // kernel entries of this thread's row, columns q, q+4, ...
    for (int jj = q; jj < kTC; jj += 4) {
      float v = 0.f;
      if (row_ok && c0 + jj < nc) {
        float r2 = 0.f;
        for (int k = 0; k < a.d; ++k) {
          float df = rc[k] - colc[k * kTC + jj];
          r2 = fmaf(df, df, r2);
        }
        v = kernel_r2(a.kp, r2);
        if (want_norm) nrm += (double)v * (double)v;
      }
      Asm[jj * kTR + r] = v;
    }
    __syncthreads();
    for (int jj = cg; jj < kTC; jj += ncg) {
      W av = (W)Asm[jj * kTR + r];
      const W* w = Wsm + jj * kColGroup + slab * 32;
#pragma unroll
      for (int c = 0; c < 32; ++c) acc[c] = fma(av, w[c], acc[c]);
    }
    __syncthreads();
  }
  // reduce over column groups through shared memory (reuses Asm/Wsm)
  if (ncg > 1) {
    W* part = Wsm;  // [4][32][64] (reuses the W chunk)
    for (int c = 0; c < 32; ++c) part[(q * 32 + c) * kTR + r] = acc[c];
    __syncthreads();
    if (cg == 0) {
      for (int g = 1; g < ncg; ++g) {
        int qq = g * nslab + slab;
        for (int c = 0; c < 32; ++c) acc[c] += part[(qq * 32 + c) * kTR + r];
      }
    }
  }
  if (cg == 0 && row_ok) {
    const int ld = mr;
    for (int c = 0; c < 32; ++c) {
      int col = slab * 32 + c;
      if (col < s) out[(size_t)col * ld + row] = acc[c];
    }
  }
  if (want_norm) {
    for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
    __syncthreads();
    if ((t & 31) == 0) red[t >> 5] = nrm;
    __syncthreads();
    if (t == 0) {
      double tot = 0;
      for (int w = 0; w < kKmmThreads / 32; ++w) tot += red[w];
      atomicAdd(&a.st[it.x].normA2, tot);
    }
  }
}

// ---------------------------------------------------------------------------
// k_kmm_tc: the same product on the tensor cores (FP32 working precision).
// CTA = 4 warps = 64 operator rows, warp = 16 rows; each lane evaluates the
// eight kernel entries of its m16n8k16 A fragment in registers and splits
// them into BF16 hi + lo (relative error ~2^-17 of an entry).  Sample pass:
// W = a Gaussian table whose entries are BF16 numbers, 2 MMAs per tile.
// Projection pass: W = Q split hi + lo, 3 MMAs per tile (hi*hi, lo*hi, hi*lo).
// ---------------------------------------------------------------------------
// k_kmm_fast: the tensor-core sketch product specialised on the dimension
// (1-3), the kernel and its derivative.  Coordinates are pre-scaled so that
// each entry costs one hardware square root and one hardware exp2 (PTX
// sqrt.approx / ex2.approx, both within a few ulp of FP32), the row
// coordinates stay in registers, and the right-hand operand (the Gaussian
// table in sampling mode, the basis Q in projection mode) is read as
// prepacked BF16 pairs straight from L1/L2 instead of being restaged per chunk.
// ---------------------------------------------------------------------------
constexpr int kCC = 128;  // columns per coordinate chunk

struct KmmFastArgs {
  const Prob* probs;
  ProbState* st;
  const int2* items;
  const float* pts;
  int npts;
  float scale;   // coordinate scale (see kval)
  float dscale;  // derivative factor
  int deriv;     // entries of dK/dl instead of K
  int bs, round;
  // right-hand operand tables in fragment order: word (k-step, column tile,
  // lane (g,t)) holds the m16n8k16 B fragment {b0, b1} with
  // b0 = {W[16 ks + 2t][8 nt + g], W[16 ks + 2t + 1][..]}, b1 = rows + 8
  const uint2* om;          // sampling: the Gaussian table, om_nt column tiles
  int om_nt;
  const uint4* qt;          // projection: {hi b0, hi b1, lo b0, lo b1} of Q, per problem
  const long long* qpoff;   // per problem (batch index), 16-byte words
  int col0;                 // projection: first basis column of this launch
  float* ws;
};

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

constexpr float kLn2f = 0.6931471805599453f;

// r2: squared distance of the scaled coordinates.
//   KIND 0 (exp):    scale = log2(e)/l,         a = r log2(e)/l,  K = 2^-a
//   KIND 1 (Matern): scale = sqrt(3) log2(e)/l,  K = (1 + a ln2) 2^-a
//   KIND 2 (Gauss):  scale = sqrt(log2(e)/2)/l,  K = 2^-r2
// derivatives dK/dl: exp a ln2 K / l, Matern (a ln2)^2 2^-a / l,
// Gauss K q / l with q = r^2/l^2 = 2 ln2 r2.
template <int KIND, bool DERIV>
__device__ __forceinline__ float kval(float r2, float dscale) {
  if (KIND == 2) {
    const float v = ex2_approx(-r2);
    return DERIV ? v * r2 * dscale : v;
  }
  const float a = sqrt_approx(r2);
  const float e = ex2_approx(-a);
  if (KIND == 1) {
    const float al = a * kLn2f;
    return DERIV ? al * al * e * dscale : fmaf(a, kLn2f, 1.0f) * e;
  }
  return DERIV ? a * e * dscale : e;
}

template <int D, int KIND, int MODE, int NT>
__global__ void __launch_bounds__(128) k_kmm_fast(KmmFastArgs a) {
  __shared__ float colc[D][kCC];
  __shared__ double red[4];
  const int2 it = a.items[blockIdx.x];
  const Prob P = a.probs[it.x];
  const ProbState S = a.st[it.x];
  if (MODE == 0 && !S.active) return;
  const int col0 = MODE ? a.col0 : 0;
  const int s = (MODE == 0 ? a.bs : S.k) - col0;  // output columns of this launch
  if (s <= 0) return;
  const int mr = MODE ? P.n : P.m;
  const int nc = MODE ? P.m : P.n;
  const int rbase = MODE ? P.c0 : P.r0;
  const int cbase = MODE ? P.r0 : P.c0;
  const int mr_ld = mr;
  float* out = a.ws + (MODE ? P.boff : P.yoff) + (size_t)col0 * mr_ld;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int ra = it.y * kTR + warp * 16 + g, rb = ra + 8;
  const bool ra_ok = ra < mr, rb_ok = rb < mr;
  const bool deriv = a.deriv != 0;
  float rca[D], rcb[D];
#pragma unroll
  for (int k = 0; k < D; ++k) {
    rca[k] = ra_ok ? a.pts[(size_t)k * a.npts + rbase + ra] * a.scale : 0.f;
    rcb[k] = rb_ok ? a.pts[(size_t)k * a.npts + rbase + rb] * a.scale : 0.f;
  }
  const int ntiles = min(NT, (s + 7) >> 3);
  const int tnt = MODE ? (S.k + 7) >> 3 : a.om_nt;  // column tiles of the table
  const uint4* qt = MODE ? a.qt + a.qpoff[it.x] + (col0 >> 3) * 32 + lane : nullptr;
  const uint2* om = MODE ? nullptr : a.om + lane;
  float acc[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
  float nrm = 0.f;
  const bool want_norm = MODE == 0 && a.round == 0;
  // B fragments of k-step kg (16 columns of the block): one word per lane and column tile
  uint32_t bh[NT][2], bl[NT][2];
  auto load_b = [&](int kg) {
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      if (nt < ntiles) {
        if (MODE == 1) {
          const uint4 v = __ldg(qt + ((size_t)kg * tnt + nt) * 32);
          bh[nt][0] = v.x;
          bh[nt][1] = v.y;
          bl[nt][0] = v.z;
          bl[nt][1] = v.w;
        } else {
          const uint2 v = __ldg(om + ((size_t)kg * tnt + nt) * 32);
          bh[nt][0] = v.x;
          bh[nt][1] = v.y;
        }
      }
    }
  };
  const int nks = (nc + 15) >> 4;
  if (MODE == 0) load_b(0);
  for (int kg = 0; kg < nks; ++kg) {
    const int c0 = (kg * 16) / kCC * kCC;
    if (kg * 16 == c0) {  // first k-step of a coordinate chunk
      __syncthreads();
      for (int e = threadIdx.x; e < D * kCC; e += blockDim.x) {
        const int k = e / kCC, jj = e % kCC;
        colc[k][jj] = c0 + jj < nc ? a.pts[(size_t)k * a.npts + cbase + c0 + jj] * a.scale : 0.f;
      }
      __syncthreads();
    }
    uint32_t ch[NT][2];
    if (MODE == 1) {
      load_b(kg);  // issued before the entries are generated, used after (no second register set)
    } else {
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        ch[nt][0] = bh[nt][0];
        ch[nt][1] = bh[nt][1];
      }
      if (kg + 1 < nks) load_b(kg + 1);  // in flight while this k-step's entries are generated
    }
    const int cb = kg * 16 - c0 + 2 * t;  // chunk columns cb, cb+1, cb+8, cb+9
    float e[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = cb + (q & 1) + ((q >> 1) << 3);
      const bool cok = c0 + c < nc;
      float r2a = 0.f, r2b = 0.f;
#pragma unroll
      for (int k = 0; k < D; ++k) {
        const float cc = colc[k][c];
        const float da = rca[k] - cc, db = rcb[k] - cc;
        r2a = fmaf(da, da, r2a);
        r2b = fmaf(db, db, r2b);
      }
      const float va = deriv ? kval<KIND, true>(r2a, a.dscale) : kval<KIND, false>(r2a, a.dscale);
      const float vb = deriv ? kval<KIND, true>(r2b, a.dscale) : kval<KIND, false>(r2b, a.dscale);
      e[q] = (ra_ok && cok) ? va : 0.f;
      e[4 + q] = (rb_ok && cok) ? vb : 0.f;
    }
    if (want_norm) {
#pragma unroll
      for (int q = 0; q < 8; ++q) nrm = fmaf(e[q], e[q], nrm);
    }
    uint32_t ah[4], al[4];
    split_bf16x2(e[0], e[1], ah[0], al[0]);  // row g, cols cb, cb+1
    split_bf16x2(e[4], e[5], ah[1], al[1]);  // row g+8
    split_bf16x2(e[2], e[3], ah[2], al[2]);  // row g, cols cb+8, cb+9
    split_bf16x2(e[6], e[7], ah[3], al[3]);  // row g+8
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      if (nt < ntiles) {
        float d[4] = {0.f, 0.f, 0.f, 0.f};
        const uint32_t b0 = MODE == 1 ? bh[nt][0] : ch[nt][0], b1 = MODE == 1 ? bh[nt][1] : ch[nt][1];
        if (MODE == 1) mma_bf16(d, ah[0], ah[1], ah[2], ah[3], bl[nt][0], bl[nt][1]);
        mma_bf16(d, al[0], al[1], al[2], al[3], b0, b1);
        mma_bf16(d, ah[0], ah[1], ah[2], ah[3], b0, b1);
        add4(acc[nt], d);
      }
    }
  }
  const int ld = mr;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    if (nt < ntiles) {
      const int c = nt * 8 + 2 * t;
      if (ra_ok) {
        if (c < s) out[(size_t)c * ld + ra] = acc[nt][0];
        if (c + 1 < s) out[(size_t)(c + 1) * ld + ra] = acc[nt][1];
      }
      if (rb_ok) {
        if (c < s) out[(size_t)c * ld + rb] = acc[nt][2];
        if (c + 1 < s) out[(size_t)(c + 1) * ld + rb] = acc[nt][3];
      }
    }
  }
  if (want_norm) {
    double dn = nrm;
    for (int o = 16; o > 0; o >>= 1) dn += __shfl_xor_sync(0xffffffffu, dn, o);
    if (lane == 0) red[warp] = dn;
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&a.st[it.x].normA2, red[0] + red[1] + red[2] + red[3]);
  }
}

// Gaussian table of one sampling round in fragment order (see KmmFastArgs):
// W[j][c] is the BF16-rounded N(0,1) value for (round, j, c), zero for c >= bs.
__global__ void k_omega_pack(uint2* om, int ksteps, int bs, int nt_tot, uint32_t seed, int round) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)ksteps * nt_tot * 32;
       e += (long long)gridDim.x * blockDim.x) {
    const int lane = (int)(e & 31), g = lane >> 2, t = lane & 3;
    const long long w = e >> 5;
    const int nt = (int)(w % nt_tot), ks = (int)(w / nt_tot);
    const int c = nt * 8 + g, j = ks * 16 + 2 * t;
    float x[4] = {0.f, 0.f, 0.f, 0.f};
    if (c < bs) {
      const uint32_t st = 0x51ed270bu + round;
      x[0] = gauss_at(seed, st, (uint32_t)j, (uint32_t)c);
      x[1] = gauss_at(seed, st, (uint32_t)(j + 1), (uint32_t)c);
      x[2] = gauss_at(seed, st, (uint32_t)(j + 8), (uint32_t)c);
      x[3] = gauss_at(seed, st, (uint32_t)(j + 9), (uint32_t)c);
    }
    om[e] = make_uint2(pack_bf16(x[0], x[1]), pack_bf16(x[2], x[3]));
  }
}

// Q (m x k, column-major, ld m) of each problem in fragment order, hi and lo
// (see KmmFastArgs): k-steps over the rows padded to whole coordinate chunks,
// column tiles over k padded to 8.
__global__ void k_pack_q(const Prob* probs, const ProbState* st, const float* ws, const long long* qpoff,
                         uint4* qt) {
  const Prob P = probs[blockIdx.x];
  const int k = st[blockIdx.x].k;
  if (k <= 0) return;
  const int ntq = (k + 7) >> 3;
  const int ksteps = (P.m + kCC - 1) / kCC * (kCC / 16);
  const float* Q = ws + P.qoff;
  uint4* q = qt + qpoff[blockIdx.x];
  for (int e = threadIdx.x; e < ksteps * ntq * 32; e += blockDim.x) {
    const int lane = e & 31, g = lane >> 2, t = lane & 3;
    const int w = e >> 5;
    const int nt = w % ntq, ks = w / ntq;
    const int c = nt * 8 + g, i = ks * 16 + 2 * t;
    float x[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = i + (r & 1) + 8 * (r >> 1);
      x[r] = (c < k && row < P.m) ? Q[(size_t)c * P.m + row] : 0.f;
    }
    uint4 o;
    split_bf16x2(x[0], x[1], o.x, o.z);
    split_bf16x2(x[2], x[3], o.y, o.w);
    q[e] = o;
  }
}

// nt: right-hand column tiles the launch must cover (sample block / 8, or
// the largest basis of the batch / 8)
template <int D, int KIND>
void launch_kmm_fast3(int mode, int nt, unsigned grid, cudaStream_t s, const KmmFastArgs& a) {
  if (mode == 0) {
    if (nt <= 2)
      k_kmm_fast<D, KIND, 0, 2><<<grid, 128, 0, s>>>(a);
    else if (nt <= 4)
      k_kmm_fast<D, KIND, 0, 4><<<grid, 128, 0, s>>>(a);
    else
      k_kmm_fast<D, KIND, 0, 8><<<grid, 128, 0, s>>>(a);
  } else {
    if (nt <= 4)
      k_kmm_fast<D, KIND, 1, 4><<<grid, 128, 0, s>>>(a);
    else if (nt <= 8)
      k_kmm_fast<D, KIND, 1, 8><<<grid, 128, 0, s>>>(a);
    else
      k_kmm_fast<D, KIND, 1, kColGroup / 8><<<grid, 128, 0, s>>>(a);
  }
}
template <int D>
void launch_kmm_fast2(int kind, int mode, int nt, unsigned grid, cudaStream_t s, const KmmFastArgs& a) {
  if (kind == HM_KERNEL_GAUSS)
    launch_kmm_fast3<D, 2>(mode, nt, grid, s, a);
  else if (kind == HM_KERNEL_MATERN32)
    launch_kmm_fast3<D, 1>(mode, nt, grid, s, a);
  else
    launch_kmm_fast3<D, 0>(mode, nt, grid, s, a);
}
void launch_kmm_fast(int d, int kind, int mode, int nt, unsigned grid, cudaStream_t s, const KmmFastArgs& a) {
  if (d == 1)
    launch_kmm_fast2<1>(kind, mode, nt, grid, s, a);
  else if (d == 2)
    launch_kmm_fast2<2>(kind, mode, nt, grid, s, a);
  else
    launch_kmm_fast2<3>(kind, mode, nt, grid, s, a);
}

// ---------------------------------------------------------------------------
// per-block orthogonalisation of the new sample
// ---------------------------------------------------------------------------
template <typename W>
struct OrthArgs {
  const Prob* probs;
  ProbState* st;
  W* ws;
  int bs;          // sample columns of this round
  int bst;         // of which the last bst are test columns (0: none)
  double thresh2;  // stop when est <= thresh2 * normA2
  int round;
};

// C[j][c] = sum_i Q[i, j] Y[i, c]  (k x bs), result in shared Csm.  Each
// thread owns a TA x 4 tile of C (rows j = 8 * TA-blocks, columns c in fours),
// so that a staged value serves TA or 4 FMAs instead of one; TA grows with k
// so that the 256 threads stay busy.  Every output sums its products in the
// same order (rows of a 32-row chunk in turn, chunks in turn) for any TA.
template <typename W, int TA>
__device__ void block_qty_t(const W* Q, const W* Y, int m, int k, int bs, W* Csm, W* stage) {
  const int t = threadIdx.x;
  const int jg = t >> 3, cg = t & 7;  // 32 row groups of TA x 8 column groups of 4
  W acc[TA][4];
#pragma unroll
  for (int a = 0; a < TA; ++a) acc[a][0] = acc[a][1] = acc[a][2] = acc[a][3] = W(0);
  W* Qs = stage;                  // [kMaxCols][33]
  W* Ys = stage + kMaxCols * 33;  // [max_bs][33]
  const bool act = jg * TA < k && cg * 4 < bs;
  for (int i0 = 0; i0 < m; i0 += 32) {
    for (int e = t; e < 32 * k; e += kOrthThreads) {
      int ii = e & 31, j = e >> 5;
      Qs[j * 33 + ii] = (i0 + ii < m) ? Q[(size_t)j * m + i0 + ii] : W(0);
    }
    for (int e = t; e < 32 * bs; e += kOrthThreads) {
      int ii = e & 31, c = e >> 5;
      Ys[c * 33 + ii] = (i0 + ii < m) ? Y[(size_t)c * m + i0 + ii] : W(0);
    }
    __syncthreads();
    if (act) {
      for (int ii = 0; ii < 32; ++ii) {
        W q[TA], y[4];
#pragma unroll
        for (int a = 0; a < TA; ++a) q[a] = Qs[(jg * TA + a) * 33 + ii];  // rows j >= k: never stored
#pragma unroll
        for (int b = 0; b < 4; ++b) y[b] = Ys[(cg * 4 + b) * 33 + ii];
#pragma unroll
        for (int a = 0; a < TA; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = fma(q[a], y[b], acc[a][b]);
      }
    }
    __syncthreads();
  }
  if (act) {
#pragma unroll
    for (int a = 0; a < TA; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int j = jg * TA + a, c = cg * 4 + b;
        if (j < k && c < bs) Csm[j * bs + c] = acc[a][b];
      }
  }
  __syncthreads();
}

template <typename W>
__device__ void block_qty(const W* Q, const W* Y, int m, int k, int bs, W* Csm, W* stage) {
  if (k <= 32)
    block_qty_t<W, 1>(Q, Y, m, k, bs, Csm, stage);
  else if (k <= 64)
    block_qty_t<W, 2>(Q, Y, m, k, bs, Csm, stage);
  else if (k <= 128)
    block_qty_t<W, 4>(Q, Y, m, k, bs, Csm, stage);
  else
    block_qty_t<W, 8>(Q, Y, m, k, bs, Csm, stage);
}

// Y -= Q C
template <typename W>
__device__ void block_update(const W* Q, W* Y, int m, int k, int bs, const W* Csm) {
  for (int i = threadIdx.x; i < m; i += kOrthThreads) {
    W y[max_bs<W>()];
    for (int c = 0; c < bs; ++c) y[c] = Y[(size_t)c * m + i];
    for (int j = 0; j < k; ++j) {
      W qv = Q[(size_t)j * m + i];
      for (int c = 0; c < bs; ++c) y[c] = fma(-qv, Csm[j * bs + c], y[c]);
    }
    for (int c = 0; c < bs; ++c) Y[(size_t)c * m + i] = y[c];
  }
  __syncthreads();
}

// G = Y^T Y in FP64 (cols x cols), into shared Gs.  Each thread owns a 2 x 2
// tile of the upper triangle (the lower one is its mirror: a product of two
// values is the same in either order), so a staged value serves two
// products; every entry sums its products in row order.
template <typename W>
__device__ void gram64(const W* Y, int m, int cols, double* Gs, W* stage) {
  static_assert(max_bs<W>() <= 32, "2 x 2 tiles of 16 x 16 threads cover 32 columns");
  const int t = threadIdx.x;
  const int ta = t >> 4, tb = t & 15;  // rows 2 ta, 2 ta + 1; columns 2 tb, 2 tb + 1
  const bool act = ta <= tb && 2 * tb < cols;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  W* Ys = stage;  // [max_bs][33]
  for (int i0 = 0; i0 < m; i0 += 32) {
    for (int e = t; e < 32 * cols; e += kOrthThreads) {
      int ii = e & 31, c = e >> 5;
      Ys[c * 33 + ii] = (i0 + ii < m) ? Y[(size_t)c * m + i0 + ii] : W(0);
    }
    __syncthreads();
    if (act) {
      for (int ii = 0; ii < 32; ++ii) {
        const double y0 = (double)Ys[(2 * ta) * 33 + ii], y1 = (double)Ys[(2 * ta + 1) * 33 + ii];
        const double z0 = (double)Ys[(2 * tb) * 33 + ii], z1 = (double)Ys[(2 * tb + 1) * 33 + ii];
        acc[0][0] += y0 * z0;
        acc[0][1] += y0 * z1;
        acc[1][0] += y1 * z0;
        acc[1][1] += y1 * z1;
      }
    }
    __syncthreads();
  }
  if (act) {
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int a = 2 * ta + u, b = 2 * tb + v;
        if (a < cols && b < cols) {
          Gs[a * cols + b] = acc[u][v];
          Gs[b * cols + a] = acc[u][v];
        }
      }
  }
  __syncthreads();
}

// Cholesky of the leading principal part of G (cols x cols, row-major), in
// place into its lower triangle, with symmetric pivoting when `pivot`; stops at
// the first pivot <= tau.  perm receives the column order.  Returns the rank.
// Runs on thread 0 (cols <= 32).
__device__ int chol_pivoted(double* G, int cols, int* perm, bool pivot, double tau) {
  for (int i = 0; i < cols; ++i) perm[i] = i;
  int rank = 0;
  for (int j = 0; j < cols; ++j) {
    int p = j;
    if (pivot) {
      for (int i = j + 1; i < cols; ++i)
        if (G[i * cols + i] > G[p * cols + p]) p = i;
    }
    if (!(G[p * cols + p] > tau)) break;
    if (p != j) {
      // symmetric swap of rows/cols j and p
      for (int c = 0; c < cols; ++c) {
        double x = G[j * cols + c];
        G[j * cols + c] = G[p * cols + c];
        G[p * cols + c] = x;
      }
      for (int r = 0; r < cols; ++r) {
        double x = G[r * cols + j];
        G[r * cols + j] = G[r * cols + p];
        G[r * cols + p] = x;
      }
      int x = perm[j];
      perm[j] = perm[p];
      perm[p] = x;
    }
    double d = sqrt(G[j * cols + j]);
    G[j * cols + j] = d;
    for (int i = j + 1; i < cols; ++i) G[i * cols + j] /= d;
    for (int i = j + 1; i < cols; ++i)
      for (int c = j + 1; c <= i; ++c) {
        G[i * cols + c] -= G[i * cols + j] * G[c * cols + j];
        G[c * cols + i] = G[i * cols + c];
      }
    rank = j + 1;
  }
  return rank;
}

// Y[:, 0:r] <- Y[:, perm[0:r]] L^{-T}  (row by row, in place)
template <typename W>
__device__ void apply_linv(W* Y, int m, int cols, const double* L, const int* perm, int r) {
  for (int i = threadIdx.x; i < m; i += kOrthThreads) {
    W y[max_bs<W>()];
    for (int c = 0; c < cols; ++c) y[c] = Y[(size_t)c * m + i];
    double x[max_bs<W>()];
    for (int a = 0; a < r; ++a) {
      double v = y[perm[a]];
      for (int b = 0; b < a; ++b) v -= L[a * cols + b] * x[b];
      x[a] = v / L[a * cols + a];
    }
    for (int a = 0; a < r; ++a) Y[(size_t)a * m + i] = (W)x[a];
  }
  __syncthreads();
}

// Orthonormalises the `cols` columns of Y (already projected against Q[0..k))
// in place: pivoted Cholesky-QR, then two Cholesky-QR refinements; R^{-1} of
// an ill-conditioned sample magnifies whatever the Gram-Schmidt left along
// the old basis, so after the first refinement the block is projected against
// Q once more.  Returns the rank r; Y[0..r) is the new orthonormal block.
template <typename W>
__device__ int cholqr_block(const W* Q, int k, W* Y, int m, int cols, double* Gs, int* perm, int* rank_sh,
                            W* Csm, W* stage) {
  gram64(Y, m, cols, Gs, stage);
  if (threadIdx.x == 0) {
    double tr = 0;
    for (int c = 0; c < cols; ++c) tr += Gs[c * cols + c];
    // columns whose norm is below FP32 resolution of the sample are noise
    *rank_sh = chol_pivoted(Gs, cols, perm, true, 1e-10 * tr);
  }
  __syncthreads();
  int r = *rank_sh;
  if (r == 0) return 0;
  apply_linv(Y, m, cols, Gs, perm, r);
  for (int pass = 0; pass < 2 && r > 0; ++pass) {
    if (pass == 1 && k > 0) {
      block_qty(Q, Y, m, k, r, Csm, stage);
      block_update(Q, Y, m, k, r, Csm);
    }
    const int rg = r;  // dimension (and row stride) of this Gram matrix
    gram64(Y, m, rg, Gs, stage);
    if (threadIdx.x == 0) *rank_sh = chol_pivoted(Gs, rg, perm, pass == 1, pass == 1 ? 1e-12 * rg : 0.0);
    __syncthreads();
    r = *rank_sh;  // a refinement that loses rank keeps the leading columns
    if (r > 0) apply_linv(Y, m, rg, Gs, perm, r);
  }
  return r;
}

template <typename W>
__device__ double trace_gram(const W* Y, int m, int cols, double* Gs, W* stage) {
  gram64(Y, m, cols, Gs, stage);
  double tr = 0;
  for (int c = 0; c < cols; ++c) tr += Gs[c * cols + c];
  return tr;
}

// One ARA round of one block.  The sample Y (m x bs) holds bs - bst basis
// columns and bst test columns (bst = 0: every column is a basis column and
// the estimate comes from the whole sample, as in the reference's ARA).
//  1. the whole sample is projected against Q (classical Gram-Schmidt, twice);
//  2. the test columns' projected norm estimates the residual
//     ||(I - QQ^T) A||_F^2 ~ ||Y_t'||^2 / bst: below the threshold, done;
//  3. the basis columns are orthonormalised and appended to Q;
//  4. the test columns, projected against the new columns as well, estimate
//     the residual left by the grown basis: below the threshold, done in this
//     round (no extra pass); otherwise they are a sample of that residual and
//     are orthonormalised and appended too.
template <typename W>
__global__ void __launch_bounds__(kOrthThreads) k_orth(OrthArgs<W> a) {
  constexpr int MB = max_bs<W>();
  extern __shared__ __align__(16) unsigned char osm[];
  double* Gs = reinterpret_cast<double*>(osm);         // [MB*MB]
  W* Csm = reinterpret_cast<W*>(Gs + MB * MB);         // [kMaxCols*MB]
  W* stage = Csm + kMaxCols * MB;                      // (kMaxCols+MB)*33
  __shared__ int perm[MB];
  __shared__ int rank_sh;
  __shared__ int decision;  // 0 continue, 1 converged, 2 cap reached

  const int p = blockIdx.x;
  ProbState S = a.st[p];
  if (!S.active) return;
  const Prob P = a.probs[p];
  const int m = P.m, bs = a.bs, bst = a.bst, bsb = bs - bst;
  W* Q = a.ws + P.qoff;
  W* Y = a.ws + P.yoff;
  W* Yt = Y + (size_t)bsb * m;
  int k = S.k;
  for (int pass = 0; pass < 2 && k > 0; ++pass) {
    block_qty(Q, Y, m, k, bs, Csm, stage);
    block_update(Q, Y, m, k, bs, Csm);
  }
  {
    const int ne = bst > 0 ? bst : bs;
    const double tr = trace_gram(bst > 0 ? Yt : Y, m, ne, Gs, stage);
    if (threadIdx.x == 0) {
      const double est = tr / ne;
      S.est = est;
      S.rounds += 1;
      if (est <= a.thresh2 * P.tscale2 * S.normA2 || S.normA2 == 0.0) decision = 1;
      else if (k + bsb > P.kmax) decision = 2;
      else decision = 0;
    }
    __syncthreads();
  }
  if (decision != 0) {
    if (threadIdx.x == 0) {
      S.active = 0;
      S.converged = decision == 1;
      a.st[p] = S;
    }
    return;
  }
  int r = cholqr_block(Q, k, Y, m, bsb, Gs, perm, &rank_sh, Csm, stage);
  for (int c = 0; c < r; ++c)
    for (int i = threadIdx.x; i < m; i += kOrthThreads) Q[(size_t)(k + c) * m + i] = Y[(size_t)c * m + i];
  __syncthreads();
  k += r;
  bool conv = false;
  if (bst > 0) {
    if (r > 0) {
      const W* Qn = Q + (size_t)(k - r) * m;
      for (int pass = 0; pass < 2; ++pass) {
        block_qty(Qn, Yt, m, r, bst, Csm, stage);
        block_update(Qn, Yt, m, r, bst, Csm);
      }
    }
    const double tr = trace_gram(Yt, m, bst, Gs, stage);
    if (threadIdx.x == 0) S.est = tr / bst;
    conv = tr / bst <= a.thresh2 * P.tscale2 * S.normA2;
    if (!conv && k < P.kmax) {
      int rt = cholqr_block(Q, k, Yt, m, bst, Gs, perm, &rank_sh, Csm, stage);
      rt = min(rt, P.kmax - k);
      for (int c = 0; c < rt; ++c)
        for (int i = threadIdx.x; i < m; i += kOrthThreads) Q[(size_t)(k + c) * m + i] = Yt[(size_t)c * m + i];
      __syncthreads();
      k += rt;
    }
  } else {
    conv = r == 0;
  }
  if (threadIdx.x == 0) {
    S.k = k;
    if (conv) {
      S.active = 0;
      S.converged = 1;
    }
    a.st[p] = S;
  }
}

// ---------------------------------------------------------------------------
// truncation: A ~ Q B^T with B = A^T Q; eig(B^T B) = W diag(lambda) W^T gives
// the singular values of A's approximation, sqrt(lambda), and
// A ~ (Q W_r)(B W_r)^T with the smallest r whose discarded sum of lambda fits
// the tolerance left after the sampling residual.  Columns come out in
// decreasing singular value, U = Q W_r orthonormal, |V_j| = sigma_j.
// ---------------------------------------------------------------------------
constexpr int kGramThreads = 256;

// G = B^T B (k x k, FP64) into global memory at goff, 8x8 register tiles
template <typename W>
__global__ void __launch_bounds__(kGramThreads) k_gram_big(const Prob* probs, const ProbState* st, const W* ws,
                                                           const long long* goff, double* G) {
  __shared__ double Bs[16][kMaxCols + 1];
  const int p = blockIdx.x;
  const int k = st[p].k;
  if (k <= 1 || k > kTruncMax) return;  // wider bases are kept as sampled
  const Prob P = probs[p];
  const W* B = ws + P.boff;
  const int nt = (k + 7) / 8;
  const int t = threadIdx.x;
  const int ti = t / 16, tj = t % 16;  // tile (ti, tj) of up to 16 x 16 tiles
  const bool active = ti < nt && tj < nt && ti <= tj;
  double acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = 0.0;
  for (int i0 = 0; i0 < P.n; i0 += 16) {
    for (int e = t; e < 16 * k; e += kGramThreads) {
      int ii = e % 16, j = e / 16;
      Bs[ii][j] = (i0 + ii < P.n) ? (double)B[(size_t)j * P.n + i0 + ii] : 0.0;
    }
    __syncthreads();
    if (active) {
      for (int ii = 0; ii < 16; ++ii) {
        double x[8], y[8];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
          int ja = ti * 8 + a, jb = tj * 8 + a;
          x[a] = ja < k ? Bs[ii][ja] : 0.0;
          y[a] = jb < k ? Bs[ii][jb] : 0.0;
        }
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
          for (int b = 0; b < 8; ++b) acc[a][b] = fma(x[a], y[b], acc[a][b]);
      }
    }
    __syncthreads();
  }
  if (active) {
    double* g = G + goff[p];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        int ja = ti * 8 + a, jb = tj * 8 + b;
        if (ja < k && jb < k) {
          g[ja * k + jb] = acc[a][b];
          g[jb * k + ja] = acc[a][b];
        }
      }
  }
}

// Parallel cyclic Jacobi on G (k x k) in shared memory; the rotations are
// accumulated into Wm (FP32).  Writes the truncated rank to st[p].r and the
// leading r eigenvectors (columns in decreasing eigenvalue) to Wr (k x r, at
// the same offset as G).
__global__ void __launch_bounds__(kGramThreads) k_jacobi(const Prob* probs, ProbState* st, const long long* goff,
                                                         const double* Gin, float* Wr, double tol2,
                                                         double rbudget) {
  extern __shared__ __align__(16) unsigned char jsm[];
  const int p = blockIdx.x;
  ProbState S = st[p];
  const int k = S.k;
  const int t = threadIdx.x;
  if (k <= 1 || k > kTruncMax) {
    // no truncation: W = identity, every column keeps its low part
    for (int e = t; e < k * k; e += kGramThreads) Wr[goff[p] + e] = (e / k == e % k) ? 1.f : 0.f;
    if (t == 0) {
      st[p].r = k;
      st[p].rhi = k;
    }
    return;
  }
  const int kp = (k + 1) & ~1;  // even size: an odd k gets a zero row and column
  double* G = reinterpret_cast<double*>(jsm);              // [kp][kp]
  float* Wm = reinterpret_cast<float*>(G + kp * kp);        // [kp][kp]
  double* cs = reinterpret_cast<double*>(Wm + kp * kp);     // [kp/2][2]
  int* pr = reinterpret_cast<int*>(cs + kp);                // [kp] tournament positions
  int* order = pr + kp;                                     // [kp]
  __shared__ double off_sh;
  const double* g = Gin + goff[p];
  for (int e = t; e < kp * kp; e += kGramThreads) {
    int a = e / kp, b = e % kp;
    G[e] = (a < k && b < k) ? g[a * k + b] : 0.0;
    Wm[e] = a == b ? 1.f : 0.f;
  }
  for (int i = t; i < kp; i += kGramThreads) pr[i] = i;
  __syncthreads();
  double scale = 0;
  for (int i = 0; i < k; ++i) scale += G[i * kp + i];
  const int npairs = kp / 2;
  for (int sweep = 0; sweep < 12; ++sweep) {
    if (t == 0) off_sh = 0;
    __syncthreads();
    for (int step = 0; step < kp - 1; ++step) {
      // pair i: (pr[i], pr[kp-1-i]); angles
      for (int i = t; i < npairs; i += kGramThreads) {
        int a = pr[i], b = pr[kp - 1 - i];
        int pp = min(a, b), qq = max(a, b);
        double apq = G[pp * kp + qq];
        double c = 1, s = 0;
        if (fabs(apq) > 1e-300 && fabs(apq) > 1e-18 * scale) {
          double th = (G[qq * kp + qq] - G[pp * kp + pp]) / (2 * apq);
          double tt = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
          c = 1.0 / sqrt(tt * tt + 1.0);
          s = tt * c;
          atomicAdd(&off_sh, apq * apq);
        }
        cs[2 * i] = c;
        cs[2 * i + 1] = s;
      }
      __syncthreads();
      // rows
      for (int e = t; e < npairs * kp; e += kGramThreads) {
        int i = e / kp, j = e % kp;
        int a = pr[i], b = pr[kp - 1 - i];
        int pp = min(a, b), qq = max(a, b);
        double c = cs[2 * i], s = cs[2 * i + 1];
        double gp = G[pp * kp + j], gq = G[qq * kp + j];
        G[pp * kp + j] = c * gp - s * gq;
        G[qq * kp + j] = s * gp + c * gq;
      }
      __syncthreads();
      // columns, and the accumulated rotation
      for (int e = t; e < npairs * kp; e += kGramThreads) {
        int i = e / kp, j = e % kp;
        int a = pr[i], b = pr[kp - 1 - i];
        int pp = min(a, b), qq = max(a, b);
        double c = cs[2 * i], s = cs[2 * i + 1];
        double gp = G[j * kp + pp], gq = G[j * kp + qq];
        G[j * kp + pp] = c * gp - s * gq;
        G[j * kp + qq] = s * gp + c * gq;
        float wp = Wm[j * kp + pp], wq = Wm[j * kp + qq];
        Wm[j * kp + pp] = (float)(c * wp - s * wq);
        Wm[j * kp + qq] = (float)(s * wp + c * wq);
      }
      __syncthreads();
      // next tournament round: keep position 0, rotate the rest
      if (t == 0) {
        int last = pr[kp - 1];
        for (int i = kp - 1; i > 1; --i) pr[i] = pr[i - 1];
        pr[1] = last;
      }
      __syncthreads();
    }
    if (off_sh <= 1e-26 * scale * scale) break;
    __syncthreads();
  }
  // order by decreasing eigenvalue (rank by counting), then the rank
  for (int i = t; i < k; i += kGramThreads) {
    double li = G[i * kp + i];
    int rk = 0;
    for (int j = 0; j < k; ++j) {
      double lj = G[j * kp + j];
      rk += (lj > li) || (lj == li && j < i);
    }
    order[rk] = i;
  }
  __syncthreads();
  __shared__ int r_sh;
  if (t == 0) {
    // discard the smallest eigenvalues while their sum fits the budget
    const double ts2 = probs[p].tscale2;
    double budget = tol2 * ts2 * S.normA2 - S.est;
    double tail = 0;
    int r = k;
    if (S.converged && budget > 0) {
      while (r > 1) {
        double l = fmax(G[order[r - 1] * kp + order[r - 1]], 0.0);
        if (tail + l > budget) break;
        tail += l;
        --r;
      }
    }
    r_sh = r;
    st[p].r = r;
    // Mixed precision: column j of U V^T carries |u_j||v_j| = sigma_j; rounding
    // both to BF16 perturbs it by at most ~2 * 2^-9 sigma_j.  The trailing
    // columns whose rounding error fits rbudget keep only their BF16 high part.
    int rhi = r;
    if (rbudget > 0) {
      double rt = 0;
      const double c = 2.0 * 0x1p-18;  // (2^-9)^2 for each of u_j and v_j
      while (rhi > 0) {
        double l = fmax(G[order[rhi - 1] * kp + order[rhi - 1]], 0.0);
        if (rt + c * l > rbudget * ts2 * S.normA2) break;
        rt += c * l;
        --rhi;
      }
    }
    st[p].rhi = rhi;
  }
  __syncthreads();
  const int r = r_sh;
  float* w = Wr + goff[p];
  for (int e = t; e < k * r; e += kGramThreads) {
    int a = e % k, c = e / k;
    w[c * k + a] = Wm[a * kp + order[c]];  // column c: eigenvector order[c]
  }
}

// U = Q W_r (m x r), V = B W_r (n x r), FP32
template <typename W>
__global__ void k_pack_trunc(const Prob* probs, const ProbState* st, const W* ws, const long long* goff,
                             const float* Wr, const long long* dst_u, const long long* dst_v, float* dst) {
  const int p = blockIdx.x;
  const int k = st[p].k, r = st[p].r;
  if (dst_u[p] < 0 || r <= 0) return;
  const Prob P = probs[p];
  if (k > kTruncMax) {  // kept as sampled (W = I): U = Q, V = B, a copy
    for (int side = 0; side < 2; ++side) {
      const size_t cnt = (size_t)(side ? P.n : P.m) * r;
      const W* src = ws + (side ? P.boff : P.qoff);
      float* out = dst + (side ? dst_v[p] : dst_u[p]);
      for (size_t e = threadIdx.x; e < cnt; e += blockDim.x) out[e] = (float)src[e];
    }
    return;
  }
  const float* w = Wr + goff[p];
  __shared__ float ws_sh[kMaxCols * 32];
  const int rc = min(r, 32);
  for (int c0 = 0; c0 < r; c0 += 32) {
    const int nc = min(32, r - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < k * nc; e += blockDim.x) ws_sh[e] = w[(size_t)(c0 + e / k) * k + e % k];
    __syncthreads();
    for (int side = 0; side < 2; ++side) {
      const int rows = side ? P.n : P.m;
      const W* src = ws + (side ? P.boff : P.qoff);
      float* out = dst + (side ? dst_v[p] : dst_u[p]);
      for (int i = threadIdx.x; i < rows; i += blockDim.x) {
        float acc[32];
        for (int c = 0; c < nc; ++c) acc[c] = 0.f;
        for (int a = 0; a < k; ++a) {
          float x = (float)src[(size_t)a * rows + i];
          for (int c = 0; c < nc; ++c) acc[c] = fmaf(x, ws_sh[c * k + a], acc[c]);
        }
        for (int c = 0; c < nc; ++c) out[(size_t)(c0 + c) * rows + i] = acc[c];
      }
    }
  }
  (void)rc;
}

size_t jacobi_smem(int kmax) {
  int kp = (kmax + 1) & ~1;
  return sizeof(double) * kp * kp + sizeof(float) * kp * kp + sizeof(double) * kp + sizeof(int) * 2 * kp + 64;
}


// ---------------------------------------------------------------------------
// packing and dense blocks
// ---------------------------------------------------------------------------
struct PackItem {
  long long src_q, src_b;  // workspace offsets
  long long dst_u, dst_v;  // offsets in the chunk
  int m, n, k;
};

template <typename W>
__global__ void k_pack(const PackItem* items, int nitems, const W* ws, float* dst) {
  const PackItem it = items[blockIdx.x];
  size_t nu = (size_t)it.m * it.k, nv = (size_t)it.n * it.k;
  for (size_t e = threadIdx.x; e < nu; e += blockDim.x) dst[it.dst_u + e] = (float)ws[it.src_q + e];
  for (size_t e = threadIdx.x; e < nv; e += blockDim.x) dst[it.dst_v + e] = (float)ws[it.src_b + e];
}

struct DenseItem {
  int r0, m, c0, n;
  long long off;
};

__global__ void k_dense_gen(const DenseItem* items, const float* pts, int npts, int d,
                            KernelParams kp, float* dst) {
  const DenseItem it = items[blockIdx.x];
  size_t tot = (size_t)it.m * it.n;
  for (size_t e = threadIdx.x; e < tot; e += blockDim.x) {
    int i = (int)(e % it.m), j = (int)(e / it.m);
    int gi = it.r0 + i, gj = it.c0 + j;
    float r2 = 0.f;
    for (int k = 0; k < d; ++k) {
      float df = pts[(size_t)k * npts + gi] - pts[(size_t)k * npts + gj];
      r2 = fmaf(df, df, r2);
    }
    float v = kernel_r2(kp, r2);
    if (gi == gj && !kp.deriv) v += kp.nugget;
    dst[it.off + e] = v;
  }
}

template <typename W>
size_t kmm_smem() {
  return sizeof(W) * (kTC * kColGroup) + sizeof(float) * (kTC * kTR + kMaxDim * kTC) +
         sizeof(double) * (kKmmThreads / 32);
}

template <typename W>
size_t orth_smem() {
  constexpr int MB = max_bs<W>();
  return sizeof(double) * MB * MB + sizeof(W) * kMaxCols * MB + sizeof(W) * (kMaxCols + MB) * 33;
}

}  // namespace

// leaf_lo, leaf_hi: the block-row shard, leaves [leaf_lo, leaf_hi) (all
// leaves for a whole matrix).  A shard compresses only the pairs whose row or
// column cluster overlaps its rows, and only its own diagonal leaves.
hm_status hmatrix_build(hm_kdtree t, hm_structure s, const double* d_points, const hm_build_opts* o,
                        cudaStream_t stream, hm_hmatrix* out, int leaf_lo, int leaf_hi) {
  if (!out) return fail(HM_ERR_INVALID, "hm_hmatrix_build: out is NULL");
  *out = nullptr;
  if (!t || !s || !o) return fail(HM_ERR_INVALID, "hm_hmatrix_build: null argument");
  if (s->tree != t) return fail(HM_ERR_INVALID, "hm_hmatrix_build: structure was built on another tree");
  if (leaf_hi < 0) leaf_hi = 1 << t->depth;
  if (leaf_lo < 0 || leaf_lo >= leaf_hi || leaf_hi > (1 << t->depth))
    return fail(HM_ERR_INVALID, "hm_hmatrix_build_rows: need 0 <= leaf_begin < leaf_end <= 2^depth");
  (void)d_points;  // the tree keeps its own tree-ordered copy of the points
  hm_build_opts opt = *o;
  if (opt.kernel < 0 || opt.kernel > 2) return fail(HM_ERR_INVALID, "hm_hmatrix_build: unknown kernel");
  if (!(opt.ell > 0) || !(opt.tol > 0) || opt.tol >= 1)
    return fail(HM_ERR_INVALID, "hm_hmatrix_build: need ell > 0 and 0 < tol < 1");
  if (opt.sample_block <= 0) opt.sample_block = 16;
  if (opt.sample_block > kMaxBs) return fail(HM_ERR_UNSUPPORTED, "hm_hmatrix_build: sample_block > 32");
  if (opt.leaf_max_rank <= 0) opt.leaf_max_rank = std::max(1, t->bucket / 2);
  if (opt.max_rank <= 0) opt.max_rank = 64;
  const int bs = opt.sample_block;
  if (opt.max_rank > kMaxCols || opt.leaf_max_rank > kMaxCols)
    return fail(HM_ERR_UNSUPPORTED, "hm_hmatrix_build: rank caps must be <= 256");
  if (opt.level_schedule != 0 && opt.level_schedule != 1)
    return fail(HM_ERR_INVALID, "hm_hmatrix_build: level_schedule must be 0 or 1");

  cudaEvent_t ev0, ev1;
  HM_CUDA(cudaEventCreate(&ev0));
  HM_CUDA(cudaEventCreate(&ev1));
  HM_CUDA(cudaEventRecord(ev0, stream));

  auto* h = new hm_hmatrix_s();
  auto cleanup = [&](hm_status st) {
    delete h;
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    return st;
  };
  h->tree = t;
  h->structure = s;
  h->n = t->n;
  h->d = t->d;
  h->depth = t->depth;
  h->opts = opt;
  h->leaf_lo = leaf_lo;
  h->leaf_hi = leaf_hi;
  h->kp.kind = opt.kernel;
  h->kp.deriv = opt.derivative ? 1 : 0;
  h->kp.ell = (float)opt.ell;
  h->kp.inv_ell = (float)(1.0 / opt.ell);
  h->kp.nugget = (float)opt.nugget;
  const int depth = t->depth;
  const std::vector<int>& lo = t->h_offsets;
  auto coff = [&](int level, int c) { return lo[(size_t)c << (depth - level)]; };
  // Rank cap and tolerance of a level-l block.  Uniform: the leaf cap at the
  // leaf level, max_rank above it, tol everywhere.  The reference's schedule
  // (level_schedule = 1): the tolerance doubles at each level above the
  // leaves (src/constructHMatrixFromStruct.cu:31,54: tol 2^(depth - l) at
  // level l) and the cap is bucket 2^i, divided by 4 beyond i = 5, with
  // i = depth - 1 - l (generateMaxRanks, src/helperFunctions.cu:67-74),
  // within this build's largest basis.
  auto level_cap = [&](int l) {
    if (l == depth) return opt.leaf_max_rank;
    if (opt.level_schedule != 1) return opt.max_rank;
    const int i = depth - 1 - l;
    long long c = (long long)t->bucket << std::min(i, 20);
    if (i > 5) c /= 4;
    return (int)std::min<long long>(c, kMaxCols);
  };
  auto level_tscale2 = [&](int l) {
    if (opt.level_schedule != 1 || l >= depth) return 1.0;
    const double f = std::ldexp(1.0, depth - l);
    return f * f;
  };
  // rows of the shard; a pair is needed when its rows or its columns overlap them
  const int row_lo = lo[leaf_lo], row_hi = lo[leaf_hi];
  auto needed = [&](int r0, int m, int c0, int n) {
    return (r0 < row_hi && r0 + m > row_lo) || (c0 < row_hi && c0 + n > row_lo);
  };

  PhaseTrace tr("build");
  // ---- the problems: stored pairs (row cluster v > column cluster u) ------
  std::vector<uint32_t> tiles(std::max<long long>(s->start[depth], 1));
  if (s->start[depth] > 0)
    HM_CUDA(cudaMemcpy(tiles.data(), s->tiles.p, 4 * (size_t)s->start[depth], cudaMemcpyDeviceToHost));
  std::vector<Prob> probs;
  for (int l = 1; l <= depth; ++l) {
    for (long long i = s->start[l - 1]; i < s->start[l]; ++i) {
      uint32_t z = tiles[i];
      int u = (int)compact16(z), v = (int)compact16(z >> 1);
      if (v <= u) continue;
      Prob P{};
      P.level = l;
      P.u = u;
      P.v = v;
      P.r0 = coff(l, v);
      P.m = coff(l, v + 1) - P.r0;
      P.c0 = coff(l, u);
      P.n = coff(l, u + 1) - P.c0;
      P.kmax = std::min(level_cap(l), std::min(P.m, P.n));
      P.tscale2 = level_tscale2(l);
      if (!needed(P.r0, P.m, P.c0, P.n)) continue;
      probs.push_back(P);
    }
  }
  const long long nprob0 = (long long)probs.size();

  tr.mark("problems", stream, -1, 0);
  // ---- batches bounded by the workspace budget -----------------------------
  size_t freeb = 0, totb = 0;
  HM_CUDA(cudaMemGetInfo(&freeb, &totb));
  const size_t budget_bytes = std::min<size_t>(freeb / 4, (size_t)24 << 30);
  // per-problem results that survive the batch: rank (-1: stored dense, -2:
  // split into its child blocks), low-part columns, and the factor location.
  // A problem that misses the tolerance at its rank cap above the leaf level
  // appends its four child pairs to `probs`, so these grow with it.
  std::vector<int> rank(nprob0, 0), conv(nprob0, 0), rhis(nprob0, 0);
  std::vector<double> nrm(nprob0, 0.0);
  long long pstart = 0;
  const double thresh2 = 0.09 * opt.tol * opt.tol;  // (0.3 tol)^2
  long long lr_count = 0, dense_count = 0, rank_sum = 0, split_count = 0;
  int max_rank_seen = 0;
  long long factor_bytes = 0, dense_bytes = 0, unconverged = 0;

  std::vector<const float*> fu(nprob0, nullptr), fv(nprob0, nullptr);
  std::vector<const float*> fd(nprob0, nullptr), fdt(nprob0, nullptr);
  auto grow = [&](size_t np) {
    rank.resize(np, 0);
    conv.resize(np, 0);
    rhis.resize(np, 0);
    nrm.resize(np, 0.0);
    fu.resize(np, nullptr);
    fv.resize(np, nullptr);
    fd.resize(np, nullptr);
    fdt.resize(np, nullptr);
  };

  // Sketches, bases and projections run in FP64 when the tolerance is below
  // what FP32 sums over a block can resolve (~u*sqrt(m) relative), else FP32.
  const bool fp64 = opt.tol < 5e-6;
  auto batch_loop = [&](auto tag) -> hm_status {
    using W = decltype(tag);
    const size_t budget_elems = budget_bytes / sizeof(W);
    HM_CUDA(cudaFuncSetAttribute(k_kmm<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kmm_smem<W>()));
    HM_CUDA(cudaFuncSetAttribute(k_orth<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)orth_smem<W>()));
    // The specialised sketch kernels draw a double-width first sample (the
    // generation of the kernel block, not its product with the sample, is
    // the cost of a pass, so blocks of rank bs..2 bs finish a pass earlier).
    // Separate test columns (k_orth's bst) are supported but measured slower
    // on the 2^20-point Matern build (wider first passes, wider bases), so
    // rounds use bst = 0, the reference ARA's estimate from the sample itself.
    constexpr bool kTensorW = std::is_same<W, float>::value;
    const bool fastW = kTensorW && t->d <= 3;
    const int bst = 0;
    const int bs_first = fastW ? std::min(2 * bs, kMaxBs) : bs;  // round 0 basis columns
    const int wmax = std::max(bs_first, bs) + bst;                // widest sample
    // greedy batches under the workspace budget; one workspace for all of
    // them (child blocks of split problems come in later batches, whose
    // workspace is no larger unless a batch of them packs tighter)
    auto next_batch = [&](long long ps, size_t* wsz_out) {
      long long pe = ps;
      size_t wsz = 0;
      while (pe < (long long)probs.size()) {
        const Prob& P = probs[pe];
        size_t need = (size_t)P.m * (P.kmax + wmax) + (size_t)P.m * wmax + (size_t)P.n * (P.kmax + wmax);
        if (pe > ps && wsz + need > budget_elems) break;
        wsz += need;
        ++pe;
      }
      *wsz_out = wsz;
      return pe;
    };
    size_t ws_max = 1;
    for (long long ps = pstart; ps < (long long)probs.size();) {
      size_t w = 0;
      ps = next_batch(ps, &w);
      ws_max = std::max(ws_max, w);
    }
    DevBuf<W> ws;
    {
      hm_status st0 = ws.alloc(ws_max);
      if (st0) return st0;
    }
    while (pstart < (long long)probs.size()) {
      size_t wsz = 0;
      const long long pend = next_batch(pstart, &wsz);
      if (wsz > ws.n) {
        hm_status st0 = ws.alloc(wsz);
        if (st0) return st0;
      }
      const int nb = (int)(pend - pstart);
      tr.mark("batch begin", stream, nb, 0);
      std::vector<Prob> bp(probs.begin() + pstart, probs.begin() + pend);
      size_t off = 0;
      std::vector<int2> items_rows, items_cols;
      for (int i = 0; i < nb; ++i) {
        Prob& P = bp[i];
        P.qoff = (long long)off;
        off += (size_t)P.m * (P.kmax + wmax);
        P.yoff = (long long)off;
        off += (size_t)P.m * wmax;
        P.boff = (long long)off;
        off += (size_t)P.n * (P.kmax + wmax);
        for (int tt = 0; tt * kTR < P.m; ++tt) items_rows.push_back(make_int2(i, tt));
        for (int tt = 0; tt * kTR < P.n; ++tt) items_cols.push_back(make_int2(i, tt));
      }
      DevBuf<Prob> dprobs;
      DevBuf<ProbState> dst;
      DevBuf<int2> drows, dcols;
      hm_status st;
      if ((st = dprobs.alloc_async(nb, stream)) || (st = dst.alloc_async(nb, stream)) ||
          (st = drows.alloc_async(items_rows.size(), stream)) || (st = dcols.alloc_async(items_cols.size(), stream)))
        return st;
      std::vector<ProbState> hst(nb);
      for (auto& x : hst) {
        x = ProbState{};
        x.active = 1;
      }
      HM_CUDA(cudaMemcpyAsync(dprobs.p, bp.data(), sizeof(Prob) * nb, cudaMemcpyHostToDevice, stream));
      HM_CUDA(cudaMemcpyAsync(dst.p, hst.data(), sizeof(ProbState) * nb, cudaMemcpyHostToDevice, stream));
      HM_CUDA(cudaMemcpyAsync(drows.p, items_rows.data(), sizeof(int2) * items_rows.size(),
                              cudaMemcpyHostToDevice, stream));
      HM_CUDA(cudaMemcpyAsync(dcols.p, items_cols.data(), sizeof(int2) * items_cols.size(),
                              cudaMemcpyHostToDevice, stream));

      KmmArgs<W> ka;
      ka.probs = dprobs.p;
      ka.st = dst.p;
      ka.pts = t->pts_tree_f.p;
      ka.npts = t->n;
      ka.d = t->d;
      ka.kp = h->kp;
      ka.bs = bs;
      ka.seed = (uint32_t)(opt.seed ^ (opt.seed >> 32)) ^ 0x5bd1e995u;
      ka.ws = ws.p;
      OrthArgs<W> oa;
      oa.probs = dprobs.p;
      oa.st = dst.p;
      oa.ws = ws.p;
      oa.bs = bs;
      oa.bst = 0;
      oa.thresh2 = thresh2;
      // FP32 working precision and d <= 3: specialised tensor-core sketch
      // kernels; otherwise the SIMT kernel in the working precision
      constexpr bool kTensor = std::is_same<W, float>::value;
      const bool fast = kTensor && t->d <= 3;
      KmmFastArgs kf{};
      DevBuf<uint2> om2;
      // round 0 basis columns: as wide as every block's rank cap allows
      int bs0 = bs_first;
      for (const Prob& P : bp)
        if (P.kmax < bs0) bs0 = std::max(bs, P.kmax / 8 * 8);
      const int bs8 = (bs0 + bst + 7) & ~7;
      int om_rows2 = 0;
      if (fast) {
        int max_n = 1;
        for (const Prob& P : bp) max_n = std::max(max_n, P.n);
        om_rows2 = (max_n + kCC - 1) / kCC * (kCC / 2);  // column pairs; k-steps = om_rows2 / 8
        if ((st = om2.alloc_async((size_t)(om_rows2 / 8) * (bs8 / 8) * 32, stream))) return st;
        const double il = 1.0 / opt.ell, log2e = 1.4426950408889634, ln2 = 0.6931471805599453;
        double sc = log2e * il, dsc = ln2 * il;
        if (opt.kernel == HM_KERNEL_MATERN32) {
          sc = std::sqrt(3.0) * log2e * il;
          dsc = il;
        } else if (opt.kernel == HM_KERNEL_GAUSS) {
          sc = std::sqrt(0.5 * log2e) * il;
          dsc = 2.0 * ln2 * il;
        }
        kf.probs = dprobs.p;
        kf.st = dst.p;
        kf.pts = t->pts_tree_f.p;
        kf.npts = t->n;
        kf.scale = (float)sc;
        kf.dscale = (float)dsc;
        kf.deriv = opt.derivative != 0;
        kf.bs = bs;
        kf.om = om2.p;
        kf.om_nt = bs8 / 8;
        kf.ws = reinterpret_cast<float*>(ws.p);
      }
      tr.mark("batch setup", stream, nb, 0);
      const int max_rounds = kMaxCols / bs + 2;
      for (int round = 0; round < max_rounds; ++round) {
        if (fast) {
          // basis + test columns: double width in the first round and again
          // from the fourth on (the blocks still active by then are the
          // high-rank ones; entry generation, not the sample width, is the
          // cost of a round, so wider rounds mean fewer of them; earlier, a
          // wider basis would cost more in the projection than it saves)
          const int rbs = (round == 1 || round == 2 ? bs : bs0) + bst;
          k_omega_pack<<<592, 256, 0, stream>>>(om2.p, om_rows2 / 8, rbs, bs8 / 8, ka.seed, round);
          HM_LAUNCH_CHECK();
          kf.round = round;
          kf.bs = rbs;
          kf.items = drows.p;
          oa.bs = rbs;
          oa.bst = bst;
          launch_kmm_fast(t->d, opt.kernel, 0, (rbs + 7) / 8, (unsigned)items_rows.size(), stream, kf);
        } else {
          ka.mode = 0;
          ka.col0 = 0;
          ka.round = round;
          ka.items = drows.p;
          k_kmm<W><<<(unsigned)items_rows.size(), kKmmThreads, kmm_smem<W>(), stream>>>(ka);
        }
        HM_LAUNCH_CHECK();
        tr.mark("  round sketch", stream, round, 1);
        oa.round = round;
        k_orth<W><<<nb, kOrthThreads, orth_smem<W>(), stream>>>(oa);
        HM_LAUNCH_CHECK();
        tr.mark("  round orth", stream, round, 2);
        HM_CUDA(cudaMemcpyAsync(hst.data(), dst.p, sizeof(ProbState) * nb, cudaMemcpyDeviceToHost, stream));
        HM_CUDA(cudaStreamSynchronize(stream));
        bool any = false;
        for (auto& x : hst) any |= x.active != 0;
        if (!any) break;
      }
      tr.mark("sample rounds", stream, nb, 2);
      // B = A^T Q
      DevBuf<uint4> qt;
      DevBuf<long long> dqpoff;
      DevBuf<int2> dcls;
      if (fast) {
        std::vector<long long> qpoff(nb);
        size_t qw = 0;
        for (int i = 0; i < nb; ++i) {
          qpoff[i] = (long long)qw;
          if (hst[i].k > 0)
            qw += (size_t)(bp[i].m + kCC - 1) / kCC * (kCC / 16) * (size_t)((hst[i].k + 7) >> 3) * 32;
        }
        if ((st = qt.alloc_async(std::max<size_t>(qw, 1), stream)) || (st = dqpoff.alloc_async(nb, stream)))
          return st;
        tr.mark("  q table alloc (MB)", stream, (long long)(qw * 16 >> 20), 3);
        HM_CUDA(cudaMemcpyAsync(dqpoff.p, qpoff.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice, stream));
        k_pack_q<<<nb, 256, 0, stream>>>(dprobs.p, dst.p, reinterpret_cast<const float*>(ws.p), dqpoff.p, qt.p);
        HM_LAUNCH_CHECK();
        tr.mark("  q pack", stream, nb, 3);
        kf.qt = qt.p;
        kf.qpoff = dqpoff.p;
        // one launch per basis-width class, so the narrow (most) blocks run
        // with few accumulator registers
        // (bases wider than 128 columns take a second launch for columns
        // 128.. of the same items)
        std::vector<int2> cls[4];
        for (const int2& ic : items_cols) {
          const int kk = hst[ic.x].k;
          if (kk <= 0) continue;
          cls[kk <= 32 ? 0 : (kk <= 64 ? 1 : (kk <= kColGroup ? 2 : 3))].push_back(ic);
        }
        const int cls_nt[4] = {4, 8, kColGroup / 8, kColGroup / 8};
        size_t ncls = 0;
        for (auto& c : cls) ncls += c.size();
        if ((st = dcls.alloc_async(std::max<size_t>(ncls, 1), stream))) return st;
        size_t o = 0;
        for (int c = 0; c < 4; ++c) {
          if (cls[c].empty()) continue;
          HM_CUDA(cudaMemcpyAsync(dcls.p + o, cls[c].data(), sizeof(int2) * cls[c].size(), cudaMemcpyHostToDevice,
                                  stream));
          kf.items = dcls.p + o;
          for (int c0 = 0; c0 < (c == 3 ? kMaxCols : kColGroup); c0 += kColGroup) {
            kf.col0 = c0;
            launch_kmm_fast(t->d, opt.kernel, 1, cls_nt[c], (unsigned)cls[c].size(), stream, kf);
            HM_LAUNCH_CHECK();
          }
          o += cls[c].size();
        }
        kf.col0 = 0;
      } else {
        ka.mode = 1;
        ka.items = dcols.p;
        int kmx = 0;
        for (int i = 0; i < nb; ++i) kmx = std::max(kmx, hst[i].k);
        for (int c0 = 0; c0 < kmx; c0 += kColGroup) {
          ka.col0 = c0;
          k_kmm<W><<<(unsigned)items_cols.size(), kKmmThreads, kmm_smem<W>(), stream>>>(ka);
          HM_LAUNCH_CHECK();
        }
        ka.col0 = 0;
      }
      HM_LAUNCH_CHECK();

      tr.mark("projection", stream, nb, 3);
      // ---- truncation: Gram of B, Jacobi eigen, truncated rank -------------
      HM_CUDA(cudaMemcpyAsync(hst.data(), dst.p, sizeof(ProbState) * nb, cudaMemcpyDeviceToHost, stream));
      HM_CUDA(cudaStreamSynchronize(stream));
      std::vector<long long> goff(nb);
      size_t gtot = 0;
      int kbig = 2;
      for (int i = 0; i < nb; ++i) {
        goff[i] = (long long)gtot;
        gtot += (size_t)hst[i].k * hst[i].k;
        if (hst[i].k <= kTruncMax) kbig = std::max(kbig, hst[i].k);
      }
      DevBuf<long long> dgoff;
      DevBuf<double> Gbuf;
      DevBuf<float> Wr;
      if ((st = dgoff.alloc_async(nb, stream)) || (st = Gbuf.alloc_async(std::max<size_t>(gtot, 1), stream)) ||
          (st = Wr.alloc_async(std::max<size_t>(gtot, 1), stream)))
        return st;
      HM_CUDA(cudaMemcpyAsync(dgoff.p, goff.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice, stream));
      k_gram_big<W><<<nb, kGramThreads, 0, stream>>>(dprobs.p, dst.p, ws.p, dgoff.p, Gbuf.p);
      HM_LAUNCH_CHECK();
      HM_CUDA(cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)jacobi_smem(kTruncMax)));
      // error budget (relative, squared): sampling residual <= 0.09 tol^2 (the
      // stopping test), truncation 0.45 tol^2 (FP32 form) or 0.35 tol^2 plus
      // 0.15 tol^2 of BF16 rounding (mixed form)
      const bool mixed = opt.precision == HM_PREC_MIXED;
      k_jacobi<<<nb, kGramThreads, jacobi_smem(kbig), stream>>>(
          dprobs.p, dst.p, dgoff.p, Gbuf.p, Wr.p, (mixed ? 0.35 : 0.45) * opt.tol * opt.tol,
          mixed ? 0.15 * opt.tol * opt.tol : 0.0);
      HM_LAUNCH_CHECK();
      HM_CUDA(cudaMemcpyAsync(hst.data(), dst.p, sizeof(ProbState) * nb, cudaMemcpyDeviceToHost, stream));
      HM_CUDA(cudaStreamSynchronize(stream));

      tr.mark("truncation", stream, nb, 4);
      // ---- results: low rank where converged; otherwise the four child
      // blocks (above the leaf level) or dense (leaf blocks) -----------------
      std::vector<long long> du(nb, -1), dv(nb, -1);
      std::vector<DenseItem> dens;
      std::vector<Prob> children;
      size_t chunk_floats = 0;
      for (int i = 0; i < nb; ++i) {
        const Prob& P = bp[i];
        const ProbState& S = hst[i];
        long long gi = pstart + i;
        nrm[gi] = S.normA2;
        const bool capped = !(S.converged || S.active);
        if (capped && P.level < depth) {
          // the pair as the reference's recursion would have recorded it had
          // it been inadmissible (src/HMatrixStructure.cu:27-89): its four
          // child pairs (2v + b, 2u + a), compressed in a later batch; every
          // child keeps row cluster > column cluster
          rank[gi] = -2;
          ++split_count;
          const int cl = P.level + 1;
          for (int b2 = 0; b2 < 2; ++b2)
            for (int a2 = 0; a2 < 2; ++a2) {
              Prob C{};
              C.level = cl;
              C.u = 2 * P.u + a2;
              C.v = 2 * P.v + b2;
              C.r0 = coff(cl, C.v);
              C.m = coff(cl, C.v + 1) - C.r0;
              C.c0 = coff(cl, C.u);
              C.n = coff(cl, C.u + 1) - C.c0;
              if (C.m <= 0 || C.n <= 0 || !needed(C.r0, C.m, C.c0, C.n)) continue;
              C.kmax = std::min(level_cap(cl), std::min(C.m, C.n));
              C.tscale2 = level_tscale2(cl);
              children.push_back(C);
            }
          continue;
        }
        if (!capped) {
          du[i] = (long long)chunk_floats;
          chunk_floats += (size_t)P.m * S.r;
          dv[i] = (long long)chunk_floats;
          chunk_floats += (size_t)P.n * S.r;
          rank[gi] = S.r;
          rhis[gi] = std::min(S.rhi, S.r);
          conv[gi] = 1;
        } else {
          // the block and its mirror, each column-major, so every dense read in
          // the matvec is coalesced
          DenseItem di;
          di.r0 = P.r0;
          di.m = P.m;
          di.c0 = P.c0;
          di.n = P.n;
          di.off = (long long)chunk_floats;
          chunk_floats += (size_t)P.m * P.n;
          dens.push_back(di);
          DenseItem dt;
          dt.r0 = P.c0;
          dt.m = P.n;
          dt.c0 = P.r0;
          dt.n = P.m;
          dt.off = (long long)chunk_floats;
          chunk_floats += (size_t)P.m * P.n;
          dens.push_back(dt);
          rank[gi] = -1;
        }
      }
      DevBuf<float> chunk;
      if ((st = chunk.alloc(std::max<size_t>(chunk_floats, 1)))) return st;
      DevBuf<long long> ddu, ddv;
      DevBuf<DenseItem> ddi;
      if ((st = ddu.alloc_async(nb, stream)) || (st = ddv.alloc_async(nb, stream))) return st;
      HM_CUDA(cudaMemcpyAsync(ddu.p, du.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice, stream));
      HM_CUDA(cudaMemcpyAsync(ddv.p, dv.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice, stream));
      k_pack_trunc<W><<<nb, 256, 0, stream>>>(dprobs.p, dst.p, ws.p, dgoff.p, Wr.p, ddu.p, ddv.p, chunk.p);
      HM_LAUNCH_CHECK();
      if (!dens.empty()) {
        if ((st = ddi.alloc_async(dens.size(), stream))) return st;
        HM_CUDA(cudaMemcpyAsync(ddi.p, dens.data(), sizeof(DenseItem) * dens.size(), cudaMemcpyHostToDevice,
                                stream));
        k_dense_gen<<<(unsigned)dens.size(), 256, 0, stream>>>(ddi.p, t->pts_tree_f.p, t->n, t->d, h->kp,
                                                               chunk.p);
        HM_LAUNCH_CHECK();
      }
      HM_CUDA(cudaStreamSynchronize(stream));
      size_t pk = 0, dk = 0;
      for (int i = 0; i < nb; ++i) {
        long long gi = pstart + i;
        if (rank[gi] == -2) continue;  // split
        if (rank[gi] >= 0) {
          fu[gi] = chunk.p + du[i];
          fv[gi] = chunk.p + dv[i];
          ++pk;
          lr_count += 2;
          rank_sum += 2 * (long long)rank[gi];
          max_rank_seen = std::max(max_rank_seen, rank[gi]);
          factor_bytes += 4ll * (bp[i].m + bp[i].n) * rank[gi];
        } else {
          fd[gi] = chunk.p + dens[dk].off;
          fdt[gi] = chunk.p + dens[dk + 1].off;
          dk += 2;
          dense_count += 2;
          dense_bytes += 8ll * bp[i].m * bp[i].n;
        }
      }
      tr.mark("factors", stream, nb, 4);
      h->storage.push_back(std::move(chunk));
      pstart = pend;
      if (!children.empty()) {
        probs.insert(probs.end(), children.begin(), children.end());
        grow(probs.size());
        tr.mark("split into children", stream, (long long)children.size(), 0);
      }
    }
    return HM_OK;
  };
  {
    hm_status bst = fp64 ? batch_loop(double(0)) : batch_loop(float(0));
    if (bst) return cleanup(bst);
  }

  // ---- diagonal leaves ------------------------------------------------------
  h->diag_fly = opt.diag_from_coords > 0 || (opt.diag_from_coords < 0 && opt.derivative != 0);
  if (!h->diag_fly) {
    const int nown = leaf_hi - leaf_lo;  // the shard's leaves (all of them for a whole matrix)
    std::vector<DenseItem> dens(nown);
    size_t tot = 0;
    for (int q = 0; q < nown; ++q) {
      const int l = leaf_lo + q;
      dens[q].r0 = lo[l];
      dens[q].m = lo[l + 1] - lo[l];
      dens[q].c0 = lo[l];
      dens[q].n = dens[q].m;
      dens[q].off = (long long)tot;
      tot += (size_t)dens[q].m * dens[q].m;
    }
    DevBuf<float> chunk;
    DevBuf<DenseItem> ddi;
    hm_status st;
    if ((st = chunk.alloc(std::max<size_t>(tot, 1))) || (st = ddi.alloc(nown))) return cleanup(st);
    HM_CUDA(cudaMemcpyAsync(ddi.p, dens.data(), sizeof(DenseItem) * nown, cudaMemcpyHostToDevice, stream));
    k_dense_gen<<<nown, 256, 0, stream>>>(ddi.p, t->pts_tree_f.p, t->n, t->d, h->kp, chunk.p);
    HM_LAUNCH_CHECK();
    HM_CUDA(cudaStreamSynchronize(stream));
    for (int l = 0; l < nown; ++l) {
      DenseBlock db;
      db.r0 = dens[l].r0;
      db.m = dens[l].m;
      db.c0 = dens[l].c0;
      db.n = dens[l].n;
      db.trans = 0;
      db.D = chunk.p + dens[l].off;
      if (db.m > 0) h->h_dense.push_back(db);
    }
    dense_count += nown;
    dense_bytes += 4ll * (long long)tot;
    h->storage.push_back(std::move(chunk));
  }

  tr.mark("diagonal leaves", stream, -1, 5);
  // ---- block lists (both orientations) --------------------------------------
  const long long nprob = (long long)probs.size();
  for (long long i = 0; i < nprob; ++i) {
    const Prob& P = probs[i];
    if (rank[i] == -2) continue;  // split: its children are in the list
    if (rank[i] >= 0) {
      LRBlock b{};
      b.level = P.level;
      b.k = rank[i];
      b.r0 = P.r0;
      b.m = P.m;
      b.c0 = P.c0;
      b.n = P.n;
      b.U = fu[i];
      b.V = fv[i];
      b.khi = std::min(rhis[i], rank[i]);
      h->h_lr.push_back(b);
      LRBlock bt = b;
      bt.r0 = P.c0;
      bt.m = P.n;
      bt.c0 = P.r0;
      bt.n = P.m;
      bt.U = fv[i];
      bt.V = fu[i];
      h->h_lr.push_back(bt);
    } else {
      DenseBlock db{P.r0, P.m, P.c0, P.n, 0, fd[i]};
      h->h_dense.push_back(db);
      DenseBlock dt{P.c0, P.n, P.r0, P.m, 0, fdt[i]};
      h->h_dense.push_back(dt);
    }
  }
  tr.mark("block lists", stream, -1, 6);
  // ---- factor panels: the mixed form's BF16 hi + lo tiles, or the FP32
  // form's FP32 tiles (both forms multiply on panels) ---------------------------
  {
    std::vector<MxPair> mp;
    for (long long i = 0; i < nprob; ++i) {
      if (rank[i] <= 0) continue;
      const Prob& P = probs[i];
      mp.push_back(MxPair{P.level, P.r0, P.m, P.c0, P.n, rank[i], std::min(rhis[i], rank[i]), fu[i], fv[i]});
    }
    std::vector<MxDenseIn> md;
    for (const DenseBlock& db : h->h_dense) md.push_back(MxDenseIn{db.r0, db.m, db.c0, db.n, db.D});
    h->mx.fmt = opt.precision == HM_PREC_MIXED ? 0 : 1;
    hm_status mst = mixed_build(h, mp, md, stream);
    if (mst) return cleanup(mst);
    if (opt.precision == HM_PREC_MIXED) {
      h->stats.mixed_bytes = h->mx.store_tiles * 512;
      release_fp32(h);
    }
  }
  h->stats.num_lowrank = lr_count;
  h->stats.num_dense = dense_count;
  h->stats.rank_sum = rank_sum;
  h->stats.max_rank_seen = max_rank_seen;
  h->stats.factor_bytes = factor_bytes;
  h->stats.dense_bytes = dense_bytes;
  h->stats.num_unconverged = unconverged;
  h->stats.num_split = split_count;
  tr.mark("mixed panels", stream, -1, 6);
  hm_status st = matvec_plan_build(h, 16, stream);
  if (st) return cleanup(st);
  tr.mark("matvec plan", stream, -1, 7);
  for (int i = 0; i < PhaseTrace::kSlots; ++i) h->stats.phase_seconds[i] = tr.sec[i];
  HM_CUDA(cudaEventRecord(ev1, stream));
  HM_CUDA(cudaEventSynchronize(ev1));
  float ms = 0;
  HM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  h->stats.build_seconds = ms * 1e-3;
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  *out = h;
  return HM_OK;
}

void release_fp32(hm_hmatrix_s* h) {
  h->chunk_meta.clear();
  for (const auto& c : h->storage) h->chunk_meta.push_back({c.p, c.n});
  h->storage.clear();
  h->fp32_released = true;
}

// Device memory held by the matrix: factor and dense storage, the mixed
// form's panels and tables, the product's plan and workspaces.
long long device_bytes(const hm_hmatrix_s* h) {
  long long b = 0;
  auto add = [&b](const auto& buf) { b += (long long)(buf.n * sizeof(*buf.p)); };
  for (const auto& c : h->storage) add(c);
  const MatvecPlan& P = h->plan;
  add(P.lr), add(P.p1), add(P.multi), add(P.groups), add(P.leaf_ptr), add(P.leaf_blk), add(P.dense);
  add(P.leaf_dptr), add(P.leaf_dblk), add(P.T), add(P.Xp), add(P.Yp);
  const MxPlan& M = h->mx;
  add(M.store), add(M.panels), add(M.pan_of), add(M.units), add(M.tile_leaf), add(M.leaf_tile0), add(M.tslot);
  add(M.mtiles), add(M.dense), add(M.leaf_dptr), add(M.leaf_dblk);
  return b;
}

}  // namespace hm

extern "C" {

void hm_build_opts_default(int d, hm_build_opts* o) {
  if (!o) return;
  o->kernel = HM_KERNEL_EXP;
  o->ell = d == 3 ? 0.2 : 0.1;  // src/TLRMatrixHelpers.cu:40-42
  o->nugget = 0.0;
  o->tol = 1e-5;                // src/config.h:127
  o->max_rank = 64;
  o->leaf_max_rank = 0;
  o->sample_block = 16;         // src/constructTLRMatrix.cu:73
  o->precision = HM_PREC_FP32;
  o->derivative = 0;
  o->seed = 0;
  o->diag_from_coords = -1;
  o->level_schedule = 0;
}

hm_status hm_hmatrix_build(hm_kdtree t, hm_structure s, const double* d_points, const hm_build_opts* opts,
                           void* stream, hm_hmatrix* out) {
  return hm::hmatrix_build(t, s, d_points, opts, hm::as_stream(stream), out, 0, -1);
}

hm_status hm_hmatrix_build_rows(hm_kdtree t, hm_structure s, const double* d_points, const hm_build_opts* opts,
                                int leaf_begin, int leaf_end, void* stream, hm_hmatrix* out) {
  if (out) *out = nullptr;
  if (!t) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_build_rows: null tree");
  if (leaf_begin < 0 || leaf_begin >= leaf_end || leaf_end > (1 << t->depth))
    return hm::fail(HM_ERR_INVALID, "hm_hmatrix_build_rows: need 0 <= leaf_begin < leaf_end <= 2^depth");
  return hm::hmatrix_build(t, s, d_points, opts, hm::as_stream(stream), out, leaf_begin, leaf_end);
}

hm_status hm_hmatrix_stats_get(hm_hmatrix h, hm_hmatrix_stats* st) {
  if (!h || !st) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_stats_get: null argument");
  *st = h->stats;
  st->device_bytes = hm::device_bytes(h);
  return HM_OK;
}

hm_status hm_hmatrix_blocks(hm_hmatrix h, long long* num_lowrank, long long* num_dense, int* lowrank,
                            int* dense) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_blocks: null matrix");
  if (num_lowrank) *num_lowrank = (long long)h->h_lr.size();
  if (num_dense) *num_dense = (long long)h->h_dense.size();
  if (lowrank)
    for (size_t i = 0; i < h->h_lr.size(); ++i) {
      const hm::LRBlock& b = h->h_lr[i];
      int* r = lowrank + 6 * i;
      r[0] = b.r0;
      r[1] = b.m;
      r[2] = b.c0;
      r[3] = b.n;
      r[4] = b.k;
      r[5] = b.level;
    }
  if (dense)
    for (size_t i = 0; i < h->h_dense.size(); ++i) {
      const hm::DenseBlock& b = h->h_dense[i];
      int* r = dense + 5 * i;
      r[0] = b.r0;
      r[1] = b.m;
      r[2] = b.c0;
      r[3] = b.n;
      r[4] = b.trans;
    }
  return HM_OK;
}

// Host copy of an FP32 array of the matrix (a factor or a dense block, count
// floats): from its storage, or rebuilt from the panels once released.
static hm_status fetch_fp32(hm_hmatrix h, const float* src, size_t count, float* dst) {
  if (!count) return HM_OK;
  if (!h->fp32_released) {
    HM_CUDA(cudaMemcpy(dst, src, sizeof(float) * count, cudaMemcpyDeviceToHost));
    return HM_OK;
  }
  const int loc = hm::mixed_find_loc(h, src);
  if (loc < 0) return hm::fail(HM_ERR_INVALID, "no panel holds this block");
  hm::DevBuf<float> tmp;
  HM_TRY(tmp.alloc(count));
  HM_TRY(hm::mixed_unpack(h, {{loc, tmp.p}}, nullptr));
  HM_CUDA(cudaMemcpy(dst, tmp.p, sizeof(float) * count, cudaMemcpyDeviceToHost));
  return HM_OK;
}

hm_status hm_hmatrix_block_factors(hm_hmatrix h, int i, float* U, float* V) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_block_factors: null matrix");
  if (i < 0 || (size_t)i >= h->h_lr.size()) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_block_factors: bad index");
  const hm::LRBlock& b = h->h_lr[i];
  if (U && b.k) HM_TRY(fetch_fp32(h, b.U, (size_t)b.m * b.k, U));
  if (V && b.k) HM_TRY(fetch_fp32(h, b.V, (size_t)b.n * b.k, V));
  return HM_OK;
}

hm_status hm_hmatrix_dense_block(hm_hmatrix h, int i, float* D) {
  if (!h) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_dense_block: null matrix");
  if (i < 0 || (size_t)i >= h->h_dense.size()) return hm::fail(HM_ERR_INVALID, "hm_hmatrix_dense_block: bad index");
  const hm::DenseBlock& b = h->h_dense[i];
  if (D && b.m && b.n) HM_TRY(fetch_fp32(h, b.D, (size_t)b.m * b.n, D));
  return HM_OK;
}

void hm_hmatrix_free(hm_hmatrix h) { delete h; }

}  // extern "C"
