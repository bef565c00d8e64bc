// hm_kdtree.cu -- KD-tree construction (FULL_TREE division), bit-exact with the
// reference's constructKDTree (src/kDTreeConstruction.cu:14-231).
//
// Reference semantics.  Per level j and segment s the reference computes the
// box (segmented min/max, :113-127), picks the first dimension of maximum span
// (ArgMax, :145-150), stably sorts the segment by the coordinate along that
// dimension (:167-174) and splits it at ceil(len/2) (src/kDTreeHelpers.cu:81-94).
// Because every level's sort is stable and the previous level left each segment
// sorted, the order at level j is the lexicographic order of the key chain
//     K_j(p) = (x_{dim_j}(p), x_{dim_{j-1}}(p), ..., x_{dim_0}(p), p)
// where dim_i is the split dimension of p's ancestor at level i.  Membership of
// the left child = the ceil(len/2) smallest elements under K_j; the final
// order of a leaf = its elements sorted by K_{depth-1}.
//
// B200 design.  Nothing is fully sorted on the wide levels: each segment's
// split element is found by a multi-word radix select over K_j (8-bit digits,
// shared-memory histograms merged with global atomics, the words after the
// first only touched when coordinates tie), then the segment is partitioned
// with warp-ballot compaction while the children's boxes are reduced on the
// fly.  Once a segment fits in shared memory (kLocal levels), one CTA per
// segment finishes the whole subtree on chip: box, split dimension and a
// bitonic sort by the key chain per level, then writes the permutation and the
// tree-ordered coordinates.  Segment offsets are data independent (sizes are
// ceil/floor halvings), so they are computed on the host.
#include <algorithm>
#include <cstdio>

#include "hm_internal.h"

namespace hm {
namespace {

constexpr int kChunk = 4096;     // elements per CTA on wide levels
constexpr int kWideThreads = 256;
constexpr int kLocalThreads = 512;
constexpr int kPassesPerBatch = 8;

struct SelState {
  unsigned long long pval;   // fixed bits of the current word
  unsigned long long pmask;  // which bits are fixed
  int shift;                 // bit position of the next digit
  int word;                  // current word of the key chain
  int target;                // rank of the split element among the candidates
  int cand;                  // number of candidates
  int done;
  int final_word;
};

struct WideArgs {
  int n, d, level, depth;
  const int* leaf_off;       // 2^depth + 1
  const int* split_dim;      // level-major, level l at [2^l - 1]
  const int* idx;            // current buffer
  const double* coord;       // current buffer, [dim * n + pos]
  SelState* st;              // per segment
  unsigned long long* chosen;  // per segment, [seg * maxw + word]
  int maxw;
  unsigned int* hist;        // per segment, 256 bins
  int cps;                   // chunks per segment
  int* err;                  // set on an internal inconsistency
};

__device__ __forceinline__ int seg_begin(const int* leaf_off, int level, int depth, int s) {
  return leaf_off[s << (depth - level)];
}

// word w of the key chain K_level for the element at position e of segment s
__device__ __forceinline__ unsigned long long key_word(const WideArgs& a, int s, int w, int e) {
  if (w <= a.level) {
    int lv = a.level - w;
    int dim = a.split_dim[(1 << lv) - 1 + (s >> w)];
    return twiddle(a.coord[(size_t)dim * a.n + e]);
  }
  return (unsigned long long)(unsigned)a.idx[e];
}

__device__ void start_word(SelState& st, int w, int level) {
  st.word = w;
  if (w == level + 1) {  // the original index: only the low 32 bits vary
    st.pmask = 0xffffffff00000000ull;
    st.pval = 0;
    st.shift = 24;
  } else {
    st.pmask = 0;
    st.pval = 0;
    st.shift = 56;
  }
}

// Called when every bit of the current word is fixed: decide whether the
// elements equal so far all go left, else move on to the next word.
__device__ void finish_word(SelState& st, unsigned long long* chosen, int level) {
  chosen[st.word] = st.pval;
  if (st.target + 1 == st.cand) {
    st.done = 1;
    st.final_word = st.word;
  } else {
    start_word(st, st.word + 1, level);
  }
}

// root box: min/max of every dimension over all points
__global__ void k_root_box(int n, int d, const double* pts, unsigned long long* bmin_tw,
                           unsigned long long* bmax_tw) {
  __shared__ unsigned long long smin[kMaxDim], smax[kMaxDim];
  if (threadIdx.x < d) {
    smin[threadIdx.x] = ~0ull;
    smax[threadIdx.x] = 0ull;
  }
  __syncthreads();
  for (int k = 0; k < d; ++k) {
    unsigned long long mn = ~0ull, mx = 0ull;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      unsigned long long t = twiddle(pts[(size_t)k * n + i]);
      mn = t < mn ? t : mn;
      mx = t > mx ? t : mx;
    }
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long a = __shfl_xor_sync(0xffffffffu, mn, o);
      unsigned long long b = __shfl_xor_sync(0xffffffffu, mx, o);
      mn = a < mn ? a : mn;
      mx = b > mx ? b : mx;
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&smin[k], mn);
      atomicMax(&smax[k], mx);
    }
  }
  __syncthreads();
  if (threadIdx.x < d) {
    atomicMin(&bmin_tw[threadIdx.x], smin[threadIdx.x]);
    atomicMax(&bmax_tw[threadIdx.x], smax[threadIdx.x]);
  }
}

// per segment: split dimension from the box, selection state for word 0
__global__ void k_select_init(WideArgs a, const unsigned long long* bmin_tw,
                              const unsigned long long* bmax_tw, int* split_dim_out) {
  int nseg = 1 << a.level;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const unsigned long long* mn = bmin_tw + (size_t)((1 << a.level) - 1 + s) * a.d;
  const unsigned long long* mx = bmax_tw + (size_t)((1 << a.level) - 1 + s) * a.d;
  int best = 0;
  double bspan = untwiddle(mx[0]) - untwiddle(mn[0]);
  for (int k = 1; k < a.d; ++k) {
    double sp = untwiddle(mx[k]) - untwiddle(mn[k]);
    if (sp > bspan) {
      bspan = sp;
      best = k;
    }
  }
  split_dim_out[(1 << a.level) - 1 + s] = best;
  int b0 = seg_begin(a.leaf_off, a.level, a.depth, s);
  int b1 = seg_begin(a.leaf_off, a.level, a.depth, s + 1);
  int len = b1 - b0;
  SelState st;
  st.done = 0;
  st.final_word = 0;
  st.target = (len + 1) / 2 - 1;
  st.cand = len;
  st.word = 0;
  // every key of word 0 lies in [tw(min), tw(max)]: their common leading
  // digits are already known
  unsigned long long lo = mn[best], hi = mx[best];
  unsigned long long x = lo ^ hi;
  int common = x ? __clzll((long long)x) : 64;
  int digits = common / 8;
  st.pmask = digits ? (~0ull << (64 - 8 * digits)) : 0ull;
  if (digits == 8) st.pmask = ~0ull;
  st.pval = lo & st.pmask;
  st.shift = 56 - 8 * digits;
  unsigned long long* ch = a.chosen + (size_t)s * a.maxw;
  if (len <= 0) {
    st.done = 1;
  } else if (st.shift < 0) {
    finish_word(st, ch, a.level);
  }
  a.st[s] = st;
}

__global__ void __launch_bounds__(kWideThreads) k_hist(WideArgs a) {
  __shared__ unsigned int h[256];
  int s = blockIdx.x / a.cps;
  int c = blockIdx.x % a.cps;
  const SelState st = a.st[s];
  if (st.done) return;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  int b0 = seg_begin(a.leaf_off, a.level, a.depth, s);
  int b1 = seg_begin(a.leaf_off, a.level, a.depth, s + 1);
  int lo = b0 + c * kChunk;
  int hi = min(b1, lo + kChunk);
  const unsigned long long* ch = a.chosen + (size_t)s * a.maxw;
  for (int e = lo + threadIdx.x; e < hi; e += blockDim.x) {
    bool match = true;
    for (int w = 0; w < st.word && match; ++w) match = key_word(a, s, w, e) == ch[w];
    if (!match) continue;
    unsigned long long k = key_word(a, s, st.word, e);
    if ((k & st.pmask) == st.pval) atomicAdd(&h[(k >> st.shift) & 255u], 1u);
  }
  __syncthreads();
  unsigned int* gh = a.hist + (size_t)s * 256;
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&gh[i], h[i]);
}

// one warp per segment
__global__ void k_select(WideArgs a, int* not_done) {
  int nseg = 1 << a.level;
  int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (s >= nseg) return;
  SelState st = a.st[s];
  if (st.done) return;
  unsigned int* gh = a.hist + (size_t)s * 256;
  unsigned int cnt[8];
  unsigned int tot = 0;
  for (int i = 0; i < 8; ++i) {
    cnt[i] = gh[lane * 8 + i];
    gh[lane * 8 + i] = 0;  // ready for the next pass
    tot += cnt[i];
  }
  unsigned int incl = tot;
  for (int o = 1; o < 32; o <<= 1) {
    unsigned int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  unsigned int excl = incl - tot;
  unsigned int target = (unsigned)st.target;
  int found_bin = -1;
  unsigned int below = 0, bcount = 0;
  if (target >= excl && target < incl) {
    unsigned int run = excl;
    for (int i = 0; i < 8; ++i) {
      if (target < run + cnt[i]) {
        found_bin = lane * 8 + i;
        below = run;
        bcount = cnt[i];
        break;
      }
      run += cnt[i];
    }
  }
  unsigned int ball = __ballot_sync(0xffffffffu, found_bin >= 0);
  if (ball == 0) {  // inconsistent histogram: stop this segment, report
    if (lane == 0) {
      st.done = 1;
      st.final_word = st.word;
      a.st[s] = st;
      atomicExch(a.err, 1);
    }
    return;
  }
  int src = __ffs(ball) - 1;
  found_bin = __shfl_sync(0xffffffffu, found_bin, src);
  below = __shfl_sync(0xffffffffu, below, src);
  bcount = __shfl_sync(0xffffffffu, bcount, src);
  if (lane != 0) return;
  st.target -= (int)below;
  st.cand = (int)bcount;
  st.pval |= (unsigned long long)found_bin << st.shift;
  st.pmask |= 0xffull << st.shift;
  st.shift -= 8;
  if (st.shift < 0) finish_word(st, a.chosen + (size_t)s * a.maxw, a.level);
  a.st[s] = st;
  if (!st.done) atomicAdd(not_done, 1);
}

struct PartArgs {
  WideArgs w;
  int* idx_out;
  double* coord_out;
  int* cursor;                 // per segment: [2*s] left, [2*s+1] right
  unsigned long long* cmin_tw; // child boxes (level+1), or null
  unsigned long long* cmax_tw;
  int* err;                    // set if a destination falls outside its child
};

// Partition one chunk of a segment into the two children (warp-ballot
// compaction, one atomic reservation per side per CTA iteration) and reduce the
// children's boxes in registers.  DMAX bounds d at compile time.
template <int DMAX>
__global__ void __launch_bounds__(kWideThreads) k_partition(PartArgs p) {
  const WideArgs& a = p.w;
  __shared__ unsigned long long bmn[2][DMAX], bmx[2][DMAX];
  __shared__ int wl[kWideThreads / 32], wr[kWideThreads / 32];
  __shared__ int base_l, base_r;
  int s = blockIdx.x / a.cps;
  int c = blockIdx.x % a.cps;
  const SelState st = a.st[s];
  int b0 = seg_begin(a.leaf_off, a.level, a.depth, s);
  int b1 = seg_begin(a.leaf_off, a.level, a.depth, s + 1);
  int m = (b1 - b0 + 1) / 2;
  int lo = b0 + c * kChunk;
  int hi = min(b1, lo + kChunk);
  const bool boxes = p.cmin_tw != nullptr;
  if (threadIdx.x < 2 * DMAX) {
    bmn[threadIdx.x / DMAX][threadIdx.x % DMAX] = ~0ull;
    bmx[threadIdx.x / DMAX][threadIdx.x % DMAX] = 0ull;
  }
  unsigned long long rmn[2][DMAX], rmx[2][DMAX];
#pragma unroll
  for (int k = 0; k < DMAX; ++k) {
    rmn[0][k] = rmn[1][k] = ~0ull;
    rmx[0][k] = rmx[1][k] = 0ull;
  }
  const unsigned long long* ch = a.chosen + (size_t)s * a.maxw;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  for (int base = lo; base < hi; base += blockDim.x) {
    int e = base + threadIdx.x;
    bool valid = e < hi;
    bool left = false;
    if (valid) {
      left = true;  // equal on every decided word -> left
      for (int w = 0; w <= st.final_word; ++w) {
        unsigned long long k = key_word(a, s, w, e);
        if (k != ch[w]) {
          left = k < ch[w];
          break;
        }
      }
    }
    unsigned int bl = __ballot_sync(0xffffffffu, valid && left);
    unsigned int br = __ballot_sync(0xffffffffu, valid && !left);
    if (lane == 0) {
      wl[warp] = __popc(bl);
      wr[warp] = __popc(br);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int tl = 0, tr = 0;
      for (int i = 0; i < kWideThreads / 32; ++i) {
        int x = wl[i], y = wr[i];
        wl[i] = tl;
        wr[i] = tr;
        tl += x;
        tr += y;
      }
      base_l = tl ? atomicAdd(&p.cursor[2 * s], tl) : 0;
      base_r = tr ? atomicAdd(&p.cursor[2 * s + 1], tr) : 0;
    }
    __syncthreads();
    if (valid) {
      unsigned int lt = (1u << lane) - 1u;
      int dst = left ? b0 + base_l + wl[warp] + __popc(bl & lt)
                     : b0 + m + base_r + wr[warp] + __popc(br & lt);
      bool in_child = left ? dst < b0 + m : dst < b1;
      if (!in_child) {
        atomicExch(p.err, 1);
      } else {
        p.idx_out[dst] = a.idx[e];
        int side = left ? 0 : 1;
#pragma unroll
        for (int k = 0; k < DMAX; ++k) {
          if (k < a.d) {
            double x = a.coord[(size_t)k * a.n + e];
            p.coord_out[(size_t)k * a.n + dst] = x;
            unsigned long long t = twiddle(x);
            if (side == 0) {
              rmn[0][k] = t < rmn[0][k] ? t : rmn[0][k];
              rmx[0][k] = t > rmx[0][k] ? t : rmx[0][k];
            } else {
              rmn[1][k] = t < rmn[1][k] ? t : rmn[1][k];
              rmx[1][k] = t > rmx[1][k] ? t : rmx[1][k];
            }
          }
        }
      }
    }
    __syncthreads();
  }
  if (!boxes) return;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
#pragma unroll
    for (int k = 0; k < DMAX; ++k) {
      if (k < a.d) {
        unsigned long long mn = rmn[side][k], mx = rmx[side][k];
        for (int o = 16; o > 0; o >>= 1) {
          unsigned long long x = __shfl_xor_sync(0xffffffffu, mn, o);
          unsigned long long y = __shfl_xor_sync(0xffffffffu, mx, o);
          mn = x < mn ? x : mn;
          mx = y > mx ? y : mx;
        }
        if (lane == 0) {
          atomicMin(&bmn[side][k], mn);
          atomicMax(&bmx[side][k], mx);
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < 2 * a.d) {
    int side = threadIdx.x / a.d, k = threadIdx.x % a.d;
    size_t node = (size_t)((1 << (a.level + 1)) - 1 + 2 * s + side);
    if (bmn[side][k] != ~0ull) atomicMin(&p.cmin_tw[node * a.d + k], bmn[side][k]);
    if (bmx[side][k] != 0ull) atomicMax(&p.cmax_tw[node * a.d + k], bmx[side][k]);
  }
}

__global__ void k_untwiddle(size_t count, const unsigned long long* tw, double* out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = untwiddle(tw[i]);
}

__global__ void k_iota(int n, int* idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) idx[i] = i;
}

// ---------------------------------------------------------------------------
// Local phase: one CTA per segment of level j0 finishes its whole subtree.
// ---------------------------------------------------------------------------
struct LocalArgs {
  int n, d, depth, j0, seg_cap, pcap;
  const int* leaf_off;
  const int* idx;        // current buffer
  const double* coord;   // current buffer
  int* split_dim;        // global, level-major
  double* bmin;          // global, level-major [(2^l-1)*d + node*d + k]
  double* bmax;
  int* perm;
  double* pts_tree;
  float* pts_tree_f;
};

struct LocalSmem {
  double* coord;          // [d][seg_cap]
  int* idx;               // [seg_cap]
  unsigned short* ord;    // [pcap] position -> slot
  unsigned short* segid;  // [seg_cap] slot -> local segment at the current level
  int* ldims;             // local levels' split dims, level j at [2^(j-j0) - 1]
  int* adims;             // ancestors' split dims for levels < j0
};

__device__ __forceinline__ int local_dim(const LocalArgs& a, const LocalSmem& sm, int root, int lv,
                                         int node) {
  // node: global index at level lv
  if (lv < a.j0) return sm.adims[lv];
  return sm.ldims[(1 << (lv - a.j0)) - 1 + (node - (root << (lv - a.j0)))];
}

// strict order of slots x, y under K_level (sentinel slots >= len sort last)
__device__ __forceinline__ bool chain_less(const LocalArgs& a, const LocalSmem& sm, int root,
                                           int level, int len, int x, int y) {
  bool sx = x >= len, sy = y >= len;
  if (sx || sy) return !sx && sy ? true : (sx && sy ? x < y : false);
  int gx = sm.segid[x], gy = sm.segid[y];
  if (gx != gy) return gx < gy;
  int node = (root << (level - a.j0)) + gx;
  for (int w = 0; w <= level; ++w) {
    int lv = level - w;
    int dim = local_dim(a, sm, root, lv, node >> w);
    double kx = sm.coord[(size_t)dim * a.seg_cap + x];
    double ky = sm.coord[(size_t)dim * a.seg_cap + y];
    if (kx < ky) return true;
    if (ky < kx) return false;
  }
  return sm.idx[x] < sm.idx[y];
}

__global__ void __launch_bounds__(kLocalThreads) k_local(LocalArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LocalSmem sm;
  size_t off = 0;
  sm.coord = reinterpret_cast<double*>(smem_raw);
  off += sizeof(double) * (size_t)a.d * a.seg_cap;
  sm.idx = reinterpret_cast<int*>(smem_raw + off);
  off += sizeof(int) * (size_t)a.seg_cap;
  int nlocal = a.depth - a.j0;  // local levels that sort
  sm.ldims = reinterpret_cast<int*>(smem_raw + off);
  off += sizeof(int) * (size_t)((1 << nlocal) + 1);
  sm.adims = reinterpret_cast<int*>(smem_raw + off);
  off += sizeof(int) * (size_t)(kMaxDepth + 1);
  sm.ord = reinterpret_cast<unsigned short*>(smem_raw + off);
  off += sizeof(unsigned short) * (size_t)a.pcap;
  sm.segid = reinterpret_cast<unsigned short*>(smem_raw + off);

  const int root = blockIdx.x;
  const int o = a.leaf_off[root << (a.depth - a.j0)];
  const int len = a.leaf_off[(root + 1) << (a.depth - a.j0)] - o;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31, nwarp = nth >> 5;

  for (int i = tid; i < len; i += nth) {
    sm.idx[i] = a.idx[o + i];
    for (int k = 0; k < a.d; ++k) sm.coord[(size_t)k * a.seg_cap + i] = a.coord[(size_t)k * a.n + o + i];
  }
  for (int i = tid; i < a.pcap; i += nth) sm.ord[i] = (unsigned short)i;
  if (tid < a.j0) sm.adims[tid] = a.split_dim[(1 << tid) - 1 + (root >> (a.j0 - tid))];
  __syncthreads();

  for (int level = a.j0; level <= a.depth; ++level) {
    const int nseg = 1 << (level - a.j0);
    const int gbase = root << (level - a.j0);
    // boxes (and split dimensions) of this level's segments: one warp each
    for (int t = warp; t < nseg; t += nwarp) {
      int p0 = a.leaf_off[(gbase + t) << (a.depth - level)] - o;
      int p1 = a.leaf_off[(gbase + t + 1) << (a.depth - level)] - o;
      int best = 0;
      double bspan = 0;
      size_t gnode = (size_t)((1 << level) - 1 + gbase + t);
      for (int k = 0; k < a.d; ++k) {
        double mn = INFINITY, mx = -INFINITY;
        for (int p = p0 + lane; p < p1; p += 32) {
          double x = sm.coord[(size_t)k * a.seg_cap + sm.ord[p]];
          mn = fmin(mn, x);
          mx = fmax(mx, x);
        }
        for (int s2 = 16; s2 > 0; s2 >>= 1) {
          mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, s2));
          mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, s2));
        }
        if (lane == 0) {
          a.bmin[gnode * a.d + k] = mn;
          a.bmax[gnode * a.d + k] = mx;
          double sp = mx - mn;
          if (k == 0 || sp > bspan) {
            bspan = sp;
            best = k;
          }
        }
      }
      if (lane == 0 && level < a.depth) {
        sm.ldims[nseg - 1 + t] = best;
        a.split_dim[(1 << level) - 1 + gbase + t] = best;
      }
    }
    if (level == a.depth) break;
    // segment of every slot by its current position
    for (int t = warp; t < nseg; t += nwarp) {
      int p0 = a.leaf_off[(gbase + t) << (a.depth - level)] - o;
      int p1 = a.leaf_off[(gbase + t + 1) << (a.depth - level)] - o;
      for (int p = p0 + lane; p < p1; p += 32) sm.segid[sm.ord[p]] = (unsigned short)t;
    }
    __syncthreads();
    // bitonic sort of the positions by (segment, K_level)
    for (int k = 2; k <= a.pcap; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = tid; i < a.pcap; i += nth) {
          int ixj = i ^ j;
          if (ixj > i) {
            int x = sm.ord[i], y = sm.ord[ixj];
            bool up = (i & k) == 0;
            bool sw = up ? chain_less(a, sm, root, level, len, y, x)
                         : chain_less(a, sm, root, level, len, x, y);
            if (sw) {
              sm.ord[i] = (unsigned short)y;
              sm.ord[ixj] = (unsigned short)x;
            }
          }
        }
        __syncthreads();
      }
    }
  }
  __syncthreads();
  for (int p = tid; p < len; p += nth) {
    int s = sm.ord[p];
    a.perm[o + p] = sm.idx[s];
    for (int k = 0; k < a.d; ++k) {
      double x = sm.coord[(size_t)k * a.seg_cap + s];
      a.pts_tree[(size_t)k * a.n + o + p] = x;
      a.pts_tree_f[(size_t)k * a.n + o + p] = (float)x;
    }
  }
}

size_t local_smem_bytes(int d, int seg_cap, int pcap, int nlocal) {
  return sizeof(double) * (size_t)d * seg_cap + sizeof(int) * (size_t)seg_cap +
         sizeof(int) * (size_t)((1 << nlocal) + 1) + sizeof(int) * (size_t)(kMaxDepth + 1) +
         sizeof(unsigned short) * (size_t)pcap + sizeof(unsigned short) * (size_t)seg_cap + 64;
}

}  // namespace

int tree_depth(int n, int bucket) {
  int it = 0;
  while (n > bucket) {
    n = (n + 1) / 2;
    ++it;
  }
  return it;
}

std::vector<int> leaf_offsets(int n, int depth) {
  std::vector<int> off = {0, n};
  for (int l = 0; l < depth; ++l) {
    std::vector<int> nx;
    nx.reserve(2 * off.size());
    for (size_t s = 0; s + 1 < off.size(); ++s) {
      nx.push_back(off[s]);
      nx.push_back(off[s] + (off[s + 1] - off[s] + 1) / 2);
    }
    nx.push_back(n);
    off.swap(nx);
  }
  return off;
}

hm_status kdtree_build(const double* d_points, int n, int d, int bucket, cudaStream_t stream,
                       hm_kdtree* out) {
  if (!out) return fail(HM_ERR_INVALID, "hm_kdtree_build: out is NULL");
  *out = nullptr;
  if (!d_points) return fail(HM_ERR_INVALID, "hm_kdtree_build: d_points is NULL");
  if (n < 1 || d < 1 || d > kMaxDim || bucket < 1)
    return fail(HM_ERR_INVALID, "hm_kdtree_build: need n >= 1, 1 <= d <= 16, bucket >= 1");
  const int depth = tree_depth(n, bucket);
  if (depth > kMaxDepth) return fail(HM_ERR_UNSUPPORTED, "hm_kdtree_build: tree too deep");

  // shared-memory capacity of the local phase: largest power of two whose
  // per-point state fits in 200 KB
  int seg_cap = 1 << 15;
  while (seg_cap > 64 && local_smem_bytes(d, seg_cap, seg_cap, 1) +
                                 sizeof(int) * (size_t)(4 * seg_cap / std::max(bucket, 1) + 4) >
                             200 * 1024)
    seg_cap >>= 1;
  // the last sorting level (depth-1) must be local: its segments hold <= 2*bucket points
  if (depth > 0 && 2 * bucket > seg_cap)
    return fail(HM_ERR_UNSUPPORTED, "hm_kdtree_build: bucket too large for this dimension");
  int j0 = 0;
  while (j0 < depth && (n + (1 << j0) - 1) / (1 << j0) > seg_cap) ++j0;
  if (depth > 0 && j0 > depth - 1) j0 = depth - 1;
  const int maxlen = (n + (1 << j0) - 1) >> j0;
  int pcap = 1;
  while (pcap < maxlen) pcap <<= 1;
  const int nlocal = depth - j0;

  hm_kdtree_s* t = new hm_kdtree_s();
  t->n = n;
  t->d = d;
  t->bucket = bucket;
  t->depth = depth;
  t->h_offsets = leaf_offsets(n, depth);
  const int nleaf = 1 << depth;
  const size_t nodes_all = (size_t)(2 * nleaf - 1);
  auto cleanup = [&](hm_status s) {
    delete t;
    return s;
  };
  hm_status s;
  if ((s = t->perm.alloc(n)) || (s = t->offsets.alloc(nleaf + 1)) ||
      (s = t->bmin.alloc(nodes_all * d)) || (s = t->bmax.alloc(nodes_all * d)) ||
      (s = t->split_dim.alloc(std::max(nleaf - 1, 1))) || (s = t->pts_tree.alloc((size_t)d * n)) ||
      (s = t->pts_tree_f.alloc((size_t)d * n)))
    return cleanup(s);

  DevBuf<int> idxA, idxB;
  DevBuf<double> coA, coB;
  if ((s = idxA.alloc_async(n, stream)) || (s = idxB.alloc_async(n, stream)) || (s = coA.alloc_async((size_t)d * n, stream)) ||
      (s = coB.alloc_async((size_t)d * n, stream)))
    return cleanup(s);
  auto cu = [&](cudaError_t e, const char* what) -> hm_status {
    if (e != cudaSuccess) return cuda_fail(e, what, __FILE__, __LINE__);
    return HM_OK;
  };
  if ((s = cu(cudaMemcpyAsync(t->offsets.p, t->h_offsets.data(), sizeof(int) * (nleaf + 1),
                              cudaMemcpyHostToDevice, stream),
              "offsets upload")))
    return cleanup(s);
  if ((s = cu(cudaMemcpyAsync(coA.p, d_points, sizeof(double) * (size_t)d * n,
                              cudaMemcpyDeviceToDevice, stream),
              "points copy")))
    return cleanup(s);
  k_iota<<<std::min((n + 255) / 256, 4096), 256, 0, stream>>>(n, idxA.p);
  if ((s = cu(cudaGetLastError(), "k_iota"))) return cleanup(s);

  if (j0 > 0) {
    const int maxw = depth + 2;
    const int nseg_max = 1 << (j0 - 1);
    const size_t wide_nodes = (size_t)((1 << j0) - 1);
    DevBuf<unsigned long long> bmin_tw, bmax_tw, chosen;
    DevBuf<SelState> st;
    DevBuf<unsigned int> hist;
    DevBuf<int> cursor, notdone, err;
    if ((s = bmin_tw.alloc(wide_nodes * d)) || (s = bmax_tw.alloc(wide_nodes * d)) ||
        (s = chosen.alloc((size_t)nseg_max * maxw)) || (s = st.alloc(nseg_max)) ||
        (s = hist.alloc((size_t)nseg_max * 256)) || (s = cursor.alloc(2 * (size_t)nseg_max)) ||
        (s = notdone.alloc(1)) || (s = err.alloc(1)))
      return cleanup(s);
    if ((s = cu(cudaMemsetAsync(bmin_tw.p, 0xff, bmin_tw.n * 8, stream), "memset")) ||
        (s = cu(cudaMemsetAsync(bmax_tw.p, 0, bmax_tw.n * 8, stream), "memset")) ||
        (s = cu(cudaMemsetAsync(hist.p, 0, hist.n * 4, stream), "memset")) ||
        (s = cu(cudaMemsetAsync(err.p, 0, 4, stream), "memset")))
      return cleanup(s);
    k_root_box<<<std::min((n + 255) / 256, 1024), 256, 0, stream>>>(n, d, d_points, bmin_tw.p,
                                                                     bmax_tw.p);
    if ((s = cu(cudaGetLastError(), "k_root_box"))) return cleanup(s);

    for (int level = 0; level < j0; ++level) {
      const int nseg = 1 << level;
      const int maxlen_l = (n + nseg - 1) / nseg;
      WideArgs a;
      a.n = n;
      a.d = d;
      a.level = level;
      a.depth = depth;
      a.leaf_off = t->offsets.p;
      a.split_dim = t->split_dim.p;
      a.idx = idxA.p;
      a.coord = coA.p;
      a.st = st.p;
      a.chosen = chosen.p;
      a.maxw = maxw;
      a.hist = hist.p;
      a.cps = (maxlen_l + kChunk - 1) / kChunk;
      a.err = err.p;
      k_select_init<<<(nseg + 127) / 128, 128, 0, stream>>>(a, bmin_tw.p, bmax_tw.p,
                                                             t->split_dim.p);
      if ((s = cu(cudaGetLastError(), "k_select_init"))) return cleanup(s);
      const int max_passes = 8 * (level + 2) + 8;
      int passes = 0;
      for (;;) {
        for (int b = 0; b < kPassesPerBatch; ++b) {
          // count the segments still active after the batch's last pass only
          if (b == kPassesPerBatch - 1 &&
              (s = cu(cudaMemsetAsync(notdone.p, 0, 4, stream), "memset")))
            return cleanup(s);
          k_hist<<<nseg * a.cps, kWideThreads, 0, stream>>>(a);
          k_select<<<(nseg * 32 + 255) / 256, 256, 0, stream>>>(a, notdone.p);
        }
        passes += kPassesPerBatch;
        if ((s = cu(cudaGetLastError(), "k_hist/k_select"))) return cleanup(s);
        int h_notdone = 0;
        if ((s = cu(cudaMemcpyAsync(&h_notdone, notdone.p, 4, cudaMemcpyDeviceToHost, stream),
                    "notdone readback")) ||
            (s = cu(cudaStreamSynchronize(stream), "sync")))
          return cleanup(s);
        if (h_notdone == 0) break;
        if (passes >= max_passes)
          return cleanup(fail(HM_ERR_INVALID, "hm_kdtree_build: selection did not converge "
                                              "(NaN coordinates?)"));
      }
      PartArgs p;
      p.w = a;
      p.idx_out = idxB.p;
      p.coord_out = coB.p;
      p.cursor = cursor.p;
      const bool child_boxes = level + 1 < j0;
      p.cmin_tw = child_boxes ? bmin_tw.p : nullptr;
      p.cmax_tw = child_boxes ? bmax_tw.p : nullptr;
      p.err = err.p;
      if ((s = cu(cudaMemsetAsync(cursor.p, 0, sizeof(int) * 2 * nseg, stream), "memset")))
        return cleanup(s);
      if (d <= 4)
        k_partition<4><<<nseg * a.cps, kWideThreads, 0, stream>>>(p);
      else
        k_partition<kMaxDim><<<nseg * a.cps, kWideThreads, 0, stream>>>(p);
      if ((s = cu(cudaGetLastError(), "k_partition"))) return cleanup(s);
      std::swap(idxA.p, idxB.p);
      std::swap(coA.p, coB.p);
    }
    k_untwiddle<<<64, 256, 0, stream>>>(wide_nodes * d, bmin_tw.p, t->bmin.p);
    k_untwiddle<<<64, 256, 0, stream>>>(wide_nodes * d, bmax_tw.p, t->bmax.p);
    if ((s = cu(cudaGetLastError(), "k_untwiddle"))) return cleanup(s);
    // the device buffers above are freed at scope exit: make sure the GPU is
    // done with them first
    int h_err = 0;
    if ((s = cu(cudaMemcpyAsync(&h_err, err.p, 4, cudaMemcpyDeviceToHost, stream), "err")) ||
        (s = cu(cudaStreamSynchronize(stream), "sync")))
      return cleanup(s);
    if (h_err)
      return cleanup(fail(HM_ERR_INVALID, "hm_kdtree_build: inconsistent split (NaN input?)"));
  }

  LocalArgs la;
  la.n = n;
  la.d = d;
  la.depth = depth;
  la.j0 = j0;
  la.seg_cap = pcap;
  la.pcap = pcap;
  la.leaf_off = t->offsets.p;
  la.idx = idxA.p;
  la.coord = coA.p;
  la.split_dim = t->split_dim.p;
  la.bmin = t->bmin.p;
  la.bmax = t->bmax.p;
  la.perm = t->perm.p;
  la.pts_tree = t->pts_tree.p;
  la.pts_tree_f = t->pts_tree_f.p;
  size_t smem = local_smem_bytes(d, pcap, pcap, nlocal);
  if ((s = cu(cudaFuncSetAttribute(k_local, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem),
              "cudaFuncSetAttribute")))
    return cleanup(s);
  k_local<<<1 << j0, kLocalThreads, smem, stream>>>(la);
  if ((s = cu(cudaGetLastError(), "k_local"))) return cleanup(s);
  if ((s = cu(cudaStreamSynchronize(stream), "sync"))) return cleanup(s);
  *out = t;
  return HM_OK;
}

}  // namespace hm
