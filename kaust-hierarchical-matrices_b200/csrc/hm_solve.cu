// hm_solve.cu -- conjugate gradients on the H-matrix: H X = B for a symmetric
// positive definite kernel matrix (a kernel with a nugget on its diagonal, as
// in kernel ridge regression or a Gaussian-process solve).  The reference has
// no solver; this is the operator's natural consumer, built on hm_hmatvec.
//
// One CG per right-hand side, all columns advancing together so that each
// iteration is one product over every column.  X, R, P and A P are FP32; the
// dot products are summed in FP64, in a fixed order (per-block partials, then
// one thread per column), so a solve is reproducible.  The scalars alpha and
// beta live on the device: a chunk of `check_every` iterations needs no host
// synchronisation, and on a created stream it is recorded once into a CUDA
// graph and relaunched.  Between chunks the host reads the residual norms
// and stops when every column meets the tolerance.  A column that meets the
// tolerance (a zero residual or right-hand side included) stops moving at
// once, on the device, while the others go on.
#include <algorithm>
#include <cmath>
#include <vector>

#include "hm_hmatrix.h"

namespace hm {
namespace {

constexpr int kCgThreads = 256;
constexpr int kCgBlocks = 296;  // partial sums per column (2 per SM)

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  v = 0.0;
  if (threadIdx.x < 32) {
    v = threadIdx.x < (int)(blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;  // valid in thread 0
}

// R = P = B, X = 0; part = partial sums of B . B
__global__ void __launch_bounds__(kCgThreads) k_cg_init(const float* __restrict__ B, int ldb, float* __restrict__ X,
                                                        int ldx, float* __restrict__ R, float* __restrict__ P, int n,
                                                        double* __restrict__ part) {
  __shared__ double sh[kCgThreads / 32];
  const int c = blockIdx.y;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float b = B[(size_t)c * ldb + i];
    R[(size_t)c * n + i] = b;
    P[(size_t)c * n + i] = b;
    X[(size_t)c * ldx + i] = 0.f;
    s += (double)b * b;
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[(size_t)c * gridDim.x + blockIdx.x] = s;
}

// part = partial sums of P . AP
__global__ void __launch_bounds__(kCgThreads) k_cg_dot(const float* __restrict__ P, const float* __restrict__ AP, int n,
                                                       double* __restrict__ part) {
  __shared__ double sh[kCgThreads / 32];
  const int c = blockIdx.y;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += (double)P[(size_t)c * n + i] * AP[(size_t)c * n + i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[(size_t)c * gridDim.x + blockIdx.x] = s;
}

// Per column, the sum of its partials, in block order.  which: 0 start
// (bb = rr = sum), 1 alpha (sum = p.Ap), 2 beta (sum = new r.r).
// sc: [bb | rr | alpha | beta], nrhs doubles each.  A column that has met the
// tolerance (rr <= tol2 bb) is frozen: alpha = beta = 0, so X and R stay as
// they are, and its p.Ap (rounding noise by then, of either sign) is not
// taken as a sign that the operator is indefinite.
__global__ void k_cg_scalars(const double* __restrict__ part, int nblk, int nrhs, int which, double tol2,
                             double* __restrict__ sc, int* __restrict__ breakdown) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nrhs) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[(size_t)c * nblk + b];
  double* bb = sc;
  double* rr = sc + nrhs;
  double* al = sc + 2 * nrhs;
  double* be = sc + 3 * nrhs;
  if (which == 0) {
    bb[c] = s;
    rr[c] = s;
  } else if (which == 1) {
    if (rr[c] <= tol2 * bb[c]) {
      al[c] = 0.0;  // met the tolerance (or a zero residual): frozen
    } else if (s > 0.0) {
      al[c] = rr[c] / s;
    } else {
      al[c] = 0.0;
      *breakdown = 1;  // p.Ap <= 0 on an unconverged column: the operator is not positive definite
    }
  } else {
    be[c] = (rr[c] > 0.0 && al[c] != 0.0) ? s / rr[c] : 0.0;
    rr[c] = s;
  }
}

// X += alpha P, R -= alpha AP; part = partial sums of the new R . R
__global__ void __launch_bounds__(kCgThreads) k_cg_update(float* __restrict__ X, int ldx, float* __restrict__ R,
                                                          const float* __restrict__ P, const float* __restrict__ AP,
                                                          int n, int nrhs, const double* __restrict__ sc,
                                                          double* __restrict__ part) {
  __shared__ double sh[kCgThreads / 32];
  const int c = blockIdx.y;
  const float a = (float)sc[2 * nrhs + c];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    X[(size_t)c * ldx + i] += a * P[(size_t)c * n + i];
    const float r = R[(size_t)c * n + i] - a * AP[(size_t)c * n + i];
    R[(size_t)c * n + i] = r;
    s += (double)r * r;
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[(size_t)c * gridDim.x + blockIdx.x] = s;
}

// P = R + beta P
__global__ void k_cg_dir(const float* __restrict__ R, float* __restrict__ P, int n, int nrhs,
                         const double* __restrict__ sc) {
  const int c = blockIdx.y;
  const float b = (float)sc[3 * nrhs + c];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    P[(size_t)c * n + i] = R[(size_t)c * n + i] + b * P[(size_t)c * n + i];
}

// part = partial sums of (B - AX) . (B - AX)
__global__ void __launch_bounds__(kCgThreads) k_cg_resid(const float* __restrict__ B, int ldb,
                                                         const float* __restrict__ AX, int n,
                                                         double* __restrict__ part) {
  __shared__ double sh[kCgThreads / 32];
  const int c = blockIdx.y;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double r = (double)B[(size_t)c * ldb + i] - AX[(size_t)c * n + i];
    s += r * r;
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[(size_t)c * gridDim.x + blockIdx.x] = s;
}

struct CgState {
  hm_hmatrix h;
  int n, nrhs, ldx;
  float *X, *R, *P, *AP;
  double *part, *sc;
  int* breakdown;
  unsigned nblk;
  double tol2;  // a column is done when r.r <= tol2 b.b
};

// one CG iteration, stream-ordered (no host synchronisation)
hm_status cg_iteration(const CgState& c, cudaStream_t s) {
  const dim3 grid(c.nblk, c.nrhs);
  HM_TRY(hm_hmatvec(c.h, 0, c.nrhs, c.P, c.n, c.AP, c.n, 0, s));
  k_cg_dot<<<grid, kCgThreads, 0, s>>>(c.P, c.AP, c.n, c.part);
  k_cg_scalars<<<(c.nrhs + 127) / 128, 128, 0, s>>>(c.part, c.nblk, c.nrhs, 1, c.tol2, c.sc, c.breakdown);
  k_cg_update<<<grid, kCgThreads, 0, s>>>(c.X, c.ldx, c.R, c.P, c.AP, c.n, c.nrhs, c.sc, c.part);
  k_cg_scalars<<<(c.nrhs + 127) / 128, 128, 0, s>>>(c.part, c.nblk, c.nrhs, 2, c.tol2, c.sc, c.breakdown);
  k_cg_dir<<<grid, kCgThreads, 0, s>>>(c.R, c.P, c.n, c.nrhs, c.sc);
  HM_LAUNCH_CHECK();
  return HM_OK;
}

}  // namespace
}  // namespace hm

extern "C" hm_status hm_cg_solve(hm_hmatrix h, int nrhs, const float* B, int ldb, float* X, int ldx, double tol,
                                 int max_iter, int check_every, void* stream, int* iterations,
                                 double* rel_residual) {
  using namespace hm;
  if (!h) return fail(HM_ERR_INVALID, "hm_cg_solve: null matrix");
  const int n = h->n;
  if (nrhs < 1 || !B || !X || ldb < n || ldx < n || !(tol > 0) || max_iter < 0 || check_every < 1)
    return fail(HM_ERR_INVALID,
                "hm_cg_solve: need nrhs >= 1, B and X with leading dimensions >= n, tol > 0, max_iter >= 0 and "
                "check_every >= 1");
  if (iterations) *iterations = 0;
  if (rel_residual) *rel_residual = 0.0;
  cudaStream_t s = as_stream(stream);
  const unsigned nblk = (unsigned)std::max(1, std::min(kCgBlocks, (n + kCgThreads - 1) / kCgThreads));
  const size_t vec = (size_t)n * nrhs;
  DevBuf<float> R, P, AP;
  DevBuf<double> part, sc;
  DevBuf<int> flag;
  HM_TRY(R.alloc_async(vec, s));
  HM_TRY(P.alloc_async(vec, s));
  HM_TRY(AP.alloc_async(vec, s));
  HM_TRY(part.alloc_async((size_t)nblk * nrhs, s));
  HM_TRY(sc.alloc_async((size_t)4 * nrhs, s));
  HM_TRY(flag.alloc_async(1, s));
  HM_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  CgState c{h, n, nrhs, ldx, X, R.p, P.p, AP.p, part.p, sc.p, flag.p, nblk, tol * tol};
  const dim3 grid(nblk, nrhs);
  k_cg_init<<<grid, kCgThreads, 0, s>>>(B, ldb, X, ldx, R.p, P.p, n, part.p);
  k_cg_scalars<<<(nrhs + 127) / 128, 128, 0, s>>>(part.p, nblk, nrhs, 0, c.tol2, sc.p, flag.p);
  HM_LAUNCH_CHECK();

  std::vector<double> hsc(2 * (size_t)nrhs);  // bb | rr
  int hflag = 0;
  auto converged = [&]() -> hm_status {
    HM_CUDA(cudaMemcpyAsync(hsc.data(), sc.p, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, s));
    HM_CUDA(cudaMemcpyAsync(&hflag, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    HM_CUDA(cudaStreamSynchronize(s));
    return HM_OK;
  };
  auto all_met = [&]() {
    for (int j = 0; j < nrhs; ++j)
      if (hsc[nrhs + j] > tol * tol * hsc[j]) return false;
    return true;
  };

  // a chunk of check_every iterations as one graph, when the stream can be captured
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  auto drop_graph = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  };
  if (s != nullptr && check_every > 1 && max_iter >= check_every) {
    HM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    hm_status st = HM_OK;
    for (int k = 0; k < check_every && st == HM_OK; ++k) st = cg_iteration(c, s);
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (st != HM_OK || ce != cudaSuccess) {
      drop_graph();
      cudaGetLastError();
      graph = nullptr;  // fall back to direct launches
    } else if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
      cudaGetLastError();
      drop_graph();
    }
  }

  int it = 0;
  hm_status st = converged();
  bool done = st == HM_OK && all_met();
  while (st == HM_OK && !done && it < max_iter) {
    const int k = std::min(check_every, max_iter - it);
    if (exec && k == check_every) {
      const cudaError_t e = cudaGraphLaunch(exec, s);
      if (e != cudaSuccess) st = cuda_fail(e, "cudaGraphLaunch", __FILE__, __LINE__);
    } else {
      for (int j = 0; j < k && st == HM_OK; ++j) st = cg_iteration(c, s);
    }
    it += k;
    if (st == HM_OK) st = converged();
    if (st == HM_OK && hflag) {
      drop_graph();
      if (iterations) *iterations = it;
      return fail(HM_ERR_UNSUPPORTED,
                  "hm_cg_solve: p.Ap <= 0 after " + std::to_string(it) +
                      " iterations: the H-matrix is not positive definite (add a nugget, or tighten the "
                      "compression tolerance)");
    }
    done = st == HM_OK && all_met();
  }
  drop_graph();
  if (st != HM_OK) return st;

  // the true residual ||B - H X|| / ||B||, worst column
  HM_TRY(hm_hmatvec(h, 0, nrhs, X, ldx, AP.p, n, 0, s));
  k_cg_resid<<<grid, kCgThreads, 0, s>>>(B, ldb, AP.p, n, part.p);
  HM_LAUNCH_CHECK();
  std::vector<double> hp((size_t)nblk * nrhs);
  HM_CUDA(cudaMemcpyAsync(hp.data(), part.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, s));
  HM_CUDA(cudaStreamSynchronize(s));
  double worst = 0.0;
  for (int j = 0; j < nrhs; ++j) {
    double r2 = 0.0;
    for (unsigned b = 0; b < nblk; ++b) r2 += hp[(size_t)j * nblk + b];
    if (hsc[j] > 0.0) worst = std::max(worst, std::sqrt(r2 / hsc[j]));
  }
  if (iterations) *iterations = it;
  if (rel_residual) *rel_residual = worst;
  if (!done)
    return fail(HM_ERR_NOT_CONVERGED, "hm_cg_solve: " + std::to_string(max_iter) +
                                          " iterations did not reach the tolerance (worst relative residual " +
                                          std::to_string(worst) + ")");
  return HM_OK;
}
