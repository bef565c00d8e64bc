/*
 * cpu_baseline.c -- the CPU path the GPU engine is timed against: dense FP64
 * kernel-matrix generation (a host restatement of `interaction`,
 * src/TLRMatrixHelpers.cu:44-58, generalised to the workloads' kernels) followed
 * by an OpenBLAS dgemm/dgemv, one row panel at a time.
 *
 * TEST / BENCHMARK INFRASTRUCTURE ONLY (bench.py's CPU-baseline leg and tests).
 * OpenBLAS is the copy shipped with scipy; its path is passed in and opened
 * with dlopen (there is no cblas.h in this image, so the two prototypes used
 * are declared here).
 */
#include <dlfcn.h>
#include <math.h>
#include <omp.h>
#include <stddef.h>
#include <stdlib.h>
#include <time.h>

double orc_kernel_r2(int kind, int deriv, double r2, double ell);

typedef void (*dgemm_fn)(int order, int ta, int tb, int m, int n, int k, double alpha,
                         const double* a, int lda, const double* b, int ldb, double beta,
                         double* c, int ldc);
typedef void (*dgemv_fn)(int order, int ta, int m, int n, double alpha, const double* a, int lda,
                         const double* x, int incx, double beta, double* y, int incy);
typedef void (*setthr_fn)(int);

static void* g_blas = NULL;
static dgemm_fn g_dgemm = NULL;
static dgemv_fn g_dgemv = NULL;
static setthr_fn g_setthr = NULL;

/* returns 0 on success */
int orc_blas_open(const char* path, int threads) {
  if (!g_blas) {
    g_blas = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!g_blas) return 1;
    g_dgemm = (dgemm_fn)dlsym(g_blas, "scipy_cblas_dgemm");
    g_dgemv = (dgemv_fn)dlsym(g_blas, "scipy_cblas_dgemv");
    g_setthr = (setthr_fn)dlsym(g_blas, "scipy_openblas_set_num_threads");
    if (!g_dgemm || !g_dgemv) return 2;
  }
  if (g_setthr) g_setthr(threads);
  omp_set_num_threads(threads);
  return 0;
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/*
 * Y(nrows x nrhs, ld nrows) = A(row0:row0+nrows, :) X, A(i, j) = K(p[perm[i]],
 * p[perm[j]]) + nugget*[i==j], X column-major n x nrhs (ld n), tree order.
 * The panel is generated into `work` (nrows*n doubles, column-major) with
 * `threads` OpenMP threads, then multiplied by OpenBLAS.  Seconds spent in each
 * part are returned through t_gen / t_blas.
 */
int orc_cpu_panel_matvec(int n, int d, const double* pts, const int* perm, int kind, double ell,
                         double nugget, int row0, int nrows, int nrhs, const double* X, double* Y,
                         double* work, double* t_gen, double* t_blas) {
  if (!g_dgemm) return 1;
  double t0 = now_s();
#pragma omp parallel for schedule(static)
  for (int j = 0; j < n; ++j) {
    int pj = perm[j];
    double* col = work + (size_t)j * nrows;
    for (int i = 0; i < nrows; ++i) {
      int pi = perm[row0 + i];
      double r2 = 0;
      for (int k = 0; k < d; ++k) {
        double t = pts[(size_t)k * n + pj] - pts[(size_t)k * n + pi];
        r2 += t * t;
      }
      double v = orc_kernel_r2(kind, 0, r2, ell);
      if (pi == pj) v += nugget;
      col[i] = v;
    }
  }
  double t1 = now_s();
  if (nrhs == 1)
    g_dgemv(102 /*col major*/, 111 /*no trans*/, nrows, n, 1.0, work, nrows, X, 1, 0.0, Y, 1);
  else
    g_dgemm(102, 111, 111, nrows, nrhs, n, 1.0, work, nrows, X, n, 0.0, Y, nrows);
  double t2 = now_s();
  *t_gen = t1 - t0;
  *t_blas = t2 - t1;
  return 0;
}
