/*
 * CBLAS forwarder for the reference build -- TEST INFRASTRUCTURE ONLY.
 * refshim_set_blas(path, threads) dlopens an OpenBLAS that exports the
 * scipy_-prefixed CBLAS names (scipy's bundled libscipy_openblas) and routes
 * cblas_dgemv / cblas_dznrm2 there; without it, plain column-major loops with
 * BLAS semantics are used.
 */
#include <dlfcn.h>
#include <math.h>
#include <stddef.h>
#include "cblas.h"

typedef void (*dgemv_t)(int, int, int, int, double, const double *, int,
                        const double *, int, double, double *, int);
typedef double (*dznrm2_t)(int, const void *, int);
typedef void (*setthr_t)(int);
static dgemv_t p_dgemv = NULL;
static dznrm2_t p_dznrm2 = NULL;
static setthr_t p_setthr = NULL;

int refshim_set_blas(const char *path, int threads) {
  if (!path) { p_dgemv = NULL; p_dznrm2 = NULL; return 0; }
  void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return -1;
  p_dgemv = (dgemv_t)dlsym(h, "scipy_cblas_dgemv");
  p_dznrm2 = (dznrm2_t)dlsym(h, "scipy_cblas_dznrm2");
  p_setthr = (setthr_t)dlsym(h, "scipy_openblas_set_num_threads");
  if (!p_dgemv || !p_dznrm2) { p_dgemv = NULL; p_dznrm2 = NULL; return -2; }
  if (p_setthr && threads > 0) p_setthr(threads);
  return 0;
}

void cblas_dgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE trans, int M,
                 int N, double alpha, const double *A, int lda,
                 const double *X, int incX, double beta, double *Y, int incY) {
  if (p_dgemv) {
    p_dgemv((int)order, (int)trans, M, N, alpha, A, lda, X, incX, beta, Y, incY);
    return;
  }
  /* column-major only (the reference uses CblasColMajor throughout) */
  if (trans == CblasNoTrans) {
    for (int i = 0; i < M; ++i) {
      double acc = 0.0;
      for (int j = 0; j < N; ++j) acc += A[(size_t)j * lda + i] * X[(size_t)j * incX];
      double *y = &Y[(size_t)i * incY];
      *y = (beta == 0.0) ? alpha * acc : beta * *y + alpha * acc;
    }
  } else {
    for (int j = 0; j < N; ++j) {
      double acc = 0.0;
      for (int i = 0; i < M; ++i) acc += A[(size_t)j * lda + i] * X[(size_t)i * incX];
      double *y = &Y[(size_t)j * incY];
      *y = (beta == 0.0) ? alpha * acc : beta * *y + alpha * acc;
    }
  }
}

double cblas_dznrm2(int N, const void *X, int incX) {
  if (p_dznrm2) return p_dznrm2(N, X, incX);
  const double *x = (const double *)X;
  double s = 0.0;
  for (int i = 0; i < N; ++i) {
    double re = x[(size_t)2 * i * incX], im = x[(size_t)2 * i * incX + 1];
    s += re * re + im * im;
  }
  return sqrt(s);
}
