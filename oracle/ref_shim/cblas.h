/*
 * Stand-in for <cblas.h> -- TEST INFRASTRUCTURE ONLY.  Declares the two CBLAS
 * routines the reference's src/tdse/tdse.cpp calls (cblas_dgemv, :28-68 and
 * :99-139; cblas_dznrm2, :194 and :277) with the standard CBLAS prototypes.
 * cblas_shim.c implements them by forwarding to an OpenBLAS loaded at run
 * time (refshim_set_blas), or with plain loops when none is loaded.
 */
#ifndef REFSHIM_CBLAS_H_
#define REFSHIM_CBLAS_H_
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
void cblas_dgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE trans, int M,
                 int N, double alpha, const double *A, int lda,
                 const double *X, int incX, double beta, double *Y, int incY);
double cblas_dznrm2(int N, const void *X, int incX);
#endif
