/* Minimal CBLAS declarations for building the reference CPU path as the oracle.
 *
 * The reference includes <cblas.h> inside an extern "C" block and uses only
 * cblas_dgemm (setup-time coordinate/Jacobian products and triangle operator
 * construction) and cblas_dgemv.  No BLAS library exists in this image, so the
 * definitions live in ref_shim.cpp.  Test infrastructure only: nothing in the
 * product links this. */
#ifndef ORACLE_SHIM_CBLAS_H
#define ORACLE_SHIM_CBLAS_H

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);

void cblas_dgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE t, int m, int n,
                 double alpha, const double *a, int lda, const double *x, int incx,
                 double beta, double *y, int incy);

#endif
