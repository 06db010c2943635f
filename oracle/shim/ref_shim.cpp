/* Definitions behind the oracle's shim headers (test infrastructure only).
 *
 *  - cblas_dgemm / cblas_dgemv: plain triple-loop BLAS, summing k in
 *    ascending order.  The reference calls them at setup time only
 *    (src/elements.cpp:365-387, 712-743, 863-868).
 *  - gimmik_mm_cpu: stand-in for the generated GiMMiK CPU kernels that are
 *    missing from the reference tree (declared include/gimmik.h:5-13).
 *    GiMMiK bakes a constant operator A into an unrolled C = A*B (+C) and
 *    drops the zero entries of A; this stand-in computes the same product
 *    with a runtime A, also skipping exact zeros, summing k in ascending
 *    order.  Results agree with GiMMiK's up to floating-point summation order.
 */
#include <cstddef>

extern "C" {
#include "cblas.h"
}
#include "H5Cpp.h"

const PredType PredType::NATIVE_DOUBLE;
const PredType PredType::NATIVE_INT;
const PredType PredType::NATIVE_INT8;
const PredType PredType::NATIVE_SHORT;

namespace {

inline double op_elem(const double *m, int ld, int row, int col, bool row_major, bool trans)
{
  /* element (row, col) of op(M) */
  if (trans) { int t = row; row = col; col = t; }
  return row_major ? m[(size_t)row * ld + col] : m[(size_t)col * ld + row];
}

}  // namespace

extern "C" void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                            int m, int n, int k, double alpha, const double *a, int lda,
                            const double *b, int ldb, double beta, double *c, int ldc)
{
  const bool rm = (order == CblasRowMajor);
  const bool at = (ta != CblasNoTrans);
  const bool bt = (tb != CblasNoTrans);
  for (int i = 0; i < m; i++)
    for (int j = 0; j < n; j++)
    {
      double s = 0.0;
      for (int p = 0; p < k; p++)
        s += op_elem(a, lda, i, p, rm, at) * op_elem(b, ldb, p, j, rm, bt);
      double &cij = rm ? c[(size_t)i * ldc + j] : c[(size_t)j * ldc + i];
      cij = (beta == 0.0 ? 0.0 : beta * cij) + alpha * s;
    }
}

extern "C" void cblas_dgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE t, int m, int n,
                            double alpha, const double *a, int lda, const double *x, int incx,
                            double beta, double *y, int incy)
{
  const bool rm = (order == CblasRowMajor);
  const bool tr = (t != CblasNoTrans);
  const int rows = tr ? n : m;
  const int cols = tr ? m : n;
  for (int i = 0; i < rows; i++)
  {
    double s = 0.0;
    for (int p = 0; p < cols; p++)
      s += op_elem(a, lda, i, p, rm, tr) * x[(size_t)p * incx];
    double &yi = y[(size_t)i * incy];
    yi = (beta == 0.0 ? 0.0 : beta * yi) + alpha * s;
  }
}

extern "C" void gimmik_mm_cpu(int m, int n, int k, const double alpha, const double *a, int lda,
                              const double *b, int ldb, const double beta, double *c, int ldc,
                              unsigned long /*operator id*/)
{
  const int kBlock = 256;
#pragma omp parallel for schedule(static)
  for (int j0 = 0; j0 < n; j0 += kBlock)
  {
    const int j1 = (j0 + kBlock < n) ? j0 + kBlock : n;
    double acc[kBlock];
    for (int i = 0; i < m; i++)
    {
      for (int j = j0; j < j1; j++) acc[j - j0] = 0.0;
      for (int p = 0; p < k; p++)
      {
        const double av = a[(size_t)i * lda + p];
        if (av == 0.0) continue;
        const double *brow = b + (size_t)p * ldb;
        for (int j = j0; j < j1; j++) acc[j - j0] += av * brow[j];
      }
      double *crow = c + (size_t)i * ldc;
      for (int j = j0; j < j1; j++)
        crow[j] = (beta == 0.0 ? 0.0 : beta * crow[j]) + alpha * acc[j - j0];
    }
  }
}
