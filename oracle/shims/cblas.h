// Project-written stand-in for the few CBLAS routines the reference's
// array.hpp calls when built with COMPMATMUL_USE_OPENBLAS
// (array.hpp:48,65,90,190,204,307): cblas_dscal, cblas_daxpy, cblas_dgemm,
// cblas_dimatcopy.  No BLAS is installed in this image.  Test
// infrastructure for the CPU oracle/baseline only; plain loops.
#ifndef CMM_SHIM_CBLAS_H
#define CMM_SHIM_CBLAS_H

#include <cstring>
#include <vector>

typedef int blasint;
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

inline void cblas_dscal(blasint n, double alpha, double* x, blasint incx) {
  for (blasint i = 0; i < n; ++i) x[(long)i * incx] *= alpha;
}

inline void cblas_daxpy(blasint n, double alpha, const double* x, blasint incx, double* y,
                        blasint incy) {
  for (blasint i = 0; i < n; ++i) y[(long)i * incy] += alpha * x[(long)i * incx];
}

// C = alpha op(A) op(B) + beta C, k-ordered sums, OpenMP over rows.
inline void cblas_dgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, blasint M,
                        blasint N, blasint K, double alpha, const double* A, blasint lda,
                        const double* B, blasint ldb, double beta, double* C, blasint ldc) {
  auto a = [&](long i, long k) {
    bool t = (ta != CblasNoTrans);
    if (order == CblasRowMajor) return t ? A[k * lda + i] : A[i * lda + k];
    return t ? A[i * lda + k] : A[k * lda + i];
  };
  auto b = [&](long k, long j) {
    bool t = (tb != CblasNoTrans);
    if (order == CblasRowMajor) return t ? B[j * ldb + k] : B[k * ldb + j];
    return t ? B[k * ldb + j] : B[j * ldb + k];
  };
#pragma omp parallel for schedule(static)
  for (long i = 0; i < M; ++i)
    for (long j = 0; j < N; ++j) {
      double s = 0.0;
      for (long k = 0; k < K; ++k) s += a(i, k) * b(k, j);
      double& c = (order == CblasRowMajor) ? C[i * ldc + j] : C[j * ldc + i];
      c = alpha * s + (beta == 0.0 ? 0.0 : beta * c);
    }
}

// In-place scaled transpose/copy; only the (alpha=1) transposes the
// reference's c_to_fortran/fortran_to_c use are meaningful here.
inline void cblas_dimatcopy(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, blasint rows,
                            blasint cols, double alpha, double* A, blasint lda, blasint ldb) {
  (void)lda; (void)ldb;
  std::vector<double> tmp(A, A + (long)rows * cols);
  if (trans == CblasNoTrans) {
    for (long i = 0; i < (long)rows * cols; ++i) A[i] = alpha * tmp[i];
    return;
  }
  // treat the input as rows x cols in the given order; write its transpose
  for (long i = 0; i < rows; ++i)
    for (long j = 0; j < cols; ++j) {
      if (order == CblasRowMajor) A[j * rows + i] = alpha * tmp[i * cols + j];
      else A[i * cols + j] = alpha * tmp[j * rows + i];
    }
}

#endif  // CMM_SHIM_CBLAS_H
