// The three CBLAS routines the reference calls (math_operations.cpp:40-42,
// 394-395), forwarded to OpenBLAS: the scipy-openblas build that numpy ships
// (OpenBLAS 0.3.x, 64-bit integers, symbols prefixed `scipy_` and suffixed
// `64_`).  This gives the timed CPU baseline the BLAS library the reference's
// build names (OpenBLAS) instead of the ordered loops of cblas_ordered.cpp.
// Test infrastructure only: OpenBLAS orders its sums its own way, so parity
// is never pinned on this build.
#include "cblas.h"

#include <cstdint>

extern "C" {

// scipy-openblas (ILP64) entry points, standard CBLAS enums.
void scipy_cblas_sgemm64_(int order, int transa, int transb, int64_t m, int64_t n, int64_t k,
                          float alpha, const float *a, int64_t lda, const float *b, int64_t ldb,
                          float beta, float *c, int64_t ldc);
void scipy_cblas_saxpy64_(int64_t n, float alpha, const float *x, int64_t incx, float *y,
                          int64_t incy);
float scipy_cblas_snrm264_(int64_t n, const float *x, int64_t incx);

void cblas_sgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const float alpha, const float *A, const int lda, const float *B,
                 const int ldb, const float beta, float *C, const int ldc) {
  scipy_cblas_sgemm64_((int)Order, (int)TransA, (int)TransB, M, N, K, alpha, A, lda, B, ldb,
                       beta, C, ldc);
}

void cblas_saxpy(const int N, const float alpha, const float *X, const int incX, float *Y,
                 const int incY) {
  scipy_cblas_saxpy64_(N, alpha, X, incX, Y, incY);
}

float cblas_snrm2(const int N, const float *X, const int incX) {
  return scipy_cblas_snrm264_(N, X, incX);
}

}  // extern "C"
