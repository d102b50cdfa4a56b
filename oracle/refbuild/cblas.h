/*
 * The three CBLAS routines the reference calls (math_operations.cpp:40-42,
 * 394-395), declared with the standard CBLAS signatures.  They are implemented
 * by cblas_ordered.cpp with one fixed, documented summation order so that the
 * reference build is deterministic.  Test infrastructure only.
 */
#ifndef DRPT_ORACLE_CBLAS_ORDERED_H
#define DRPT_ORACLE_CBLAS_ORDERED_H

#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

void cblas_sgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const float alpha, const float *A, const int lda, const float *B,
                 const int ldb, const float beta, float *C, const int ldc);

void cblas_saxpy(const int N, const float alpha, const float *X, const int incX, float *Y,
                 const int incY);

float cblas_snrm2(const int N, const float *X, const int incX);

#ifdef __cplusplus
}
#endif

#endif
