// Deterministic CBLAS subset for the reference build (test infrastructure).
//
// Summation order, which the GPU parity kernels reproduce bit for bit:
//  * sgemm: every C[i][j] is acc = 0.0f; for k = 0..K-1 ascending:
//    acc = acc + op(A)[i][k] * op(B)[k][j] (one rounded multiply, one rounded
//    add; this file is compiled with -ffp-contract=off); then
//    C = alpha * acc (+ beta * C when beta != 0).
//    A term whose op(B) entry is zero is skipped: for a finite op(A) entry it
//    adds +-0 to an accumulator that starts at +0 and therefore never becomes
//    -0, so skipping it leaves every bit of C unchanged.  When op(A) holds a
//    non-finite value nothing is skipped.
//    Rows of C are split over OpenMP threads; each element keeps its order, so
//    the result does not depend on the thread count.
//  * saxpy: y[i] = alpha * x[i] + y[i], rounded multiply then rounded add.
//  * snrm2: s = 0.0f; s = s + x[i] * x[i] ascending; return sqrtf(s).
// OpenBLAS (the reference's real dependency, version unpinned) may order these
// differently; parity is pinned to this order.
#include "cblas.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

extern "C" {

void cblas_sgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const float alpha, const float *A, const int lda, const float *B,
                 const int ldb, const float beta, float *C, const int ldc) {
  if (Order != CblasRowMajor) {
    std::fprintf(stderr, "cblas_ordered: only CblasRowMajor is implemented\n");
    std::abort();
  }
  if (M <= 0 || N <= 0) return;
  const bool ta = TransA != CblasNoTrans, tb = TransB != CblasNoTrans;
  auto a_at = [&](long i, long k) -> float { return ta ? A[k * lda + i] : A[i * lda + k]; };
  auto b_at = [&](long k, long j) -> float { return tb ? B[j * ldb + k] : B[k * ldb + j]; };

  bool a_finite = true;
  if (K > 0) {
    const long total = (long)(ta ? K : M) * (long)lda;
    for (long t = 0; t < total && a_finite; ++t) a_finite = std::isfinite(A[t]);
  }
  // Per k, the columns j whose op(B)[k][j] takes part in the sum.
  std::vector<std::vector<int>> cols(K > 0 ? K : 0);
  for (int k = 0; k < K; ++k)
    for (int j = 0; j < N; ++j)
      if (!a_finite || b_at(k, j) != 0.0f) cols[k].push_back(j);

  const int RB = 64;  // rows of C accumulated together
#pragma omp parallel for schedule(dynamic, 1)
  for (int i0 = 0; i0 < M; i0 += RB) {
    const int rb = (M - i0) < RB ? (M - i0) : RB;
    std::vector<float> acc((size_t)rb * N, 0.0f);
    for (int k = 0; k < K; ++k) {
      const std::vector<int> &cj = cols[k];
      if (cj.empty()) continue;
      for (int r = 0; r < rb; ++r) {
        const float a = a_at(i0 + r, k);
        float *row = &acc[(size_t)r * N];
        for (int j : cj) {
          const float prod = a * b_at(k, j);
          row[j] = row[j] + prod;
        }
      }
    }
    for (int r = 0; r < rb; ++r)
      for (int j = 0; j < N; ++j) {
        float *c = &C[(long)(i0 + r) * ldc + j];
        const float v = alpha * acc[(size_t)r * N + j];
        *c = (beta == 0.0f) ? v : v + beta * (*c);
      }
  }
}

void cblas_saxpy(const int N, const float alpha, const float *X, const int incX, float *Y,
                 const int incY) {
  for (int i = 0; i < N; ++i) {
    const float prod = alpha * X[(long)i * incX];
    Y[(long)i * incY] = prod + Y[(long)i * incY];
  }
}

float cblas_snrm2(const int N, const float *X, const int incX) {
  float s = 0.0f;
  for (int i = 0; i < N; ++i) {
    const float x = X[(long)i * incX];
    const float sq = x * x;
    s = s + sq;
  }
  return std::sqrt(s);
}

}  // extern "C"
