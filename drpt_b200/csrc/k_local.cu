// K5 -- positional local split (MDRPT::grow_local_trees, mdrpt.cpp:321-400,
// with DRPTLocal, drpt_local.cpp:49-180).  The reference's local projection
// matrix is all zero (its density parameter is an int and truncates to 0), so
// every local split runs std::nth_element on equal keys and the resulting
// final leaves are a fixed permutation of the global leaf's positions that
// depends only on the leaf size.  The host computes that permutation once
// per distinct size with the same standard library; this kernel applies it.
// Final leaf id of local leaf l of global leaf j is j * 2^ld + l
// (mdrpt.cpp:390-392 at one rank).
#include "kernels.cuh"

namespace drpt {
namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_local(LocalArgs a) {
  const int t = blockIdx.x / a.nleaf, j = blockIdx.x - t * a.nleaf;
  const int32_t *goff = a.goff + (int64_t)t * (a.nleaf + 1);
  const int32_t b = goff[j], sz = goff[j + 1] - b;
  const int32_t *perm = a.pool + a.perm_base[(int64_t)t * a.nleaf + j];
  const int32_t *first = a.pool + a.first_base[(int64_t)t * a.nleaf + j];
  const int32_t *src = a.order + (int64_t)t * a.n + b;
  int32_t *dst = a.final_order + (int64_t)t * a.n + b;
  for (int q = threadIdx.x; q < sz; q += kThreads) dst[q] = __ldg(src + __ldg(perm + q));
  const int nl = 1 << a.ld;
  int32_t *fo = a.final_off + (int64_t)t * ((int64_t)a.nleaf * nl + 1);
  for (int l = threadIdx.x; l < nl; l += kThreads) fo[(int64_t)j * nl + l] = b + first[l];
  if (threadIdx.x == 0 && j == a.nleaf - 1) fo[(int64_t)a.nleaf * nl] = b + sz;
}

}  // namespace

drpt_status launch_local(const LocalArgs &a, cudaStream_t s) {
  const int64_t blocks = (int64_t)a.T * a.nleaf;
  if (blocks <= 0) return DRPT_OK;
  k_local<<<(unsigned)blocks, kThreads, 0, s>>>(a);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt
