// Out-of-sample queries against the trees of a built index (no reference
// counterpart: the reference stores its splits, drpt_global.cpp:290 and
// drpt_local.cpp:142-155, but never reads them back).
//
//   Q1 k_descend  per (query, tree): walk the heap from the root with the
//                 query's projected values and the stored node medians,
//                 `value <= median` going left as in the build
//                 (drpt_global.cpp:308); ends at a global leaf
//   Q2 k_query    per query one warp: the members of its leaf in every tree,
//                 32 at a time (one per lane), exact FP32 distances
//                 (sequential fused multiply-adds over the dimensions,
//                 square root), a warp-wide list of the k best by
//                 (distance, id): a batch that beats the k-th is sorted
//                 with a shuffle bitonic network and merged into the list;
//                 members already in the list are skipped, so a point found
//                 in several trees counts once
#include "kernels.cuh"

namespace drpt {
namespace {

__global__ void k_descend(const float *__restrict__ Pq, int64_t nq, int T, int gd,
                          const float *__restrict__ medians, int32_t *__restrict__ leaf) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nq * T) return;
  const int64_t q = e / T;
  const int t = (int)(e - q * T);
  const int nleaf = 1 << (gd - 1);
  const float *med = medians + (int64_t)t * (nleaf - 1);
  int node = 0;  // heap index; children of h are 2h+1 (left), 2h+2 (right)
  for (int l = 0; l + 1 < gd; ++l) {
    const float v = Pq[((int64_t)t * (gd - 1) + l) * nq + q];
    node = 2 * node + 1 + ((v <= __ldg(med + node)) ? 0 : 1);
  }
  leaf[e] = node - (nleaf - 1);
}

__device__ __forceinline__ bool qbefore(float da, int32_t ia, float db, int32_t ib) {
  return da < db || (da == db && (uint32_t)ia < (uint32_t)ib);
}

// Bitonic sort of 32 (d, id) pairs held one per lane, ascending.
__device__ __forceinline__ void warp_sort32(float &d, int32_t &id, int lane) {
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const float od = __shfl_xor_sync(kFull, d, stride);
      const int32_t oi = __shfl_xor_sync(kFull, id, stride);
      const bool up = (lane & size) == 0 || size == 32;
      const bool lower = (lane & stride) == 0;
      const bool mine_first = qbefore(d, id, od, oi);
      const bool keep = (lower == up) ? mine_first : !mine_first;
      if (!keep) {
        d = od;
        id = oi;
      }
    }
}

template <typename T>
__device__ __forceinline__ float4 ld4(const T *p);
template <>
__device__ __forceinline__ float4 ld4<float>(const float *p) {
  return __ldg(reinterpret_cast<const float4 *>(p));
}
template <>
__device__ __forceinline__ float4 ld4<uint8_t>(const uint8_t *p) {
  const uchar4 v = __ldg(reinterpret_cast<const uchar4 *>(p));
  return make_float4(v.x, v.y, v.z, v.w);
}

template <typename T, typename TQ>
__global__ void __launch_bounds__(256) k_query(const T *__restrict__ X, int d, int64_t n,
                                               const TQ *__restrict__ Qx, int64_t nq, int T_,
                                               const int32_t *__restrict__ order,
                                               const int32_t *__restrict__ goff, int nleaf,
                                               const int32_t *__restrict__ leaf, int k,
                                               int32_t *__restrict__ oi, float *__restrict__ od) {
  extern __shared__ float qs[];  // 8 warps x d query values
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t q = (int64_t)blockIdx.x * 8 + warp;
  if (q >= nq) return;  // warp-uniform; no block barrier below
  float *qv = qs + (int64_t)warp * d;
  for (int c = lane; c < d; c += 32) qv[c] = (float)Qx[q * d + c];
  __syncwarp();
  const float inf = __int_as_float(0x7f800000);
  float ld = inf;  // the list: lane j holds the j-th best (j < 32)
  int32_t li = -1;
  for (int t = 0; t < T_; ++t) {
    const int lf = leaf[q * T_ + t];
    const int32_t *go = goff + (int64_t)t * (nleaf + 1);
    const int32_t lo = go[lf], hi = go[lf + 1];
    const int32_t *ord = order + (int64_t)t * n;
    for (int32_t base = lo; base < hi; base += 32) {
      const int32_t pos = base + lane;
      const int32_t p = pos < hi ? __ldg(ord + pos) : -1;
      float dist = inf;
      if (p >= 0) {
        const T *row = X + (int64_t)p * d;
        float acc = 0.0f;
        for (int c = 0; c < d; c += 4) {  // d % 4 == 0
          const float4 x = ld4<T>(row + c);
          const float4 y = *reinterpret_cast<const float4 *>(qv + c);
          float df = x.x - y.x;
          acc = fmaf(df, df, acc);
          df = x.y - y.y;
          acc = fmaf(df, df, acc);
          df = x.z - y.z;
          acc = fmaf(df, df, acc);
          df = x.w - y.w;
          acc = fmaf(df, df, acc);
        }
        dist = sqrtf(acc);
      }
      // skip members the list already holds, and those that cannot enter it
      const float kd = __shfl_sync(kFull, ld, k - 1);
      const int32_t ki = __shfl_sync(kFull, li, k - 1);
      // every lane takes part in every shuffle (a full-mask shuffle that some
      // lanes skip never completes)
      bool dup = false;
#pragma unroll 8
      for (int j = 0; j < 32; ++j) {
        const int32_t lj = __shfl_sync(kFull, li, j);
        dup |= (p >= 0 && lj == p);
      }
      int32_t cid = p;
      if (dup || p < 0 || !qbefore(dist, p, kd, ki)) {
        dist = inf;
        cid = -1;
      }
      if (!__any_sync(kFull, cid >= 0)) continue;
      warp_sort32(dist, cid, lane);
      // the 32 smallest of list and batch: min of the list and the reversed
      // batch is bitonic; a bitonic clean sorts it
      const float rd = __shfl_sync(kFull, dist, 31 - lane);
      const int32_t ri = __shfl_sync(kFull, cid, 31 - lane);
      if (qbefore(rd, ri, ld, li)) {
        ld = rd;
        li = ri;
      }
#pragma unroll
      for (int stride = 16; stride > 0; stride >>= 1) {
        const float odv = __shfl_xor_sync(kFull, ld, stride);
        const int32_t oiv = __shfl_xor_sync(kFull, li, stride);
        const bool lower = (lane & stride) == 0;
        const bool mine_first = qbefore(ld, li, odv, oiv);
        if (lower != mine_first) {
          ld = odv;
          li = oiv;
        }
      }
    }
  }
  if (lane < k) {
    oi[q * k + lane] = li;
    od[q * k + lane] = li >= 0 ? ld : inf;
  }
}

template <typename T, typename TQ>
void query_t(const void *X, int d, int64_t n, const void *Qx, int64_t nq, int T_,
             const int32_t *order, const int32_t *goff, int nleaf, const int32_t *leaf, int k,
             int32_t *oi, float *od, cudaStream_t s) {
  const size_t smem = (size_t)8 * d * sizeof(float);
  k_query<T, TQ><<<(unsigned)ceil_div(nq, 8), 256, smem, s>>>(
      (const T *)X, d, n, (const TQ *)Qx, nq, T_, order, goff, nleaf, leaf, k, oi, od);
}

}  // namespace

drpt_status launch_descend(const float *Pq, int64_t nq, int T, int gd, const float *medians,
                           int32_t *leaf, cudaStream_t s) {
  if (nq <= 0) return DRPT_OK;
  k_descend<<<(unsigned)ceil_div(nq * T, 256), 256, 0, s>>>(Pq, nq, T, gd, medians, leaf);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_query(const void *X, int dtype, int d, int64_t n, const void *Qx, int64_t nq,
                         int T, const int32_t *order, const int32_t *goff, int nleaf,
                         const int32_t *leaf, int k, int32_t *oi, float *od, cudaStream_t s) {
  if (nq <= 0) return DRPT_OK;
  if (k <= 0 || k > 32 || d % 4 != 0 || d > 1024) {
    set_error("queries: k in [1, 32] and d %% 4 == 0, d <= 1024 (got k %d, d %d)", k, d);
    return DRPT_ERR_UNSUPPORTED;
  }
  if (dtype == DRPT_DTYPE_U8)
    query_t<uint8_t, uint8_t>(X, d, n, Qx, nq, T, order, goff, nleaf, leaf, k, oi, od, s);
  else
    query_t<float, float>(X, d, n, Qx, nq, T, order, goff, nleaf, leaf, k, oi, od, s);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt
