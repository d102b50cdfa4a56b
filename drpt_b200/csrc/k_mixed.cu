// Mixed-precision form of the leaf brute force.
//
// The reference scores every leaf row exactly in FP32 (mdrpt.cpp:123-212).
// The mixed form keeps its global trees (projection + histogram-median
// splits) but brute-forces each whole global leaf with BF16 Gram tiles on the
// tensor cores and wins the accuracy back afterwards:
//
//   K8  k_leaf_index    per tree and point: its row in the tree's leaf order
//                       and its leaf
//       k_leaf_mean     per tree and global leaf: the mean of its first rows
//       k_leaf_stage    per point, read once in index order, for every tree of
//                       a chunk: subtract its leaf's mean (FP32), round to
//                       BF16, store at its row in that tree's leaf order, norm
//                       of the rounded row
//   K9  k_tile_plan     row tiles of 128 points of every leaf
//   K10 k_leaf_mma      per row tile: TMA-fed tcgen05 MMAs (BF16 x BF16 ->
//                       FP32 in Tensor Memory, M = 128 rows, N = 64 columns
//                       per tile, K = the padded dimension), epilogue scores
//                       ||y||^2 - 2 x.y per column and keeps each row's KP
//                       best in registers (threshold filter seeded from the
//                       running list, per-thread shared-memory buffer,
//                       bitonic sort + merge), then folds them into the
//                       point's running list of the KP best distinct
//                       candidates over the trees built so far
//   K11 k_rerank        per point: the running list's KP candidates rescored with the
//                       exact sequential FP32 distance of the plain form, the
//                       k best kept; candidates whose FP32 distance lies within
//                       a relative 2^-16 of the k-th are re-ordered by an FP64
//                       distance
//
// Centring on the leaf mean keeps the BF16 rounding error of x.y small next
// to the squared distances that are ranked (values of a few tens instead of a
// few hundreds for the synthetic workloads).
#include <cuda.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <type_traits>

#include "kernels.cuh"
#include "sm100.cuh"

namespace drpt {
namespace {

using namespace sm100;

constexpr int kTM = 128;            // rows per tile (M)
constexpr int kTN = 64;             // columns per tile (N) of the streamed form
// Per list width KP and A layout: columns per tile (N), accumulator buffers
// (together 128 TMEM columns), B-tile stages, per-row pending-key slots,
// epilogue groups of four warps and the CTAs per SM the kernel is built for.
// The epilogue bounds the kernel: with 16 keys per row and a resident A,
// one group, 3 CTAs per SM (d <= 128: 68 KB of shared memory each) on one
// 64-column B stage and 32 slots.  Measured slower on the 1M x 128 bench
// build (leaf kernel, 6 trees): two groups taking the column tiles in turn
// at 2 CTAs per SM (5.96 ms against 4.96: their split lists need more
// flushes), three 32-column stages with four accumulators (5.35 ms: twice
// the per-tile epilogue overhead), one group at 2 CTAs per SM with two or
// three stages (5.48 ms).  With 32 keys or a streamed A: one group, 2 CTAs,
// two stages, 64 or 32 slots.
template <int KP, bool STREAM>
struct MmaCfg {
  static constexpr bool dense = KP == 16 && !STREAM;
  static constexpr int tn = 64;
  static constexpr int nacc = 128 / tn;
  static constexpr int stages = dense ? 1 : 2;
  static constexpr int slots = KP == 16 ? 32 : 64;
  static constexpr int groups = 1;
  static constexpr int epi_warps = 4 * groups;
  static constexpr int threads = 32 * (epi_warps + 2);
  static constexpr int min_blocks = dense ? 3 : 2;
};
constexpr int kColBits = 13;        // low key bits holding the column in the leaf
constexpr uint32_t kColMask = (1u << kColBits) - 1;
constexpr int kMaxLeaf = 1 << kColBits;  // largest leaf the key can address
constexpr int kCheck = 16;          // columns between flush checks
constexpr int kCentreRows = 64;     // rows averaged for a leaf's centre

__device__ __forceinline__ bool before(float da, int32_t ia, float db, int32_t ib) {
  return da < db || (da == db && (uint32_t)ia < (uint32_t)ib);
}

// ------------------------------------------------------------------ K8
template <typename T>
__device__ __forceinline__ void load4(const T *p, float *v);
template <>
__device__ __forceinline__ void load4<float>(const float *p, float *v) {
  const float4 q = __ldg(reinterpret_cast<const float4 *>(p));
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
template <>
__device__ __forceinline__ void load4<uint8_t>(const uint8_t *p, float *v) {
  const uchar4 q = __ldg(reinterpret_cast<const uchar4 *>(p));
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}

// Streaming variants for data read or written once (evict-first in L2, so
// that the leaf centres stay resident).
template <typename T>
__device__ __forceinline__ void load4_cs(const T *p, float *v);
template <>
__device__ __forceinline__ void load4_cs<float>(const float *p, float *v) {
  const float4 q = __ldcs(reinterpret_cast<const float4 *>(p));
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
template <>
__device__ __forceinline__ void load4_cs<uint8_t>(const uint8_t *p, float *v) {
  const uchar4 q = __ldcs(reinterpret_cast<const uchar4 *>(p));
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}

// k_leaf_index: block (j, t) writes, for every point of leaf j of tree t,
// its position in the tree's leaf order and the leaf.
__global__ void __launch_bounds__(256) k_leaf_index(const int32_t *__restrict__ order,
                                                    const int32_t *__restrict__ goff, int64_t n,
                                                    int nleaf, int32_t *__restrict__ pos,
                                                    int32_t *__restrict__ lf) {
  const int j = blockIdx.x, t = blockIdx.y;
  const int32_t *o = order + (int64_t)t * n;
  const int32_t *g = goff + (int64_t)t * (nleaf + 1);
  const int32_t lo = g[j], hi = g[j + 1];
  for (int32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const int32_t p = __ldg(o + i);
    pos[(int64_t)t * n + p] = i;
    lf[(int64_t)t * n + p] = j;
  }
}

// k_leaf_mean: block (j, t) for leaf j of tree t.  The centre is the mean of
// the leaf's first (up to) kCentreRows rows -- it only has to bring the
// values near zero -- summed per warp, the eight warp partials added in warp
// order, so the result does not depend on scheduling.  In both this kernel
// and k_leaf_stage lane l owns the four dimensions 4l..4l+3 of every 128-wide
// chunk (NCH chunks, d <= 128 * NCH, d % 4 == 0).
template <typename T, int NCH>
__global__ void __launch_bounds__(256) k_leaf_mean(const T *__restrict__ X, int64_t n, int d,
                                                   const int32_t *__restrict__ order,
                                                   const int32_t *__restrict__ goff, int nleaf,
                                                   float *__restrict__ mu) {
  constexpr int W = NCH * 128;
  __shared__ float part[8][W];
  const int j = blockIdx.x, t = blockIdx.y;
  const int32_t *ord = order + (int64_t)t * n;
  const int32_t *g = goff + (int64_t)t * (nleaf + 1);
  const int32_t lo = g[j], m = g[j + 1] - lo;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float acc[NCH][4];
#pragma unroll
  for (int h = 0; h < NCH; ++h) acc[h][0] = acc[h][1] = acc[h][2] = acc[h][3] = 0.0f;
  const int mc = min(m, kCentreRows);
  // warp w adds rows w, w + 8, ... in order; CB rows' loads in flight at once
  constexpr int CB = NCH <= 2 ? kCentreRows / 8 : 2;
  for (int rb = warp; rb < mc; rb += 8 * CB) {
    float v[CB][NCH][4];
#pragma unroll
    for (int i = 0; i < CB; ++i) {
      const int r = rb + 8 * i;
      const T *src = r < mc ? X + (int64_t)__ldg(ord + lo + r) * d : nullptr;
#pragma unroll
      for (int h = 0; h < NCH; ++h) {
        const int c0 = h * 128 + 4 * lane;
        v[i][h][0] = v[i][h][1] = v[i][h][2] = v[i][h][3] = 0.0f;
        if (src && c0 < d) load4<T>(src + c0, v[i][h]);
      }
    }
#pragma unroll
    for (int i = 0; i < CB; ++i)
      if (rb + 8 * i < mc)
#pragma unroll
        for (int h = 0; h < NCH; ++h)
#pragma unroll
          for (int e = 0; e < 4; ++e) acc[h][e] += v[i][h][e];
  }
#pragma unroll
  for (int h = 0; h < NCH; ++h)
#pragma unroll
    for (int e = 0; e < 4; ++e) part[warp][h * 128 + 4 * lane + e] = acc[h][e];
  __syncthreads();
  float *out = mu + ((int64_t)t * nleaf + j) * d;
  for (int i = threadIdx.x; i < d; i += 256) {
    float s = 0.0f;
    for (int w = 0; w < 8; ++w) s += part[w][i];
    out[i] = mc > 0 ? s / (float)mc : 0.0f;
  }
}

// k_leaf_stage: warps take RB consecutive points at a time (grid-stride) and
// read their rows once; for every tree t of the chunk each point's row is
// centred on its leaf's mean and stored at its position in tree t's leaf
// order (slice t of Xq, nrm, scl).  The positions and leaves of RB points
// and up to 32 / RB trees are loaded by one lane each and broadcast.
//
// BF16 output: the centred row rounded to BF16 (d_pad elements, zero-padded).
// E4M3 output (FP8): the centred row divided by its scale
// s = max|x - c| / 448 (448 = largest finite E4M3 value) and rounded to E4M3
// with saturation (d_pad bytes, zero-padded); the scale goes to `scl`.  In
// both cases `nrm` receives the squared norm of the row the tensor cores see
// (dequantised for FP8), so that ||y||^2 - 2 x.y ranks the same values.
// Sums of RB (a power of two, <= 32) per-lane values s[q] over the warp, all
// at once: while more than one value is left, each lane keeps half of its
// values and sends the other half to the lane that keeps those (log2 RB
// steps of RB/2, ..., 1 shuffles), then a plain butterfly over the lanes
// that hold the same value.  Lane l returns the sum for q = l >> (5 - log2 RB).
template <int RB>
__device__ __forceinline__ float warp_sum_rows(float *s, int lane) {
  int bit = 16;
#pragma unroll
  for (int cnt = RB; cnt > 1; cnt >>= 1, bit >>= 1) {
    const bool up = (lane & bit) != 0;
#pragma unroll
    for (int i = 0; i < cnt / 2; ++i) {
      const float keep = up ? s[i + cnt / 2] : s[i];
      const float send = up ? s[i] : s[i + cnt / 2];
      s[i] = keep + __shfl_xor_sync(kFull, send, bit);
    }
  }
  float v = s[0];
#pragma unroll
  for (int o = bit; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

template <int NCH>
struct StageCfg {
  static constexpr int rb = NCH <= 2 ? 4 / NCH : 1;           // points per warp step
  static constexpr int min_blocks = NCH == 1 ? 4 : (NCH == 2 ? 3 : 2);
};

// FULL: d == d_pad == 128 * NCH, so no dimension needs a bounds check.
template <typename T, int NCH, bool FP8, bool FULL>
__global__ void __launch_bounds__(256, StageCfg<NCH>::min_blocks) k_leaf_stage(const T *__restrict__ X, int64_t n, int d,
                                                    int d_pad, const int32_t *__restrict__ pos,
                                                    const int32_t *__restrict__ lf,
                                                    const float *__restrict__ mu, int nleaf,
                                                    int tc, void *__restrict__ Xq,
                                                    float *__restrict__ nrm,
                                                    float *__restrict__ scl) {
  constexpr int RB = StageCfg<NCH>::rb;  // points per warp step, loaded together
  constexpr int TG = 32 / RB;            // trees per broadcast group
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r0 = gw * RB; r0 < n; r0 += nw * RB) {
    float v[RB][NCH][4];
#pragma unroll
    for (int q = 0; q < RB; ++q) {
      const int64_t r = r0 + q;
      const T *src = r < n ? X + r * d : nullptr;
#pragma unroll
      for (int h = 0; h < NCH; ++h) {
        const int c0 = h * 128 + 4 * lane;
        v[q][h][0] = v[q][h][1] = v[q][h][2] = v[q][h][3] = 0.0f;
        if (src && (FULL || c0 < d)) load4_cs<T>(src + c0, v[q][h]);
      }
    }
    for (int tg = 0; tg < tc; tg += TG) {
      int32_t my_pos = -1, my_lf = 0;
      {
        const int tt = tg + lane / RB;
        const int64_t r = r0 + lane % RB;
        if (lane < TG * RB && tt < tc && r < n) {
          my_pos = __ldg(pos + (int64_t)tt * n + r);
          my_lf = __ldg(lf + (int64_t)tt * n + r);
        }
      }
      const int tend = min(tg + TG, tc);
      for (int t = tg; t < tend; ++t) {
        // the RB points' leaf centres are all requested before the first use
        int32_t rows[RB];
        float m4[RB][NCH][4];
#pragma unroll
        for (int q = 0; q < RB; ++q) {
          const int src_lane = (t - tg) * RB + q;
          rows[q] = __shfl_sync(kFull, my_pos, src_lane);
          const int32_t leaf = __shfl_sync(kFull, my_lf, src_lane);  // 0 past the end
          const float *mr = mu + ((int64_t)t * nleaf + leaf) * d;
#pragma unroll
          for (int h = 0; h < NCH; ++h) {
            const int c0 = h * 128 + 4 * lane;
            m4[q][h][0] = m4[q][h][1] = m4[q][h][2] = m4[q][h][3] = 0.0f;
            if (FULL || c0 < d) load4<float>(mr + c0, m4[q][h]);
          }
        }
        float sqs[RB];  // BF16: this lane's part of each point's squared norm
#pragma unroll
        for (int q = 0; q < RB; ++q) {
          sqs[q] = 0.0f;
          const int32_t row = rows[q];
          if (row < 0) continue;  // warp-uniform: a point past the end
          float c[NCH][4];
#pragma unroll
          for (int h = 0; h < NCH; ++h) {
            const int c0 = h * 128 + 4 * lane;
            if constexpr (FULL) {
              // two differences per packed FP32x2 multiply-add (-1 * m + v,
              // one rounding: the same value as v - m)
#pragma unroll
              for (int e = 0; e < 4; e += 2) {
                const float2 r = fma2(make_float2(m4[q][h][e], m4[q][h][e + 1]),
                                      make_float2(-1.0f, -1.0f),
                                      make_float2(v[q][h][e], v[q][h][e + 1]));
                c[h][e] = r.x;
                c[h][e + 1] = r.y;
              }
            } else {
#pragma unroll
              for (int e = 0; e < 4; ++e)
                c[h][e] = c0 + e < d ? v[q][h][e] - m4[q][h][e] : 0.0f;
            }
          }
          const int64_t orow = (int64_t)t * n + row;
          float sq = 0.0f;
          if constexpr (FP8) {
            float amax = 0.0f;
#pragma unroll
            for (int h = 0; h < NCH; ++h)
#pragma unroll
              for (int e = 0; e < 4; ++e) amax = fmaxf(amax, fabsf(c[h][e]));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(kFull, amax, o));
            const float sc = amax > 0.0f ? amax / 448.0f : 1.0f;
            const float inv = amax > 0.0f ? 448.0f / amax : 1.0f;
            uint8_t *dst = static_cast<uint8_t *>(Xq) + orow * d_pad;
#pragma unroll
            for (int h = 0; h < NCH; ++h) {
              const int c0 = h * 128 + 4 * lane;
              if (FULL || c0 < d_pad) {
                const __nv_fp8x2_storage_t lo2 = __nv_cvt_float2_to_fp8x2(
                    make_float2(c[h][0] * inv, c[h][1] * inv), __NV_SATFINITE, __NV_E4M3);
                const __nv_fp8x2_storage_t hi2 = __nv_cvt_float2_to_fp8x2(
                    make_float2(c[h][2] * inv, c[h][3] * inv), __NV_SATFINITE, __NV_E4M3);
                const float2 a = __half22float2(__nv_cvt_fp8x2_to_halfraw2(lo2, __NV_E4M3));
                const float2 b = __half22float2(__nv_cvt_fp8x2_to_halfraw2(hi2, __NV_E4M3));
                sq = fmaf(a.x, a.x, sq);
                sq = fmaf(a.y, a.y, sq);
                sq = fmaf(b.x, b.x, sq);
                sq = fmaf(b.y, b.y, sq);
                __stcs(reinterpret_cast<unsigned int *>(dst + c0),
                       (unsigned int)lo2 | ((unsigned int)hi2 << 16));
              }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(kFull, sq, o);
            if (lane == 0) {
              __stcs(nrm + orow, sq * sc * sc);
              __stcs(scl + orow, sc);
            }
          } else {
            __nv_bfloat16 *dst = static_cast<__nv_bfloat16 *>(Xq) + orow * d_pad;
            // squares of the rounded values, even and odd dimensions in the
            // two halves of a packed FP32x2 sum
            float2 sq2 = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int h = 0; h < NCH; ++h) {
              const int c0 = h * 128 + 4 * lane;
              if (FULL || c0 < d_pad) {
                const __nv_bfloat162 b01 = __floats2bfloat162_rn(c[h][0], c[h][1]);
                const __nv_bfloat162 b23 = __floats2bfloat162_rn(c[h][2], c[h][3]);
                const float2 r01 = __bfloat1622float2(b01), r23 = __bfloat1622float2(b23);
                sq2 = fma2(r01, r01, sq2);
                sq2 = fma2(r23, r23, sq2);
                uint2 pk;
                pk.x = *reinterpret_cast<const uint32_t *>(&b01);
                pk.y = *reinterpret_cast<const uint32_t *>(&b23);
                __stcs(reinterpret_cast<uint2 *>(dst + c0), pk);
              }
            }
            sqs[q] = sq2.x + sq2.y;
          }
        }
        if constexpr (!FP8) {
          // the RB norms summed over the warp together: lane l ends with
          // point (l >> (5 - log2 RB)); the first lane of each group stores it
          const float nv = warp_sum_rows<RB>(sqs, lane);
          constexpr int kGroup = 32 / RB;
          if ((lane & (kGroup - 1)) == 0) {
            const int32_t row = rows[lane / kGroup];
            if (row >= 0) __stcs(nrm + (int64_t)t * n + row, nv);
          }
        }
      }
    }
  }
}

// ------------------------------------------------------------------ K9
// Row tiles of `rows` rows of every leaf, in leaf order.
__global__ void __launch_bounds__(1024) k_tile_plan(const int32_t *__restrict__ goff, int nleaf,
                                                    int rows, int32_t *tile_leaf,
                                                    int32_t *tile_r0, int32_t *n_tiles) {
  __shared__ int warp_tot[32];
  const int per = (nleaf + 1023) / 1024;
  const int j0 = threadIdx.x * per;
  int cnt = 0;
  for (int i = 0; i < per; ++i)
    if (j0 + i < nleaf) cnt += (goff[j0 + i + 1] - goff[j0 + i] + rows - 1) / rows;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    int v = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, v, o);
      if (lane >= o) v += y;
    }
    warp_tot[lane] = v;
  }
  __syncthreads();
  int base = x - cnt + (w > 0 ? warp_tot[w - 1] : 0);
  for (int i = 0; i < per; ++i) {
    const int j = j0 + i;
    if (j >= nleaf) break;
    const int nt = (goff[j + 1] - goff[j] + rows - 1) / rows;
    for (int q = 0; q < nt; ++q) {
      tile_leaf[base + q] = j;
      tile_r0[base + q] = q * rows;
    }
    base += nt;
  }
  if (threadIdx.x == 1023) *n_tiles = base;
}

// ------------------------------------------------------------------ K10
// Register-resident sorting networks (all indices compile-time constants).
__device__ __forceinline__ void cmp_swap(float *d, int32_t *id, int a, int b) {  // d[a] <= d[b]
  const bool sw = d[b] < d[a];
  const float x = d[a], y = d[b];
  const int32_t p = id[a], q = id[b];
  d[a] = sw ? y : x;
  d[b] = sw ? x : y;
  id[a] = sw ? q : p;
  id[b] = sw ? p : q;
}

// Bitonic sort, ascending.
template <int N>
__device__ __forceinline__ void bitonic_sort(float *d, int32_t *id) {
#pragma unroll
  for (int k = 2; k <= N; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const int l = i ^ j;
        if (l > i) {
          if ((i & k) == 0) cmp_swap(d, id, i, l);
          else cmp_swap(d, id, l, i);
        }
      }
}

// L (ascending, N) <- the N smallest of L and S (ascending, M <= N): the
// element-wise minimum of L and reversed S is bitonic and holds them, a
// bitonic clean sorts it.
template <int N, int M>
__device__ __forceinline__ void bitonic_merge_into(float *L, int32_t *Li, const float *S,
                                                   const int32_t *Si) {
#pragma unroll
  for (int i = N - M; i < N; ++i) {
    const float sv = S[N - 1 - i];
    const int32_t si = Si[N - 1 - i];
    const bool take = sv < L[i];
    L[i] = take ? sv : L[i];
    Li[i] = take ? si : Li[i];
  }
#pragma unroll
  for (int j = N >> 1; j > 0; j >>= 1)
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const int l = i ^ j;
      if (l > i) cmp_swap(L, Li, i, l);
    }
}

// Sorting networks on single float keys (min / max pairs).
__device__ __forceinline__ void key_cmp_swap(float *d, int a, int b) {  // d[a] <= d[b]
  const float x = fminf(d[a], d[b]), y = fmaxf(d[a], d[b]);
  d[a] = x;
  d[b] = y;
}

template <int N>
__device__ __forceinline__ void key_sort(float *d) {
#pragma unroll
  for (int k = 2; k <= N; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const int l = i ^ j;
        if (l > i) {
          if ((i & k) == 0) key_cmp_swap(d, i, l);
          else key_cmp_swap(d, l, i);
        }
      }
}

// L (ascending, N) <- the N smallest of L and S (ascending, M <= N).
template <int N, int M>
__device__ __forceinline__ void key_merge_into(float *L, const float *S) {
#pragma unroll
  for (int i = N - M; i < N; ++i) L[i] = fminf(L[i], S[N - 1 - i]);
#pragma unroll
  for (int j = N >> 1; j > 0; j >>= 1)
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const int l = i ^ j;
      if (l > i) key_cmp_swap(L, i, l);
    }
}

// L (ascending, N) <- the N smallest of L and `key`.
template <int N>
__device__ __forceinline__ void key_insert(float *L, float key) {
  // entry i becomes max(old i - 1, min(old i, key)): every entry from the
  // old list at once, no chain through the key
  float prev = L[0];
  L[0] = fminf(prev, key);
#pragma unroll
  for (int i = 1; i < N; ++i) {
    const float cur = L[i];
    L[i] = fmaxf(prev, fminf(cur, key));
    prev = cur;
  }
}

// Shared-memory layout.  Every operand tile is rows of 128 bytes (64 BF16 or
// 128 E4M3 values of one 128-byte K block), 128-byte swizzled, 1024-byte
// aligned.
//   resident A (kb <= 2): A = kb K blocks of the 128 rows, loaded once per row
//     tile; `stages` stages of the kb K blocks of a tn-column B tile;
//   streamed A (larger kb): kSStages stages, each one K block of A (16 KB)
//     and of B (8 KB), so A is re-read from L2 for every column tile.
constexpr int kSStages = 3;
constexpr uint32_t kStreamA = kTM * 128, kStreamStage = kTM * 128 + kTN * 128;

struct MmaSmem {
  uint32_t a_off, b_off, buf_off, nrm_off, scl_off, thr_off, bar_off, total;
};

__host__ __device__ inline MmaSmem mma_smem_layout(int kb, bool stream, int stages, int slots,
                                                   int tn, int groups) {
  MmaSmem L;
  L.a_off = 0;
  if (stream) {
    L.b_off = kStreamA;  // inside each stage
    L.buf_off = kSStages * kStreamStage;
  } else {
    L.b_off = L.a_off + (uint32_t)kb * kTM * 128;
    L.buf_off = L.b_off + (uint32_t)stages * kb * tn * 128;
  }
  L.nrm_off = L.buf_off + kTM * (uint32_t)slots * groups * 4;
  L.scl_off = L.nrm_off + 4 * groups * (uint32_t)tn * 4;
  L.thr_off = L.scl_off + 4 * groups * (uint32_t)tn * 4;
  L.bar_off = L.thr_off + (uint32_t)groups * kTM * 4;
  L.total = L.bar_off + 24 * 8 + 16;
  return L;
}

// KP: candidates kept per row and tree.  STREAM: streamed A.  FP8: E4M3
// operands with per-row scales `scl` (scores are then scaled by the row's and
// the column's scale); otherwise BF16.
template <int KP, bool STREAM, bool FP8>
__global__ void __launch_bounds__(MmaCfg<KP, STREAM>::threads,
                                  MmaCfg<KP, STREAM>::min_blocks) k_leaf_mma(
    const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
    const int32_t *__restrict__ goff, const int32_t *__restrict__ order,
    const float *__restrict__ nrm, const float *__restrict__ scl,
    const int32_t *__restrict__ tile_leaf, const int32_t *__restrict__ tile_r0,
    const int32_t *__restrict__ n_tiles, int kb, int tree, int32_t *__restrict__ run_idx,
    float *__restrict__ run_dist, int32_t *__restrict__ tree_idx, float *__restrict__ tree_dist,
    int *err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  using Cfg = MmaCfg<KP, STREAM>;
  constexpr int kBufSlots = Cfg::slots;
  constexpr int TN = Cfg::tn, NACC = Cfg::nacc, G = Cfg::groups, EPI = Cfg::epi_warps;
  static_assert(!STREAM || TN == kTN, "streamed stages hold kTN-column B blocks");
  static_assert(NACC % G == 0, "a group owns whole accumulators");
  const MmaSmem L = mma_smem_layout(kb, STREAM, Cfg::stages, Cfg::slots, TN, G);
  uint8_t *sA = smem + L.a_off;
  uint8_t *sB = smem + L.b_off;
  uint32_t *buf = reinterpret_cast<uint32_t *>(smem + L.buf_off);  // [group][slot][row] keys
  float *thr_sh = reinterpret_cast<float *>(smem + L.thr_off);  // [group][row] KP-th best key
  float *nbuf = reinterpret_cast<float *>(smem + L.nrm_off);  // [warp][TN] column norms of a tile
  float *sbuf = reinterpret_cast<float *>(smem + L.scl_off);  // [warp][TN] column scales (FP8)
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L.bar_off);
  static_assert(kSStages <= 4 && Cfg::stages <= 4 && NACC <= 4, "barrier slots");
  uint64_t *full_a = bars + 0;
  uint64_t *full_b = bars + 1;     // up to 4 stages
  uint64_t *empty_b = bars + 5;    // up to 4 stages
  uint64_t *acc_full = bars + 9;   // up to 4 accumulators
  uint64_t *acc_empty = bars + 13; // up to 4 accumulators
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 24);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 24) + 1;
  constexpr int NS = STREAM ? kSStages : Cfg::stages;
  constexpr int kKE = FP8 ? 128 : 64;  // elements per 128-byte K block

  const int u = blockIdx.x;
  if (u >= *n_tiles) return;  // uniform for the whole block
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int leaf = tile_leaf[u], r0 = tile_r0[u];
  const int32_t lo = goff[leaf], m = goff[leaf + 1] - lo;
  if (m > kMaxLeaf) {  // the candidate keys address at most kMaxLeaf columns
    if (threadIdx.x == 0) atomicOr(err, 2);
    return;  // uniform for the whole block
  }
  const int nct = (m + TN - 1) / TN;
  const uint32_t a_bytes = (uint32_t)kb * kTM * 128, b_bytes = (uint32_t)kb * TN * 128;

  if (threadIdx.x == 0) {
    mbar_init(full_a, 1);
    for (int s = 0; s < NS; ++s) {
      mbar_init(full_b + s, 1);
      mbar_init(empty_b + s, 1);
    }
    for (int b = 0; b < NACC; ++b) {
      mbar_init(acc_full + b, 1);
      mbar_init(acc_empty + b, 4 * 32);  // the owning group's 128 threads
    }
    *abort_flag = 0;
    fence_barrier_init();
  }
  for (int i = threadIdx.x; i < G * kTM; i += blockDim.x) thr_sh[i] = __int_as_float(0x7f800000);
  if (warp == EPI + 1) tmem_alloc(tmem_slot, 128);  // NACC accumulators x TN columns
  if (warp == EPI && lane == 0) {
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == EPI) {
    // ---- TMA producer
    if (lane == 0) {
      if constexpr (STREAM) {
        // stage i = (column tile c, K block q) with i = c * kb + q
        const int total = nct * kb;
        for (int i = 0; i < total && !*abort_flag; ++i) {
          const int s = i % NS, c = i / kb, q = i - c * kb;
          if (i >= NS && !mbar_wait(empty_b + s, ((i / NS) - 1) & 1)) {
            *abort_flag = 1;
            break;
          }
          uint8_t *st = smem + (size_t)s * kStreamStage;
          mbar_arrive_expect_tx(full_b + s, kStreamStage);
          tma_load_2d(st, &tmA, full_b + s, q * kKE, lo + r0);
          tma_load_2d(st + kStreamA, &tmB, full_b + s, q * kKE, lo + c * TN);
        }
      } else {
        mbar_arrive_expect_tx(full_a, a_bytes);
        for (int q = 0; q < kb; ++q)
          tma_load_2d(sA + q * kTM * 128, &tmA, full_a, q * kKE, lo + r0);
        for (int c = 0; c < nct && !*abort_flag; ++c) {
          const int s = c % NS;
          if (c >= NS && !mbar_wait(empty_b + s, ((c / NS) - 1) & 1)) {
            *abort_flag = 1;
            break;
          }
          uint8_t *dst = sB + s * b_bytes;
          mbar_arrive_expect_tx(full_b + s, b_bytes);
          for (int q = 0; q < kb; ++q)
            tma_load_2d(dst + q * TN * 128, &tmB, full_b + s, q * kKE, lo + c * TN);
        }
      }
    }
  } else if (warp == EPI + 1) {
    // ---- MMA issuer: 4 instructions per 128-byte K block (K = 16 BF16 or
    // 32 E4M3 values, 32 bytes each)
    if (lane == 0) {
      constexpr uint32_t idesc = FP8 ? idesc_e4m3_f32(kTM, TN) : idesc_bf16_f32(kTM, TN);
      auto mma = [&](uint32_t d, uint64_t ad, uint64_t bd, uint32_t acc) {
        if constexpr (FP8) mma_e4m3(d, ad, bd, idesc, acc);
        else mma_bf16(d, ad, bd, idesc, acc);
      };
      bool ok = true;
      if constexpr (STREAM) {
        for (int c = 0; ok && c < nct && !*abort_flag; ++c) {
          const int b = c % NACC;
          if (c >= NACC) ok = mbar_wait(acc_empty + b, ((c / NACC) - 1) & 1);
          for (int q = 0; ok && q < kb; ++q) {
            const int i = c * kb + q, s = i % NS;
            ok = mbar_wait(full_b + s, (i / NS) & 1);
            if (!ok) break;
            tc_fence_after();
            const uint32_t as = smem_u32(smem + (size_t)s * kStreamStage), bs = as + kStreamA;
#pragma unroll
            for (int k = 0; k < 4; ++k)
              mma(tmem + b * TN, desc_k_sw128(as + k * 32), desc_k_sw128(bs + k * 32),
                  (q | k) ? 1u : 0u);
            mma_commit(empty_b + s);
          }
          if (ok) mma_commit(acc_full + b);
        }
      } else {
        const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
        ok = mbar_wait(full_a, 0);
        for (int c = 0; ok && c < nct && !*abort_flag; ++c) {
          const int s = c % NS, b = c % NACC;
          ok = mbar_wait(full_b + s, (c / NS) & 1);
          if (ok && c >= NACC) ok = mbar_wait(acc_empty + b, ((c / NACC) - 1) & 1);
          if (!ok) break;
          tc_fence_after();
          const uint32_t bs = b_base + s * b_bytes;
          for (int q = 0; q < kb; ++q)
#pragma unroll
            for (int k = 0; k < 4; ++k)
              mma(tmem + b * TN, desc_k_sw128(a_base + q * kTM * 128 + k * 32),
                  desc_k_sw128(bs + q * TN * 128 + k * 32), (q | k) ? 1u : 0u);
          mma_commit(empty_b + s);
          mma_commit(acc_full + b);
        }
      }
      if (!ok) *abort_flag = 1;
    }
  } else {
    // ---- epilogue: thread = row (TMEM lane).  A candidate is one 32-bit
    // key: its score (an FP32 value, ordered as a float) with the low
    // kColBits mantissa bits replaced by its column in the leaf, so keys sort
    // with plain min/max and equal scores order by column.  Keys below the
    // row's current KP-th best go to a slot-major shared buffer
    // (conflict-free: consecutive rows are consecutive words); when any row
    // of the warp has too many pending, every row sorts its pending keys in
    // batches of 16 and merges them into its sorted list of KP keys with a
    // bitonic network.  With two groups, group g takes the column tiles
    // c = g, g + 2, ... (accumulator g) and keeps its own list per row; each
    // group filters with the smaller of the groups' KP-th best keys (a key
    // above another group's KP-th best cannot be among the KP best of the
    // union), and group 0 merges the lists at the end.
    const int grp = warp / 4, wq = warp % 4;
    const int row = wq * 32 + lane;
    const bool rvalid = r0 + row < m;
    float td[KP];
#pragma unroll
    for (int j = 0; j < KP; ++j) td[j] = __int_as_float(0x7f800000);
    // Candidates that cannot beat the KP-th of the point's running list
    // (approximate squared distances of the earlier trees) are never kept.
    // (rows past the leaf get -inf and keep nothing)
    float thr = rvalid ? __int_as_float(0x7f800000) : -__int_as_float(0x7f800000);
    int32_t my_pos = -1, my_pt = -1;
    float nr = 0.0f, m2s = -2.0f;  // FP8: -2 x the row's scale
    if (rvalid) {
      my_pos = lo + r0 + row;
      my_pt = __ldg(order + my_pos);
      nr = __ldg(nrm + my_pos);
      if constexpr (FP8) m2s = -2.0f * __ldg(scl + my_pos);
      if (tree > 0) thr = run_dist[(int64_t)my_pt * KP + KP - 1] - nr;
    }
    const float thr0 = thr;
    const uint32_t my_col = (uint32_t)(r0 + row);  // the row's own point, dropped when read
    // Pending keys: a passing key is stored at the next free slot of one of
    // two per-row lanes of the buffer (even and odd columns, two independent
    // append chains) by a predicated shared-memory store, no branch; slot
    // addresses are 32-bit shared-window offsets.
    constexpr int kChains = 2, kLane = kBufSlots / kChains, kPerBatch = 16 / kChains;
    uint32_t *const pbase = buf + grp * kBufSlots * kTM + row;
    const uint32_t abase = smem_u32(pbase);
    uint32_t aslot[kChains], alim[kChains];
#pragma unroll
    for (int q = 0; q < kChains; ++q) {
      aslot[q] = abase + q * kLane * kTM * 4;
      // after a check that does not flush a chain holds at most
      // kLane - kCheck / kChains keys, so the next kCheck / kChains stores
      // stay inside its kLane slots
      alim[q] = aslot[q] + (kLane - kCheck / kChains) * kTM * 4;
    }
    auto pending = [&](int q) {
      return (int)((aslot[q] - abase - q * kLane * kTM * 4) / (kTM * 4));
    };
    auto flush = [&]() {
      int cnt[kChains], mine = 0;
#pragma unroll
      for (int q = 0; q < kChains; ++q) {
        cnt[q] = pending(q);
        mine = max(mine, cnt[q]);
      }
      const int mx = __reduce_max_sync(kFull, mine);
      if (mx <= 3) {
        // few pending keys (the common case once a threshold is set): insert
        // them one by one (2 KP min/max each) rather than sort a batch of 16
        // and merge it (about 240); the kept keys are the same
#pragma unroll
        for (int q = 0; q < kChains; ++q)
          for (int slot = 0; slot < mx; ++slot) {
            uint32_t key = 0x7f800000u;
            if (slot < cnt[q]) key = pbase[(q * kLane + slot) * kTM];
            if ((key & kColMask) == my_col && key != 0x7f800000u) key = 0x7f800000u;
            key_insert<KP>(td, __uint_as_float(key));
          }
      }
      for (int base = 0; mx > 3 && base < mx; base += kPerBatch) {
        float sd[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int q = e / kPerBatch, slot = base + e % kPerBatch;
          uint32_t key = 0x7f800000u;
          if (slot < cnt[q]) key = pbase[(q * kLane + slot) * kTM];
          if ((key & kColMask) == my_col && key != 0x7f800000u) key = 0x7f800000u;
          sd[e] = __uint_as_float(key);
        }
        key_sort<16>(sd);
        key_merge_into<KP, 16>(td, sd);
      }
#pragma unroll
      for (int q = 0; q < kChains; ++q) aslot[q] = abase + q * kLane * kTM * 4;
      float lim = td[KP - 1];
      if constexpr (G > 1) {
        volatile float *ts = thr_sh;
        ts[grp * kTM + row] = lim;
#pragma unroll
        for (int g2 = 0; g2 < G; ++g2)
          if (g2 != grp) lim = fminf(lim, ts[g2 * kTM + row]);
      }
      thr = fminf(thr0, lim);
    };
    // key = the score's high bits and the column bits of the packed norm
    // (one bit-select), stored only when the score beats the threshold
    auto append = [&](uint32_t &slot, float sv, float ncp) {
      const uint32_t key = (__float_as_uint(sv) & ~kColMask) | (__float_as_uint(ncp) & kColMask);
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.lt.f32 p, %1, %2;\n\t"
          "@p st.shared.u32 [%0], %3;\n\t"
          "@p add.u32 %0, %0, %4;\n\t}"
          : "+r"(slot)
          : "f"(sv), "f"(thr), "r"(key), "n"(kTM * 4)
          : "memory");
    };
    // one 32-column chunk of scores; the packed norms (and E4M3 scales) of
    // each kCheck columns are read into registers before that group's
    // stores, so the loads do not wait behind them
    auto scan = [&](const float *v, const float *wn, const float *ws) {
#pragma unroll
      for (int h = 0; h < 32; h += kCheck) {
        float nc[kCheck], sc[kCheck];
#pragma unroll
        for (int j4 = 0; j4 < kCheck; j4 += 4) {
          const float4 a = *reinterpret_cast<const float4 *>(wn + h + j4);
          nc[j4] = a.x;
          nc[j4 + 1] = a.y;
          nc[j4 + 2] = a.z;
          nc[j4 + 3] = a.w;
          if constexpr (FP8) {
            const float4 b = *reinterpret_cast<const float4 *>(ws + h + j4);
            sc[j4] = b.x;
            sc[j4 + 1] = b.y;
            sc[j4 + 2] = b.z;
            sc[j4 + 3] = b.w;
          }
        }
        (void)sc;
#pragma unroll
        for (int e = 0; e < kCheck; e += 2) {
          const int j = h + e;
          float2 sv;
          if constexpr (FP8) {
            sv.x = fmaf(m2s * sc[e], v[j], nc[e]);
            sv.y = fmaf(m2s * sc[e + 1], v[j + 1], nc[e + 1]);
          } else {
            // two scores per packed FP32x2 multiply-add
            sv = fma2(make_float2(v[j], v[j + 1]), make_float2(-2.0f, -2.0f),
                      make_float2(nc[e], nc[e + 1]));
          }
          append(aslot[j % kChains], sv.x, nc[e]);
          append(aslot[(j + 1) % kChains], sv.y, nc[e + 1]);
        }
        bool over = false;
#pragma unroll
        for (int q = 0; q < kChains; ++q) over |= aslot[q] > alim[q];
        if (__any_sync(kFull, over)) flush();
      }
    };
    const uint32_t lane_base = tmem + ((uint32_t)(wq * 32) << 16);
    // column norms (and E4M3 scales) of a tile: lane l holds columns l and
    // l + 32, loaded one tile ahead; columns past the leaf carry an infinite
    // norm (a NaN once packed) and so never pass
    float pn[TN / 32], ps[TN / 32];
    auto load_cols = [&](int c) {
#pragma unroll
      for (int h = 0; h < TN / 32; ++h) {
        const int col = c * TN + h * 32 + lane;
        const bool in = c < nct && col < m;
        pn[h] = in ? __ldg(nrm + lo + col) : __int_as_float(0x7f800000);
        ps[h] = 0.0f;
        if constexpr (FP8) ps[h] = in ? __ldg(scl + lo + col) : 0.0f;
      }
    };
    load_cols(grp);
    for (int c = grp; c < nct; c += G) {
      const int b = c % NACC;
      // this tile's column norms, staged per warp (16-byte aligned reads)
      float *wn = nbuf + warp * TN;
      float *ws = sbuf + warp * TN;
      __syncwarp();
#pragma unroll
      for (int h = 0; h < TN / 32; ++h) {
        // the norm's low kColBits bits replaced by the column (a relative
        // change below 2^-10 of the norm, next to the BF16 rounding of x.y);
        // a past-the-leaf column's infinite norm becomes a NaN, which
        // fails every comparison
        wn[h * 32 + lane] = __uint_as_float((__float_as_uint(pn[h]) & ~kColMask) |
                                            (uint32_t)(c * TN + h * 32 + lane));
        if constexpr (FP8) ws[h * 32 + lane] = ps[h];
      }
      __syncwarp();
      load_cols(c + G);
      if (!__all_sync(kFull, mbar_wait(acc_full + b, (c / NACC) & 1))) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
#pragma unroll
      for (int q = 0; q < TN / 32; ++q) {
        float v[32];
        tmem_ld32(lane_base + b * TN + q * 32, v);
        scan(v, wn + q * 32, ws + q * 32);
      }
      tc_fence_before();
      mbar_arrive(acc_empty + b);
    }
    flush();
    if constexpr (G > 1) {
      // groups g > 0 hand their sorted lists to group 0 through their own
      // buffer slots (KP <= slots); a barrier over the epilogue warps only
      if (grp > 0) {
#pragma unroll
        for (int j = 0; j < KP; ++j) pbase[j * kTM] = __float_as_uint(td[j]);
      }
      asm volatile("bar.sync 1, %0;" ::"n"(EPI * 32) : "memory");
      if (grp == 0) {
        for (int g2 = 1; g2 < G; ++g2) {
          float sd[KP];
#pragma unroll
          for (int j = 0; j < KP; ++j) sd[j] = __uint_as_float(buf[(g2 * kBufSlots + j) * kTM + row]);
          key_merge_into<KP, KP>(td, sd);
        }
      }
    }
    if (grp == 0 && rvalid) {
      // this tree's list, keys back to (squared distance, point id), already
      // ascending by key, i.e. by distance: tree 0's is the running list;
      // later trees' go to the tree list, which k_fold_lists merges into the
      // running list (a separate, fully parallel pass: folding here kept the
      // CTA, its idle TMA and MMA warps and its shared memory for the
      // latency of the running list's reads)
      float rd[KP];
      int32_t ri[KP];
#pragma unroll
      for (int j = 0; j < KP; ++j) {
        const uint32_t key = __float_as_uint(td[j]);
        const bool have = key != 0x7f800000u;
        const int32_t q = have ? __ldg(order + lo + (int32_t)(key & kColMask)) : -1;
        rd[j] = have ? nr + __uint_as_float(key & ~kColMask) : __int_as_float(0x7f800000);
        ri[j] = q;
      }
      const int64_t o = (int64_t)my_pt * KP;
      float4 *dd = reinterpret_cast<float4 *>((tree > 0 ? tree_dist : run_dist) + o);
      int4 *di = reinterpret_cast<int4 *>((tree > 0 ? tree_idx : run_idx) + o);
#pragma unroll
      for (int j = 0; j < KP; j += 4) {
        dd[j / 4] = make_float4(rd[j], rd[j + 1], rd[j + 2], rd[j + 3]);
        di[j / 4] = make_int4(ri[j], ri[j + 1], ri[j + 2], ri[j + 3]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == EPI + 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 128);
  }
  if (threadIdx.x == 0 && *abort_flag) atomicOr(err, 1);
}

// k_fold_lists: per point (one thread each), fold this tree's list (KP
// candidates ascending by approximate distance) into the running list of the
// KP best distinct candidates of the trees before: neighbours the running
// list already holds are dropped from the new list, which is re-sorted, and a
// bitonic merge keeps the KP best by distance.
template <int KP>
__global__ void __launch_bounds__(256) k_fold_lists(const float *__restrict__ tree_dist,
                                                    const int32_t *__restrict__ tree_idx,
                                                    int64_t n, float *__restrict__ run_dist,
                                                    int32_t *__restrict__ run_idx) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int64_t o = p * KP;
  float rd[KP], od[KP];
  int32_t ri[KP], oi[KP];
#pragma unroll
  for (int j = 0; j < KP; j += 4) {
    const float4 a = __ldcs(reinterpret_cast<const float4 *>(tree_dist + o) + j / 4);
    const int4 b = __ldcs(reinterpret_cast<const int4 *>(tree_idx + o) + j / 4);
    const float4 c = reinterpret_cast<const float4 *>(run_dist + o)[j / 4];
    const int4 e = reinterpret_cast<const int4 *>(run_idx + o)[j / 4];
    rd[j] = a.x; rd[j + 1] = a.y; rd[j + 2] = a.z; rd[j + 3] = a.w;
    ri[j] = b.x; ri[j + 1] = b.y; ri[j + 2] = b.z; ri[j + 3] = b.w;
    od[j] = c.x; od[j + 1] = c.y; od[j + 2] = c.z; od[j + 3] = c.w;
    oi[j] = e.x; oi[j + 1] = e.y; oi[j + 2] = e.z; oi[j + 3] = e.w;
  }
#pragma unroll
  for (int j = 0; j < KP; ++j) {
    bool dup = false;
#pragma unroll
    for (int i = 0; i < KP; ++i) dup |= (ri[j] >= 0 && oi[i] == ri[j]);
    if (dup) {
      ri[j] = -1;
      rd[j] = __int_as_float(0x7f800000);
    }
  }
  bitonic_sort<KP>(rd, ri);
  bitonic_merge_into<KP, KP>(od, oi, rd, ri);
#pragma unroll
  for (int j = 0; j < KP; j += 4) {
    reinterpret_cast<float4 *>(run_dist + o)[j / 4] = make_float4(od[j], od[j + 1], od[j + 2], od[j + 3]);
    reinterpret_cast<int4 *>(run_idx + o)[j / 4] = make_int4(oi[j], oi[j + 1], oi[j + 2], oi[j + 3]);
  }
}

// ------------------------------------------------------------------ K11
// One warp per point.  d <= 256: four candidates at a time, eight lanes
// each, every lane reading 16-byte pieces of the candidate row (a group reads
// 128 contiguous bytes per load); d > 256: one candidate at a time over the
// whole warp (lane l holds dimensions 4l..4l+3 of every 128-wide chunk).
// Each lane adds its squared differences with fused multiply-adds and a
// fixed butterfly adds the lane sums: an FP32 distance with pairwise
// summation, the same on every run.  Lane j then holds candidate j (j < K2)
// and the K2 pairs are sorted with a bitonic network; candidates whose
// distance lies within 2^-16 of the k-th are re-ordered by an FP64
// distance.  d must be a multiple of 4.
template <typename T, int D, int K2>
__global__ void __launch_bounds__(256) k_rerank(const T *__restrict__ X, int d,
                                                const int32_t *__restrict__ visit, int64_t n,
                                                const int32_t *__restrict__ ci, int k,
                                                int32_t *__restrict__ oi, float *__restrict__ od) {
  const int lane = threadIdx.x & 31;
  const int g = 0, j = lane;  // one point per warp: the group is the warp
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n) return;  // warp-uniform
  const bool live = true;
  const int32_t p = visit ? __ldg(visit + w) : (int32_t)w;
  const float inf = __int_as_float(0x7f800000);
  const int32_t c = lane < K2 ? __ldg(ci + (int64_t)p * K2 + lane) : -1;
  float dist = inf;
  if constexpr (D <= 256) {
    // four candidates per pass, eight lanes each: lane s of group g holds
    // dimensions 4s + 32t .. +3 (t < D / 32) of the query and adds the
    // squared differences of those dimensions of candidate 4 pass + g; a
    // fixed butterfly over the group's lanes completes the sum
    constexpr int NQ = D / 32;
    const int grp = lane >> 3, sl = lane & 7;
    float q[NQ][4];
    const T *xp = X + (int64_t)p * d;
#pragma unroll
    for (int t = 0; t < NQ; ++t) {
      const int c0 = 32 * t + 4 * sl;
      q[t][0] = q[t][1] = q[t][2] = q[t][3] = 0.0f;
      if (c0 < d) load4<T>(xp + c0, q[t]);
    }
#pragma unroll
    for (int pass = 0; pass < K2 / 4; ++pass) {
      const int32_t cj = __shfl_sync(kFull, c, 4 * pass + grp);
      float acc = 0.0f;
      if (cj >= 0) {
        const T *xc = X + (int64_t)cj * d;
#pragma unroll
        for (int t = 0; t < NQ; ++t) {
          const int c0 = 32 * t + 4 * sl;
          if (c0 < d) {
            float v[4];
            load4<T>(xc + c0, v);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const float df = v[e] - q[t][e];
              acc = fmaf(df, df, acc);
            }
          }
        }
      }
      acc += __shfl_xor_sync(kFull, acc, 4);
      acc += __shfl_xor_sync(kFull, acc, 2);
      acc += __shfl_xor_sync(kFull, acc, 1);
      const float got = __shfl_sync(kFull, acc, 8 * (lane & 3));
      if ((lane >> 2) == pass && c >= 0) dist = sqrtf(got);
    }
  } else {
    constexpr int NC = (D + 127) / 128;  // 128-wide chunks (d <= D <= 1024)
    float q[NC][4];
    const T *xp = X + (int64_t)p * d;
#pragma unroll
    for (int h = 0; h < NC; ++h) {
      const int c0 = h * 128 + 4 * lane;
      q[h][0] = q[h][1] = q[h][2] = q[h][3] = 0.0f;
      if (c0 < d) load4<T>(xp + c0, q[h]);
    }
#pragma unroll 4
    for (int jj = 0; jj < K2; ++jj) {
      const int32_t cj = __shfl_sync(kFull, c, jj);
      if (cj < 0) continue;  // warp-uniform
      const T *xc = X + (int64_t)cj * d;
      float acc = 0.0f;
#pragma unroll
      for (int h = 0; h < NC; ++h) {
        const int c0 = h * 128 + 4 * lane;
        if (c0 < d) {
          float v[4];
          load4<T>(xc + c0, v);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float df = v[e] - q[h][e];
            acc = fmaf(df, df, acc);
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
      if (lane == jj) dist = sqrtf(acc);
    }
  }
  int32_t id = c;
  // bitonic sort of K2 (dist, id) pairs inside the group, ascending
#pragma unroll
  for (int size = 2; size <= K2; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const float od_ = __shfl_xor_sync(kFull, dist, stride);
      const int32_t oi_ = __shfl_xor_sync(kFull, id, stride);
      const bool up = ((j & size) == 0);
      const bool lower = (j & stride) == 0;
      const bool mine_first = before(dist, id, od_, oi_);
      const bool keep = (lower == up) ? mine_first : !mine_first;
      if (!keep) {
        dist = od_;
        id = oi_;
      }
    }
  }
  // FP64 check of the candidates near the k-th distance
  const float dk = __shfl_sync(kFull, dist, g * K2 + k - 1);
  const float eps = 1.52587890625e-05f;  // 2^-16
  const bool near = id >= 0 && isfinite(dk) && fabsf(dist - dk) <= eps * dk;
  const unsigned gmask = (K2 == 32 ? 0xffffffffu : ((1u << K2) - 1u)) << (g * K2);
  const unsigned wmask = __ballot_sync(kFull, near) & gmask;
  const unsigned below = gmask & ((1u << (g * K2 + k)) - 1u);
  if (__any_sync(kFull, (wmask & below) != 0 && (wmask & ~below) != 0)) {
    const bool act = (wmask & below) != 0 && (wmask & ~below) != 0;  // group-uniform
    double d64 = 1e300;
    if (act && near) {
      const T *xp = X + (int64_t)p * d, *xc = X + (int64_t)id * d;
      double s = 0.0;
      for (int i = 0; i < d; ++i) {
        const double df = (double)xc[i] - (double)xp[i];
        s += df * df;
      }
      d64 = sqrt(s);
    }
    // re-order the window by (FP64 distance, id); other lanes keep their place
    const int first = act ? __ffs(wmask) - 1 : lane;
    int rank = 0;
    for (int q = 0; q < 32; ++q) {
      const double oq = __shfl_sync(kFull, d64, q);
      const int32_t iq = __shfl_sync(kFull, id, q);
      if (act && near && ((wmask >> q) & 1u) &&
          (oq < d64 || (oq == d64 && (uint32_t)iq < (uint32_t)id)))
        ++rank;
    }
    const int dest = (act && near) ? first + rank : lane;
    float nd = dist;
    int32_t ni = id;
    for (int q = 0; q < 32; ++q) {
      const int dq = __shfl_sync(kFull, dest, q);
      const float dv = __shfl_sync(kFull, dist, q);
      const int32_t iv = __shfl_sync(kFull, id, q);
      if (act && ((wmask >> q) & 1u) && dq == lane) {
        nd = dv;
        ni = iv;
      }
    }
    dist = nd;
    id = ni;
  }
  if (live && j < k) {
    oi[(int64_t)p * k + j] = id;
    od[(int64_t)p * k + j] = id >= 0 ? dist : inf;
  }
}

template <typename T, int D, int K2>
drpt_status launch_rerank_t(const void *X, int d, const int32_t *visit, int64_t n,
                            const int32_t *cand, int k, int32_t *out_idx, float *out_dist,
                            cudaStream_t s) {
  const int64_t warps = n;
  const unsigned grid = (unsigned)ceil_div(warps * 32, 256);
  k_rerank<T, D, K2><<<grid, 256, 0, s>>>((const T *)X, d, visit, n, cand, k, out_idx, out_dist);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

template <typename T, int K2>
drpt_status launch_rerank_d(const void *X, int d, const int32_t *visit, int64_t n,
                            const int32_t *cand, int k, int32_t *out_idx, float *out_dist,
                            cudaStream_t s) {
  // D: an upper bound of d in whole 128-value chunks (the kernel guards c0 < d)
  if (d <= 128) return launch_rerank_t<T, 128, K2>(X, d, visit, n, cand, k, out_idx, out_dist, s);
  if (d <= 256) return launch_rerank_t<T, 256, K2>(X, d, visit, n, cand, k, out_idx, out_dist, s);
  if (d <= 512) return launch_rerank_t<T, 512, K2>(X, d, visit, n, cand, k, out_idx, out_dist, s);
  return launch_rerank_t<T, 1024, K2>(X, d, visit, n, cand, k, out_idx, out_dist, s);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

drpt_status make_tmap(CUtensorMap *map, const void *base, int64_t rows, int d_pad, int box_rows,
                      bool fp8) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available");
    return DRPT_ERR_CUDA;
  }
  const int esz = fp8 ? 1 : 2;
  cuuint64_t dims[2] = {(cuuint64_t)d_pad, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)d_pad * esz};
  cuuint32_t box[2] = {(cuuint32_t)(128 / esz), (cuuint32_t)box_rows};  // 128-byte rows
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, fp8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                  const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return DRPT_ERR_CUDA;
  }
  return DRPT_OK;
}

template <typename T, int NCH>
void stage_t(const LeafStageArgs &a, bool means, cudaStream_t s) {
  const T *X = (const T *)a.X;
  if (means) {
    const dim3 g((unsigned)a.nleaf, (unsigned)a.T);
    k_leaf_index<<<g, 256, 0, s>>>(a.order, a.goff, a.n, a.nleaf, a.pos, a.lf);
    k_leaf_mean<T, NCH><<<g, 256, 0, s>>>(X, a.n, a.d, a.order, a.goff, a.nleaf, a.mu);
    return;
  }
  constexpr int RB = StageCfg<NCH>::rb;
  // one resident round of blocks, each warp looping over its points
  const bool full = a.d == NCH * 128 && a.d_pad == NCH * 128;
  auto kern = a.fp8 ? (full ? k_leaf_stage<T, NCH, true, true> : k_leaf_stage<T, NCH, true, false>)
                    : (full ? k_leaf_stage<T, NCH, false, true> : k_leaf_stage<T, NCH, false, false>);
  static int per_sm = 0;  // the four forms use the same registers within a few
  if (per_sm == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
  }
  const int sms = device_sm_count();
  const unsigned grid =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(a.n, 8 * RB), (int64_t)sms * per_sm));
  const int64_t toff = (int64_t)a.t0 * a.n;
  const float *mu = a.mu + (int64_t)a.t0 * a.nleaf * a.d;
  kern<<<grid, 256, 0, s>>>(X, a.n, a.d, a.d_pad, a.pos + toff, a.lf + toff, mu, a.nleaf, a.tc,
                            a.Xb, a.nrm, a.scl);
}

template <typename T>
void stage_d(const LeafStageArgs &a, bool means, cudaStream_t s) {
  if (a.d_pad <= 128) stage_t<T, 1>(a, means, s);
  else if (a.d_pad <= 256) stage_t<T, 2>(a, means, s);
  else if (a.d_pad <= 512) stage_t<T, 4>(a, means, s);
  else stage_t<T, 8>(a, means, s);
}

template <int KP, bool STREAM, bool FP8>
drpt_status mma_t(const MixedTreeArgs &a, const CUtensorMap &tmA, int kb, cudaStream_t s) {
  using Cfg = MmaCfg<KP, STREAM>;
  CUtensorMap tmB;
  DRPT_TRY(make_tmap(&tmB, a.Xb, a.n, a.d_pad, Cfg::tn, a.fp8));
  const MmaSmem L = mma_smem_layout(kb, STREAM, Cfg::stages, Cfg::slots, Cfg::tn, Cfg::groups);
  const size_t smem = L.total + 1024;
  if (smem > 227 * 1024) {
    set_error("mixed leaf kernel: %zu bytes of shared memory needed", smem);
    return DRPT_ERR_UNSUPPORTED;
  }
  const unsigned grid = (unsigned)(ceil_div(a.n, kTM) + a.nleaf);
  DRPT_CUDA(cudaFuncSetAttribute(k_leaf_mma<KP, STREAM, FP8>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_leaf_mma<KP, STREAM, FP8><<<grid, Cfg::threads, smem, s>>>(
      tmA, tmB, a.goff, a.order, a.nrm, a.scl, a.tile_leaf, a.tile_r0, a.n_tiles, kb, a.tree,
      a.cand_idx, a.cand_dist, a.tree_idx, a.tree_dist, a.err);
  DRPT_LAUNCH_CHECK();
  if (a.tree > 0) DRPT_TRY(launch_fold_lists(a, s));
  return DRPT_OK;
}

template <int KP>
drpt_status mma_kp(const MixedTreeArgs &a, const CUtensorMap &tmA, int kb, cudaStream_t s) {
  // Resident A only for up to two K blocks: beyond that the streamed
  // stages fit two CTAs per SM where a resident A tile fits one.
  const bool stream = kb > 2;
  if (a.fp8)
    return stream ? mma_t<KP, true, true>(a, tmA, kb, s) : mma_t<KP, false, true>(a, tmA, kb, s);
  return stream ? mma_t<KP, true, false>(a, tmA, kb, s) : mma_t<KP, false, false>(a, tmA, kb, s);
}

}  // namespace

// Padded row length of the mixed form's tensor-core operand: whole 128-byte
// K blocks (64 BF16 or 128 E4M3 values).
int mixed_d_pad(int d, int fp8) { return fp8 ? (d + 127) / 128 * 128 : (d + 63) / 64 * 64; }

static drpt_status stage_check(const LeafStageArgs &a) {
  if (a.d % 4 != 0 || a.d > 1024 || a.d_pad != mixed_d_pad(a.d, a.fp8)) {
    set_error("mixed mode needs d %% 4 == 0 and d <= 1024 (got %d)", a.d);
    return DRPT_ERR_UNSUPPORTED;
  }
  return DRPT_OK;
}

drpt_status launch_leaf_means(const LeafStageArgs &a, cudaStream_t s) {
  DRPT_TRY(stage_check(a));
  if (a.dtype == DRPT_DTYPE_U8) stage_d<uint8_t>(a, true, s);
  else stage_d<float>(a, true, s);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_leaf_stage(const LeafStageArgs &a, cudaStream_t s) {
  DRPT_TRY(stage_check(a));
  if (a.dtype == DRPT_DTYPE_U8) stage_d<uint8_t>(a, false, s);
  else stage_d<float>(a, false, s);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

int mixed_stage_trees(int64_t n, int d_pad, int fp8, int T) {
  // centred rows of as many trees as fit in 8 GiB
  const int64_t per_tree = n * d_pad * (fp8 ? 1 : 2);
  const int64_t fit = per_tree > 0 ? ((int64_t)8 << 30) / per_tree : T;
  return (int)std::max<int64_t>(1, std::min<int64_t>(T, fit));
}

drpt_status launch_leaf_mma(const MixedTreeArgs &a, cudaStream_t s) {
  const int esz = a.fp8 ? 1 : 2;
  if ((a.d_pad * esz) % 128 != 0 || a.d_pad > 1024) {
    set_error("mixed leaf kernel: padded dimension %d unsupported", a.d_pad);
    return DRPT_ERR_UNSUPPORTED;
  }
  k_tile_plan<<<1, 1024, 0, s>>>(a.goff, a.nleaf, kTM, a.tile_leaf, a.tile_r0, a.n_tiles);
  DRPT_LAUNCH_CHECK();
  CUtensorMap tmA;
  DRPT_TRY(make_tmap(&tmA, a.Xb, a.n, a.d_pad, kTM, a.fp8));
  const int kb = a.d_pad * esz / 128;
  if (a.kp == 16) return mma_kp<16>(a, tmA, kb, s);
  if (a.kp == 32) return mma_kp<32>(a, tmA, kb, s);
  set_error("mixed leaf kernel: %d candidates per tree unsupported (16 or 32)", a.kp);
  return DRPT_ERR_UNSUPPORTED;
}

drpt_status launch_tile_plan(const int32_t *goff, int nleaf, int rows, int32_t *tile_leaf,
                             int32_t *tile_r0, int32_t *n_tiles, cudaStream_t s) {
  k_tile_plan<<<1, 1024, 0, s>>>(goff, nleaf, rows, tile_leaf, tile_r0, n_tiles);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_fold_lists(const MixedTreeArgs &a, cudaStream_t s) {
  const unsigned grid = (unsigned)ceil_div(a.n, 256);
  if (a.kp == 16)
    k_fold_lists<16><<<grid, 256, 0, s>>>(a.tree_dist, a.tree_idx, a.n, a.cand_dist, a.cand_idx);
  else if (a.kp == 32)
    k_fold_lists<32><<<grid, 256, 0, s>>>(a.tree_dist, a.tree_idx, a.n, a.cand_dist, a.cand_idx);
  else {
    set_error("fold: %d candidates per tree unsupported (16 or 32)", a.kp);
    return DRPT_ERR_UNSUPPORTED;
  }
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_rerank(const void *X, int dtype, int d, const int32_t *visit, int64_t n,
                          const int32_t *cand, int K2, int k, int32_t *out_idx, float *out_dist,
                          cudaStream_t s) {
  if ((K2 != 16 && K2 != 32) || k > K2 || k <= 0) {
    set_error("re-rank: %d candidates for k = %d unsupported (16 or 32)", K2, k);
    return DRPT_ERR_UNSUPPORTED;
  }
  if (d % 4 != 0 || d > 1024) {
    set_error("re-rank needs d %% 4 == 0 and d <= 1024 (got %d)", d);
    return DRPT_ERR_UNSUPPORTED;
  }
  if (dtype == DRPT_DTYPE_U8)
    return K2 == 16 ? launch_rerank_d<uint8_t, 16>(X, d, visit, n, cand, k, out_idx, out_dist, s)
                    : launch_rerank_d<uint8_t, 32>(X, d, visit, n, cand, k, out_idx, out_dist, s);
  return K2 == 16 ? launch_rerank_d<float, 16>(X, d, visit, n, cand, k, out_idx, out_dist, s)
                  : launch_rerank_d<float, 32>(X, d, visit, n, cand, k, out_idx, out_dist, s);
}

}  // namespace drpt
