// K6 -- exact FP32 brute force inside every final leaf (MDRPT::calculate_nns,
// mdrpt.cpp:123-212, with MathOp::calculate_distance, math_operations.cpp:
// 385-396).
//
// One thread block per (tree, final leaf).  The leaf's rows are gathered from
// X in chunks of 32 dimensions into shared memory; 256 threads each own a 4x4
// block of (row, column) pairs of a 64x64 tile and keep the distance chains
// in registers:  acc = acc + (q_i - p_i)^2 for i ascending, each subtract,
// multiply and add rounded on its own, then sqrt -- the reference's saxpy
// (-1) + snrm2 sequence, so every distance is bit-identical to the
// reference's.  One thread per row then folds the tile's 64 candidates into
// the row's running k nearest by (distance, index), skipping the point
// itself.  Leaves larger than 64 loop over 64x64 tiles.
//
// Output: for point p and tree t, cand[(p*T + t)*k + j], j < k, sorted; slots
// beyond the leaf size hold index -1 and distance +inf.
#include "kernels.cuh"

namespace drpt {
namespace {

constexpr int kThreads = 256;
constexpr int kTile = 64;
constexpr int kChunk = 32;             // dimensions staged per step
constexpr int kLd = kChunk + 1;        // padded row stride in shared memory

template <typename T>
__device__ __forceinline__ void stage_rows(float *dst, const T *__restrict__ X, int d,
                                           const int32_t *ids, int rows, int k0, int kc) {
  for (int e = threadIdx.x; e < kTile * kChunk; e += kThreads) {
    const int r = e / kChunk, kk = e - r * kChunk;
    float v = 0.0f;
    if (r < rows && kk < kc) v = (float)X[(int64_t)ids[r] * d + k0 + kk];
    dst[r * kLd + kk] = v;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_leaf_knn(LeafKnnArgs a) {
  extern __shared__ float smem[];
  float *xr = smem;                          // kTile x kLd
  float *xc = xr + kTile * kLd;              // kTile x kLd
  float *dt = xc + kTile * kLd;              // kTile x (kTile + 1)
  float *topd = dt + kTile * (kTile + 1);    // kTile x (k + 1)
  int32_t *topi = (int32_t *)(topd + kTile * (a.k + 1));
  int32_t *rid = topi + kTile * (a.k + 1);   // kTile
  int32_t *cid = rid + kTile;                // kTile

  const int t = blockIdx.x / a.n_final, f = blockIdx.x - t * a.n_final;
  const int32_t *off = a.final_off + (int64_t)t * (a.n_final + 1);
  const int32_t b = off[f], m = off[f + 1] - b;
  const int32_t *members = a.final_order + (int64_t)t * a.n + b;
  const T *X = (const T *)a.X;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int kp1 = a.k + 1;

  for (int r0 = 0; r0 < m; r0 += kTile) {
    const int rows = min(kTile, m - r0);
    for (int i = threadIdx.x; i < kTile * kp1; i += kThreads) {
      topd[i] = __int_as_float(0x7f800000);  // +inf
      topi[i] = INT32_MAX;
    }
    if (threadIdx.x < kTile) rid[threadIdx.x] = threadIdx.x < rows ? members[r0 + threadIdx.x] : -1;
    for (int c0 = 0; c0 < m; c0 += kTile) {
      const int cols = min(kTile, m - c0);
      const bool same = (c0 == r0);
      if (threadIdx.x < kTile) cid[threadIdx.x] = threadIdx.x < cols ? members[c0 + threadIdx.x] : -1;
      __syncthreads();
      float acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
      const float *xcol = same ? xr : xc;
      for (int k0 = 0; k0 < a.d; k0 += kChunk) {
        const int kc = min(kChunk, a.d - k0);
        stage_rows(xr, X, a.d, rid, rows, k0, kc);
        if (!same) stage_rows(xc, X, a.d, cid, cols, k0, kc);
        __syncthreads();
        for (int kk = 0; kk < kc; ++kk) {
          float av[4], bv[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) av[i] = xr[(ty + 16 * i) * kLd + kk];
#pragma unroll
          for (int j = 0; j < 4; ++j) bv[j] = xcol[(tx + 16 * j) * kLd + kk];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const float df = __fsub_rn(bv[j], av[i]);
              acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(df, df));
            }
        }
        __syncthreads();
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dt[(ty + 16 * i) * (kTile + 1) + tx + 16 * j] = __fsqrt_rn(acc[i][j]);
      __syncthreads();
      if (threadIdx.x < rows) {
        const int r = threadIdx.x;
        const int32_t p = rid[r];
        float *ld = topd + r * kp1;
        int32_t *li = topi + r * kp1;
        for (int c = 0; c < cols; ++c) {
          const int32_t q = cid[c];
          if (q == p) continue;
          const float dv = dt[r * (kTile + 1) + c];
          const float wd = ld[a.k - 1];
          if (!(dv < wd || (dv == wd && q < li[a.k - 1]))) continue;
          int j = a.k - 1;
          while (j > 0 && (dv < ld[j - 1] || (dv == ld[j - 1] && q < li[j - 1]))) {
            ld[j] = ld[j - 1];
            li[j] = li[j - 1];
            --j;
          }
          ld[j] = dv;
          li[j] = q;
        }
      }
      __syncthreads();
    }
    if (threadIdx.x < rows) {
      const int r = threadIdx.x;
      const int64_t o = ((int64_t)rid[r] * a.T + t) * a.k;
      for (int j = 0; j < a.k; ++j) {
        const bool have = topi[r * kp1 + j] != INT32_MAX;
        a.cand_idx[o + j] = have ? topi[r * kp1 + j] : -1;
        a.cand_dist[o + j] = have ? topd[r * kp1 + j] : __int_as_float(0x7f800000);
      }
    }
    __syncthreads();
  }
}

}  // namespace

drpt_status launch_leaf_knn_exact(const LeafKnnArgs &a, cudaStream_t s) {
  if (a.k <= 0 || a.k > kMaxK) {
    set_error("leaf k-NN: k = %d outside [1, %d]", a.k, kMaxK);
    return DRPT_ERR_UNSUPPORTED;
  }
  const int64_t blocks = (int64_t)a.T * a.n_final;
  if (blocks <= 0) return DRPT_OK;
  const size_t smem = sizeof(float) * (2 * kTile * kLd + kTile * (kTile + 1)) +
                      (sizeof(float) + sizeof(int32_t)) * kTile * (a.k + 1) + sizeof(int32_t) * 2 * kTile;
  if (a.dtype == DRPT_DTYPE_U8) {
    DRPT_CUDA(cudaFuncSetAttribute(k_leaf_knn<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    k_leaf_knn<uint8_t><<<(unsigned)blocks, kThreads, smem, s>>>(a);
  } else {
    DRPT_CUDA(cudaFuncSetAttribute(k_leaf_knn<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    k_leaf_knn<float><<<(unsigned)blocks, kThreads, smem, s>>>(a);
  }
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt
