// K6 -- exact FP32 brute force inside every final leaf (MDRPT::calculate_nns,
// mdrpt.cpp:123-212, with MathOp::calculate_distance, math_operations.cpp:
// 385-396).
//
// One thread block per (tree, final leaf).  The leaf's rows are gathered from
// X in chunks of 32 dimensions into shared memory (zero-padded past d); 256
// threads on a 16 x 16 grid each own an MT x MT block of (row, column) pairs
// of a TM x TM tile (TM = 16 * MT) and keep the distance chains in
// registers:  acc = acc + (q_i - p_i)^2 for i ascending, each subtract,
// multiply and add rounded on its own, then sqrt -- the reference's saxpy
// (-1) + snrm2 sequence, so every distance is bit-identical to the
// reference's (a zero-padded dimension adds (0 - 0)^2 = +0, which leaves a
// non-negative sum unchanged).  One thread per row then folds the tile's
// candidates into the row's running k nearest by (distance, index), skipping
// the point itself.  Two instantiations: TM = 64 serves leaves of up to 64
// points and those above 128 (looping over 64 x 64 tiles), TM = 128 the
// leaves of 65 to 128 points in one tile; each launch covers every leaf and
// returns at once for the other class.
//
// Output: for point p and tree t, cand[(p*T + t)*k + j], j < k, sorted; slots
// beyond the leaf size hold index -1 and distance +inf.
#include "kernels.cuh"

namespace drpt {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 32;             // dimensions staged per step
constexpr int kLd = kChunk + 1;        // padded row stride in shared memory

template <int TM, typename T>
__device__ __forceinline__ void stage_rows(float *dst, const T *__restrict__ X, int d,
                                           const int32_t *ids, int rows, int k0) {
  for (int e = threadIdx.x; e < TM * kChunk; e += kThreads) {
    const int r = e / kChunk, kk = e - r * kChunk;
    float v = 0.0f;
    if (r < rows && k0 + kk < d) v = (float)X[(int64_t)ids[r] * d + k0 + kk];
    dst[r * kLd + kk] = v;
  }
}

template <int TM>
constexpr size_t leaf_smem(int k) {
  return sizeof(float) * (2 * TM * kLd + TM * (TM + 1)) +
         (sizeof(float) + sizeof(int32_t)) * TM * (k + 1) + sizeof(int32_t) * 2 * TM;
}

template <int TM, typename T>
__global__ void __launch_bounds__(kThreads) k_leaf_knn(LeafKnnArgs a) {
  constexpr int MT = TM / 16;
  // TM = 128 serves 64 < m <= 128 (one tile); TM = 64 serves m <= 64 and,
  // with less padding than 128-wide tiles, every leaf above 128.
  extern __shared__ float smem[];
  float *xr = smem;                          // TM x kLd
  float *xc = xr + TM * kLd;                 // TM x kLd
  float *dt = xc + TM * kLd;                 // TM x (TM + 1)
  float *topd = dt + TM * (TM + 1);          // TM x (k + 1)
  int32_t *topi = (int32_t *)(topd + TM * (a.k + 1));
  int32_t *rid = topi + TM * (a.k + 1);      // TM
  int32_t *cid = rid + TM;                   // TM

  const int t = blockIdx.x / a.n_final, f = blockIdx.x - t * a.n_final;
  const int32_t *off = a.final_off + (int64_t)t * (a.n_final + 1);
  const int32_t b = off[f], m = off[f + 1] - b;
  const bool mine = TM == 128 ? (m > 64 && m <= 128) : (m <= 64 || m > 128);
  if (!mine) return;
  const int32_t *members = a.final_order + (int64_t)t * a.n + b;
  const T *X = (const T *)a.X;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int kp1 = a.k + 1;
  const float inf = __int_as_float(0x7f800000);

  for (int r0 = 0; r0 < m; r0 += TM) {
    const int rows = min(TM, m - r0);
    for (int i = threadIdx.x; i < TM * kp1; i += kThreads) {
      topd[i] = inf;
      topi[i] = INT32_MAX;
    }
    if (threadIdx.x < TM) rid[threadIdx.x] = threadIdx.x < rows ? members[r0 + threadIdx.x] : -1;
    for (int c0 = 0; c0 < m; c0 += TM) {
      const int cols = min(TM, m - c0);
      const bool same = (c0 == r0);
      if (threadIdx.x < TM) cid[threadIdx.x] = threadIdx.x < cols ? members[c0 + threadIdx.x] : -1;
      __syncthreads();
      float acc[MT][MT];
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < MT; ++j) acc[i][j] = 0.0f;
      const float *xcol = same ? xr : xc;
      for (int k0 = 0; k0 < a.d; k0 += kChunk) {
        stage_rows<TM>(xr, X, a.d, rid, rows, k0);
        if (!same) stage_rows<TM>(xc, X, a.d, cid, cols, k0);
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < kChunk; ++kk) {
          float av[MT], bv[MT];
#pragma unroll
          for (int i = 0; i < MT; ++i) av[i] = xr[(ty + 16 * i) * kLd + kk];
#pragma unroll
          for (int j = 0; j < MT; ++j) bv[j] = xcol[(tx + 16 * j) * kLd + kk];
#pragma unroll
          for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < MT; ++j) {
              const float df = __fsub_rn(bv[j], av[i]);
              acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(df, df));
            }
        }
        __syncthreads();
      }
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < MT; ++j) dt[(ty + 16 * i) * (TM + 1) + tx + 16 * j] = __fsqrt_rn(acc[i][j]);
      __syncthreads();
      if (threadIdx.x < rows) {
        const int r = threadIdx.x;
        const int32_t p = rid[r];
        float *ld = topd + r * kp1;
        int32_t *li = topi + r * kp1;
        float wd = ld[a.k - 1];
        int32_t wi = li[a.k - 1];
        for (int c = 0; c < cols; ++c) {
          const int32_t q = cid[c];
          const float dv = dt[r * (TM + 1) + c];
          if (q == p || !(dv < wd || (dv == wd && q < wi))) continue;
          int j = a.k - 1;
          while (j > 0 && (dv < ld[j - 1] || (dv == ld[j - 1] && q < li[j - 1]))) {
            ld[j] = ld[j - 1];
            li[j] = li[j - 1];
            --j;
          }
          ld[j] = dv;
          li[j] = q;
          wd = ld[a.k - 1];
          wi = li[a.k - 1];
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
        a.cand_dist[o + j] = have ? topd[r * kp1 + j] : inf;
      }
    }
    __syncthreads();
  }
}

template <int TM, typename T>
drpt_status launch_one(const LeafKnnArgs &a, unsigned blocks, cudaStream_t s) {
  const size_t smem = leaf_smem<TM>(a.k);
  DRPT_CUDA(cudaFuncSetAttribute(k_leaf_knn<TM, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  k_leaf_knn<TM, T><<<blocks, kThreads, smem, s>>>(a);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace

drpt_status launch_leaf_knn_exact(const LeafKnnArgs &a, cudaStream_t s) {
  if (a.k <= 0 || a.k > kMaxK) {
    set_error("leaf k-NN: k = %d outside [1, %d]", a.k, kMaxK);
    return DRPT_ERR_UNSUPPORTED;
  }
  const int64_t blocks = (int64_t)a.T * a.n_final;
  if (blocks <= 0) return DRPT_OK;
  if (blocks > 0x7fffffff) return DRPT_ERR_UNSUPPORTED;
  if (a.dtype == DRPT_DTYPE_U8) {
    DRPT_TRY((launch_one<64, uint8_t>(a, (unsigned)blocks, s)));
    DRPT_TRY((launch_one<128, uint8_t>(a, (unsigned)blocks, s)));
  } else {
    DRPT_TRY((launch_one<64, float>(a, (unsigned)blocks, s)));
    DRPT_TRY((launch_one<128, float>(a, (unsigned)blocks, s)));
  }
  return DRPT_OK;
}

int leaf_knn_exact_kernels() { return 2; }

}  // namespace drpt
