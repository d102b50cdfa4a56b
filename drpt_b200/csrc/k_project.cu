// K1 -- sparse random projection P = X.B (math_operations.cpp:15-46 through
// an ordered sgemm).  HBM-bound: each point row is read once, coalesced, into
// shared memory; each output column is written once, coalesced.
//
// Per output element the sum runs over the nonzeros of B's column in
// ascending k with one rounded multiply and one rounded add per term
// (__fmul_rn / __fadd_rn, never contracted).  Zero entries of B are skipped:
// for finite inputs they add +-0 to an accumulator that starts at +0 and so
// never changes it, which keeps P bit-identical to the sequential sum over
// all d terms.
#include "kernels.cuh"

namespace drpt {
namespace {

constexpr int kThreads = 256;

template <typename T>
__device__ __forceinline__ float to_f(T v) { return (float)v; }

// Four consecutive elements (16-byte or 4-byte aligned: d % 4 == 0) as floats.
__device__ __forceinline__ float4 load4v(const float *p) {
  return __ldg(reinterpret_cast<const float4 *>(p));
}
__device__ __forceinline__ float4 load4v(const uint8_t *p) {
  const uchar4 q = __ldg(reinterpret_cast<const uchar4 *>(p));
  return make_float4(q.x, q.y, q.z, q.w);
}

// Block: `pts` consecutive points (or the block table's entry: first point,
// points, column set); thread pairs (point, column) with the point index
// fastest so a warp writes 32 consecutive P entries of a column.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_project(const T *__restrict__ X, int64_t n, int d,
                                                      CscDev csc, float *__restrict__ P, int pts) {
  extern __shared__ float xs[];  // pts x (d + 1), padded against bank conflicts
  int64_t p0 = (int64_t)blockIdx.x * pts;
  int np = (int)min64(pts, n - p0);
  if (csc.blocks) {
    const int32_t *b = csc.blocks + 3 * (int64_t)blockIdx.x;
    p0 = b[0];
    np = b[1];
    csc.colptr += (int64_t)b[2] * (csc.ncols + 1);
  }
  const int ld = d + 1;
  const T *src = X + p0 * d;
  if (d % 4 == 0) {
    // Stage the rows with 4-element loads: warp w takes rows w, w + 8, ...,
    // lane l the quads l, l + 32, ... of a row (no index division).
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q4 = d >> 2;
#pragma unroll 2
    for (int r = warp; r < np; r += kThreads / 32) {
      const T *row = src + (int64_t)r * d;
      float *dst = xs + r * ld;
      for (int c4 = lane; c4 < q4; c4 += 32) {
        const float4 v = load4v(row + 4 * c4);
        dst[4 * c4] = v.x;
        dst[4 * c4 + 1] = v.y;
        dst[4 * c4 + 2] = v.z;
        dst[4 * c4 + 3] = v.w;
      }
    }
  } else {
    // consecutive threads read consecutive elements of a row
    const int total = np * d;
    for (int e = threadIdx.x; e < total; e += kThreads) {
      const int r = e / d, c = e - r * d;
      xs[r * ld + c] = to_f(src[e]);
    }
  }
  __syncthreads();
  // pairs q = col * np + r, walked in steps of the block size without division
  const int pairs = np * csc.ncols;
  int col = threadIdx.x / np, r = threadIdx.x - col * np;
  for (int q = threadIdx.x; q < pairs; q += kThreads) {
    const int e0 = __ldg(csc.colptr + col), e1 = __ldg(csc.colptr + col + 1);
    const float *x = xs + r * ld;
    float acc = 0.0f;
    for (int e = e0; e < e1; ++e) acc = __fadd_rn(acc, __fmul_rn(x[__ldg(csc.row + e)], __ldg(csc.val + e)));
    P[(int64_t)col * n + p0 + r] = acc;
    r += kThreads;
    while (r >= np) {
      r -= np;
      ++col;
    }
  }
}

}  // namespace

int project_points_per_block(int d) {
  // About 96 KB of staged rows per block, at least 8 and at most 128 points.
  const int pts = (int)(96 * 1024 / ((d + 1) * (int)sizeof(float)));
  return pts < 8 ? 8 : (pts > 128 ? 128 : pts);
}

drpt_status launch_project(const void *X, int dtype, int64_t n, int d, const CscDev &csc,
                           float *P, cudaStream_t s) {
  if (n <= 0 || csc.ncols <= 0) return DRPT_OK;
  const int pts = project_points_per_block(d);
  const size_t smem = (size_t)pts * (d + 1) * sizeof(float);
  if (smem > 227 * 1024) {
    set_error("projection: d = %d too large for one staged row block", d);
    return DRPT_ERR_UNSUPPORTED;
  }
  const unsigned grid = csc.blocks ? (unsigned)csc.nblocks : (unsigned)ceil_div(n, pts);
  if (dtype == DRPT_DTYPE_U8) {
    DRPT_CUDA(cudaFuncSetAttribute(k_project<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    k_project<uint8_t><<<grid, kThreads, smem, s>>>((const uint8_t *)X, n, d, csc, P, pts);
  } else {
    DRPT_CUDA(cudaFuncSetAttribute(k_project<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    k_project<float><<<grid, kThreads, smem, s>>>((const float *)X, n, d, csc, P, pts);
  }
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt
