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
// points, column set).  The rows are staged as floats with a row stride of
// d + 1 (odd for even d, so 32 lanes reading one dimension of 32 rows hit 32
// banks).  Staging: the block's rows are one contiguous range of d / 4 quads
// per row; thread t takes quads t, t + 256, ..., eight loads in flight
// before their stores.  Products: warp w takes output columns w, w + 8, ...;
// lane l the points l + 32 i (i < PPL, PPL * 32 >= points), PPL independent
// sums that share each nonzero of the column.
template <typename T, int PPL>
__global__ void __launch_bounds__(kThreads) k_project(const T *__restrict__ X, int64_t n, int d,
                                                      CscDev csc, float *__restrict__ P, int pts) {
  extern __shared__ float xs[];  // pts x (d + 1)
  int64_t p0 = (int64_t)blockIdx.x * pts;
  int np = (int)min64(pts, n - p0);
  if (csc.blocks) {
    const int32_t *b = csc.blocks + 3 * (int64_t)blockIdx.x;
    p0 = b[0];
    np = b[1];
    csc.colptr += (int64_t)b[2] * (csc.ncols + 1);
  }
  if (np <= 0) return;  // uniform for the whole block
  const int ld = d + 1;
  const T *src = X + p0 * d;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (d % 4 == 0) {
    constexpr int kBatch = 8;
    const int q4 = d >> 2, total = np * q4;
    // quad qi = r * q4 + c4, walked in steps of kThreads without division
    int r = threadIdx.x / q4, c4 = threadIdx.x - r * q4;
    const int dr = kThreads / q4, dc = kThreads - dr * q4;
    for (int qb = threadIdx.x; qb < total; qb += kBatch * kThreads) {
      float4 v[kBatch];
      int rr[kBatch], cc[kBatch];
#pragma unroll
      for (int i = 0; i < kBatch; ++i) {
        rr[i] = r;
        cc[i] = c4;
        if (qb + i * kThreads < total) v[i] = load4v(src + (int64_t)r * d + 4 * c4);
        r += dr;
        c4 += dc;
        if (c4 >= q4) {
          c4 -= q4;
          ++r;
        }
      }
#pragma unroll
      for (int i = 0; i < kBatch; ++i) {
        if (qb + i * kThreads < total) {
          float *dst = xs + rr[i] * ld + 4 * cc[i];
          dst[0] = v[i].x;
          dst[1] = v[i].y;
          dst[2] = v[i].z;
          dst[3] = v[i].w;
        }
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
  // rows past the block's points read its last row and are not written
  int off[PPL];
#pragma unroll
  for (int i = 0; i < PPL; ++i) off[i] = min(lane + 32 * i, np - 1) * ld;
  for (int col = warp; col < csc.ncols; col += kThreads / 32) {
    const int e0 = __ldg(csc.colptr + col), e1 = __ldg(csc.colptr + col + 1);
    float acc[PPL];
#pragma unroll
    for (int i = 0; i < PPL; ++i) acc[i] = 0.0f;
    for (int e = e0; e < e1; ++e) {
      const int k = __ldg(csc.row + e);
      const float b = __ldg(csc.val + e);
#pragma unroll
      for (int i = 0; i < PPL; ++i) acc[i] = __fadd_rn(acc[i], __fmul_rn(xs[off[i] + k], b));
    }
    float *out = P + (int64_t)col * n + p0;
#pragma unroll
    for (int i = 0; i < PPL; ++i)
      if (lane + 32 * i < np) out[lane + 32 * i] = acc[i];
  }
}

template <typename T>
void project_t(const void *X, int64_t n, int d, const CscDev &csc, float *P, int pts,
               unsigned grid, size_t smem, cudaStream_t s) {
  auto launch = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<grid, kThreads, smem, s>>>((const T *)X, n, d, csc, P, pts);
  };
  if (pts <= 32) launch(k_project<T, 1>);
  else if (pts <= 64) launch(k_project<T, 2>);
  else launch(k_project<T, 4>);
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
  if (dtype == DRPT_DTYPE_U8) project_t<uint8_t>(X, n, d, csc, P, pts, grid, smem, s);
  else project_t<float>(X, n, d, csc, P, pts, grid, smem, s);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt
