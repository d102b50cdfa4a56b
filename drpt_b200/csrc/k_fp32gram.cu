// FP32 CUDA-core form of the whole-leaf brute force (DRPT_MODE_FP32_GRAM):
// the same trees, running list and exact FP32 re-rank as the mixed form, with
// the leaf Gram tiles computed in FP32 by fused multiply-adds on the CUDA
// cores (packed FP32x2 multiply-adds) instead of BF16 tiles on the tensor
// cores.  It is the fastest plain FP32 counterpart of the mixed form (the
// reference's own per-pair subtract / multiply / add sequence, kept bit for
// bit by k_leaf_knn, takes three FP32 operations per dimension and pair; this
// takes one).
//
//   k_row_norms   ||x||^2 of every row in FP32 (once per build)
//   k_leaf_f32    per CTA one 128-row tile of a global leaf against every
//                 128-column tile of the leaf: rows and columns gathered from
//                 X in 32-dimension chunks into shared memory (the next chunk
//                 loaded into registers while the current one is used), an
//                 8 x 8 register block of FFMA dot products per thread, then
//                 score ||y||^2 - 2 x.y per pair; two threads per row keep
//                 the KP best (score, column) pairs of their half of the
//                 columns, merged at the end of the row tile into the tree's
//                 list of the row's point.  (The rows are not centred, so
//                 the scores are large next to the gaps between neighbours:
//                 the mixed form's packed keys, which give up the score's low
//                 13 bits to the column, would rank them too coarsely.)
//
// Reference: the leaf brute force MDRPT::calculate_nns (mdrpt.cpp:123-212)
// with MathOp::calculate_distance (math_operations.cpp:385-396).
#include "kernels.cuh"
#include "sm100.cuh"

namespace drpt {
namespace {

constexpr int kRows = 128;       // rows per tile
constexpr int kCols = 128;       // columns per tile
constexpr int kKc = 32;          // dimensions per staged chunk
constexpr int kThreads = 256;
constexpr int kParts = 2;        // threads per row in the selection
constexpr int kPitch = kCols + 2;  // score-tile row pitch (words)
constexpr int kPool = kRows * kPitch;  // floats of the shared pool
static_assert(2 * kKc * (kRows + kCols) <= kPool, "two buffers of staged chunks fit the pool");
static_assert(2 * 32 * kRows <= kPool, "a 32-entry hand-over list fits the pool");
constexpr size_t kSmem = sizeof(float) * (kPool + kCols) + sizeof(int32_t) * kRows;
constexpr int kMaxLeaf = 1 << 13;  // the mixed form's leaf limit

template <typename T>
__device__ __forceinline__ void load_row8(const T *p, bool in, float *v);
template <>
__device__ __forceinline__ void load_row8<float>(const float *p, bool in, float *v) {
  float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
  if (in) {
    a = __ldg(reinterpret_cast<const float4 *>(p));
    b = __ldg(reinterpret_cast<const float4 *>(p) + 1);
  }
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
template <>
__device__ __forceinline__ void load_row8<uint8_t>(const uint8_t *p, bool in, float *v) {
  uchar4 a = make_uchar4(0, 0, 0, 0), b = a;
  if (in) {
    a = __ldg(reinterpret_cast<const uchar4 *>(p));
    b = __ldg(reinterpret_cast<const uchar4 *>(p) + 1);
  }
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}

// ||x||^2 per row: a warp per row, lanes over 4-value groups, a fixed
// butterfly for the lane sums.
template <typename T>
__global__ void __launch_bounds__(256) k_row_norms(const T *__restrict__ X, int64_t n, int d,
                                                   float *__restrict__ out) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;
  const T *row = X + w * d;
  float s = 0.0f;
  for (int c = 4 * lane; c < d; c += 128)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float v = (float)row[c + e];
      s = fmaf(v, v, s);
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
  if (lane == 0) out[w] = s;
}

// Ascending list of N (score, column) pairs <- the N smallest of it and
// (v, c) by (score, column): one compare-exchange sweep (used to merge two
// lists, where columns interleave).
template <int N>
__device__ __forceinline__ void pair_insert(float *Lv, int32_t *Lc, float v, int32_t c) {
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const bool sw = v < Lv[i] || (v == Lv[i] && c < Lc[i]);
    const float tv = sw ? v : Lv[i];
    const int32_t tc = sw ? c : Lc[i];
    v = sw ? Lv[i] : v;
    c = sw ? Lc[i] : c;
    Lv[i] = tv;
    Lc[i] = tc;
  }
}

// The same for a (v, c) whose column is above every column in the list (the
// scan order): entry i becomes entry i - 1 where v < old entry i - 1, (v, c)
// where it falls between them, else stays; every entry from the old list at
// once, no chain through (v, c).  Equal scores keep the earlier column.
template <int N>
__device__ __forceinline__ void pair_shift_in(float *Lv, int32_t *Lc, float v, int32_t c) {
  bool below[N];
#pragma unroll
  for (int i = 0; i < N; ++i) below[i] = v < Lv[i];
#pragma unroll
  for (int i = N - 1; i > 0; --i) {
    Lv[i] = below[i - 1] ? Lv[i - 1] : (below[i] ? v : Lv[i]);
    Lc[i] = below[i - 1] ? Lc[i - 1] : (below[i] ? c : Lc[i]);
  }
  Lv[0] = below[0] ? v : Lv[0];
  Lc[0] = below[0] ? c : Lc[0];
}

template <typename T, int KP>
__global__ void __launch_bounds__(kThreads, 1) k_leaf_f32(
    const T *__restrict__ X, int d, const int32_t *__restrict__ goff,
    const int32_t *__restrict__ order, const float *__restrict__ xnorm,
    const int32_t *__restrict__ tile_leaf, const int32_t *__restrict__ tile_r0,
    const int32_t *__restrict__ n_tiles, int tree, int32_t *__restrict__ run_idx,
    float *__restrict__ run_dist, int32_t *__restrict__ tree_idx, float *__restrict__ tree_dist,
    int *err) {
  // One dynamic pool, three uses in turn: the staged chunks (As: rows, Bs:
  // columns, dimension-major), the tile's scores St (row pitch kPitch = 2
  // mod 32 words, so that the 16 rows x 2 parts of a warp reading columns
  // 2j + part hit 32 distinct banks), and at the end the list part 1 hands
  // to part 0.
  extern __shared__ __align__(16) float pool[];
  // two buffers of staged chunks: chunk i is used from buffer i & 1 while
  // chunk i + 1 is stored into the other
  auto As = [&](int b) { return reinterpret_cast<float(*)[kRows]>(pool + b * kKc * (kRows + kCols)); };
  auto Bs = [&](int b) {
    return reinterpret_cast<float(*)[kCols]>(pool + b * kKc * (kRows + kCols) + kKc * kRows);
  };
  float(*St)[kPitch] = reinterpret_cast<float(*)[kPitch]>(pool);
  float(*hv)[kRows] = reinterpret_cast<float(*)[kRows]>(pool);                 // [KP][row]
  int32_t(*hc)[kRows] = reinterpret_cast<int32_t(*)[kRows]>(pool + KP * kRows);
  float *cnorm = pool + kPool;                                                 // kCols
  int32_t *rid = reinterpret_cast<int32_t *>(cnorm + kCols);                  // kRows
  const int u = blockIdx.x;
  if (u >= *n_tiles) return;  // uniform for the whole block
  const int leaf = tile_leaf[u], r0 = tile_r0[u];
  const int32_t lo = goff[leaf], m = goff[leaf + 1] - lo;
  if (m > kMaxLeaf) {
    if (threadIdx.x == 0) atomicOr(err, 2);
    return;
  }
  const int rows = min(kRows, m - r0);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  if (tid < kRows) rid[tid] = tid < rows ? __ldg(order + lo + r0 + tid) : -1;
  // selection: row sr, columns 2j + sp of every column tile
  const int sr = tid >> 1, sp = tid & 1;
  float tv[KP];
  int32_t tcol[KP];
#pragma unroll
  for (int j = 0; j < KP; ++j) {
    tv[j] = __int_as_float(0x7f800000);
    tcol[j] = -1;
  }
  const bool svalid = sr < rows;
  const int my_col = r0 + sr;
  __syncthreads();
  // later trees: candidates at or above the KP-th of the point's running
  // list (score = squared distance - ||x||^2) are never kept
  float thr0 = __int_as_float(0x7f800000);
  if (tree > 0 && svalid) {
    const int32_t pt = rid[sr];
    thr0 = run_dist[(int64_t)pt * KP + KP - 1] - __ldg(xnorm + pt);
  }
  // staging: thread takes 16 dimensions of row (or column) tid / 2
  const int sg = tid >> 1, sk = (tid & 1) * 16;
  const int32_t arow = rid[sg];
  // The next column tile's ids, norm and first chunk are loaded while the
  // current tile is computed, so that no tile starts on global-memory
  // latency (the id, then the row it names).
  auto col_id = [&](int c0, int i) {
    return c0 < m && i < min(kCols, m - c0) ? __ldg(order + lo + c0 + i) : -1;
  };
  float pa[16], pb[16];
  auto fetch = [&](int32_t bc, int k0) {
    const T *ra = X + (int64_t)max(arow, 0) * d + k0 + sk;
    const T *rb = X + (int64_t)max(bc, 0) * d + k0 + sk;
    load_row8<T>(ra, arow >= 0 && k0 + sk < d, pa);
    load_row8<T>(ra + 8, arow >= 0 && k0 + sk + 8 < d, pa + 8);
    load_row8<T>(rb, bc >= 0 && k0 + sk < d, pb);
    load_row8<T>(rb + 8, bc >= 0 && k0 + sk + 8 < d, pb + 8);
  };
  auto store = [&](int b) {
    float(*A)[kRows] = As(b);
    float(*B)[kCols] = Bs(b);
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      A[sk + e][sg] = pa[e];
      B[sk + e][sg] = pb[e];
    }
  };
  int32_t bcol = col_id(0, sg);                 // staged column sg of this tile
  int32_t qn = tid < kCols ? col_id(0, tid) : -1;  // column tid (its norm)
  float cn = qn >= 0 ? __ldg(xnorm + qn) : __int_as_float(0x7f800000);
  fetch(bcol, 0);
  for (int c0 = 0; c0 < m; c0 += kCols) {
    const int cols = min(kCols, m - c0);
    const int nc0 = c0 + kCols;
    // the next tile's ids now, its norms a chunk later
    const int32_t bcol_next = col_id(nc0, sg);
    const int32_t qn_next = tid < kCols ? col_id(nc0, tid) : -1;
    float cn_next = __int_as_float(0x7f800000);
    // thread (ty, tx) owns rows 4ty + i and 64 + 4ty + i, columns 4tx + j
    // and 64 + 4tx + j (i, j < 4): conflict-free 16-byte reads of a chunk row
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
    __syncthreads();  // the previous tile's scores are no longer read
    if (tid < kCols) cnorm[tid] = cn;
    store(0);
    __syncthreads();
    int cur = 0;
    for (int k0 = 0; k0 < d; k0 += kKc, cur ^= 1) {
      const bool more = k0 + kKc < d;
      // in flight while this chunk is used: the next chunk, or the next
      // tile's first one
      if (more) fetch(bcol, k0 + kKc);
      else if (nc0 < m) fetch(bcol_next, 0);
      if (k0 == 0 && qn_next >= 0) cn_next = __ldg(xnorm + qn_next);
      const float(*A)[kRows] = As(cur);
      const float(*B)[kCols] = Bs(cur);
#pragma unroll 4
      for (int kk = 0; kk < kKc; ++kk) {
        const float4 a0 = *reinterpret_cast<const float4 *>(&A[kk][4 * ty]);
        const float4 a1 = *reinterpret_cast<const float4 *>(&A[kk][64 + 4 * ty]);
        const float4 b0 = *reinterpret_cast<const float4 *>(&B[kk][4 * tx]);
        const float4 b1 = *reinterpret_cast<const float4 *>(&B[kk][64 + 4 * tx]);
        const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
        // two columns per packed FP32x2 multiply-add (each product rounded
        // once into its own sum, in the same order as scalar FMAs)
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float2 ai = make_float2(av[i], av[i]);
#pragma unroll
          for (int j = 0; j < 8; j += 2) {
            const float2 r = sm100::fma2(ai, make_float2(bv[j], bv[j + 1]),
                                         make_float2(acc[i][j], acc[i][j + 1]));
            acc[i][j] = r.x;
            acc[i][j + 1] = r.y;
          }
        }
      }
      // the other buffer was last read in the previous chunk, before the
      // barrier that ended it
      if (more) store(cur ^ 1);
      __syncthreads();
    }
    bcol = bcol_next;
    cn = cn_next;
    // scores ||y||^2 - 2 x.y (columns past the leaf: +inf)
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int r = (i < 4 ? 0 : 64) + 4 * ty + (i & 3);
        const int c = (j < 4 ? 0 : 64) + 4 * tx + (j & 3);
        St[r][c] = fmaf(-2.0f, acc[i][j], cnorm[c]);
      }
    __syncthreads();
    if (svalid) {
      // a mask of the row's scores below the threshold at the tile's start
      // (a superset of those that enter the list), then its set bits in
      // column order, each tested again against the current threshold:
      // the warp runs the insertion as often as its busiest lane, not once
      // per column where any lane inserts
      const float *srow = St[sr];
      float thr = fminf(thr0, tv[KP - 1]);
      uint64_t pass = 0;
#pragma unroll
      for (int jj = 0; jj < kCols / kParts; ++jj) {
        const int j = kParts * jj + sp;
        if (srow[j] < thr && j < cols && c0 + j != my_col) pass |= 1ull << jj;
      }
      while (pass) {
        const int j = kParts * (__ffsll((long long)pass) - 1) + sp;
        pass &= pass - 1;
        const float v = srow[j];
        if (v < thr) {  // (ties with the KP-th keep the earlier column)
          pair_shift_in<KP>(tv, tcol, v, c0 + j);
          thr = fminf(thr0, tv[KP - 1]);
        }
      }
    }
  }
  __syncthreads();
  // part 1 hands its list to part 0, which merges and writes the row's
  // list: tree 0 straight into the running list, later trees into the tree
  // list (folded by k_fold_lists)
  if (sp == 1)
#pragma unroll
    for (int j = 0; j < KP; ++j) {
      hv[j][sr] = tv[j];
      hc[j][sr] = tcol[j];
    }
  __syncthreads();
  if (sp == 0 && svalid) {
#pragma unroll
    for (int j = 0; j < KP; ++j)
      if (hc[j][sr] >= 0) pair_insert<KP>(tv, tcol, hv[j][sr], hc[j][sr]);
    const int32_t pt = rid[sr];
    const float nr = __ldg(xnorm + pt);
    const int64_t o = (int64_t)pt * KP;
    float *dd = (tree > 0 ? tree_dist : run_dist) + o;
    int32_t *di = (tree > 0 ? tree_idx : run_idx) + o;
#pragma unroll
    for (int j = 0; j < KP; ++j) {
      const bool have = tcol[j] >= 0;
      di[j] = have ? __ldg(order + lo + tcol[j]) : -1;
      dd[j] = have ? nr + tv[j] : __int_as_float(0x7f800000);
    }
  }
}

template <typename T, int KP>
drpt_status f32_launch(const MixedTreeArgs &a, const float *xnorm, unsigned grid, cudaStream_t s) {
  DRPT_CUDA(cudaFuncSetAttribute(k_leaf_f32<T, KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmem));
  k_leaf_f32<T, KP><<<grid, kThreads, kSmem, s>>>((const T *)a.X, a.d, a.goff, a.order, xnorm,
                                                  a.tile_leaf, a.tile_r0, a.n_tiles, a.tree,
                                                  a.cand_idx, a.cand_dist, a.tree_idx,
                                                  a.tree_dist, a.err);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace

drpt_status launch_row_norms(const void *X, int dtype, int64_t n, int d, float *out,
                             cudaStream_t s) {
  const unsigned grid = (unsigned)ceil_div(n * 32, 256);
  if (dtype == DRPT_DTYPE_U8)
    k_row_norms<uint8_t><<<grid, 256, 0, s>>>((const uint8_t *)X, n, d, out);
  else
    k_row_norms<float><<<grid, 256, 0, s>>>((const float *)X, n, d, out);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_leaf_f32(const MixedTreeArgs &a, const float *xnorm, cudaStream_t s) {
  if (a.d % 8 != 0) {
    set_error("FP32 Gram leaf kernel: d %% 8 == 0 needed (got %d)", a.d);
    return DRPT_ERR_UNSUPPORTED;
  }
  DRPT_TRY(launch_tile_plan(a.goff, a.nleaf, kRows, a.tile_leaf, a.tile_r0, a.n_tiles, s));
  const unsigned grid = (unsigned)(ceil_div(a.n, kRows) + a.nleaf);
  drpt_status st;
  if (a.kp == 16)
    st = a.dtype == DRPT_DTYPE_U8 ? f32_launch<uint8_t, 16>(a, xnorm, grid, s)
                                  : f32_launch<float, 16>(a, xnorm, grid, s);
  else if (a.kp == 32)
    st = a.dtype == DRPT_DTYPE_U8 ? f32_launch<uint8_t, 32>(a, xnorm, grid, s)
                                  : f32_launch<float, 32>(a, xnorm, grid, s);
  else {
    set_error("FP32 Gram leaf kernel: %d candidates per tree unsupported (16 or 32)", a.kp);
    return DRPT_ERR_UNSUPPORTED;
  }
  DRPT_TRY(st);
  DRPT_LAUNCH_CHECK();
  if (a.tree > 0) DRPT_TRY(launch_fold_lists(a, s));
  return DRPT_OK;
}

}  // namespace drpt
