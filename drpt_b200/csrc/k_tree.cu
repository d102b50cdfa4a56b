// K2-K4 -- one level of every global tree: node statistics, 16-slot
// histogram median and stable partition (drpt_global.cpp:228-352 with
// MathOp::distributed_mean/_variance/_median, math_operations.cpp:121-383, at
// one rank).
//
// A node's points are a contiguous range of the tree's `ord` array in
// ascending point index (the root starts in index order and every partition
// is stable); `val` holds the matching split values.  The work of a level is
// cut into units of up to kUnit consecutive positions that never straddle a
// node, so large nodes near the root spread over the whole GPU and small
// nodes near the leaves cost one unit each:
//
//   plan      one block: units per node, their prefix, unit -> (node, start)
//   stats     exact: one block per node runs the reference's sequential FP32
//             sums (a single dependent add chain: warp 0 adds the values in
//             list order from a shared-memory double buffer that the other
//             warps fill); fast: FP64 partial sums per unit, combined per
//             node in unit order
//   bounds    16 histogram boundaries per node (exact float arithmetic)
//   hist      per unit, 16 integer counts
//   median    per node: counts summed in unit order, selection and the
//             double-precision interpolation of the reference
//   count     per unit, values <= median
//   scan      per node: unit prefix of the left counts, child offsets
//   scatter   per unit: warp-ballot stable partition through shared memory,
//             coalesced writes of the point ids and of their next-level values
//
// Every operation that the reference performs in float or double rounds on
// its own here (__f*_rn / __d*_rn), so with exact = 1 the medians, and hence
// the trees, are bit-identical to the reference's.
#include "kernels.cuh"

namespace drpt {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kUnit = 4096;                  // positions per unit
constexpr int kPer = kUnit / kThreads;       // positions per thread in a unit
constexpr int kChainChunk = 2048;            // values per shared-memory buffer of the chain

// ------------------------------------------------------------------ helpers
// Histogram boundaries (math_operations.cpp:252-288, factor 1, 7 bins):
// slots 0..13 around the mean at multiples of sigma/30, sigma/6 and sigma/2;
// slots 14 and 15 stay 0.
__device__ void node_bounds(float mu, float sigma, float *D) {
  const float s1 = __double2float_rn(__ddiv_rn((double)sigma, 30.0));
  const float s2 = __double2float_rn(__ddiv_rn((double)sigma, 6.0));
  const float s3 = __double2float_rn(__ddiv_rn((double)sigma, 2.0));
#pragma unroll
  for (int j = 1; j <= 4; ++j) {
    const float r = __fmul_rn((float)j, s1);
    D[6 + j] = __fadd_rn(mu, r);
    D[7 - j] = __fsub_rn(mu, r);
  }
#pragma unroll
  for (int j = 1; j <= 2; ++j) {
    const float r = __fadd_rn(sigma, __fmul_rn((float)j, s2));
    D[10 + j] = __fadd_rn(mu, r);
    D[3 - j] = __fsub_rn(mu, r);
  }
  const float r3 = __fadd_rn(__fmul_rn(2.0f, sigma), __fmul_rn(1.0f, s3));
  D[13] = __fadd_rn(mu, r3);
  D[0] = __fsub_rn(mu, r3);
  D[14] = 0.0f;
  D[15] = 0.0f;
}

// Slot of x (math_operations.cpp:292-308): slot j in 1..15 when
// D[j-1] < x <= D[j]; slot 0 when no slot takes it.  D[0..13] never
// decrease (offsets from the mean in increasing order, rounded
// monotonically) and D[14] = D[15] = 0, so for x <= D[13] the slot is the
// number of D[0..12] below x (0 when x <= D[0], and for a NaN x); above
// D[13] only slot 14 can take x, when x <= 0.  That count is found by a
// branch-free binary search over D[0..12] (a lower bound in a non-decreasing
// array; D[13] >= x closes it): four compares instead of thirteen, the same
// slot for every x, NaNs included (every compare with a NaN is false).
__device__ __forceinline__ int bin_of(const float *D, float x) {
  if (x > D[13]) return x <= 0.0f ? 14 : 0;
  const bool c8 = D[7] < x;                                              // >= 8 below
  const bool c4 = (c8 ? D[11] : D[3]) < x;                               // + 4
  const bool c2 = (c8 ? (c4 ? D[13] : D[9]) : (c4 ? D[5] : D[1])) < x;  // + 2
  const int s = (c8 ? 8 : 0) + (c4 ? 4 : 0) + (c2 ? 2 : 0);
  const float t = c8 ? (c4 ? D[12] : (c2 ? D[10] : D[8]))
                     : (c4 ? (c2 ? D[6] : D[4]) : (c2 ? D[2] : D[0]));
  return s + (t < x ? 1 : 0);                                           // + 1
}

// Median selection and interpolation (math_operations.cpp:333-375): the
// first slot whose running count (a float) reaches int(50*n/100); the
// interpolation runs in double from float boundaries and is stored as float.
// Slot -1 (read when slot 0 is selected) is 0, the preceding node's D[15].
__device__ float node_median(const float *D, const unsigned *hist, int64_t n) {
  float cfreq = 0.0f;
  const float target = (float)((50 * n) / 100);
  int sel = kBins - 1;
  for (int k = 0; k < kBins; ++k) {
    cfreq = __double2float_rn(__dadd_rn((double)cfreq, (double)hist[k]));
    if (cfreq >= target) {
      sel = k;
      break;
    }
  }
  const double count = (double)hist[sel];
  const float lo = sel > 0 ? D[sel - 1] : 0.0f;
  const float width = __fsub_rn(D[sel], lo);
  const double frac =
      __ddiv_rn(__dsub_rn((double)(n / 2), __dsub_rn((double)cfreq, count)), count);
  return __double2float_rn(__dadd_rn((double)lo, __dmul_rn(frac, (double)width)));
}

struct NodeRange {
  int64_t lo, hi;
};

__device__ __forceinline__ NodeRange node_range(const TreeLevelArgs &a, int g) {
  const int nodes = 1 << a.level;
  const int t = g >> a.level, s = g & (nodes - 1);
  if (!a.off_in) return {0, a.n};
  const int32_t *o = a.off_in + (int64_t)t * (nodes + 1);
  return {o[s], o[s + 1]};
}

__device__ __forceinline__ const float *tree_vals(const TreeLevelArgs &a, int t) {
  // The first level (p_level0) reads its values straight from P (column
  // t*(gd-1)): the points are still in index order there.
  return a.level == a.p_level0 ? a.P + (int64_t)t * (a.gd - 1) * a.n
                               : a.val_in + (int64_t)t * a.n;
}

// ------------------------------------------------------------------ plan
__global__ void __launch_bounds__(1024) k_plan(TreeLevelArgs a) {
  __shared__ int warp_tot[32];
  const int G = a.T << a.level;  // nodes of all trees
  const int per = (G + 1023) / 1024;
  const int g0 = threadIdx.x * per;
  int cnt = 0;
  for (int i = 0; i < per; ++i) {
    const int g = g0 + i;
    if (g < G) {
      const NodeRange r = node_range(a, g);
      cnt += (int)ceil_div(r.hi - r.lo, kUnit);
    }
  }
  // block-wide exclusive scan of cnt
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
    const int g = g0 + i;
    if (g >= G) break;
    const NodeRange r = node_range(a, g);
    const int nu = (int)ceil_div(r.hi - r.lo, kUnit);
    a.node_ubase[g] = base;
    for (int c = 0; c < nu; ++c) {
      a.unit_node[base + c] = g;
      a.unit_lo[base + c] = (int32_t)(r.lo + (int64_t)c * kUnit);
    }
    base += nu;
  }
  if (threadIdx.x == 1023) {
    a.node_ubase[G] = base;
    *a.n_units = base;
  }
}

// ------------------------------------------------------------------ exact stats
// Sequential FP32 sum of v[0..n) (or of (v - mu)^2), warp 0 adding from a
// shared-memory double buffer that warps 1..7 fill.  All of warp 0 computes
// the same chain; every thread returns it after the final barrier.
template <bool kSq>
__device__ float block_chain(const float *__restrict__ v, int64_t n, float mu, float *buf,
                             float *result) {
  const int warp = threadIdx.x >> 5;
  const int64_t chunks = ceil_div(n, kChainChunk);
  float s = 0.0f;
  auto load = [&](int64_t c) {
    float *dst = buf + (c & 1) * kChainChunk;
    const int64_t base = c * kChainChunk;
    const int len = (int)min64(kChainChunk, n - base);
    for (int i = threadIdx.x - 32; i < len; i += kThreads - 32) {
      float x = __ldg(v + base + i);
      if (kSq) {
        const float df = __fsub_rn(x, mu);
        x = __fmul_rn(df, df);
      }
      dst[i] = x;
    }
  };
  if (warp != 0 && chunks > 0) load(0);
  for (int64_t c = 0; c < chunks; ++c) {
    __syncthreads();  // buffer c complete; buffer c+1 free
    if (warp != 0) {
      if (c + 1 < chunks) load(c + 1);
    } else {
      const float *src = buf + (c & 1) * kChainChunk;
      const int len = (int)min64(kChainChunk, n - c * kChainChunk);
      const int len4 = len & ~3;
      const float4 *src4 = reinterpret_cast<const float4 *>(src);
#pragma unroll 8
      for (int i = 0; i < len4 / 4; ++i) {
        const float4 q = src4[i];
        s = __fadd_rn(s, q.x);
        s = __fadd_rn(s, q.y);
        s = __fadd_rn(s, q.z);
        s = __fadd_rn(s, q.w);
      }
      for (int i = len4; i < len; ++i) s = __fadd_rn(s, src[i]);
    }
  }
  if (threadIdx.x == 0) *result = s;
  __syncthreads();
  return *result;
}

__global__ void __launch_bounds__(kThreads) k_stats_exact(TreeLevelArgs a) {
  __shared__ __align__(16) float buf[2 * kChainChunk];
  __shared__ float sh[2];
  const int g = blockIdx.x;
  const int t = g >> a.level;
  const NodeRange r = node_range(a, g);
  const int64_t cnt = r.hi - r.lo;
  const float *v = tree_vals(a, t) + r.lo;
  const float sum = block_chain<false>(v, cnt, 0.0f, buf, &sh[0]);     // :137-142
  const float mu = __fdiv_rn(sum, __int2float_rn((int)cnt));          // :164
  const float sq = block_chain<true>(v, cnt, mu, buf, &sh[1]);        // :186-192
  if (threadIdx.x == 0) {
    const float var = __fdiv_rn(sq, __int2float_rn((int)cnt - 1));    // :201
    float Dl[kBins];
    node_bounds(mu, __fsqrt_rn(var), Dl);
    float *D = a.node_D + (int64_t)g * kBins;
#pragma unroll
    for (int j = 0; j < kBins; ++j) D[j] = Dl[j];
  }
}

// ------------------------------------------------------------------ fast stats
__global__ void __launch_bounds__(kThreads) k_stats_partial(TreeLevelArgs a) {
  __shared__ double sh[2 * kWarps];
  const int n_units = *a.n_units;
  for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
    const int g = a.unit_node[u];
    const int t = g >> a.level;
    const NodeRange r = node_range(a, g);
    const int64_t lo = a.unit_lo[u];
    const int len = (int)min64(kUnit, r.hi - lo);
    const float *v = tree_vals(a, t) + lo;
    // all kPer loads of a thread in flight before the sums (same order of adds)
    float xs[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int i = threadIdx.x + j * kThreads;
      xs[j] = i < len ? __ldg(v + i) : 0.0f;
    }
    double s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      if (threadIdx.x + j * kThreads < len) {
        const double x = (double)xs[j];
        s1 += x;
        s2 += x * x;
      }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1 += __shfl_down_sync(kFull, s1, o);
      s2 += __shfl_down_sync(kFull, s2, o);
    }
    if (lane == 0) {
      sh[2 * w] = s1;
      sh[2 * w + 1] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t1 = 0.0, t2 = 0.0;
      for (int i = 0; i < kWarps; ++i) {
        t1 += sh[2 * i];
        t2 += sh[2 * i + 1];
      }
      a.unit_s[2 * u] = t1;
      a.unit_s[2 * u + 1] = t2;
    }
    __syncthreads();  // sh is reused by the next unit
  }
}

// One warp per node: lanes take the node's units in turn, the lane partials
// are then added in a fixed tree order.
__global__ void k_bounds_fast(TreeLevelArgs a) {
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= (a.T << a.level)) return;  // warp-uniform
  const NodeRange r = node_range(a, g);
  double s1 = 0.0, s2 = 0.0;
  for (int u = a.node_ubase[g] + lane; u < a.node_ubase[g + 1]; u += 32) {
    s1 += a.unit_s[2 * u];
    s2 += a.unit_s[2 * u + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(kFull, s1, o);
    s2 += __shfl_xor_sync(kFull, s2, o);
  }
  if (lane != 0) return;
  const double dn = (double)(r.hi - r.lo);
  double var = (s2 - s1 * (s1 / dn)) / (dn - 1.0);
  if (var < 0.0) var = 0.0;  // rounding can push a zero variance below 0 (NaN stays NaN)
  float Dl[kBins];
  node_bounds((float)(s1 / dn), __fsqrt_rn((float)var), Dl);
  float *D = a.node_D + (int64_t)g * kBins;
#pragma unroll
  for (int j = 0; j < kBins; ++j) D[j] = Dl[j];
}

// ------------------------------------------------------------------ histogram
// Per thread, the 16 counts are 8-bit fields of two 64-bit registers (at
// most kPer = 16 values per thread), widened to 16-bit fields of four
// registers (a warp's sum is at most 512) and added over the warp with
// shuffles; no atomics.
__global__ void __launch_bounds__(kThreads) k_hist(TreeLevelArgs a) {
  __shared__ unsigned hist[kWarps][kBins];
  __shared__ float Ds[kBins];
  const int n_units = *a.n_units;
  for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
    const int g = a.unit_node[u];
    const int t = g >> a.level;
    const NodeRange r = node_range(a, g);
    const int64_t lo = a.unit_lo[u];
    const int len = (int)min64(kUnit, r.hi - lo);
    const float *v = tree_vals(a, t) + lo;
    if (threadIdx.x < kBins) Ds[threadIdx.x] = a.node_D[(int64_t)g * kBins + threadIdx.x];
    __syncthreads();
    float D[kBins];
#pragma unroll
    for (int j = 0; j < kBins; ++j) D[j] = Ds[j];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    static_assert(kPer < 256, "a thread's counts fit 8-bit fields");
    uint64_t c2[2] = {0ull, 0ull};
    float xs[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int i = threadIdx.x + j * kThreads;
      xs[j] = i < len ? __ldg(v + i) : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      if (threadIdx.x + j * kThreads < len) {
        const int b = bin_of(D, xs[j]);
        const uint64_t inc = 1ull << (8 * (b & 7));
        c2[0] += b < 8 ? inc : 0ull;
        c2[1] += b < 8 ? 0ull : inc;
      }
    }
    // bins 4q .. 4q + 3 as 16-bit fields of c4[q]
    uint64_t c4[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t x = (uint32_t)(c2[q >> 1] >> (32 * (q & 1)));
      c4[q] = (uint64_t)(x & 0xffu) | ((uint64_t)((x >> 8) & 0xffu) << 16) |
              ((uint64_t)((x >> 16) & 0xffu) << 32) | ((uint64_t)(x >> 24) << 48);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c4[q] += __shfl_xor_sync(kFull, c4[q], o);
    const int q = lane >> 2;
    const uint64_t mine = q == 0 ? c4[0] : q == 1 ? c4[1] : q == 2 ? c4[2] : c4[3];
    if (lane < kBins) hist[w][lane] = (unsigned)((mine >> (16 * (lane & 3))) & 0xffffu);
    __syncthreads();
    if (threadIdx.x < kBins) {
      unsigned tot = 0;
      for (int k = 0; k < kWarps; ++k) tot += hist[k][threadIdx.x];
      a.unit_hist[(int64_t)u * kBins + threadIdx.x] = tot;
    }
    __syncthreads();  // hist and Ds are reused by the next unit
  }
}

// ------------------------------------------------------------------ median
// One warp per node: lanes add the counts of the node's units in turn
// (integer counts, so the order is immaterial), lane 0 selects the median.
__global__ void k_median(TreeLevelArgs a) {
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= (a.T << a.level)) return;  // warp-uniform
  const NodeRange r = node_range(a, g);
  unsigned h[kBins];
#pragma unroll
  for (int j = 0; j < kBins; ++j) h[j] = 0u;
  for (int u = a.node_ubase[g] + lane; u < a.node_ubase[g + 1]; u += 32)
#pragma unroll
    for (int j = 0; j < kBins; ++j) h[j] += a.unit_hist[(int64_t)u * kBins + j];
#pragma unroll
  for (int j = 0; j < kBins; ++j)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h[j] += __shfl_xor_sync(kFull, h[j], o);
  if (lane != 0) return;
  float D[kBins];
#pragma unroll
  for (int j = 0; j < kBins; ++j) D[j] = a.node_D[(int64_t)g * kBins + j];
  float med = node_median(D, h, r.hi - r.lo);
  if (a.stop) {
    // root slot s0 of the first level owns the nodes s0 << depth .. below it;
    // from depth stop[s0] on its nodes keep every point (median +inf)
    const int nodes = 1 << a.level, depth = a.level - a.p_level0;
    if (depth >= a.stop[(g & (nodes - 1)) >> depth]) med = __int_as_float(0x7f800000);
  }
  a.node_med[g] = med;
  if (a.medians) {
    const int nodes = 1 << a.level, t = g >> a.level, s = g & (nodes - 1);
    a.medians[(int64_t)t * ((1 << (a.gd - 1)) - 1) + (nodes - 1) + s] = med;
  }
}

// ------------------------------------------------------------------ count
__global__ void __launch_bounds__(kThreads) k_count(TreeLevelArgs a) {
  __shared__ int sh[kWarps];
  const int n_units = *a.n_units;
  for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
    const int g = a.unit_node[u];
    const int t = g >> a.level;
    const NodeRange r = node_range(a, g);
    const int64_t lo = a.unit_lo[u];
    const int len = (int)min64(kUnit, r.hi - lo);
    const float *v = tree_vals(a, t) + lo;
    const float med = a.node_med[g];
    float xs[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int i = threadIdx.x + j * kThreads;
      xs[j] = i < len ? __ldg(v + i) : 0.0f;
    }
    int c = 0;
#pragma unroll
    for (int j = 0; j < kPer; ++j)  // value <= median goes left (drpt_global.cpp:308)
      c += (threadIdx.x + j * kThreads < len && xs[j] <= med) ? 1 : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int k = 0; k < kWarps; ++k) tot += sh[k];
      a.unit_left[u] = tot;
    }
    __syncthreads();  // sh is reused by the next unit
  }
}

// ------------------------------------------------------------------ node scan
// One warp per node: exclusive prefix of the units' left counts in unit
// order, 32 units per step with a running carry.
__global__ void k_node_scan(TreeLevelArgs a) {
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= (a.T << a.level)) return;  // warp-uniform
  const NodeRange r = node_range(a, g);
  int carry = 0;
  for (int u0 = a.node_ubase[g]; u0 < a.node_ubase[g + 1]; u0 += 32) {
    const int u = u0 + lane;
    const int c = u < a.node_ubase[g + 1] ? a.unit_left[u] : 0;
    int x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    if (u < a.node_ubase[g + 1]) a.unit_lbase[u] = carry + x - c;
    carry += __shfl_sync(kFull, x, 31);
  }
  if (lane != 0) return;
  a.node_nleft[g] = carry;
  const int nodes = 1 << a.level, t = g >> a.level, s = g & (nodes - 1);
  int32_t *oo = a.off_out + (int64_t)t * (2 * nodes + 1);
  oo[2 * s] = (int32_t)r.lo;
  oo[2 * s + 1] = (int32_t)(r.lo + carry);
  if (s == nodes - 1) oo[2 * nodes] = (int32_t)r.hi;
}

// ------------------------------------------------------------------ scatter
// Warp-ballot stable partition of a unit through shared memory.  Position
// p = threadIdx.x + j * kThreads is chunk c = j * kWarps + warp of 32
// positions (so c-major order is position order); each warp's ballot of
// "value <= median" gives the chunk's left count and, per lane, the left-goers
// before it in the chunk; one warp scans the kUnit / 32 chunk counts.  A
// left-goer lands at (left-goers before it), a right-goer at (left total +
// right-goers before it): left-goers in position order, then right-goers in
// position order.  All loads are coalesced; the point ids and their next-level
// values then leave in coalesced writes.
__global__ void __launch_bounds__(kThreads) k_scatter(TreeLevelArgs a) {
  constexpr int kChunks = kUnit / 32;
  static_assert(kChunks == 4 * 32, "one warp scans the chunk counts, four per lane");
  __shared__ int32_t sid[kUnit];
  __shared__ float sval[kUnit];
  __shared__ int cbase[kChunks];  // chunk left counts, then their exclusive prefix
  __shared__ int ltot_sh;
  const int n_units = *a.n_units;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
    const int g = a.unit_node[u];
    const int t = g >> a.level;
    const NodeRange r = node_range(a, g);
    const int64_t lo = a.unit_lo[u];
    const int len = (int)min64(kUnit, r.hi - lo);
    const float *v = tree_vals(a, t) + lo;
    const float med = a.node_med[g];
    const int32_t *oin = a.ord_in ? a.ord_in + (int64_t)t * a.n + lo : nullptr;
    // every value and id of the thread in flight before the ballots
    float xs[kPer];
    int32_t ids[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int p = threadIdx.x + j * kThreads;
      xs[j] = p < len ? __ldg(v + p) : 0.0f;
      ids[j] = p < len ? (oin ? __ldg(oin + p) : (int32_t)(lo + p)) : 0;
    }
    unsigned bal[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int p = threadIdx.x + j * kThreads;
      bal[j] = __ballot_sync(kFull, p < len && xs[j] <= med);  // drpt_global.cpp:308
      if (lane == 0) cbase[j * kWarps + w] = __popc(bal[j]);
    }
    __syncthreads();
    if (w == 0) {
      int c4[4], sum = 0;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        c4[e] = cbase[4 * lane + e];
        sum += c4[e];
      }
      int x = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
      }
      int run = x - sum;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        cbase[4 * lane + e] = run;
        run += c4[e];
      }
      if (lane == 31) ltot_sh = x;
    }
    __syncthreads();
    const int ltot = ltot_sh;
    const bool want_val = a.val_out != nullptr;
    const float *pnext =
        want_val ? a.P + ((int64_t)t * (a.gd - 1) + a.level - a.p_level0 + 1) * a.n : nullptr;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int p = threadIdx.x + j * kThreads;
      if (p < len) {
        const int lbefore = cbase[j * kWarps + w] + __popc(bal[j] & lt_mask);
        const int slot = ((bal[j] >> lane) & 1u) ? lbefore : ltot + (p - lbefore);
        sid[slot] = ids[j];
        if (want_val) sval[slot] = __ldg(pnext + ids[j]);
      }
    }
    __syncthreads();
    // left-goers -> [node lo + unit lbase, ...), right-goers -> [node lo + nleft + rbase, ...)
    const int64_t lbase = r.lo + a.unit_lbase[u];
    const int64_t rbase = r.lo + a.node_nleft[g] + (lo - r.lo - a.unit_lbase[u]);
    int32_t *oout = a.ord_out + (int64_t)t * a.n;
    float *vout = want_val ? a.val_out + (int64_t)t * a.n : nullptr;
    for (int i = threadIdx.x; i < len; i += kThreads) {
      const int64_t dst = i < ltot ? lbase + i : rbase + (i - ltot);
      oout[dst] = sid[i];
      if (want_val) vout[dst] = sval[i];
    }
    __syncthreads();  // sid, sval and cbase are reused by the next unit
  }
}

}  // namespace

drpt_status launch_tree_level(const TreeLevelArgs &a, int64_t max_units, cudaStream_t s) {
  const int64_t G = (int64_t)a.T << a.level;
  if (G > (1 << 20) || max_units > 0x7fffffff) {
    set_error("too many tree nodes at level %d", a.level);
    return DRPT_ERR_UNSUPPORTED;
  }
  // unit kernels loop over the units actually planned (grid-stride)
  const unsigned U = (unsigned)min64(max_units, (int64_t)device_sm_count() * 16);
  const unsigned gn = (unsigned)ceil_div(G * 32, 256);  // warp per node
  k_plan<<<1, 1024, 0, s>>>(a);
  if (a.exact) {
    k_stats_exact<<<(unsigned)G, kThreads, 0, s>>>(a);
  } else {
    k_stats_partial<<<U, kThreads, 0, s>>>(a);
    k_bounds_fast<<<gn, 256, 0, s>>>(a);
  }
  k_hist<<<U, kThreads, 0, s>>>(a);
  k_median<<<gn, 256, 0, s>>>(a);
  k_count<<<U, kThreads, 0, s>>>(a);
  k_node_scan<<<gn, 256, 0, s>>>(a);
  k_scatter<<<U, kThreads, 0, s>>>(a);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

int64_t tree_level_max_units(int64_t n, int T, int level) {
  return (int64_t)T * (ceil_div(n, kUnit) + ((int64_t)1 << level));
}

int tree_level_kernels(int exact) { return exact ? 7 : 8; }

}  // namespace drpt
