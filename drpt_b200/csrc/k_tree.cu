// K2-K4 -- one level of every global tree: node statistics, 16-slot
// histogram median and stable partition (drpt_global.cpp:228-352 with
// MathOp::distributed_mean/_variance/_median, math_operations.cpp:121-383, at
// one rank).
//
// One thread block per (tree, node).  A node's points are a contiguous range
// of the tree's `ord` array in ascending point index, because the partition
// below is stable and the root starts in index order; their split values are
// the matching range of `val`.
//
// exact = 1 reproduces the reference bit for bit: the mean and the squared
// deviations are summed one value at a time in list order in FP32 (a single
// dependent add chain per node, run by warp 0; the warp loads 256 values per
// step coalesced and broadcasts them with shuffles), and every float or
// double operation of the boundaries and of the median interpolation rounds
// on its own (__f*_rn / __d*_rn).
// exact = 0 sums in FP64 with a fixed block-wide reduction order (the same
// result on every run, not the reference's).
#include "kernels.cuh"

namespace drpt {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// Dependent FP32 chain over v[0..n): s = s + f(v[i]) in index order, where
// f is the identity or (v - mu)^2 with a rounded subtract and multiply.
// Called by one full warp; every lane returns the sum.
template <bool kSq>
__device__ float warp_chain(const float *__restrict__ v, int64_t n, float mu) {
  const int lane = threadIdx.x & 31;
  constexpr int U = 8;
  constexpr int STEP = 32 * U;
  const int64_t full = (n / STEP) * STEP;
  float s = 0.0f;
  float cur[U], nxt[U];
#pragma unroll
  for (int u = 0; u < U; ++u) cur[u] = full > 0 ? __ldg(v + u * 32 + lane) : 0.0f;
  for (int64_t b = 0; b < full; b += STEP) {
    const int64_t nb = b + STEP;
#pragma unroll
    for (int u = 0; u < U; ++u) nxt[u] = nb < full ? __ldg(v + nb + u * 32 + lane) : 0.0f;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      float x = cur[u];
      if (kSq) {
        const float df = __fsub_rn(x, mu);
        x = __fmul_rn(df, df);
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) s = __fadd_rn(s, __shfl_sync(kFull, x, j));
    }
#pragma unroll
    for (int u = 0; u < U; ++u) cur[u] = nxt[u];
  }
  for (int64_t b = full; b < n; b += 32) {
    float x = (b + lane < n) ? __ldg(v + b + lane) : 0.0f;
    if (kSq) {
      const float df = __fsub_rn(x, mu);
      x = __fmul_rn(df, df);
    }
    const int cnt = (int)min64(32, n - b);
    for (int j = 0; j < cnt; ++j) s = __fadd_rn(s, __shfl_sync(kFull, x, j));
  }
  return s;
}

// Fixed-order block reduction of two doubles; result valid in all threads.
__device__ void block_sum2(double &a, double &b, double *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(kFull, a, o);
    b += __shfl_down_sync(kFull, b, o);
  }
  if (lane == 0) {
    sh[2 * w] = a;
    sh[2 * w + 1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int i = 0; i < kWarps; ++i) {
      ta += sh[2 * i];
      tb += sh[2 * i + 1];
    }
    sh[2 * kWarps] = ta;
    sh[2 * kWarps + 1] = tb;
  }
  __syncthreads();
  a = sh[2 * kWarps];
  b = sh[2 * kWarps + 1];
  __syncthreads();
}

__device__ int block_count(int c, int *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(kFull, c, o);
  if (lane == 0) sh[w] = c;
  __syncthreads();
  int tot = 0;
  for (int i = 0; i < kWarps; ++i) tot += sh[i];
  __syncthreads();
  return tot;
}

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
// D[j-1] < x <= D[j]; slot 0 when no slot takes it.
__device__ __forceinline__ int bin_of(const float *D, float x) {
  int slot = 0;
#pragma unroll
  for (int j = 1; j < kBins; ++j)
    if (D[j - 1] < x && D[j] >= x) slot = j;
  return slot;
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

__global__ void __launch_bounds__(kThreads) k_level(LevelArgs a, int64_t val_stride) {
  __shared__ float sD[kBins];
  __shared__ unsigned sHist[kWarps][kBins];
  __shared__ float sStat[2];
  __shared__ double sRed[2 * kWarps + 2];
  __shared__ int sCnt[kWarps];
  __shared__ int sScan[kWarps + 1];

  const int nodes = 1 << a.level;
  const int t = blockIdx.x / nodes, node = blockIdx.x - t * nodes;
  const int64_t lo = a.off_in ? a.off_in[(int64_t)t * (nodes + 1) + node] : 0;
  const int64_t hi = a.off_in ? a.off_in[(int64_t)t * (nodes + 1) + node + 1] : a.n;
  const int64_t cnt = hi - lo;
  const float *v = a.val_in + (int64_t)t * val_stride + lo;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // 1. mean and variance
  if (a.exact) {
    if (warp == 0) {
      const float sum = warp_chain<false>(v, cnt, 0.0f);
      const float mu = __fdiv_rn(sum, __int2float_rn((int)cnt));
      const float sq = warp_chain<true>(v, cnt, mu);
      const float var = __fdiv_rn(sq, __int2float_rn((int)cnt - 1));
      if (lane == 0) {
        sStat[0] = mu;
        sStat[1] = var;
      }
    }
  } else {
    double s1 = 0.0, s2 = 0.0;
    for (int64_t i = threadIdx.x; i < cnt; i += kThreads) {
      const double x = (double)__ldg(v + i);
      s1 += x;
      s2 += x * x;
    }
    block_sum2(s1, s2, sRed);
    if (threadIdx.x == 0) {
      const double dn = (double)cnt;
      sStat[0] = (float)(s1 / dn);
      double var = (s2 - s1 * (s1 / dn)) / (dn - 1.0);
      if (var < 0.0) var = 0.0;  // rounding can push an exact 0 below 0 (NaN stays NaN)
      sStat[1] = (float)var;
    }
  }
  for (int i = threadIdx.x; i < kWarps * kBins; i += kThreads) (&sHist[0][0])[i] = 0u;
  __syncthreads();
  if (threadIdx.x == 0) node_bounds(sStat[0], __fsqrt_rn(sStat[1]), sD);
  __syncthreads();

  // 2. histogram (integer counts: order does not matter)
  float D[kBins];
#pragma unroll
  for (int j = 0; j < kBins; ++j) D[j] = sD[j];
  for (int64_t i = threadIdx.x; i < cnt; i += kThreads) atomicAdd(&sHist[warp][bin_of(D, __ldg(v + i))], 1u);
  __syncthreads();
  if (threadIdx.x < kBins) {
    unsigned tot = 0;
    for (int w = 0; w < kWarps; ++w) tot += sHist[w][threadIdx.x];
    sHist[0][threadIdx.x] = tot;
  }
  __syncthreads();

  // 3. median
  if (threadIdx.x == 0) {
    const float med = node_median(sD, sHist[0], cnt);
    sStat[0] = med;
    if (a.medians) a.medians[(int64_t)t * ((1 << (a.gd - 1)) - 1) + (nodes - 1) + node] = med;
  }
  __syncthreads();
  const float med = sStat[0];

  // 4. stable partition: value <= median goes left (drpt_global.cpp:308)
  int c = 0;
  for (int64_t i = threadIdx.x; i < cnt; i += kThreads) c += (__ldg(v + i) <= med) ? 1 : 0;
  const int64_t nleft = block_count(c, sCnt);

  const int32_t *oin = a.ord_in ? a.ord_in + (int64_t)t * a.n + lo : nullptr;
  int32_t *oout = a.ord_out + (int64_t)t * a.n + lo;
  float *vout = a.val_out ? a.val_out + (int64_t)t * a.n + lo : nullptr;
  const float *pnext =
      vout ? a.P + ((int64_t)t * (a.gd - 1) + a.level + 1) * a.n : nullptr;
  int64_t lbase = 0, rbase = 0;
  for (int64_t b = 0; b < cnt; b += kThreads) {
    const int64_t i = b + threadIdx.x;
    const bool valid = i < cnt;
    const bool left = valid && __ldg(v + i) <= med;
    const unsigned bl = __ballot_sync(kFull, left);
    const unsigned bv = __ballot_sync(kFull, valid);
    if (lane == 0) sCnt[warp] = __popc(bl) | (__popc(bv) << 16);
    __syncthreads();
    if (threadIdx.x == 0) {
      int accl = 0, accv = 0;
      for (int w = 0; w < kWarps; ++w) {
        sScan[w] = accl | (accv << 16);
        accl += sCnt[w] & 0xffff;
        accv += sCnt[w] >> 16;
      }
      sScan[kWarps] = accl | (accv << 16);
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const int wl = sScan[warp] & 0xffff, wv = sScan[warp] >> 16;
    const int rl = wl + __popc(bl & lt);                  // left-goers before i in the chunk
    const int rr = (wv + __popc(bv & lt)) - rl;            // right-goers before i
    if (valid) {
      const int64_t pos = left ? lbase + rl : nleft + rbase + rr;
      const int32_t id = oin ? __ldg(oin + i) : (int32_t)(lo + i);
      oout[pos] = id;
      if (vout) vout[pos] = __ldg(pnext + id);
    }
    const int tl = sScan[kWarps] & 0xffff, tv = sScan[kWarps] >> 16;
    lbase += tl;
    rbase += tv - tl;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int32_t *oo = a.off_out + (int64_t)t * (2 * nodes + 1);
    oo[2 * node] = (int32_t)lo;
    oo[2 * node + 1] = (int32_t)(lo + nleft);
    if (node == nodes - 1) oo[2 * nodes] = (int32_t)hi;
  }
}

}  // namespace

drpt_status launch_level(const LevelArgs &a, cudaStream_t s) {
  const int64_t blocks = (int64_t)a.T << a.level;
  if (blocks > 0x7fffffff) {
    set_error("too many tree nodes at level %d", a.level);
    return DRPT_ERR_UNSUPPORTED;
  }
  // Level 0 reads the root values straight from P (stride (gd-1)*n per tree).
  const int64_t stride = a.level == 0 ? (int64_t)(a.gd - 1) * a.n : a.n;
  k_level<<<(unsigned)blocks, kThreads, 0, s>>>(a, stride);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt
