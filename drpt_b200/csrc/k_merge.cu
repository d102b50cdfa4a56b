// K7 -- cross-tree merge (the std::merge + std::unique of calculate_nns,
// mdrpt.cpp:179-198, and the one-rank pass-through of communicate_nns,
// mdrpt.cpp:580-631).  Each point has T lists of its k nearest leaf-mates
// (one per tree, sorted by (distance, index), the point itself excluded); the
// result is its k nearest distinct candidates over all trees.  The same
// neighbour found in several trees carries the same distance bits (the
// distance is a deterministic function of the two rows), so a duplicate
// always meets its twin at the same sort position.
//
// One warp per point: lane j holds slot j of the running list (k <= 32) or
// slots j and j+32 (k <= 64); each tree contributes a list of `lk` entries.  Candidates are streamed tree by tree; a
// candidate enters when it beats the current k-th entry and is not already
// present, and the lanes shift to make room.
#include "kernels.cuh"

namespace drpt {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ bool before(float da, int32_t ia, float db, int32_t ib) {
  return da < db || (da == db && (uint32_t)ia < (uint32_t)ib);
}

template <int S>  // slots per lane
__global__ void __launch_bounds__(kThreads) k_merge(const int32_t *__restrict__ ci,
                                                    const float *__restrict__ cd, int64_t n, int T,
                                                    int lk, int k, int32_t *__restrict__ oi,
                                                    float *__restrict__ od) {
  const int lane = threadIdx.x & 31;
  const int64_t p = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  if (p >= n) return;  // warp-uniform: a warp owns one point
  const float inf = __int_as_float(0x7f800000);
  float d[S];
  int32_t id[S];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    d[s] = inf;
    id[s] = -1;  // -1 sorts after every index (compared as unsigned)
  }
  const int wl = (k - 1) & 31, ws = (k - 1) >> 5;
  // Tree by tree: each list is sorted, so once an entry fails to beat the
  // current k-th, the rest of that list cannot enter either.
  for (int t = 0; t < T; ++t) {
    const int32_t *pi = ci + (p * T + t) * lk;
    const float *pd = cd + (p * T + t) * lk;
    float ld[S];
    int32_t li[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int e = s * 32 + lane;
      ld[s] = e < lk ? __ldg(pd + e) : inf;
      li[s] = e < lk ? __ldg(pi + e) : -1;
    }
    for (int j = 0; j < lk; ++j) {
      float cdv = inf;
      int32_t civ = -1;
#pragma unroll
      for (int s = 0; s < S; ++s) {
        const float td = __shfl_sync(kFull, ld[s], j & 31);
        const int32_t ti = __shfl_sync(kFull, li[s], j & 31);
        if (s == (j >> 5)) {
          cdv = td;
          civ = ti;
        }
      }
      if (civ < 0) break;  // the rest of this list is empty (warp-uniform)
      float wd = inf;
      int32_t wi = -1;
#pragma unroll
      for (int s = 0; s < S; ++s) {
        const float td = __shfl_sync(kFull, d[s], wl);
        const int32_t ti = __shfl_sync(kFull, id[s], wl);
        if (s == ws) {
          wd = td;
          wi = ti;
        }
      }
      if (!before(cdv, civ, wd, wi)) break;  // not better than the k-th entry
      bool dup = false;
      int pos = 0;
#pragma unroll
      for (int s = 0; s < S; ++s) {
        const bool live = s * 32 + lane < k;
        dup |= live && id[s] == civ;
        pos += __popc(__ballot_sync(kFull, live && before(d[s], id[s], cdv, civ)));
      }
      if (__any_sync(kFull, dup)) continue;
      // slot pos takes the candidate, later slots take their predecessor
      float prev_d = inf;
      int32_t prev_i = -1;
#pragma unroll
      for (int s = 0; s < S; ++s) {
        float up_d = __shfl_up_sync(kFull, d[s], 1);
        int32_t up_i = __shfl_up_sync(kFull, id[s], 1);
        const float last_d = __shfl_sync(kFull, d[s], 31);
        const int32_t last_i = __shfl_sync(kFull, id[s], 31);
        if (lane == 0) {
          up_d = prev_d;
          up_i = prev_i;
        }
        prev_d = last_d;
        prev_i = last_i;
        const int slot = s * 32 + lane;
        if (slot == pos) {
          d[s] = cdv;
          id[s] = civ;
        } else if (slot > pos) {
          d[s] = up_d;
          id[s] = up_i;
        }
      }
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int slot = s * 32 + lane;
    if (slot < k) {
      oi[p * k + slot] = id[s];
      od[p * k + slot] = d[s];
    }
  }
}

}  // namespace

drpt_status launch_merge(const int32_t *cand_idx, const float *cand_dist, int64_t n, int T, int lk,
                         int k, int32_t *out_idx, float *out_dist, cudaStream_t s) {
  if (k <= 0 || k > kMaxK || lk <= 0 || lk > kMaxK) {
    set_error("merge: k = %d outside [1, %d]", k, kMaxK);
    return DRPT_ERR_UNSUPPORTED;
  }
  if (n <= 0) return DRPT_OK;
  const unsigned grid = (unsigned)ceil_div(n * 32, kThreads);
  if (k <= 32 && lk <= 32)
    k_merge<1><<<grid, kThreads, 0, s>>>(cand_idx, cand_dist, n, T, lk, k, out_idx, out_dist);
  else
    k_merge<2><<<grid, kThreads, 0, s>>>(cand_idx, cand_dist, n, T, lk, k, out_idx, out_dist);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt

namespace drpt {
namespace {

// Batches: point p of dataset s (rows [off[s], off[s+1])) gets its
// neighbours' ids relative to off[s].
__global__ void k_localize(int32_t *__restrict__ idx, int64_t n, int k,
                           const int64_t *__restrict__ off, int nsets) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int lo = 0, hi = nsets;  // largest s with off[s] <= p
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= p) lo = mid;
    else hi = mid;
  }
  const int32_t base = (int32_t)__ldg(off + lo);
  int32_t *row = idx + p * k;
  for (int j = 0; j < k; ++j) {
    const int32_t v = row[j];
    if (v >= 0) row[j] = v - base;
  }
}

}  // namespace

drpt_status launch_localize(int32_t *idx, int64_t n, int k, const int64_t *set_off, int nsets,
                            cudaStream_t s) {
  if (n <= 0) return DRPT_OK;
  k_localize<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(idx, n, k, set_off, nsets);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt
