// Mixed-precision form of the leaf brute force.
//
// The reference scores every leaf row exactly in FP32 (mdrpt.cpp:123-212).
// The mixed form keeps its global trees (projection + histogram-median
// splits) but brute-forces each whole global leaf with BF16 Gram tiles on the
// tensor cores and wins the accuracy back afterwards:
//
//   K8  k_leaf_center   per global leaf: subtract the leaf mean (FP32), round
//                       to BF16 in leaf order, row norms of the rounded rows
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

#include <algorithm>
#include <type_traits>

#include "kernels.cuh"
#include "sm100.cuh"

namespace drpt {
namespace {

using namespace sm100;

constexpr int kTM = 128;            // rows per tile (M)
constexpr int kTN = 64;             // columns per tile (N)
constexpr int kStages = 2;          // B-tile pipeline depth
constexpr int kBufCap = 32;         // per-row pending candidates
constexpr int kCheck = 16;          // columns between flush checks
constexpr int kEpiWarps = 4;
constexpr int kMmaThreads = 32 * (kEpiWarps + 2);
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

// One block per global leaf.  Warps take rows in turn; lane l owns the four
// dimensions 4l..4l+3 of every 128-wide chunk (d <= 256, d % 4 == 0).  The
// centre is the mean of the leaf's first (up to) kCentreRows rows -- it only
// has to bring the values near zero -- summed per warp, the eight warp
// partials added in warp order, so the result does not depend on scheduling.
template <typename T>
__global__ void __launch_bounds__(256) k_leaf_center(const T *__restrict__ X, int d, int d_pad,
                                                     const int32_t *__restrict__ order,
                                                     const int32_t *__restrict__ goff,
                                                     __nv_bfloat16 *__restrict__ Xb,
                                                     float *__restrict__ nrm) {
  __shared__ float part[8][256];
  __shared__ float mu[256];
  const int j = blockIdx.x;
  const int32_t lo = goff[j], hi = goff[j + 1];
  const int m = hi - lo;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
  const int mc = min(m, kCentreRows);
  for (int r = warp; r < mc; r += 8) {
    const T *src = X + (int64_t)__ldg(order + lo + r) * d;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c0 = h * 128 + 4 * lane;
      if (c0 < d) {
        float v[4];
        load4<T>(src + c0, v);
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[h][e] += v[e];
      }
    }
  }
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int e = 0; e < 4; ++e) part[warp][h * 128 + 4 * lane + e] = acc[h][e];
  __syncthreads();
  if (threadIdx.x < 256) {
    float s = 0.0f;
    for (int w = 0; w < 8; ++w) s += part[w][threadIdx.x];
    mu[threadIdx.x] = mc > 0 ? s / (float)mc : 0.0f;
  }
  __syncthreads();
  constexpr int RB = 4;  // rows per warp step, loaded together
  for (int r0w = warp * RB; r0w < m; r0w += 8 * RB) {
    float v[RB][2][4];
#pragma unroll
    for (int q = 0; q < RB; ++q) {
      const int r = r0w + q;
      const T *src = r < m ? X + (int64_t)__ldg(order + lo + r) * d : nullptr;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c0 = h * 128 + 4 * lane;
        v[q][h][0] = v[q][h][1] = v[q][h][2] = v[q][h][3] = 0.0f;
        if (src && c0 < d) load4<T>(src + c0, v[q][h]);
      }
    }
#pragma unroll
    for (int q = 0; q < RB; ++q) {
      const int r = r0w + q;
      float sq = 0.0f;
      __nv_bfloat16 *dst = Xb + (int64_t)(lo + (r < m ? r : 0)) * d_pad;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c0 = h * 128 + 4 * lane;
        if (c0 < d_pad) {
          __nv_bfloat16 b[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            b[e] = __float2bfloat16_rn(c0 + e < d ? v[q][h][e] - mu[c0 + e] : 0.0f);
            const float vr = __bfloat162float(b[e]);
            sq = fmaf(vr, vr, sq);
          }
          if (r < m) *reinterpret_cast<uint2 *>(dst + c0) = *reinterpret_cast<const uint2 *>(b);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(kFull, sq, o);
      if (lane == 0 && r < m) nrm[lo + r] = sq;
    }
  }
}

// ------------------------------------------------------------------ K9
__global__ void __launch_bounds__(1024) k_tile_plan(const int32_t *__restrict__ goff, int nleaf,
                                                    int32_t *tile_leaf, int32_t *tile_r0,
                                                    int32_t *n_tiles) {
  __shared__ int warp_tot[32];
  const int per = (nleaf + 1023) / 1024;
  const int j0 = threadIdx.x * per;
  int cnt = 0;
  for (int i = 0; i < per; ++i)
    if (j0 + i < nleaf) cnt += (goff[j0 + i + 1] - goff[j0 + i] + kTM - 1) / kTM;
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
    const int nt = (goff[j + 1] - goff[j] + kTM - 1) / kTM;
    for (int q = 0; q < nt; ++q) {
      tile_leaf[base + q] = j;
      tile_r0[base + q] = q * kTM;
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

struct MmaSmem {
  uint32_t a_off, b_off, buf_off, nrm_off, bar_off, total;
};

__host__ __device__ inline MmaSmem mma_smem_layout(int kb) {
  MmaSmem L;
  L.a_off = 0;
  L.b_off = L.a_off + (uint32_t)kb * kTM * 128;
  L.buf_off = L.b_off + (uint32_t)kStages * kb * kTN * 128;
  L.nrm_off = L.buf_off + kTM * kBufCap * 8;
  L.bar_off = L.nrm_off + kEpiWarps * kTN * 4;
  L.total = L.bar_off + 16 * 8 + 16;
  return L;
}

template <int KP>
__global__ void __launch_bounds__(kMmaThreads, 2) k_leaf_mma(
    const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
    const int32_t *__restrict__ goff, const int32_t *__restrict__ order,
    const float *__restrict__ nrm, const int32_t *__restrict__ tile_leaf,
    const int32_t *__restrict__ tile_r0, const int32_t *__restrict__ n_tiles, int kb, int tree,
    int32_t *__restrict__ run_idx, float *__restrict__ run_dist, int *err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const MmaSmem L = mma_smem_layout(kb);
  uint8_t *sA = smem + L.a_off;
  uint8_t *sB = smem + L.b_off;
  uint2 *buf = reinterpret_cast<uint2 *>(smem + L.buf_off);  // [slot][row]: (value bits, position)
  float *nbuf = reinterpret_cast<float *>(smem + L.nrm_off);  // [warp][kTN] column norms of a tile
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L.bar_off);
  uint64_t *full_a = bars + 0;
  uint64_t *full_b = bars + 1;             // kStages
  uint64_t *empty_b = bars + 1 + kStages;  // kStages
  uint64_t *acc_full = bars + 1 + 2 * kStages;
  uint64_t *acc_empty = acc_full + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 16);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 16) + 1;

  const int u = blockIdx.x;
  if (u >= *n_tiles) return;  // uniform for the whole block
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int leaf = tile_leaf[u], r0 = tile_r0[u];
  const int32_t lo = goff[leaf], m = goff[leaf + 1] - lo;
  const int nct = (m + kTN - 1) / kTN;
  const uint32_t a_bytes = (uint32_t)kb * kTM * 128, b_bytes = (uint32_t)kb * kTN * 128;

  if (threadIdx.x == 0) {
    mbar_init(full_a, 1);
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full_b + s, 1);
      mbar_init(empty_b + s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + b, 1);
      mbar_init(acc_empty + b, kEpiWarps * 32);
    }
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == kEpiWarps + 1) tmem_alloc(tmem_slot, 128);  // 2 accumulators x 64 columns
  if (warp == kEpiWarps && lane == 0) {
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kEpiWarps) {
    // ---- TMA producer
    if (lane == 0) {
      mbar_arrive_expect_tx(full_a, a_bytes);
      for (int q = 0; q < kb; ++q) tma_load_2d(sA + q * kTM * 128, &tmA, full_a, q * 64, lo + r0);
      for (int c = 0; c < nct && !*abort_flag; ++c) {
        const int s = c % kStages;
        if (c >= kStages && !mbar_wait(empty_b + s, ((c / kStages) - 1) & 1)) {
          *abort_flag = 1;
          break;
        }
        uint8_t *dst = sB + s * b_bytes;
        mbar_arrive_expect_tx(full_b + s, b_bytes);
        for (int q = 0; q < kb; ++q)
          tma_load_2d(dst + q * kTN * 128, &tmB, full_b + s, q * 64, lo + c * kTN);
      }
    }
  } else if (warp == kEpiWarps + 1) {
    // ---- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16_f32(kTM, kTN);
      const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
      bool ok = mbar_wait(full_a, 0);
      for (int c = 0; ok && c < nct && !*abort_flag; ++c) {
        const int s = c % kStages, b = c & 1;
        ok = mbar_wait(full_b + s, (c / kStages) & 1);
        if (ok && c >= 2) ok = mbar_wait(acc_empty + b, ((c >> 1) - 1) & 1);
        if (!ok) break;
        tc_fence_after();
        const uint32_t bs = b_base + s * b_bytes;
        for (int q = 0; q < kb; ++q)
#pragma unroll
          for (int k = 0; k < 4; ++k)
            mma_bf16(tmem + b * kTN, desc_k_sw128(a_base + q * kTM * 128 + k * 32),
                     desc_k_sw128(bs + q * kTN * 128 + k * 32), idesc, (q | k) ? 1u : 0u);
        mma_commit(empty_b + s);
        mma_commit(acc_full + b);
      }
      if (!ok) *abort_flag = 1;
    }
  } else {
    // ---- epilogue: thread = row (TMEM lane).  Candidates below the row's
    // current KP-th best go to a slot-major shared buffer (conflict-free:
    // consecutive rows are consecutive words); when any row of the warp has
    // kCheck pending, every row sorts its pending entries in batches of 16
    // and merges them into its sorted list with a bitonic network.
    const int row = warp * 32 + lane;
    const bool rvalid = r0 + row < m;
    float td[KP];
    int32_t ti[KP];
#pragma unroll
    for (int j = 0; j < KP; ++j) {
      td[j] = __int_as_float(0x7f800000);
      ti[j] = -1;
    }
    // Candidates that cannot beat the KP-th of the point's running list
    // (approximate squared distances of the earlier trees) are never kept.
    // (rows past the leaf get -inf and keep nothing)
    float thr = rvalid ? __int_as_float(0x7f800000) : -__int_as_float(0x7f800000);
    int32_t my_pos = -1, my_pt = -1;
    float nr = 0.0f;
    if (rvalid) {
      my_pos = lo + r0 + row;
      my_pt = __ldg(order + my_pos);
      nr = __ldg(nrm + my_pos);
      if (tree > 0) thr = run_dist[(int64_t)my_pt * KP + KP - 1] - nr;
    }
    const float thr0 = thr;
    // Pending candidates: a passing candidate is stored at the next free slot
    // of one of two per-row lanes of the buffer (even and odd columns, so two
    // independent append chains) by a predicated shared-memory store, no
    // branch; slot addresses are 32-bit shared-window offsets.
    constexpr int kHalf = kBufCap / 2;
    uint2 *const pbase = buf + row;
    const uint32_t abase0 = smem_u32(pbase), abase1 = abase0 + kHalf * kTM * 8;
    uint32_t aslot0 = abase0, aslot1 = abase1;
    auto pending0 = [&]() { return (int)((aslot0 - abase0) / (kTM * 8)); };
    auto pending1 = [&]() { return (int)((aslot1 - abase1) / (kTM * 8)); };
    auto flush = [&]() {
      const int c0 = pending0(), c1 = pending1();
      const int mx = __reduce_max_sync(kFull, max(c0, c1));
      for (int base = 0; base < mx; base += 8) {
        // 8 slots of each half make one batch of 16
        float sd[16];
        int32_t si[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int half = e >> 3, slot = base + (e & 7);
          const bool have = slot < (half ? c1 : c0);
          const uint2 ent = have ? pbase[(half * kHalf + slot) * kTM]
                                 : make_uint2(0x7f800000u, 0xffffffffu);
          sd[e] = __uint_as_float(ent.x);
          si[e] = (int32_t)ent.y;
        }
        bitonic_sort<16>(sd, si);
        bitonic_merge_into<KP, 16>(td, ti, sd, si);
      }
      aslot0 = abase0;
      aslot1 = abase1;
      thr = fminf(thr0, td[KP - 1]);
    };
    auto append = [&](uint32_t &aslot, float sv, uint32_t pos) {
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.lt.f32 p, %1, %2;\n\t"
          "@p st.shared.v2.u32 [%0], {%3, %4};\n\t"
          "@p add.u32 %0, %0, %5;\n\t}"
          : "+r"(aslot)
          : "f"(sv), "f"(thr), "r"(__float_as_uint(sv)), "r"(pos), "n"(kTM * 8)
          : "memory");
    };
    // one 32-column chunk of scores; DIAG: the warp's diagonal chunk, where
    // lane l's own point is column l and is skipped
    auto scan = [&](const float *v, const float *wn, int cb, auto diag_tag) {
      constexpr bool DIAG = decltype(diag_tag)::value;
#pragma unroll
      for (int h = 0; h < 32; h += kCheck) {
#pragma unroll
        for (int j4 = h; j4 < h + kCheck; j4 += 4) {
          const float4 nc4 = *reinterpret_cast<const float4 *>(wn + j4);
          const float ncs[4] = {nc4.x, nc4.y, nc4.z, nc4.w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int j = j4 + e;
            float sv = fmaf(-2.0f, v[j], ncs[e]);
            if (DIAG) sv = (j == lane) ? __int_as_float(0x7f800000) : sv;
            if (j & 1) append(aslot1, sv, (uint32_t)(cb + j));
            else append(aslot0, sv, (uint32_t)(cb + j));
          }
        }
        if (__any_sync(kFull, max(pending0(), pending1()) >= kHalf - kCheck / 2)) flush();
      }
    };
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c = 0; c < nct; ++c) {
      const int b = c & 1;
      if (!__all_sync(kFull, mbar_wait(acc_full + b, (c >> 1) & 1))) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      // this tile's column norms, staged per warp (16-byte aligned reads);
      // columns past the leaf carry an infinite norm and so never pass
      float *wn = nbuf + warp * kTN;
      __syncwarp();
#pragma unroll
      for (int h = 0; h < kTN; h += 32) {
        const int col = c * kTN + h + lane;
        wn[h + lane] = col < m ? __ldg(nrm + lo + col) : __int_as_float(0x7f800000);
      }
      __syncwarp();
#pragma unroll
      for (int q = 0; q < kTN / 32; ++q) {
        float v[32];
        tmem_ld32(lane_base + b * kTN + q * 32, v);
        const int cb = c * kTN + q * 32;
        // the warp's 32 rows sit in one 32-column chunk of the diagonal
        if (cb == r0 + warp * 32)
          scan(v, wn + q * 32, lo + cb, std::true_type{});
        else
          scan(v, wn + q * 32, lo + cb, std::false_type{});
      }
      tc_fence_before();
      mbar_arrive(acc_empty + b);
    }
    flush();
    if (rvalid) {
      // fold this tree's list into the running list: drop neighbours it
      // already holds, then a bitonic merge keeps the KP best
      const int64_t o = (int64_t)my_pt * KP;
      float rd[KP];
      int32_t ri[KP];
#pragma unroll
      for (int j = 0; j < KP; ++j) {
        rd[j] = tree > 0 ? run_dist[o + j] : __int_as_float(0x7f800000);
        ri[j] = tree > 0 ? run_idx[o + j] : -1;
      }
#pragma unroll
      for (int j = 0; j < KP; ++j) {
        int32_t q = ti[j] >= 0 ? __ldg(order + ti[j]) : -1;
        bool dup = false;
#pragma unroll
        for (int i = 0; i < KP; ++i) dup |= (q >= 0 && ri[i] == q);
        ti[j] = dup ? -1 : q;
        td[j] = (dup || q < 0) ? __int_as_float(0x7f800000) : nr + td[j];
      }
      bitonic_sort<KP>(td, ti);
      bitonic_merge_into<KP, KP>(rd, ri, td, ti);
#pragma unroll
      for (int j = 0; j < KP; ++j) {
        run_dist[o + j] = rd[j];
        run_idx[o + j] = ri[j];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kEpiWarps + 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 128);
  }
  if (threadIdx.x == 0 && *abort_flag) atomicOr(err, 1);
}

// ------------------------------------------------------------------ K11
// One warp per point.  The warp stages the query row and its K2 candidate
// rows in shared memory with coalesced loads (rows padded to d + 4 floats so
// that the float4 reads below hit distinct banks), then lane j computes the
// exact FP32 distance of candidate j: the sequential sum, in dimension order,
// of rounded squares of rounded differences, and its rounded square root.
// d must be a multiple of 4.
// One warp per point.  For each candidate the warp reads the candidate row
// with one coalesced pass (lane l holds dimensions 4l..4l+3 of every
// 128-wide chunk), each lane adds its squared differences with fused
// multiply-adds and a fixed butterfly adds the 32 lane sums: an FP32 distance
// with pairwise summation, the same on every run.  Lane j then holds
// candidate j (j < K2) and the K2 pairs are sorted with a bitonic network;
// candidates whose distance lies within 2^-16 of the k-th are re-ordered by
// an FP64 distance.  d must be a multiple of 4 and at most 256.
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
  constexpr int NC = D > 0 ? (D + 127) / 128 : 2;  // 128-wide chunks (d <= 256)
  float q[NC][4];
  const T *xp = X + (int64_t)p * d;
#pragma unroll
  for (int h = 0; h < NC; ++h) {
    const int c0 = h * 128 + 4 * lane;
    q[h][0] = q[h][1] = q[h][2] = q[h][3] = 0.0f;
    if (c0 < d) load4<T>(xp + c0, q[h]);
  }
  float dist = inf;
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
  switch (d) {
    case 128: return launch_rerank_t<T, 128, K2>(X, d, visit, n, cand, k, out_idx, out_dist, s);
    case 96: return launch_rerank_t<T, 128, K2>(X, d, visit, n, cand, k, out_idx, out_dist, s);
    case 256: return launch_rerank_t<T, 256, K2>(X, d, visit, n, cand, k, out_idx, out_dist, s);
    default: return launch_rerank_t<T, 0, K2>(X, d, visit, n, cand, k, out_idx, out_dist, s);
  }
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

drpt_status make_tmap(CUtensorMap *map, const void *base, int64_t rows, int d_pad, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available");
    return DRPT_ERR_CUDA;
  }
  cuuint64_t dims[2] = {(cuuint64_t)d_pad, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)d_pad * 2};
  cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return DRPT_ERR_CUDA;
  }
  return DRPT_OK;
}

}  // namespace

drpt_status launch_leaf_center(const MixedTreeArgs &a, cudaStream_t s) {
  if (a.d % 4 != 0 || a.d > 256) {
    set_error("mixed mode needs d %% 4 == 0 and d <= 256 (got %d)", a.d);
    return DRPT_ERR_UNSUPPORTED;
  }
  const size_t smem = 0;
  if (a.dtype == DRPT_DTYPE_U8)
    k_leaf_center<uint8_t><<<a.nleaf, 256, smem, s>>>((const uint8_t *)a.X, a.d, a.d_pad, a.order,
                                                       a.goff, a.Xb, a.nrm);
  else
    k_leaf_center<float><<<a.nleaf, 256, smem, s>>>((const float *)a.X, a.d, a.d_pad, a.order,
                                                     a.goff, a.Xb, a.nrm);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_leaf_mma(const MixedTreeArgs &a, cudaStream_t s) {
  if (a.d_pad % 64 != 0 || a.d_pad > 256) {
    set_error("mixed leaf kernel: padded dimension %d unsupported (multiple of 64, <= 256)", a.d_pad);
    return DRPT_ERR_UNSUPPORTED;
  }
  k_tile_plan<<<1, 1024, 0, s>>>(a.goff, a.nleaf, a.tile_leaf, a.tile_r0, a.n_tiles);
  DRPT_LAUNCH_CHECK();
  CUtensorMap tmA, tmB;
  DRPT_TRY(make_tmap(&tmA, a.Xb, a.n, a.d_pad, kTM));
  DRPT_TRY(make_tmap(&tmB, a.Xb, a.n, a.d_pad, kTN));
  const int kb = a.d_pad / 64;
  const MmaSmem L = mma_smem_layout(kb);
  const size_t smem = L.total + 1024;
  const unsigned grid = (unsigned)(ceil_div(a.n, kTM) + a.nleaf);
  if (a.kp == 16) {
    DRPT_CUDA(cudaFuncSetAttribute(k_leaf_mma<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    k_leaf_mma<16><<<grid, kMmaThreads, smem, s>>>(tmA, tmB, a.goff, a.order, a.nrm, a.tile_leaf,
                                                   a.tile_r0, a.n_tiles, kb, a.tree, a.cand_idx,
                                                   a.cand_dist, a.err);
  } else if (a.kp == 32) {
    DRPT_CUDA(cudaFuncSetAttribute(k_leaf_mma<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    k_leaf_mma<32><<<grid, kMmaThreads, smem, s>>>(tmA, tmB, a.goff, a.order, a.nrm, a.tile_leaf,
                                                   a.tile_r0, a.n_tiles, kb, a.tree, a.cand_idx,
                                                   a.cand_dist, a.err);
  } else {
    set_error("mixed leaf kernel: %d candidates per tree unsupported (16 or 32)", a.kp);
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
  if (d % 4 != 0 || d > 256) {
    set_error("re-rank needs d %% 4 == 0 and d <= 256 (got %d)", d);
    return DRPT_ERR_UNSUPPORTED;
  }
  if (dtype == DRPT_DTYPE_U8)
    return K2 == 16 ? launch_rerank_d<uint8_t, 16>(X, d, visit, n, cand, k, out_idx, out_dist, s)
                    : launch_rerank_d<uint8_t, 32>(X, d, visit, n, cand, k, out_idx, out_dist, s);
  return K2 == 16 ? launch_rerank_d<float, 16>(X, d, visit, n, cand, k, out_idx, out_dist, s)
                  : launch_rerank_d<float, 32>(X, d, visit, n, cand, k, out_idx, out_dist, s);
}

}  // namespace drpt
