// Learned splits: per tree level an MLP d -> 64 -> 1 whose output replaces the
// random projection as the split value of a learned tree (no reference
// counterpart; the method is otherwise the mixed form's).
//
// Training (one level of all learned trees at a time, on a sample of S points
// grouped by the level's nodes, neighbour pairs from the method's own leaf
// brute force of the sample):
//   L1 k_mlp_fwd        z = bf16(W1) x + b1, a = tanh z, f = bf16(w2) . a + b2
//   L2 k_node_moments   per node: mean and variance of f (FP64, fixed order)
//   L3 k_point_pairs    per point: its out- and in-pairs inside its node
//   L4 k_node_pairsum   per node: S_n = sum of squared pair differences
//   L5 k_point_grad     dL/df of every sample point
//   L6 k_mlp_bwd        partial weight gradients per row chunk
//   L7 k_adam           chunk partials added in order, Adam step
// with L = (1/P) sum_n S_n / V_n over the P same-node ordered pairs.  Every
// reduction runs in a fixed order, so training is deterministic.  Small
// kernels around it (sample moments, weight initialisation, pair counts, loss
// sums, node labels, weight stacking) keep the whole level loop on the
// device.
//
// Inference over all n points (L8 k_mlp_infer): TMA-fed tcgen05 BF16 MMAs of
// 128 standardised rows against each MLP's 64 x d weights (FP32 accumulators
// in TMEM), epilogue tanh + output layer per row, one projected column per
// MLP.
#include <cuda.h>

#include "kernels.cuh"
#include "sm100.cuh"

namespace drpt {
namespace {

using namespace sm100;

constexpr int kH = kLearnHidden;  // 64 hidden units

__device__ __forceinline__ float rbf(float w) { return __bfloat162float(__float2bfloat16_rn(w)); }

// ------------------------------------------------------------------ L1
// Block: 128 sample rows x 64 hidden units of one tree; thread (ty, tx) holds
// rows 8ty..8ty+7 and units 4tx..4tx+3 (ty 0..15, tx 0..15); d in chunks of
// 32 through shared memory stored k-major, so a thread reads its 8 rows and 4
// units as float4s.  Output A (T x S x 64) and f (T x S).
__global__ void __launch_bounds__(256) k_mlp_fwd(const float *__restrict__ Xs, int S, int d,
                                                 const float *__restrict__ params, int np,
                                                 float *__restrict__ A, float *__restrict__ f) {
  __shared__ __align__(16) float xs[32][128 + 4];
  __shared__ __align__(16) float ws[32][64 + 4];
  const int t = blockIdx.y;
  const float *W1 = params + (int64_t)t * np;
  const float *b1 = W1 + kH * d, *w2 = b1 + kH, *b2 = w2 + kH;
  const int r0 = blockIdx.x * 128;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[8][4] = {};
  for (int k0 = 0; k0 < d; k0 += 32) {
    for (int e = threadIdx.x; e < 128 * 32; e += 256) {
      const int r = e >> 5, k = e & 31;
      xs[k][r] = (r0 + r < S && k0 + k < d) ? Xs[(int64_t)(r0 + r) * d + k0 + k] : 0.0f;
    }
    for (int e = threadIdx.x; e < 64 * 32; e += 256) {
      const int h = e >> 5, k = e & 31;
      ws[k][h] = (k0 + k < d) ? rbf(W1[(int64_t)h * d + k0 + k]) : 0.0f;
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const float4 x0 = *reinterpret_cast<const float4 *>(&xs[k][8 * ty]);
      const float4 x1 = *reinterpret_cast<const float4 *>(&xs[k][8 * ty + 4]);
      const float4 w = *reinterpret_cast<const float4 *>(&ws[k][4 * tx]);
      const float xv[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
      const float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(xv[i], wv[j], acc[i][j]);
    }
    __syncthreads();
  }
  float bb[4], ww[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    bb[j] = b1[4 * tx + j];
    ww[j] = rbf(w2[4 * tx + j]);
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = r0 + 8 * ty + i;
    float a[4], part = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      a[j] = tanhf(acc[i][j] + bb[j]);
      part = fmaf(ww[j], a[j], part);
    }
    if (r < S)
      *reinterpret_cast<float4 *>(A + ((int64_t)t * S + r) * kH + 4 * tx) =
          make_float4(a[0], a[1], a[2], a[3]);
    // the 16 threads of a row are 16 consecutive lanes: fixed butterfly
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
    if (tx == 0 && r < S) f[(int64_t)t * S + r] = part + b2[0];
  }
}

// Block reduction of a double in a fixed order (256 threads).
__device__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  const int w = threadIdx.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < 8; ++i) s += sh[i];
  return s;
}

// ------------------------------------------------------------------ L2
// Block (node, tree): mean and variance (+ eps) of f over the node's points.
// Node tables have `nodes` entries per tree (noff: nodes + 1).
__global__ void __launch_bounds__(256) k_node_moments(const float *__restrict__ f, int S,
                                                      const int32_t *__restrict__ perm,
                                                      const int32_t *__restrict__ noff, int nodes,
                                                      float *__restrict__ mu,
                                                      float *__restrict__ var) {
  __shared__ double sh[8];
  const int n = blockIdx.x, t = blockIdx.y;
  const int32_t *off = noff + (int64_t)t * (nodes + 1);
  const int lo = off[n], hi = off[n + 1];
  if (lo >= hi) return;  // block-uniform
  const int32_t *pm = perm + (int64_t)t * S;
  const float *ft = f + (int64_t)t * S;
  double s1 = 0.0;
  for (int i = lo + threadIdx.x; i < hi; i += 256) s1 += ft[pm[i]];
  const double m = block_sum(s1, sh) / (hi - lo);
  double s2 = 0.0;
  for (int i = lo + threadIdx.x; i < hi; i += 256) {
    const double df = ft[pm[i]] - m;
    s2 += df * df;
  }
  const double v = block_sum(s2, sh) / (hi - lo) + kLearnEps;
  if (threadIdx.x == 0) {
    mu[(int64_t)t * nodes + n] = (float)m;
    var[(int64_t)t * nodes + n] = (float)v;
  }
}

// ------------------------------------------------------------------ L3
// Per point i: pair part of dL/df_i, 2/(P V_n) * sum over its out- and
// in-pairs in its node of (f_i - f_j), and s_i = sum over its out-pairs of
// (f_i - f_j)^2.
__global__ void k_point_pairs(const float *__restrict__ f, int S, const int32_t *__restrict__ node_of,
                              const int32_t *__restrict__ nbr, int k,
                              const int32_t *__restrict__ in_ptr, const int32_t *__restrict__ in_idx,
                              const float *__restrict__ var, int nodes,
                              const float *__restrict__ inv_pairs, float *__restrict__ gp,
                              float *__restrict__ sp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, t = blockIdx.y;
  if (i >= S) return;
  const float *ft = f + (int64_t)t * S;
  const int32_t *no = node_of + (int64_t)t * S;
  const int n = no[i];
  const float fi = ft[i];
  float lin = 0.0f, sq = 0.0f;
  for (int q = 0; q < k; ++q) {
    const int j = nbr[(int64_t)i * k + q];
    if (j >= 0 && no[j] == n) {
      const float df = fi - ft[j];
      lin += df;
      sq = fmaf(df, df, sq);
    }
  }
  for (int e = in_ptr[i]; e < in_ptr[i + 1]; ++e) {
    const int j = in_idx[e];
    if (no[j] == n) lin += fi - ft[j];
  }
  const float V = var[(int64_t)t * nodes + n];
  gp[(int64_t)t * S + i] = 2.0f * inv_pairs[t] * lin / V;
  sp[(int64_t)t * S + i] = sq;
}

// ------------------------------------------------------------------ L4
// Block (node, tree): S_n, and the node's loss term S_n / (P V_n).
__global__ void __launch_bounds__(256) k_node_pairsum(const float *__restrict__ sp, int S,
                                                      const int32_t *__restrict__ perm,
                                                      const int32_t *__restrict__ noff, int nodes,
                                                      const float *__restrict__ var,
                                                      const float *__restrict__ inv_pairs,
                                                      float *__restrict__ sn,
                                                      float *__restrict__ lterm) {
  __shared__ double sh[8];
  const int n = blockIdx.x, t = blockIdx.y;
  const int32_t *off = noff + (int64_t)t * (nodes + 1);
  const int lo = off[n], hi = off[n + 1];
  const int64_t o = (int64_t)t * nodes + n;
  if (lo >= hi) {
    if (threadIdx.x == 0) lterm[o] = 0.0f;
    return;
  }
  const int32_t *pm = perm + (int64_t)t * S;
  double s = 0.0;
  for (int i = lo + threadIdx.x; i < hi; i += 256) s += sp[(int64_t)t * S + pm[i]];
  const double tot = block_sum(s, sh);
  if (threadIdx.x == 0) {
    sn[o] = (float)tot;
    lterm[o] = (float)(tot / var[o] * inv_pairs[t]);
  }
}

// ------------------------------------------------------------------ L5
__global__ void k_point_grad(const float *__restrict__ f, int S, const int32_t *__restrict__ node_of,
                             const int32_t *__restrict__ noff, int nodes,
                             const float *__restrict__ mu, const float *__restrict__ var,
                             const float *__restrict__ sn, const float *__restrict__ inv_pairs,
                             float *__restrict__ g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, t = blockIdx.y;
  if (i >= S) return;
  const int n = node_of[(int64_t)t * S + i];
  const int64_t o = (int64_t)t * nodes + n;
  const int32_t *off = noff + (int64_t)t * (nodes + 1);
  const float m = (float)(off[n + 1] - off[n]);
  const float V = var[o];
  const float fi = f[(int64_t)t * S + i];
  g[(int64_t)t * S + i] -= 2.0f * inv_pairs[t] * sn[o] * (fi - mu[o]) / (V * V * m);
}

// ------------------------------------------------------------------ L6
// Block (row chunk, tree, 128-dimension tile): partial dW1 over the chunk's
// rows for 64 units x 128 dimensions (thread (ty, tx): units 4ty..4ty+3,
// dimensions 4tx..4tx+3 and 64+4tx..64+4tx+3, so that the 16 lanes' float4
// reads of a row cover 64 consecutive floats: no bank conflicts), rows in
// steps of 32 through shared memory.
// Dimension tile 0 also writes the partials of b1, w2 and b2.  Partials:
// T x R x np.
__global__ void __launch_bounds__(256) k_mlp_bwd(const float *__restrict__ Xs, int S, int d,
                                                 const float *__restrict__ params, int np,
                                                 const float *__restrict__ A,
                                                 const float *__restrict__ g, int rows_per_chunk,
                                                 float *__restrict__ part) {
  __shared__ __align__(16) float dz[32][64 + 4];
  __shared__ __align__(16) float xs[32][128 + 4];
  __shared__ float as[32][64 + 1];
  __shared__ float gs[32];
  const int r = blockIdx.x, t = blockIdx.y, k0 = blockIdx.z * 128;
  const int R = gridDim.x;
  const float *w2 = params + (int64_t)t * np + kH * d + kH;
  const int i0 = r * rows_per_chunk, i1 = min(S, i0 + rows_per_chunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][8] = {};
  float db1 = 0.0f, dw2 = 0.0f, db2 = 0.0f;  // thread h < 64: unit h
  for (int b = i0; b < i1; b += 32) {
    for (int e = threadIdx.x; e < 32 * 64; e += 256) {
      const int q = e >> 6, h = e & 63, i = b + q;
      float v = 0.0f, a = 0.0f;
      if (i < i1) {
        a = A[((int64_t)t * S + i) * kH + h];
        v = g[(int64_t)t * S + i] * rbf(w2[h]) * (1.0f - a * a);
      }
      dz[q][h] = v;
      as[q][h] = a;
    }
    for (int e = threadIdx.x; e < 32 * 128; e += 256) {
      const int q = e >> 7, k = e & 127, i = b + q;
      xs[q][k] = (i < i1 && k0 + k < d) ? Xs[(int64_t)i * d + k0 + k] : 0.0f;
    }
    if (threadIdx.x < 32)
      gs[threadIdx.x] = b + threadIdx.x < i1 ? g[(int64_t)t * S + b + threadIdx.x] : 0.0f;
    __syncthreads();
#pragma unroll 4
    for (int q = 0; q < 32; ++q) {
      const float4 z = *reinterpret_cast<const float4 *>(&dz[q][4 * ty]);
      const float4 x0 = *reinterpret_cast<const float4 *>(&xs[q][4 * tx]);
      const float4 x1 = *reinterpret_cast<const float4 *>(&xs[q][64 + 4 * tx]);
      const float zv[4] = {z.x, z.y, z.z, z.w};
      const float xv[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = fmaf(zv[u], xv[v], acc[u][v]);
    }
    if (blockIdx.z == 0 && threadIdx.x < kH) {
      const int h = threadIdx.x;
      for (int q = 0; q < 32 && b + q < i1; ++q) {
        db1 += dz[q][h];
        dw2 = fmaf(gs[q], as[q][h], dw2);
        if (h == 0) db2 += gs[q];
      }
    }
    __syncthreads();
  }
  float *out = part + ((int64_t)t * R + r) * np;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const int h = 4 * ty + u, k = k0 + (v < 4 ? 4 * tx + v : 64 + 4 * tx + v - 4);
      if (k < d) out[(int64_t)h * d + k] = acc[u][v];
    }
  if (blockIdx.z == 0 && threadIdx.x < kH) {
    out[kH * d + threadIdx.x] = db1;
    out[kH * d + kH + threadIdx.x] = dw2;
    if (threadIdx.x == 0) out[kH * d + 2 * kH] = db2;
  }
}

// ------------------------------------------------------------------ L7
// Gradient = chunk partials added in chunk order; Adam (b1 0.9, b2 0.999) on
// the FP32 master weights.  lr = 0 only writes the gradient.
__global__ void k_adam(float *__restrict__ params, float *__restrict__ m1, float *__restrict__ m2,
                       const float *__restrict__ part, int R, int np, int T, float lr, float bc1,
                       float bc2, float *__restrict__ grad_out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)T * np) return;
  const int t = (int)(e / np), p = (int)(e - (int64_t)t * np);
  float gsum = 0.0f;
  for (int r = 0; r < R; ++r) gsum += part[((int64_t)t * R + r) * np + p];
  if (grad_out) grad_out[e] = gsum;
  if (lr == 0.0f) return;
  const float a = 0.9f * m1[e] + 0.1f * gsum;
  const float b = 0.999f * m2[e] + 0.001f * gsum * gsum;
  m1[e] = a;
  m2[e] = b;
  params[e] -= lr * (a / bc1) / (sqrtf(b / bc2) + 1e-8f);
}

// ------------------------------------------------------------------ init
// Initial weights of one level of every tree: W1 ~ N(0, 1/d), b1 = 0,
// w2 ~ N(0, 1/64), b2 = 0.  Normal deviates by the Box-Muller transform of
// two uniforms from a counter-based hash (splitmix64 finaliser) of (seed,
// tree, level, parameter), so the draw does not depend on the launch shape.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void k_init_params(float *__restrict__ params, int T, int d, int np, uint64_t seed,
                              int level) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)T * np) return;
  const int t = (int)(e / np), p = (int)(e - (int64_t)t * np);
  float v = 0.0f;
  const bool is_w1 = p < kH * d, is_w2 = p >= kH * d + kH && p < kH * d + 2 * kH;
  if (is_w1 || is_w2) {
    const uint64_t h =
        mix64(seed ^ mix64(((uint64_t)t << 40) ^ ((uint64_t)level << 32) ^ (uint64_t)p));
    const float u1 = ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);  // (0, 1)
    const float u2 = (float)((h >> 16) & 0xFFFFFFull) * (1.0f / 16777216.0f);
    const float z = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
    v = is_w1 ? z * rsqrtf((float)d) : z * 0.125f;
  }
  params[e] = v;
}

// ------------------------------------------------------------------ pairs
// Same-node ordered pairs of every tree (integer counts: order-free), then
// inv[t] = 1 / max(count, 1).
__global__ void k_pair_count(const int32_t *__restrict__ node_of, int S,
                             const int32_t *__restrict__ nbr, int k, int *__restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, t = blockIdx.y;
  int c = 0;
  if (i < S) {
    const int32_t *no = node_of + (int64_t)t * S;
    const int n = no[i];
    for (int q = 0; q < k; ++q) {
      const int j = nbr[(int64_t)i * k + q];
      c += (j >= 0 && no[j] == n) ? 1 : 0;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt + t, c);
}

__global__ void k_pair_inv(const int *__restrict__ cnt, int T, float *__restrict__ inv) {
  const int t = threadIdx.x;
  if (t < T) inv[t] = 1.0f / (float)max(cnt[t], 1);
}

// Loss of the level (sum of node terms per tree, trees added in order) added
// to acc[slot].
__global__ void k_loss_sum(const float *__restrict__ lterm, int T, int nodes, float *acc,
                           int slot) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < nodes; ++j) s += lterm[(int64_t)t * nodes + j];
  acc[slot] += (float)s;
}

// f in the order of perm (the level kernels' node-grouped values).
__global__ void k_gather_f(const float *__restrict__ f, const int32_t *__restrict__ perm, int S,
                           int T, float *__restrict__ fp) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)T * S) return;
  const int t = (int)(e / S);
  fp[e] = f[(int64_t)t * S + perm[e]];
}

// Block (node, tree): the node's points get label j.
__global__ void k_node_label(const int32_t *__restrict__ perm, const int32_t *__restrict__ noff,
                             int nodes, int S, int32_t *__restrict__ node_of) {
  const int j = blockIdx.x, t = blockIdx.y;
  const int32_t *off = noff + (int64_t)t * (nodes + 1);
  for (int i = off[j] + threadIdx.x; i < off[j + 1]; i += blockDim.x)
    node_of[(int64_t)t * S + perm[(int64_t)t * S + i]] = j;
}

// Inference weights of MLP m = t * levels + level: W1 to BF16 rows of d_pad
// (padding stays 0 from an earlier clear), b1, w2 rounded as in training, b2.
__global__ void k_stack(const float *__restrict__ params, int T, int d, int np, int d_pad,
                        int levels, int level, __nv_bfloat16 *__restrict__ W1b,
                        float *__restrict__ b1, float *__restrict__ w2, float *__restrict__ b2) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)T * np) return;
  const int t = (int)(e / np), p = (int)(e - (int64_t)t * np);
  const int64_t m = (int64_t)t * levels + level;
  const float v = params[e];
  if (p < kH * d) {
    const int h = p / d, k = p - h * d;
    W1b[(m * kH + h) * d_pad + k] = __float2bfloat16_rn(v);
  } else if (p < kH * d + kH) {
    b1[m * kH + (p - kH * d)] = v;
  } else if (p < kH * d + 2 * kH) {
    w2[m * kH + (p - kH * d - kH)] = rbf(v);
  } else {
    b2[m] = v;
  }
}

// Per-dimension mean of the sample rows and the scalar scale
// 1 / sqrt(mean over dimensions of the variance), FP64 in fixed order.
// Block: 32 dimensions (lane tx) x 8 row phases (ty): thread (tx, ty) adds
// rows ty, ty + 8, ... of dimension k0 + tx in order (coalesced 128-byte row
// pieces per warp), the 8 phase sums are added in phase order; the squared
// deviations from the mean follow in a second pass.
__global__ void __launch_bounds__(256) k_sample_mean(const float *__restrict__ Xr, int S, int d,
                                                     float *__restrict__ c,
                                                     double *__restrict__ var) {
  __shared__ double part[8][32];
  __shared__ double mean[32];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int k = blockIdx.x * 32 + tx;
  double s = 0.0;
  if (k < d)
    for (int i = ty; i < S; i += 8) s += Xr[(int64_t)i * d + k];
  part[ty][tx] = s;
  __syncthreads();
  if (ty == 0) {
    double t = 0.0;
    for (int p = 0; p < 8; ++p) t += part[p][tx];
    mean[tx] = t / S;
  }
  __syncthreads();
  const double m = mean[tx];
  double q = 0.0;
  if (k < d)
    for (int i = ty; i < S; i += 8) {
      const double df = Xr[(int64_t)i * d + k] - m;
      q += df * df;
    }
  __syncthreads();  // part is reused
  part[ty][tx] = q;
  __syncthreads();
  if (ty == 0 && k < d) {
    double t = 0.0;
    for (int p = 0; p < 8; ++p) t += part[p][tx];
    c[k] = (float)m;
    var[k] = t / S;
  }
}

__global__ void k_sample_scale(const double *__restrict__ var, int d, float *__restrict__ inv_sigma) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int k = 0; k < d; ++k) s += var[k];
  const double sig = sqrt(s / d);
  *inv_sigma = sig > 0.0 ? (float)(1.0 / sig) : 1.0f;
}

// ------------------------------------------------------------------ standardise
// Out row i = (X[rows ? rows[i] : i] - c) * inv_sigma (c, inv_sigma device
// pointers, nullptr = 0 and 1): as BF16 rows of d_pad (zero-padded) and/or
// FP32 rows of d.
template <typename T>
__global__ void k_standardise(const T *__restrict__ X, int64_t n, int d, int d_pad,
                              const int32_t *__restrict__ rows, const float *__restrict__ c,
                              const float *__restrict__ inv_sigma, __nv_bfloat16 *__restrict__ Xb,
                              float *__restrict__ Xf) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * d_pad) return;
  const int64_t i = e / d_pad;
  const int k = (int)(e - i * d_pad);
  float v = 0.0f;
  if (k < d) {
    const int64_t src = rows ? rows[i] : i;
    v = (float)X[src * d + k];
    if (c) v -= c[k];
    if (inv_sigma) v *= *inv_sigma;
  }
  if (Xb) Xb[e] = __float2bfloat16_rn(v);
  if (Xf && k < d) Xf[i * d + k] = v;
}

// ------------------------------------------------------------------ L8
constexpr int kIM = 128;  // rows per CTA
constexpr int kIN = 64;   // hidden units per MLP (MMA N)
constexpr int kIStages = 2;
constexpr int kIEpi = 4;
constexpr int kIThreads = 32 * (kIEpi + 2);

__global__ void __launch_bounds__(kIThreads, 1) k_mlp_infer(
    const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmW, int64_t n,
    int kb, int nmlp, const float *__restrict__ b1, const float *__restrict__ w2,
    const float *__restrict__ b2, float *__restrict__ P, int *err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t a_bytes = (uint32_t)kb * kIM * 128, b_bytes = (uint32_t)kb * kIN * 128;
  uint8_t *sA = smem;
  uint8_t *sB = smem + a_bytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(sB + kIStages * b_bytes);
  uint64_t *full_a = bars, *full_b = bars + 1, *empty_b = bars + 1 + kIStages;
  uint64_t *acc_full = bars + 1 + 2 * kIStages, *acc_empty = acc_full + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 12);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(bars + 12) + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r0 = (int64_t)blockIdx.x * kIM;
  if (threadIdx.x == 0) {
    mbar_init(full_a, 1);
    for (int s = 0; s < kIStages; ++s) {
      mbar_init(full_b + s, 1);
      mbar_init(empty_b + s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(acc_full + b, 1);
      mbar_init(acc_empty + b, kIEpi * 32);
    }
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == kIEpi + 1) tmem_alloc(tmem_slot, 128);
  if (warp == kIEpi && lane == 0) {
    prefetch_tmap(&tmX);
    prefetch_tmap(&tmW);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  if (warp == kIEpi) {
    if (lane == 0) {
      mbar_arrive_expect_tx(full_a, a_bytes);
      for (int q = 0; q < kb; ++q)
        tma_load_2d(sA + q * kIM * 128, &tmX, full_a, q * 64, (int32_t)r0);
      for (int c = 0; c < nmlp && !*abort_flag; ++c) {
        const int s = c % kIStages;
        if (c >= kIStages && !mbar_wait(empty_b + s, ((c / kIStages) - 1) & 1)) {
          *abort_flag = 1;
          break;
        }
        mbar_arrive_expect_tx(full_b + s, b_bytes);
        for (int q = 0; q < kb; ++q)
          tma_load_2d(sB + s * b_bytes + q * kIN * 128, &tmW, full_b + s, q * 64, c * kIN);
      }
    }
  } else if (warp == kIEpi + 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16_f32(kIM, kIN);
      const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
      bool ok = mbar_wait(full_a, 0);
      for (int c = 0; ok && c < nmlp && !*abort_flag; ++c) {
        const int s = c % kIStages, b = c & 1;
        ok = mbar_wait(full_b + s, (c / kIStages) & 1);
        if (ok && c >= 2) ok = mbar_wait(acc_empty + b, ((c >> 1) - 1) & 1);
        if (!ok) break;
        tc_fence_after();
        const uint32_t bs = b_base + s * b_bytes;
        for (int q = 0; q < kb; ++q)
#pragma unroll
          for (int k = 0; k < 4; ++k)
            mma_bf16(tmem + b * kIN, desc_k_sw128(a_base + q * kIM * 128 + k * 32),
                     desc_k_sw128(bs + q * kIN * 128 + k * 32), idesc, (q | k) ? 1u : 0u);
        mma_commit(empty_b + s);
        mma_commit(acc_full + b);
      }
      if (!ok) *abort_flag = 1;
    }
  } else {
    // epilogue: thread = row; per MLP the 64 pre-activations of the row
    const int64_t row = r0 + warp * 32 + lane;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c = 0; c < nmlp; ++c) {
      const int b = c & 1;
      if (!__all_sync(kFull, mbar_wait(acc_full + b, (c >> 1) & 1))) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      float z[64];
      tmem_ld32(lane_base + b * kIN, z);
      tmem_ld32(lane_base + b * kIN + 32, z + 32);
      tc_fence_before();
      mbar_arrive(acc_empty + b);
      const float *bb = b1 + (int64_t)c * kIN, *ww = w2 + (int64_t)c * kIN;
      float fv = __ldg(b2 + c);
#pragma unroll
      for (int h = 0; h < kIN; ++h) fv = fmaf(__ldg(ww + h), tanhf(z[h] + __ldg(bb + h)), fv);
      if (row < n) P[(int64_t)c * n + row] = fv;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kIEpi + 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 128);
  }
  if (threadIdx.x == 0 && *abort_flag) atomicOr(err, 1);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

drpt_status bf16_tmap(CUtensorMap *map, const void *base, int64_t rows, int d_pad, int box_rows) {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available");
    return DRPT_ERR_CUDA;
  }
  cuuint64_t dims[2] = {(cuuint64_t)d_pad, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)d_pad * 2};
  cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return DRPT_ERR_CUDA;
  }
  return DRPT_OK;
}

}  // namespace

drpt_status launch_learn_step(const LearnArgs &a, float lr, float bc1, float bc2, float *grad_out,
                              cudaStream_t s) {
  const dim3 g128((unsigned)ceil_div(a.S, 128), (unsigned)a.T);
  k_mlp_fwd<<<g128, 256, 0, s>>>(a.Xs, a.S, a.d, a.params, a.np, a.A, a.f);
  const dim3 gn((unsigned)a.nodes, (unsigned)a.T);
  k_node_moments<<<gn, 256, 0, s>>>(a.f, a.S, a.perm, a.noff, a.nodes, a.mu, a.var);
  const dim3 gp((unsigned)ceil_div(a.S, 256), (unsigned)a.T);
  k_point_pairs<<<gp, 256, 0, s>>>(a.f, a.S, a.node_of, a.nbr, a.k, a.in_ptr, a.in_idx, a.var,
                                   a.nodes, a.inv_pairs, a.g, a.sp);
  k_node_pairsum<<<gn, 256, 0, s>>>(a.sp, a.S, a.perm, a.noff, a.nodes, a.var, a.inv_pairs,
                                    a.sn, a.lterm);
  k_point_grad<<<gp, 256, 0, s>>>(a.f, a.S, a.node_of, a.noff, a.nodes, a.mu, a.var, a.sn,
                                  a.inv_pairs, a.g);
  const int rows = (int)ceil_div(a.S, a.R);
  const dim3 gb((unsigned)a.R, (unsigned)a.T, (unsigned)ceil_div(a.d, 128));
  k_mlp_bwd<<<gb, 256, 0, s>>>(a.Xs, a.S, a.d, a.params, a.np, a.A, a.g, rows, a.part);
  const int64_t total = (int64_t)a.T * a.np;
  k_adam<<<(unsigned)ceil_div(total, 256), 256, 0, s>>>(a.params, a.m1, a.m2, a.part, a.R, a.np,
                                                        a.T, lr, bc1, bc2, grad_out);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

int learn_step_kernels() { return 7; }

drpt_status launch_learn_init(const LearnArgs &a, uint64_t seed, int level, cudaStream_t s) {
  const int64_t total = (int64_t)a.T * a.np;
  k_init_params<<<(unsigned)ceil_div(total, 256), 256, 0, s>>>(a.params, a.T, a.d, a.np, seed,
                                                               level);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_learn_pairs(const LearnArgs &a, int *cnt, cudaStream_t s) {
  DRPT_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * a.T, s));
  const dim3 gp((unsigned)ceil_div(a.S, 256), (unsigned)a.T);
  k_pair_count<<<gp, 256, 0, s>>>(a.node_of, a.S, a.nbr, a.k, cnt);
  k_pair_inv<<<1, 32 * (int)ceil_div(a.T, 32), 0, s>>>(cnt, a.T, (float *)a.inv_pairs);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_learn_loss(const LearnArgs &a, float *acc, int slot, cudaStream_t s) {
  k_loss_sum<<<1, 32, 0, s>>>(a.lterm, a.T, a.nodes, acc, slot);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_gather_f(const LearnArgs &a, float *fp, cudaStream_t s) {
  const int64_t total = (int64_t)a.T * a.S;
  k_gather_f<<<(unsigned)ceil_div(total, 256), 256, 0, s>>>(a.f, a.perm, a.S, a.T, fp);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_node_label(const int32_t *perm, const int32_t *noff, int nodes, int S, int T,
                              int32_t *node_of, cudaStream_t s) {
  k_node_label<<<dim3((unsigned)nodes, (unsigned)T), 256, 0, s>>>(perm, noff, nodes, S, node_of);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_stack(const LearnArgs &a, int d_pad, int levels, int level,
                         __nv_bfloat16 *W1b, float *b1, float *w2, float *b2, cudaStream_t s) {
  const int64_t total = (int64_t)a.T * a.np;
  k_stack<<<(unsigned)ceil_div(total, 256), 256, 0, s>>>(a.params, a.T, a.d, a.np, d_pad, levels,
                                                         level, W1b, b1, w2, b2);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_sample_scale(const float *Xr, int S, int d, float *c, double *var,
                                float *inv_sigma, cudaStream_t s) {
  k_sample_mean<<<(unsigned)ceil_div(d, 32), 256, 0, s>>>(Xr, S, d, c, var);
  k_sample_scale<<<1, 32, 0, s>>>(var, d, inv_sigma);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_standardise(const void *X, int dtype, int64_t n, int d, int d_pad,
                               const int32_t *rows, const float *c, const float *inv_sigma,
                               __nv_bfloat16 *Xb, float *Xf, cudaStream_t s) {
  const int64_t total = n * d_pad;
  const unsigned grid = (unsigned)ceil_div(total, 256);
  if (dtype == DRPT_DTYPE_U8)
    k_standardise<uint8_t><<<grid, 256, 0, s>>>((const uint8_t *)X, n, d, d_pad, rows, c,
                                                inv_sigma, Xb, Xf);
  else
    k_standardise<float><<<grid, 256, 0, s>>>((const float *)X, n, d, d_pad, rows, c, inv_sigma,
                                              Xb, Xf);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

drpt_status launch_mlp_infer(const __nv_bfloat16 *Xb, int64_t n, int d_pad,
                             const __nv_bfloat16 *W1b, int nmlp, const float *b1, const float *w2,
                             const float *b2, float *P, int *err, cudaStream_t s) {
  if (d_pad % 64 != 0 || d_pad > 256) {
    set_error("learned splits: padded dimension %d unsupported (<= 256)", d_pad);
    return DRPT_ERR_UNSUPPORTED;
  }
  CUtensorMap tmX, tmW;
  DRPT_TRY(bf16_tmap(&tmX, Xb, n, d_pad, kIM));
  DRPT_TRY(bf16_tmap(&tmW, W1b, (int64_t)nmlp * kIN, d_pad, kIN));
  const int kb = d_pad / 64;
  const size_t smem = (size_t)kb * kIM * 128 + (size_t)kIStages * kb * kIN * 128 + 16 * 8 + 1024;
  DRPT_CUDA(cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  k_mlp_infer<<<(unsigned)ceil_div(n, kIM), kIThreads, smem, s>>>(tmX, tmW, n, kb, nmlp, b1, w2,
                                                                  b2, P, err);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt
