// CPU oracle for the DRPT k-NN-graph path -- test infrastructure only (a
// checker for tests/, smoke() and the CPU-baseline leg of bench.py).
//
// A plain single-threaded restatement of the reference algorithm.  Each
// function cites the reference lines (relative to the reference project
// root) whose arithmetic it reproduces.  Compiled with -ffp-contract=off and
// without -march=native, so every float operation below rounds on its own.
// The libstdc++ calls (std::mt19937, the two distributions, std::nth_element)
// are the same library calls the reference makes; their results define the
// projection matrix and the positional local split.
#include "drpt_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <utility>
#include <vector>

namespace {

constexpr int kBins = 16;  // dist_length = 2*factor*(4+2+1)+2 with 7 bins (math_operations.cpp:228-236)

// Boundaries of the 16-slot histogram (math_operations.cpp:252-288).
void node_bounds(float mu, float sigma, float D[kBins]) {
  for (int i = 0; i < kBins; ++i) D[i] = 0.0f;
  const float step1 = (float)((double)sigma / 30.0);  // sigma / (2*2^4 - 2), double division
  for (int j = 1; j <= 4; ++j) {
    const float rate = (float)j * step1;
    D[6 + j] = mu + rate;
    D[7 - j] = mu - rate;
  }
  const float step2 = (float)((double)sigma / 6.0);  // sigma / (2*2^2 - 2)
  for (int j = 1; j <= 2; ++j) {
    const float rate = sigma + (float)j * step2;
    D[10 + j] = mu + rate;
    D[3 - j] = mu - rate;
  }
  const float step3 = (float)((double)sigma / 2.0);  // sigma / (2*2^1 - 2)
  {
    const float rate = 2.0f * sigma + 1.0f * step3;
    D[13] = mu + rate;
    D[0] = mu - rate;
  }
  // D[14] and D[15] keep the 0 the vector was created with (math_operations.cpp:238).
}

// Counting rule of math_operations.cpp:292-308: slot j (1..15) takes x when
// D[j-1] < x <= D[j]; a value no slot takes goes to slot 0.
int bin_of(const float D[kBins], float x) {
  int slot = 0;
  for (int j = 1; j < kBins; ++j)
    if (D[j - 1] < x && D[j] >= x) slot = j;  // at most one j matches
  return slot;
}

struct NodeResult {
  float mean, var, sigma, median;
  float D[kBins];
  double freq[kBins];
};

// distributed_median with its mean and variance at one rank
// (math_operations.cpp:121-168, 170-206, 208-383).
NodeResult node_median(const float *vals, int64_t n) {
  NodeResult r;
  float sum = 0.0f;
  for (int64_t i = 0; i < n; ++i) sum = sum + vals[i];  // :137-142
  const float mu = sum / (float)(int)n;                  // :164
  float vsum = 0.0f;
  for (int64_t i = 0; i < n; ++i) {                      // :186-192
    const float diff = vals[i] - mu;
    const float sq = diff * diff;
    vsum = vsum + sq;
  }
  const float var = vsum / (float)((int)n - 1);           // :201
  const float sigma = std::sqrt(var);                     // :252
  r.mean = mu;
  r.var = var;
  r.sigma = sigma;
  node_bounds(mu, sigma, r.D);
  for (int j = 0; j < kBins; ++j) r.freq[j] = 0.0;
  for (int64_t i = 0; i < n; ++i) r.freq[bin_of(r.D, vals[i])] += 1.0;
  // Selection (:333-375).  cfreq is a float accumulating double counts.
  float cfreq = 0.0f;
  const float val = (float)(50 * (int)n / 100);
  int sel = -1;
  for (int k = 0; k < kBins; ++k) {
    cfreq = (float)((double)cfreq + r.freq[k]);
    if (cfreq >= val) {
      sel = k;
      break;
    }
  }
  const double count = r.freq[sel];
  // Slot -1 is read when sel == 0: for node i > 0 it is the previous node's
  // D[15] (always 0); for node 0 it is the float before the heap block, the
  // high half of glibc's chunk-size word, 0 for any block below 4 GiB.
  const float lo = sel > 0 ? r.D[sel - 1] : 0.0f;
  const float width = r.D[sel] - lo;  // float subtraction
  const double frac = ((double)((int)n / 2) - ((double)cfreq - count)) / count;
  r.median = (float)((double)lo + frac * (double)width);
  return r;
}

template <typename T>
void project(const T *X, int64_t n, int d, const float *B, int L, float *P) {
  // math_operations.cpp:15-46 through the ordered cblas_sgemm: per output
  // element acc = acc + x*b for k ascending; zero b terms add +-0 and are
  // skipped (exact for finite x).
  std::vector<std::vector<std::pair<int, float>>> nz(L);
  for (int k = 0; k < d; ++k)
    for (int j = 0; j < L; ++j)
      if (B[(int64_t)k * L + j] != 0.0f) nz[j].push_back({k, B[(int64_t)k * L + j]});
  for (int64_t i = 0; i < n; ++i) {
    const T *x = X + i * d;
    for (int j = 0; j < L; ++j) {
      float acc = 0.0f;
      for (const auto &kb : nz[j]) {
        const float prod = (float)x[kb.first] * kb.second;
        acc = acc + prod;
      }
      P[i * L + j] = acc;
    }
  }
}

float distance(const float *p, const float *q, int d) {
  // calculate_distance (math_operations.cpp:385-396): saxpy(-1) gives
  // q - p, snrm2 sums squares in order and takes the square root.
  float s = 0.0f;
  for (int i = 0; i < d; ++i) {
    const float diff = q[i] - p[i];
    const float sq = diff * diff;
    s = s + sq;
  }
  return std::sqrt(s);
}

// drpt_local.cpp:49-59 (leaf sizes) and :61-69 (prefix sums).
void leaf_sizes(int64_t n, int level, int depth, std::vector<int32_t> &out) {
  if (level == depth) {
    out.push_back((int32_t)n);
    return;
  }
  leaf_sizes(n - n / 2, level + 1, depth, out);
  leaf_sizes(n / 2, level + 1, depth, out);
}

// drpt_local.cpp:121-161: nth_element at n/2 on keys that are all equal
// (the local projection is all zero), recursion on [begin, end - n/2) and
// [end - n/2, end).  Only the comparator's results matter to nth_element, and
// every comparison of equal keys is false.
void local_split(std::vector<int32_t>::iterator b, std::vector<int32_t>::iterator e, int depth,
                 int ld) {
  if (depth == ld) return;
  const int64_t sz = e - b;
  std::nth_element(b, b + sz / 2, e, [](int32_t, int32_t) { return false; });
  auto mid = e - sz / 2;
  local_split(b, mid, depth + 1, ld);
  local_split(mid, e, depth + 1, ld);
}

}  // namespace

extern "C" {

void drpt_oracle_projection_matrix(uint32_t seed, int d, int L, float density, float *B) {
  // math_operations.cpp:48-76: row-major over d rows x L columns; a uniform
  // draw above `density` leaves a zero, otherwise a N(0,1) draw is stored.
  std::mt19937 gen(seed);
  std::uniform_real_distribution<float> uni(0, 1);
  std::normal_distribution<float> norm(0, 1);
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < L; ++i) B[i + (int64_t)j * L] = (uni(gen) > density) ? 0.0f : norm(gen);
}

void drpt_oracle_project_f32(const float *X, int64_t n, int d, const float *B, int L, float *P) {
  project(X, n, d, B, L, P);
}

void drpt_oracle_project_u8(const uint8_t *X, int64_t n, int d, const float *B, int L, float *P) {
  project(X, n, d, B, L, P);
}

void drpt_oracle_node_median(const float *vals, int64_t n, float *out4, float *bounds16,
                             double *counts16) {
  NodeResult r = node_median(vals, n);
  if (out4) {
    out4[0] = r.mean;
    out4[1] = r.var;
    out4[2] = r.sigma;
    out4[3] = r.median;
  }
  if (bounds16) std::memcpy(bounds16, r.D, sizeof(r.D));
  if (counts16) std::memcpy(counts16, r.freq, sizeof(r.freq));
}

int drpt_oracle_global_tree(const float *P, int64_t n, int T, int gd, int32_t *order,
                            int32_t *offsets, float *medians) {
  // drpt_global.cpp:153-352 at one rank.  Column t*gd + depth of P holds the
  // value tree t splits on at `depth` (:196-204); nodes keep their points in
  // ascending index order because the partition is stable at one thread.
  if (gd <= 0 || gd > std::log2((double)n) || T <= 0) return -2;  // :155-163
  const int L = T * gd;
  const int nleaf = 1 << (gd - 1);
  for (int t = 0; t < T; ++t) {
    std::vector<std::vector<int32_t>> nodes(1);
    nodes[0].resize(n);
    std::iota(nodes[0].begin(), nodes[0].end(), 0);
    for (int depth = 0; depth < gd - 1; ++depth) {  // :220-224
      std::vector<std::vector<int32_t>> next(nodes.size() * 2);
      for (size_t i = 0; i < nodes.size(); ++i) {
        const std::vector<int32_t> &pts = nodes[i];
        std::vector<float> vals(pts.size());
        for (size_t q = 0; q < pts.size(); ++q) vals[q] = P[(int64_t)pts[q] * L + t * gd + depth];
        const NodeResult r = node_median(vals.data(), (int64_t)vals.size());
        if (medians) medians[(int64_t)t * (nleaf - 1) + ((1 << depth) - 1) + i] = r.median;
        for (size_t q = 0; q < pts.size(); ++q)  // :301-326
          (vals[q] <= r.median ? next[2 * i] : next[2 * i + 1]).push_back(pts[q]);
      }
      nodes.swap(next);
    }
    int64_t pos = 0;
    for (int j = 0; j < nleaf; ++j) {
      if (offsets) offsets[(int64_t)t * (nleaf + 1) + j] = (int32_t)pos;
      for (int32_t p : nodes[j]) {
        if (order) order[(int64_t)t * n + pos] = p;
        ++pos;
      }
    }
    if (offsets) offsets[(int64_t)t * (nleaf + 1) + nleaf] = (int32_t)pos;
  }
  return 0;
}

int drpt_oracle_local_depth(int64_t min_leaf, int nn, int local_tree_offset) {
  // mdrpt.cpp:324: int(log2(min) - (log2(nn) + offset)), double arithmetic.
  return (int)(std::log2((double)(int)min_leaf) - (std::log2((double)nn) + local_tree_offset));
}

int drpt_oracle_local_perm(int64_t n, int ld, int32_t *perm, int32_t *first) {
  if (ld <= 0 || ld > std::log2((double)n)) return -2;  // drpt_local.cpp:84-88
  std::vector<int32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  local_split(idx.begin(), idx.end(), 0, ld);
  std::vector<int32_t> sizes;
  leaf_sizes(n, 0, ld, sizes);
  if (perm) std::copy(idx.begin(), idx.end(), perm);
  if (first) {
    first[0] = 0;
    for (size_t l = 0; l < sizes.size(); ++l) first[l + 1] = first[l] + sizes[l];
  }
  return 0;
}

float drpt_oracle_distance(const float *p, const float *q, int d) { return distance(p, q, d); }

int drpt_oracle_build(const drpt_oracle_desc *desc, const void *X, const uint32_t *local_seeds,
                      drpt_oracle_info *info, int32_t *final_order, int32_t *final_offsets,
                      int32_t *knn_idx, float *knn_dist) {
  if (!desc || !X || desc->n <= 0 || desc->d <= 0 || desc->ntrees <= 0 || desc->nn <= 0)
    return -1;
  const int64_t n = desc->n;
  const int d = desc->d, T = desc->ntrees, nn = desc->nn;
  const double density_d = desc->density == 0 ? 1.0 / std::sqrt((double)d) : desc->density;
  const float density = (float)density_d;                       // grow_trees takes float
  const int tree_depth = (int)(std::log2((double)n) - 2);      // main.cpp:143
  const int gd = (int)(tree_depth * desc->tree_depth_ratio);   // mdrpt.cpp:52
  if (gd <= 0 || gd > std::log2((double)n)) return -2;
  const int L = gd * T;

  std::vector<float> Xf((size_t)n * d);
  if (desc->is_u8) {
    const uint8_t *xu = (const uint8_t *)X;
    for (size_t i = 0; i < Xf.size(); ++i) Xf[i] = (float)xu[i];
  } else {
    std::memcpy(Xf.data(), X, Xf.size() * sizeof(float));
  }
  std::vector<float> B((size_t)d * L), P((size_t)n * L);
  drpt_oracle_projection_matrix(desc->seed, d, L, density, B.data());
  project(Xf.data(), n, d, B.data(), L, P.data());

  const int nleaf = 1 << (gd - 1);
  std::vector<int32_t> gorder((size_t)T * n), goff((size_t)T * (nleaf + 1));
  int st = drpt_oracle_global_tree(P.data(), n, T, gd, gorder.data(), goff.data(), nullptr);
  if (st) return st;

  // Smallest non-empty global leaf over all trees (mdrpt.cpp:293-319).
  int64_t min_leaf = INT32_MAX;
  bool empty_leaf = false;
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < nleaf; ++j) {
      const int64_t sz = goff[(size_t)t * (nleaf + 1) + j + 1] - goff[(size_t)t * (nleaf + 1) + j];
      if (sz == 0) empty_leaf = true;
      else min_leaf = std::min(min_leaf, sz);
    }
  const int ld = drpt_oracle_local_depth(min_leaf, nn, desc->local_tree_offset);
  if (info) {
    info->tree_depth = tree_depth;
    info->global_depth = gd;
    info->local_depth = ld;
    info->n_global_leaves = nleaf;
    info->n_final_leaves = ld > 0 ? nleaf << ld : 0;
    info->min_global_leaf = min_leaf;
  }
  if (ld <= 0) return -2;
  if (empty_leaf) return -3;

  if (local_seeds) {  // mdrpt.cpp:348-352 with density 0 (int parameter)
    std::vector<float> C((size_t)d * ld);
    for (int t = 0; t < T; ++t) {
      drpt_oracle_projection_matrix(local_seeds[t], d, ld, 0.0f, C.data());
      for (float c : C)
        if (c != 0.0f) return -4;
    }
  }

  const int nfinal = nleaf << ld;
  std::vector<int32_t> forder((size_t)T * n), foff((size_t)T * (nfinal + 1));
  for (int t = 0; t < T; ++t) {
    int64_t pos = 0;
    for (int j = 0; j < nleaf; ++j) {
      const int32_t b = goff[(size_t)t * (nleaf + 1) + j];
      const int64_t sz = goff[(size_t)t * (nleaf + 1) + j + 1] - b;
      if (ld > std::log2((double)sz)) return -2;  // drpt_local.cpp:84-88
      std::vector<int32_t> perm(sz), first((1 << ld) + 1);
      drpt_oracle_local_perm(sz, ld, perm.data(), first.data());
      for (int l = 0; l < (1 << ld); ++l) {  // mdrpt.cpp:381-393: id = j*2^ld + l
        foff[(size_t)t * (nfinal + 1) + (size_t)j * (1 << ld) + l] = (int32_t)pos;
        for (int32_t q = first[l]; q < first[l + 1]; ++q)
          forder[(size_t)t * n + pos++] = gorder[(size_t)t * n + b + perm[q]];
      }
    }
    foff[(size_t)t * (nfinal + 1) + nfinal] = (int32_t)pos;
  }
  if (final_order) std::copy(forder.begin(), forder.end(), final_order);
  if (final_offsets)
    for (int t = 0; t < T; ++t)
      std::copy(foff.begin() + (size_t)t * (nfinal + 1), foff.begin() + (size_t)(t + 1) * (nfinal + 1),
                final_offsets + (size_t)t * (nfinal + 1));

  if (knn_idx || knn_dist) {
    // Leaf brute force and cross-tree merge (mdrpt.cpp:123-212).  Per tree a
    // point keeps the first 2*nn of its sorted leaf row; the merged list keeps
    // every distinct candidate.  Its first nn non-self entries are the nn
    // nearest distinct leaf-mates over all trees, which is what is returned
    // here, with ties ordered by index.
    std::vector<std::vector<std::pair<float, int32_t>>> cand(n);
    for (int t = 0; t < T; ++t)
      for (int f = 0; f < nfinal; ++f) {
        const int32_t b = foff[(size_t)t * (nfinal + 1) + f];
        const int32_t e = foff[(size_t)t * (nfinal + 1) + f + 1];
        for (int32_t a = b; a < e; ++a) {
          const int32_t p = forder[(size_t)t * n + a];
          std::vector<std::pair<float, int32_t>> row;
          for (int32_t c = b; c < e; ++c) {
            const int32_t q = forder[(size_t)t * n + c];
            row.push_back({distance(&Xf[(size_t)p * d], &Xf[(size_t)q * d], d), q});
          }
          std::sort(row.begin(), row.end());
          if ((int)row.size() > 2 * nn) row.resize(2 * nn);
          cand[p].insert(cand[p].end(), row.begin(), row.end());
        }
      }
    for (int64_t p = 0; p < n; ++p) {
      auto &c = cand[p];
      std::sort(c.begin(), c.end());
      c.erase(std::unique(c.begin(), c.end(),
                          [](const std::pair<float, int32_t> &x, const std::pair<float, int32_t> &y) {
                            return x.second == y.second;
                          }),
              c.end());
      int w = 0;
      for (const auto &e : c) {
        if (e.second == (int32_t)p) continue;
        if (w == nn) break;
        if (knn_idx) knn_idx[p * nn + w] = e.second;
        if (knn_dist) knn_dist[p * nn + w] = e.first;
        ++w;
      }
      for (; w < nn; ++w) {
        if (knn_idx) knn_idx[p * nn + w] = -1;
        if (knn_dist) knn_dist[p * nn + w] = std::numeric_limits<float>::infinity();
      }
    }
  }
  return 0;
}

}  // extern "C"
