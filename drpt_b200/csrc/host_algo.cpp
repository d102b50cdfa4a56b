// Host-side, libstdc++-defined parts of the DRPT path (see host_algo.h).
#include "host_algo.h"

#include <algorithm>
#include <numeric>
#include <random>

namespace drpt {

void host_projection_matrix(uint32_t seed, int d, int L, float density, float *B) {
  // Row-major over d rows and L columns; one uniform draw per entry, and a
  // normal draw only for the entries the uniform draw keeps.
  std::mt19937 gen(seed);
  std::uniform_real_distribution<float> keep(0, 1);
  std::normal_distribution<float> gauss(0, 1);
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < L; ++c) {
      const float u = keep(gen);
      B[(int64_t)r * L + c] = (u > density) ? 0.0f : gauss(gen);
    }
}

bool host_local_matrix_is_zero(uint32_t seed, int d, int L) {
  std::mt19937 gen(seed);
  std::uniform_real_distribution<float> keep(0, 1);
  std::normal_distribution<float> gauss(0, 1);
  for (int64_t e = 0; e < (int64_t)d * L; ++e) {
    const float u = keep(gen);
    if (!(u > 0.0f)) {
      if (gauss(gen) != 0.0f) return false;
    }
  }
  return true;
}

namespace {

void split_range(std::vector<int32_t>::iterator b, std::vector<int32_t>::iterator e, int depth,
                 int ld) {
  if (depth == ld) return;
  const int64_t size = e - b;
  // All local keys are zero, so the reference's `<` comparator is false for
  // every pair; nth_element's permutation then depends on the size only.
  std::nth_element(b, b + size / 2, e, [](int32_t, int32_t) { return false; });
  const auto mid = e - size / 2;  // left half keeps ceil(size / 2)
  split_range(b, mid, depth + 1, ld);
  split_range(mid, e, depth + 1, ld);
}

void sizes_rec(int64_t n, int level, int ld, std::vector<int32_t> &out) {
  if (level == ld) {
    out.push_back((int32_t)n);
    return;
  }
  sizes_rec(n - n / 2, level + 1, ld, out);
  sizes_rec(n / 2, level + 1, ld, out);
}

}  // namespace

void host_local_permutation(int64_t n, int ld, std::vector<int32_t> &perm,
                            std::vector<int32_t> &first) {
  perm.resize(n);
  std::iota(perm.begin(), perm.end(), 0);
  split_range(perm.begin(), perm.end(), 0, ld);
  std::vector<int32_t> sizes;
  sizes.reserve((size_t)1 << ld);
  sizes_rec(n, 0, ld, sizes);
  first.assign(sizes.size() + 1, 0);
  for (size_t l = 0; l < sizes.size(); ++l) first[l + 1] = first[l] + sizes[l];
}

namespace {

// The reference's candidate record (drpt_global.hpp:17-20): the same field
// order, so that std::sort sees the same sequence of comparisons and moves.
struct PriorityMap {
  int leaf_index;
  float priority;
};

}  // namespace

bool host_locality_slots(int T, int nleaf, int64_t n, const int32_t *order, const int32_t *goff,
                         int32_t *slot_leaf) {
  // every point's leaf in every tree (index_to_tree_leaf_mapper,
  // drpt_global.cpp:314, 323)
  std::vector<int32_t> leaf_of((size_t)n * T, 0);
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < nleaf; ++j)
      for (int32_t i = goff[(size_t)t * (nleaf + 1) + j]; i < goff[(size_t)t * (nleaf + 1) + j + 1];
           ++i)
        leaf_of[(size_t)order[(size_t)t * n + i] * T + t] = j;
  // sel[(tree * nleaf + leaf) * T + c]: the first leaf of tree c holding the
  // largest share (count / size * 100, in float) of the points of `leaf` of
  // `tree` (drpt_global.cpp:607-652)
  std::vector<int32_t> sel((size_t)T * nleaf * T);
  std::vector<float> cnt((size_t)T * nleaf);
  for (int tree = 0; tree < T; ++tree)
    for (int leaf = 0; leaf < nleaf; ++leaf) {
      std::fill(cnt.begin(), cnt.end(), 0.0f);
      const int32_t lo = goff[(size_t)tree * (nleaf + 1) + leaf];
      const int32_t hi = goff[(size_t)tree * (nleaf + 1) + leaf + 1];
      const int size = hi - lo;
      for (int32_t i = lo; i < hi; ++i) {
        const int32_t p = order[(size_t)tree * n + i];
        for (int j = 0; j < T; ++j) cnt[(size_t)j * nleaf + leaf_of[(size_t)p * T + j]] += 1.0f;
      }
      for (int c = 0; c < T; ++c) {
        const float *x = cnt.data() + (size_t)c * nleaf;
        int best = 0;
        float bv = (x[0] / size) * 100;
        for (int l = 1; l < nleaf; ++l) {  // std::max_element: the first largest
          const float v = (x[l] / size) * 100;
          if (bv < v) {
            bv = v;
            best = l;
          }
        }
        sel[((size_t)tree * nleaf + leaf) * T + c] = best;
      }
    }
  // At one rank every candidate list holds one leaf at priority 1 (its
  // frequency among the ranks, sortByFreq) and the others at 0
  // (drpt_global.cpp:667-688).
  auto candidates = [&](int tree, int leaf, int m, std::vector<PriorityMap> &v) {
    v.resize(nleaf);
    const int s = sel[((size_t)tree * nleaf + leaf) * T + m];
    for (int q = 0; q < nleaf; ++q) v[q] = PriorityMap{q, q == s ? 1.0f : 0.0f};
  };
  // slots in ascending order, trees in order: the leaf of tree m at slot k
  // follows the leaf chosen for slot k in tree m - 1 (select_next_candidate,
  // drpt_global.cpp:104-151, and the loop at :690-699)
  std::vector<uint8_t> taken((size_t)T * nleaf, 0);  // leaf of tree m used by a lower slot
  std::vector<int32_t> zero_sel((size_t)T * T, 0);   // leaves of tree cur choosing leaf 0 of m
  for (int cur = 0; cur < T; ++cur)
    for (int j = 0; j < nleaf; ++j)
      for (int m = 0; m < T; ++m)
        if (sel[((size_t)cur * nleaf + j) * T + m] == 0) ++zero_sel[(size_t)cur * T + m];
  std::vector<PriorityMap> vec;
  for (int k = 0; k < nleaf; ++k) {
    int prev = k;
    for (int m = 0; m < T; ++m) {
      const int cur = m == 0 ? 0 : m - 1;
      // the sorted list starts with its one priority-1 leaf: when that leaf
      // is free it is the choice and the order of the rest does not matter
      const int top = sel[((size_t)cur * nleaf + prev) * T + m];
      if (!taken[(size_t)m * nleaf + top]) {
        slot_leaf[(size_t)k * T + m] = top;
        taken[(size_t)m * nleaf + top] = 1;
        prev = top;
        continue;
      }
      candidates(cur, prev, m, vec);
      std::sort(vec.begin(), vec.end(), [](const PriorityMap &lhs, const PriorityMap &rhs) {
        if (lhs.priority > rhs.priority) return true;
        return false;
      });
      int chosen = -1;
      for (const PriorityMap &can : vec) {
        const int id = can.leaf_index;
        if (taken[(size_t)m * nleaf + id]) continue;
        // another leaf j != prev of tree cur whose candidate list starts with
        // a higher-priority entry for the same leaf: only entry 0 is looked
        // at, which is leaf 0 with priority 1 exactly when j chose leaf 0
        if (id == 0 && can.priority < 1.0f) {
          const int others = zero_sel[(size_t)cur * T + m] -
                             (sel[((size_t)cur * nleaf + prev) * T + m] == 0 ? 1 : 0);
          if (others > 0) continue;
        }
        chosen = id;
        break;
      }
      if (chosen < 0) return false;
      slot_leaf[(size_t)k * T + m] = chosen;
      taken[(size_t)m * nleaf + chosen] = 1;
      prev = chosen;
    }
  }
  return true;
}

}  // namespace drpt
