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

}  // namespace drpt
