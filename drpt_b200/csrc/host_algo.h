// Host-side parts of the path that the reference computes with libstdc++:
// the seeded projection matrix, the positional local split and the locality
// relabelling.  They call the same libstdc++ facilities the reference calls,
// so they reproduce its results bit for bit on the same standard library.
#pragma once

#include <stdint.h>

#include <vector>

namespace drpt {

// d x L row-major sparse Gaussian matrix (math_operations.cpp:48-76).
void host_projection_matrix(uint32_t seed, int d, int L, float density, float *B);

// True when the d x L matrix drawn with `density` = 0 from `seed` is all
// zero (the local matrices, mdrpt.cpp:348-352, whose int density is 0).
bool host_local_matrix_is_zero(uint32_t seed, int d, int L);

// Positional split of a global leaf of `n` points to depth `ld`
// (drpt_local.cpp:49-69 and :121-161 with all-equal keys).  perm[q] is the
// position inside the global leaf of the q-th point in final-leaf order;
// first has 2^ld + 1 entries (leaf starts).
void host_local_permutation(int64_t n, int ld, std::vector<int32_t> &perm,
                            std::vector<int32_t> &first);

// The locality relabelling of the global leaves at one rank and one thread
// (drpt_global.cpp:64-151, 572-732).  order (T x n) and goff (T x (nleaf + 1))
// are every tree's global leaves; slot_leaf[k * T + t] receives the leaf of
// tree t placed at slot k.  Returns false when a slot finds no free leaf
// (the reference then indexes its tables with -1).
bool host_locality_slots(int T, int nleaf, int64_t n, const int32_t *order, const int32_t *goff,
                         int32_t *slot_leaf);

}  // namespace drpt
