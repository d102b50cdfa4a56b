// Launch wrappers of the device kernels (one .cu file each).
#pragma once

#include "common.cuh"

namespace drpt {

// ---- K1: sparse projection (k_project.cu) -------------------------------
// Column c of P (column-major, ncols x n) is sum over the nonzeros (k, b) of
// B's column, in ascending k, of x[k] * b with one rounding per operation.
struct CscDev {
  const int32_t *colptr;  // ncols + 1
  const int32_t *row;     // nnz, ascending within a column
  const float *val;       // nnz
  int32_t ncols;
};
drpt_status launch_project(const void *X, int dtype, int64_t n, int d, const CscDev &csc,
                           float *P, cudaStream_t s);

// ---- K2-K4: one global-tree level of all trees (k_tree.cu) ---------------
struct LevelArgs {
  const float *P;          // projected columns, (T*(gd-1)) x n
  int64_t n;
  int T, gd, level;
  const int32_t *ord_in;   // T x n, grouped by node, ascending within a node
  const float *val_in;     // T x n, the level's value of ord_in[.]
  const int32_t *off_in;   // T x (2^level + 1)
  int32_t *ord_out;        // T x n, grouped by child
  float *val_out;          // T x n, next level's value (unused at the last level)
  int32_t *off_out;        // T x (2^(level+1) + 1)
  float *medians;          // T x (2^(gd-1) - 1) heap order, or nullptr
  int exact;               // sequential FP32 statistics
};
drpt_status launch_level(const LevelArgs &a, cudaStream_t s);
// val_out[t][i] = P[t*(gd-1)][i], ord_out[t][i] = i, off[t] = {0, n}
drpt_status launch_tree_init(const float *P, int64_t n, int T, int gd, int32_t *ord,
                             float *val, int32_t *off, cudaStream_t s);

// ---- K5: positional local split (k_local.cu) ------------------------------
struct LocalArgs {
  const int32_t *order;        // T x n global-leaf order
  const int32_t *goff;         // T x (nleaf + 1)
  const int64_t *perm_base;    // T x nleaf: offset of the leaf's permutation
  const int64_t *first_base;   // T x nleaf: offset of the leaf's 2^ld+1 starts
  const int32_t *pool;         // permutations and leaf starts
  int64_t n;
  int T, nleaf, ld;
  int32_t *final_order;        // T x n
  int32_t *final_off;          // T x (nleaf * 2^ld + 1)
};
drpt_status launch_local(const LocalArgs &a, cudaStream_t s);

// ---- K6: exact leaf brute force (k_leafknn.cu) -----------------------------
struct LeafKnnArgs {
  const void *X;
  int dtype;
  int64_t n;
  int d, T, k;
  const int32_t *final_order;  // T x n
  const int32_t *final_off;    // T x (n_final + 1)
  int n_final;
  int32_t *cand_idx;           // n x T x k
  float *cand_dist;            // n x T x k
};
drpt_status launch_leaf_knn_exact(const LeafKnnArgs &a, cudaStream_t s);

// ---- K7: cross-tree merge (k_merge.cu) -------------------------------------
drpt_status launch_merge(const int32_t *cand_idx, const float *cand_dist, int64_t n, int T, int k,
                         int32_t *out_idx, float *out_dist, cudaStream_t s);

}  // namespace drpt
