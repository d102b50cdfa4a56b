/*
 * CPU oracle for the DRPT k-NN-graph path: a plain, single-threaded
 * restatement of the reference algorithm, used ONLY as a checker by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg.  The product
 * (libdrpt_gpu.so) never links or calls it.
 *
 * Every function names the reference lines it follows (paths relative to the
 * reference project root).  Parity of this restatement is pinned against the
 * reference itself, built from its own sources by `make -C oracle ref`
 * (golden fixtures in tests/golden/).
 */
#ifndef DRPT_ORACLE_H
#define DRPT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Sparse Gaussian projection matrix, d x L row-major
 * (cpp/src/drpt/math/math_operations.cpp:48-76). */
void drpt_oracle_projection_matrix(uint32_t seed, int d, int L, float density, float *B);

/* P = X.B, n x L row-major, sequential-k FP32 order of the ordered cblas
 * (math_operations.cpp:15-46). X is n x d row-major (f32 or u8). */
void drpt_oracle_project_f32(const float *X, int64_t n, int d, const float *B, int L, float *P);
void drpt_oracle_project_u8(const uint8_t *X, int64_t n, int d, const float *B, int L, float *P);

/* Histogram median of one node's values in list order
 * (math_operations.cpp:121-383).  out4 = {mean, variance, sigma, median};
 * bounds16 = the 16 bin boundaries; counts16 = the 16 bin counts. */
void drpt_oracle_node_median(const float *vals, int64_t n, float *out4, float *bounds16,
                             double *counts16);

/* Global tree of every tree (drpt_global.cpp:153-352).  P is n x (T*gd).
 * order[t*n + p]: point ids grouped by global leaf (heap order), ascending
 * within a leaf; offsets[t*(nleaf+1) + j]: start of leaf j, nleaf = 2^(gd-1).
 * medians[t*(2^(gd-1)-1) + node] (heap numbering) may be NULL. */
int drpt_oracle_global_tree(const float *P, int64_t n, int T, int gd, int32_t *order,
                            int32_t *offsets, float *medians);

/* Local depth from the smallest non-empty global leaf (mdrpt.cpp:324). */
int drpt_oracle_local_depth(int64_t min_leaf, int nn, int local_tree_offset);

/* Positional local split of a global leaf of size n to depth ld
 * (drpt_local.cpp:49-180 with the all-zero local projection,
 * mdrpt.cpp:343-393).  perm[q]: position inside the global leaf of the q-th
 * member in final-leaf order; first[l]: start of local leaf l (2^ld + 1). */
int drpt_oracle_local_perm(int64_t n, int ld, int32_t *perm, int32_t *first);

/* Euclidean distance sqrt(sum (q_i - p_i)^2), sequential FP32
 * (math_operations.cpp:385-396 with the ordered saxpy/snrm2). */
float drpt_oracle_distance(const float *p, const float *q, int d);

typedef struct {
  int64_t n;
  int d;
  int is_u8;                  /* 1: X is uint8, 0: float32 */
  int ntrees;
  int nn;
  double tree_depth_ratio;    /* default 0.6 (main.cpp:35) */
  int local_tree_offset;      /* default 2 (main.cpp:37) */
  double density;             /* 0 -> 1/sqrt(d) (main.cpp:129-132) */
  uint32_t seed;              /* global projection seed (mdrpt.cpp:55) */
} drpt_oracle_desc;

typedef struct {
  int tree_depth;             /* int(log2(n) - 2) (main.cpp:141-145) */
  int global_depth;           /* gd = int(tree_depth * ratio) (mdrpt.cpp:52) */
  int local_depth;            /* ld (mdrpt.cpp:324) */
  int n_global_leaves;        /* 2^(gd-1) */
  int n_final_leaves;         /* 2^(gd-1+ld) */
  int64_t min_global_leaf;
} drpt_oracle_info;

/* Whole path: projection, global trees, positional local split and the
 * leaf brute force with the cross-tree merge (mdrpt.cpp:46-212, 273-291).
 * Outputs (any may be NULL):
 *   final_order   T*n      point ids grouped by final leaf (leaf id order)
 *   final_offsets T*(n+1)  capacity; row t holds n_final+1 leaf starts at
 *                          stride n_final+1
 *   knn_idx/knn_dist n*nn  each point's nn nearest distinct non-self
 *                          candidates ordered by (distance, index); -1/+inf pad.
 * local_seeds (ntrees values, may be NULL) are the seeds of the local
 * matrices (mdrpt.cpp:341); when given, every local matrix is regenerated and
 * must be all zero, as the positional split assumes.
 * Returns 0 or a negative status:
 *   -1 invalid argument, -2 depth out of range (the reference throws
 *   std::out_of_range, drpt_global.cpp:155-163, drpt_local.cpp:84-92),
 *   -3 empty global leaf (the same throw, reached through log2(0)),
 *   -4 a local matrix is not all zero. */
int drpt_oracle_build(const drpt_oracle_desc *desc, const void *X, const uint32_t *local_seeds,
                      drpt_oracle_info *info, int32_t *final_order, int32_t *final_offsets,
                      int32_t *knn_idx, float *knn_dist);

#ifdef __cplusplus
}
#endif

#endif
