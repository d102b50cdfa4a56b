// Launch wrappers of the device kernels (one .cu file each).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace drpt {

// ---- K1: sparse projection (k_project.cu) -------------------------------
// Column c of P (column-major, ncols x n) is sum over the nonzeros (k, b) of
// B's column, in ascending k, of x[k] * b with one rounding per operation.
struct CscDev {
  const int32_t *colptr;  // ncols + 1 (x column sets with a block table)
  const int32_t *row;     // nnz, ascending within a column
  const float *val;       // nnz
  int32_t ncols;
  // Optional block table (batches): nblocks entries {first point, points
  // (<= project_points_per_block), column set}; column set c uses colptr
  // entries [c * (ncols + 1), (c + 1) * (ncols + 1)).
  const int32_t *blocks = nullptr;
  int32_t nblocks = 0;
};
int project_points_per_block(int d);
drpt_status launch_project(const void *X, int dtype, int64_t n, int d, const CscDev &csc,
                           float *P, cudaStream_t s);

// ---- K2-K4: one global-tree level of all trees (k_tree.cu) ---------------
struct TreeLevelArgs {
  const float *P;          // projected columns, (T*(gd-1)) x n
  int64_t n;
  int T, gd, level;
  const int32_t *ord_in;   // T x n grouped by node (nullptr at level 0: identity)
  const float *val_in;     // T x n, the level's value of ord_in[.] (unused at level 0)
  const int32_t *off_in;   // T x (2^level + 1) (nullptr at level 0: {0, n})
  int32_t *ord_out;        // T x n, grouped by child
  float *val_out;          // T x n, next level's value (nullptr at the last level)
  int32_t *off_out;        // T x (2^(level+1) + 1)
  float *medians;          // T x (2^(gd-1) - 1) heap order, or nullptr
  int exact;               // sequential FP32 statistics
  int p_level0;            // level that reads P directly (0; a batch's root level)
  const int8_t *stop;      // batches: per root slot of level p_level0, the depth
                           // from which its nodes keep all points; nullptr = none
  // scratch (G = T * 2^level nodes, U = tree_level_max_units units)
  int32_t *node_ubase;     // G + 1
  int32_t *unit_node;      // U
  int32_t *unit_lo;        // U
  int32_t *n_units;        // 1
  float *node_D;           // G x 16
  double *unit_s;          // 2U
  unsigned *unit_hist;     // U x 16
  float *node_med;         // G
  int32_t *unit_left;      // U
  int32_t *unit_lbase;     // U
  int32_t *node_nleft;     // G
};
drpt_status launch_tree_level(const TreeLevelArgs &a, int64_t max_units, cudaStream_t s);
int64_t tree_level_max_units(int64_t n, int T, int level);
int tree_level_kernels(int exact);

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
int leaf_knn_exact_kernels();

// ---- K7: cross-tree merge (k_merge.cu) -------------------------------------
// T sorted lists of `lk` entries per point (n x T x lk) -> the k best distinct.
drpt_status launch_merge(const int32_t *cand_idx, const float *cand_dist, int64_t n, int T, int lk,
                         int k, int32_t *out_idx, float *out_dist, cudaStream_t s);

// ---- K8-K11: mixed-precision leaf brute force (k_mixed.cu) ---------------------
struct MixedTreeArgs {
  const void *X;
  int dtype;
  int64_t n;
  int d, d_pad;
  const int32_t *order;      // this tree's global-leaf order (n)
  const int32_t *goff;       // this tree's leaf starts (nleaf + 1)
  int nleaf;
  int T, tree, kp;           // trees, this tree, candidates kept per point
  int fp8;                   // 0: BF16 tiles; 1: E4M3 tiles with per-row scales
  void *Xb;                  // n x d_pad centred rows in leaf order (BF16 or E4M3)
  float *nrm;                // n, squared norms of the rows the tensor cores see
  float *scl;                // n, per-row E4M3 scales (FP8 only)
  int32_t *tile_leaf, *tile_r0, *n_tiles;  // n / 128 + nleaf
  int32_t *cand_idx;         // n x kp running list (point ids), updated tree by tree
  float *cand_dist;          // n x kp approximate squared distances, ascending
  int32_t *tree_idx;         // n x kp: this tree's list (trees after the first),
  float *tree_dist;          // folded into the running list after the leaf kernel
  int *err;                  // set when a bounded wait gave up
};
int mixed_d_pad(int d, int fp8);
// The mixed form's staging of centred rows for the trees t0 .. t0 + tc - 1
// (launch_leaf_means covers every tree; launch_leaf_stage one chunk).
struct LeafStageArgs {
  const void *X;
  int dtype;
  int64_t n;
  int d, d_pad, fp8;
  const int32_t *order, *goff;  // every tree: T x n leaf orders, T x (nleaf + 1) starts
  int nleaf, T;
  int32_t *pos, *lf;            // T x n: each point's row in the tree's leaf order, its leaf
  float *mu;                    // T x nleaf x d leaf centres
  int t0, tc;                   // the chunk
  void *Xb;                     // tc x n x d_pad centred rows, slice t in tree t0 + t's order
  float *nrm, *scl;             // tc x n
};
drpt_status launch_leaf_means(const LeafStageArgs &a, cudaStream_t s);
drpt_status launch_leaf_stage(const LeafStageArgs &a, cudaStream_t s);
// trees per staging chunk: as many as 8 GiB of centred rows hold, at least 1
int mixed_stage_trees(int64_t n, int d_pad, int fp8, int T);
// Batches: ids of point p's neighbours made relative to its dataset's first
// row (set_off: nsets + 1 row offsets, device).
drpt_status launch_localize(int32_t *idx, int64_t n, int k, const int64_t *set_off, int nsets,
                            cudaStream_t s);
drpt_status launch_leaf_mma(const MixedTreeArgs &a, cudaStream_t s);
// K1u (k_project_i8.cu): P (nc x n, column-major) = X (n x d u8) . S^T with S
// (ncp x d signed bytes, ncp = nc rounded up to 16, extra rows zero) on the
// tensor cores in s32; d % 16 == 0, nc <= project_i8_max_cols().
int project_i8_max_cols();
drpt_status launch_project_i8(const uint8_t *X, int64_t n, int d, const int8_t *S, int nc,
                              float *P, int *err, cudaStream_t s);
// Row tiles of `rows` rows of every leaf (tile_leaf, tile_r0, *n_tiles).
drpt_status launch_tile_plan(const int32_t *goff, int nleaf, int rows, int32_t *tile_leaf,
                             int32_t *tile_r0, int32_t *n_tiles, cudaStream_t s);
// Folds a.tree_idx / a.tree_dist (this tree's lists) into the running list.
drpt_status launch_fold_lists(const MixedTreeArgs &a, cudaStream_t s);
// FP32 CUDA-core form of the leaf phase (k_fp32gram.cu): ||x||^2 of every
// row, then per tree the Gram tiles of whole leaves in FP32 (a.X rows, not
// staged) into the running list as launch_leaf_mma does.
drpt_status launch_row_norms(const void *X, int dtype, int64_t n, int d, float *out,
                             cudaStream_t s);
drpt_status launch_leaf_f32(const MixedTreeArgs &a, const float *xnorm, cudaStream_t s);
drpt_status launch_rerank(const void *X, int dtype, int d, const int32_t *visit, int64_t n,
                          const int32_t *cand, int K2, int k, int32_t *out_idx, float *out_dist,
                          cudaStream_t s);


// ---- out-of-sample queries (k_query.cu) ---------------------------------------
drpt_status launch_descend(const float *Pq, int64_t nq, int T, int gd, const float *medians,
                           int32_t *leaf, cudaStream_t s);
drpt_status launch_query(const void *X, int dtype, int d, int64_t n, const void *Qx, int64_t nq,
                         int T, const int32_t *order, const int32_t *goff, int nleaf,
                         const int32_t *leaf, int k, int32_t *oi, float *od, cudaStream_t s);

// ---- learned splits (k_learned.cu) ------------------------------------------
constexpr int kLearnHidden = 64;
constexpr double kLearnEps = 1e-6;  // floor added to a node's variance
// Training state of one level of T learned trees on a sample of S points.
// Node tables hold `nodes` entries per tree (noff: nodes + 1), the level's
// node count.
struct LearnArgs {
  const float *Xs;          // S x d standardised sample rows
  int S, d, T, k;
  int np;                   // parameters per tree: 64 d + 64 + 64 + 1
  float *params, *m1, *m2;  // T x np: W1 (64 x d), b1, w2, b2; Adam moments
  const int32_t *perm;      // T x S: sample ids grouped by node
  const int32_t *noff;      // T x (nodes + 1) node starts in perm
  const int32_t *node_of;   // T x S: node of every sample point
  int nodes;
  const int32_t *nbr;       // S x k sample-local neighbour ids (-1 = none)
  const int32_t *in_ptr, *in_idx;  // reverse pairs (CSR over S)
  const float *inv_pairs;   // T: 1 / (same-node ordered pairs)
  float *A, *f;             // T x S x 64 activations, T x S outputs
  float *mu, *var, *sn, *lterm;  // T x nodes node statistics
  float *g, *sp;            // T x S: dL/df, squared pair sums
  int R;                    // row chunks of the backward pass
  float *part;              // T x R x np partial gradients
};
drpt_status launch_learn_step(const LearnArgs &a, float lr, float bc1, float bc2, float *grad_out,
                              cudaStream_t s);
int learn_step_kernels();
drpt_status launch_learn_init(const LearnArgs &a, uint64_t seed, int level, cudaStream_t s);
drpt_status launch_learn_pairs(const LearnArgs &a, int *cnt, cudaStream_t s);
drpt_status launch_learn_loss(const LearnArgs &a, float *acc, int slot, cudaStream_t s);
drpt_status launch_gather_f(const LearnArgs &a, float *fp, cudaStream_t s);
drpt_status launch_node_label(const int32_t *perm, const int32_t *noff, int nodes, int S, int T,
                              int32_t *node_of, cudaStream_t s);
drpt_status launch_stack(const LearnArgs &a, int d_pad, int levels, int level,
                         __nv_bfloat16 *W1b, float *b1, float *w2, float *b2, cudaStream_t s);
drpt_status launch_sample_scale(const float *Xr, int S, int d, float *c, double *var,
                                float *inv_sigma, cudaStream_t s);
drpt_status launch_standardise(const void *X, int dtype, int64_t n, int d, int d_pad,
                               const int32_t *rows, const float *c, const float *inv_sigma,
                               __nv_bfloat16 *Xb, float *Xf, cudaStream_t s);
drpt_status launch_mlp_infer(const __nv_bfloat16 *Xb, int64_t n, int d_pad,
                             const __nv_bfloat16 *W1b, int nmlp, const float *b1, const float *w2,
                             const float *b2, float *P, int *err, cudaStream_t s);

}  // namespace drpt
