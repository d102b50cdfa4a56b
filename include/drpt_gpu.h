/*
 * drpt_gpu.h -- C ABI of libdrpt_gpu.so, the B200 (sm_100a) k-NN-graph path
 * of DRPT (sparse random projection trees).
 *
 * Plain pointers and sizes only; no C++ or framework types cross this
 * boundary.  Every call returns a drpt_status and never exits or throws;
 * drpt_last_error() describes the last failure on the calling thread.
 *
 * Reference interface each entry point replaces (paths relative to the
 * reference project root):
 *   drpt_build_graph      MDRPT::MDRPT + MDRPT::grow_trees + MDRPT::gather_nns
 *                         (cpp/src/drpt/algo/mdrpt.hpp:102-110, called from
 *                         cpp/src/main.cpp:198-217); the returned lists feed
 *                         the edge-list writer (main.cpp:227-228).
 *   drpt_host_projection  MathOp::build_sparse_projection_matrix
 *                         (cpp/src/drpt/math/math_operations.hpp:24-26).
 *   drpt_project          MathOp::multiply_mat (math_operations.hpp:20-21).
 *   drpt_global_trees     DRPTGlobal::grow_global_tree
 *                         (cpp/src/drpt/algo/drpt_global.hpp:59-62).
 *   drpt_local_leaves     MDRPT::grow_local_trees + DRPTLocal
 *                         (mdrpt.hpp:61-62, drpt_local.hpp:58-69).
 *   drpt_leaf_knn         MDRPT::calculate_nns (mdrpt.hpp:54-55).
 *   drpt_merge_candidates the cross-tree merge of calculate_nns /
 *                         communicate_nns at one rank (mdrpt.hpp:50-52).
 */
#ifndef DRPT_GPU_H
#define DRPT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DRPT_OK = 0,
  DRPT_ERR_INVALID_ARG = 1,         /* bad descriptor field or pointer */
  DRPT_ERR_DEPTH_OUT_OF_RANGE = 2,  /* the reference throws std::out_of_range
                                       (drpt_global.cpp:155-163,
                                       drpt_local.cpp:84-92) */
  DRPT_ERR_EMPTY_LEAF = 3,          /* a global leaf is empty; the reference
                                       throws from DRPTLocal (log2(0)) */
  DRPT_ERR_LOCAL_MATRIX_NONZERO = 4,/* exact mode only: a local projection
                                       matrix is not all zero, so the
                                       positional local split does not hold */
  DRPT_ERR_OOM = 5,
  DRPT_ERR_CUDA = 6,
  DRPT_ERR_TIMEOUT = 7,             /* a bounded device wait gave up */
  DRPT_ERR_UNSUPPORTED = 8
} drpt_status;

typedef enum { DRPT_DTYPE_F32 = 0, DRPT_DTYPE_U8 = 1 } drpt_dtype;

typedef enum {
  /* Reference-exact plain form: the reference's projection matrix, its
   * sequential FP32 node statistics and histogram median, its positional
   * local split and sequential FP32 distances.  Tree assignments are bit-exact
   * with the reference; neighbour lists match it up to exact-distance ties. */
  DRPT_MODE_EXACT = 0,
  /* Plain form with parallel (deterministic, FP64) node statistics; same
   * algorithm otherwise.  Not bit-exact in tree assignment. */
  DRPT_MODE_FAST = 1,
  /* Mixed-precision form: the same global trees (fast statistics), grown to
   * leaves of about `leaf_size` points; every global leaf is brute-forced
   * with BF16 (or FP8-E4M3, `precision`) tensor-core Gram tiles with FP32
   * accumulation, keeping 16 (nn <= 10) or 32 (nn <= 32) candidates per point
   * across the trees; those are re-ranked with FP32 distances and the k-th
   * boundary is checked in FP64.  No positional local split.  nn <= 32,
   * d <= 1024 and a multiple of 4. */
  DRPT_MODE_MIXED = 2,
  /* The mixed form's method in plain FP32: the same global trees and whole
   * global leaves, brute-forced with the exact sequential FP32 distance of
   * the plain form on the CUDA cores (no tensor cores, no re-rank).  The
   * equal-recall FP32 counterpart of DRPT_MODE_MIXED. */
  DRPT_MODE_FP32_LEAF = 3,
  /* The mixed form with its leaf Gram tiles in FP32 on the CUDA cores:
   * ||y||^2 - 2 x.y by fused multiply-adds (one per dimension and pair) over
   * the unstaged rows, the same candidates per point and tree, running list,
   * FP32 re-rank and FP64 boundary check.  The fastest plain FP32
   * counterpart of DRPT_MODE_MIXED.  d a multiple of 8, no learned trees. */
  DRPT_MODE_FP32_GRAM = 4
} drpt_mode;

/* Operand type of the mixed form's tensor-core leaf tiles (FP32 accumulation
 * in both cases). */
typedef enum {
  DRPT_PRECISION_BF16 = 0,      /* centred rows rounded to BF16 */
  DRPT_PRECISION_FP8_E4M3 = 1   /* centred rows scaled per row to the E4M3 range
                                   (scale = max |x - centre| / 448) and rounded */
} drpt_precision;

typedef struct drpt_ctx drpt_ctx;

typedef enum {
  /* The reference's sparse Gaussian matrix in FP32 (every mode). */
  DRPT_PROJECTION_GAUSSIAN = 0,
  /* Its sign (+1 / -1 where it is non-zero, the same sparsity mask) applied
   * to u8 rows as an exact u8 x s8 -> s32 product on the tensor cores
   * (tcgen05.mma kind::i8); d a multiple of 16.  A fast form: the trees are
   * not the reference's and are judged by recall. */
  DRPT_PROJECTION_SIGN = 1
} drpt_projection;

typedef struct {
  int64_t n;                  /* points */
  int32_t d;                  /* dimensions */
  int32_t dtype;              /* drpt_dtype of the input rows */
  int32_t ntrees;             /* -ntrees (main.cpp:61-64) */
  int32_t nn;                 /* -nn (main.cpp:73-76) */
  double tree_depth_ratio;    /* -tree-depth-ratio, default 0.6 (main.cpp:35) */
  int32_t local_tree_offset;  /* -local-tree-offset, default 2 (main.cpp:37) */
  int32_t tree_depth;         /* 0: int(log2(n) - 2) as main.cpp:141-145 */
  double density;             /* 0: 1/sqrt(d) (main.cpp:129-132) */
  uint32_t seed;              /* seed of the global projection matrix */
  const uint32_t *local_seeds;/* ntrees seeds of the local matrices, or NULL
                                 (exact mode then skips the all-zero check) */
  int32_t mode;               /* drpt_mode */
  int32_t data_on_device;     /* 1: `data` is device memory; 0: host memory */
  int32_t out_on_device;      /* 1: outputs are device memory; 0: host */
  void *stream;               /* cudaStream_t to run on; NULL = legacy default */
  int32_t leaf_size;          /* mixed and FP32-leaf modes: target global leaf
                                 size (0 = 512) */
  int32_t precision;          /* mixed mode: drpt_precision of the leaf tiles */
  int32_t learned_trees;      /* mixed mode: how many of the ntrees (the last
                                 ones) split on learned MLP values instead of
                                 random projections (0 = none; d <= 256) */
  int32_t learn_sample;       /* sample points the split MLPs train on
                                 (0 = 8,192; at most 2^20; a sample above
                                 8,192 finds its neighbour pairs in chunks of
                                 at most 8,192 points sorted along a random
                                 direction) */
  int32_t learn_iters;        /* Adam steps per level (0 = 10) */
  int32_t locality;           /* exact and fast modes: 1 runs the locality
                                 relabelling (-locality 1) between the global
                                 and the local trees; at one rank it only
                                 renumbers global leaves, the graph is the same */
  int32_t list_width;         /* mixed mode: candidates kept per point and tree
                                 for the final re-rank, 16 or 32 and >= nn
                                 (0 = 16 for nn <= 10, else 32) */
  int32_t projection;         /* drpt_projection: mixed and FP32 Gram forms may
                                 project u8 rows with the sign matrix */
} drpt_build_desc;

typedef struct {
  int32_t tree_depth;         /* total depth before the local split */
  int32_t global_depth;       /* gd = int(tree_depth * ratio) (mdrpt.cpp:52) */
  int32_t local_depth;        /* ld (mdrpt.cpp:324) */
  int32_t n_global_leaves;    /* 2^(gd-1) per tree */
  int32_t n_final_leaves;     /* 2^(gd-1+ld) per tree */
  int32_t max_final_leaf;     /* largest final leaf */
  int64_t min_global_leaf;    /* smallest non-empty global leaf */
  int64_t sum_leaf_sq;        /* sum over trees and final leaves of m^2 */
  int32_t kernels_launched;   /* device kernels this call launched */
  int32_t reserved;
  float ms_project, ms_global, ms_local, ms_leaf_knn, ms_merge, ms_total;
  /* mixed mode: time of the tensor-core leaf kernels alone (all trees) and
   * of the BF16 staging kernels; padded Gram-tile multiply-adds per call */
  float ms_leaf_mma, ms_leaf_stage;
  int64_t mma_pairs_padded;
  /* learned trees: training time (sample neighbours, all levels) and the
   * mean split loss over trees and levels before and after training */
  float ms_learn, learn_loss_start, learn_loss_end;
  int32_t reserved2;
} drpt_stats;

/* Library version string. */
const char *drpt_version(void);

/* Description of the last failure on the calling thread ("" if none). */
const char *drpt_last_error(void);

/* A context owns the device workspace reused across calls on one device.
 * One host thread at a time per context. */
drpt_status drpt_ctx_create(drpt_ctx **ctx, int device);
void drpt_ctx_destroy(drpt_ctx *ctx);

/* The whole path: projection, global trees, local split, leaf brute force
 * and cross-tree merge.  `data` is n x d row-major (u8 or f32).  Outputs:
 * out_idx (int32, n x nn) and out_dist (float, n x nn, may be NULL): for every
 * point its nn nearest distinct candidates other than itself found in any
 * tree's final leaf, ordered by (distance, index); missing slots hold -1 and
 * +inf.  The reference's edge list (file_writer.cpp:36-184, called with
 * nn-1 at main.cpp:228) is the first nn-1 of them per point. */
drpt_status drpt_build_graph(drpt_ctx *ctx, const drpt_build_desc *desc, const void *data,
                             int32_t *out_idx, float *out_dist, drpt_stats *stats);

/* Many k-NN-graph builds of the same shape from host memory, pipelined (no
 * reference counterpart: the reference reads one dataset, builds and writes
 * its edge list per run, main.cpp:156-233).  desc->mode must be
 * DRPT_MODE_MIXED with host inputs and outputs (data_on_device and
 * out_on_device 0); desc->stream (NULL = legacy default) carries the device
 * work.  Job j reads data[j] (n x d rows) and writes out_idx[j] and, when
 * out_dist and out_dist[j] are not NULL, out_dist[j] (n x nn each), as
 * drpt_build_graph would.  The input copy of job j + 1 and the output copy of
 * job j - 1 run on their own streams while job j builds; pinned host memory
 * lets them overlap.  Returns when every job has finished; stats (may be
 * NULL) gets the kernels launched and, in ms_total, the device time from the
 * first input copy to the last output copy. */
drpt_status drpt_build_graph_stream(drpt_ctx *ctx, const drpt_build_desc *desc, int32_t count,
                                    const void *const *data, int32_t *const *out_idx,
                                    float *const *out_dist, drpt_stats *stats);

/* A batch of independent k-NN-graph builds (no reference counterpart: the
 * reference builds one dataset per process run).  The datasets share d,
 * dtype and the build parameters and lie row-wise one after another in
 * `data`; dataset s is rows [offsets[s], offsets[s+1]). */
typedef struct {
  int32_t nsets;              /* datasets in the batch (1 .. 65536) */
  int32_t d;                  /* dimensions of every dataset */
  int32_t dtype;              /* drpt_dtype */
  int32_t ntrees;
  int32_t nn;
  int32_t mode;               /* DRPT_MODE_MIXED or DRPT_MODE_FP32_LEAF */
  int32_t precision;          /* drpt_precision (mixed mode) */
  int32_t leaf_size;          /* target global leaf size (0 = 512) */
  uint32_t seed;              /* projection seed, the same for every dataset */
  int32_t use_graph;          /* 1: capture the device work of this batch in a
                                 CUDA graph and replay it on later calls with
                                 the same offsets, parameters and pointers
                                 (device pointers only) */
  double density;             /* 0: 1/sqrt(d) */
  int32_t data_on_device;     /* 1: data is device memory */
  int32_t out_on_device;      /* 1: outputs are device memory */
  void *stream;               /* cudaStream_t; NULL = legacy default */
  int32_t list_width;         /* mixed mode: as drpt_build_desc.list_width */
  int32_t reserved;
} drpt_batch_desc;

/* Builds every dataset of the batch together: one projection launch, one
 * launch per kernel and tree level, one leaf-kernel launch per tree and one
 * re-rank launch over all datasets.  Each dataset's graph equals
 * drpt_build_graph's for that dataset alone with the same parameters.
 * `offsets` is a host array of nsets + 1 row offsets (offsets[0] = 0,
 * non-decreasing, every dataset at least 2 rows).  out_idx / out_dist
 * (total rows x nn) hold neighbour ids relative to their dataset's first
 * row. */
drpt_status drpt_build_graph_batched(drpt_ctx *ctx, const drpt_batch_desc *desc,
                                     const int64_t *offsets, const void *data, int32_t *out_idx,
                                     float *out_dist, drpt_stats *stats);

/* Loss and gradient of one learned split (no reference counterpart; the
 * training kernels of the learned trees, one step with learning rate 0).
 * Host arrays: Xs (S x d sample rows), params (64 d + 129 values: W1 64 x d,
 * b1 64, w2 64, b2), node (S: node of every sample point, 0 .. S-1), nbr
 * (S x k sample-local neighbour ids, -1 = none).  Outputs grad (64 d + 129)
 * and *loss.  The weights are rounded to BF16 in the forward pass. */
drpt_status drpt_learn_gradient(drpt_ctx *ctx, const float *Xs, int32_t S, int32_t d,
                                const float *params, const int32_t *node, const int32_t *nbr,
                                int32_t k, float *grad, float *loss);

/* An index: a mixed-form build that keeps its trees for out-of-sample
 * queries (no reference counterpart; the reference stores its node splits,
 * drpt_global.cpp:290 and drpt_local.cpp:142-155, but never reads them).
 * drpt_index_build runs drpt_build_graph (desc->mode must be
 * DRPT_MODE_MIXED, learned trees allowed) and returns its graph and an index
 * holding device copies of the rows, the trees' leaves and node medians and
 * their split functions.  drpt_index_query routes each of nq query rows (d
 * values of the index's dtype, host or device memory) down every tree by the
 * stored medians and returns its k <= 32 nearest points among its leaves'
 * members by exact FP32 distance, ordered by (distance, id), each point
 * once.  The index owns its memory until drpt_index_destroy; one host thread
 * at a time per index.  Query calls keep their scratch in the index, so the
 * device work of two query calls on one index must not overlap, whatever
 * the streams they run on: wait for one call's stream before issuing the
 * next call on another stream (a call that grows the scratch frees the old
 * buffers). */
typedef struct drpt_index drpt_index;
drpt_status drpt_index_build(drpt_ctx *ctx, const drpt_build_desc *desc, const void *data,
                             int32_t *out_idx, float *out_dist, drpt_stats *stats,
                             drpt_index **index);
drpt_status drpt_index_query(drpt_index *index, const void *queries, int64_t nq, int32_t k,
                             int32_t on_device, int32_t *out_idx, float *out_dist, void *stream);
void drpt_index_destroy(drpt_index *index);

/* The reference's sparse Gaussian projection matrix on the host, d x L
 * row-major, from std::mt19937(seed) (math_operations.cpp:48-76). */
drpt_status drpt_host_projection(uint32_t seed, int32_t d, int32_t L, float density, float *B);

/* Kernel-level entry points (device pointers, stream-ordered on `stream`). */

/* P[c][i] = sum_k X[i][k] * B[k][col(c)] for the listed columns, FP32 in
 * ascending k without fused multiply-add; P is column-major (ncols x n). */
drpt_status drpt_project(drpt_ctx *ctx, const void *X, int64_t n, int32_t d, int32_t dtype,
                         const float *B_host, int32_t L, const int32_t *cols_host,
                         int32_t ncols, float *P, void *stream);

/* The sign-matrix projection (no reference counterpart; the fast form of
 * MathOp::multiply_mat for u8 rows): P[c][i] = sum_k X[i][k] * sign(B[k][col(c)])
 * over the non-zero entries, exact in 32-bit integers on the tensor cores
 * (tcgen05.mma kind::i8) and stored as float; X is u8 (n x d, d % 16 == 0)
 * on the device, P column-major (ncols x n).  Synchronises the stream to
 * read the kernel's error flag. */
drpt_status drpt_project_sign(drpt_ctx *ctx, const uint8_t *X, int64_t n, int32_t d,
                              const float *B_host, int32_t L, const int32_t *cols_host,
                              int32_t ncols, float *P, void *stream);

/* Global trees of all T trees from the projected columns P (column t*(gd-1)
 * + level, n values each).  order (T x n): point ids grouped by global leaf in
 * heap order, ascending within a leaf; offsets (T x (2^(gd-1)+1)).  medians
 * (T x (2^(gd-1)-1), heap numbering) may be NULL.  exact != 0 uses the
 * reference's sequential FP32 statistics. */
drpt_status drpt_global_trees(drpt_ctx *ctx, const float *P, int64_t n, int32_t T, int32_t gd,
                              int32_t exact, int32_t *order, int32_t *offsets, float *medians,
                              void *stream);

/* Locality relabelling of the global leaves, one rank and one thread
 * (replaces DRPTGlobal::calculate_tree_leaf_correlation, drpt_global.cpp:572-732,
 * with sortByFreq and select_next_candidate, :64-151).  HOST memory: order and
 * offsets as drpt_global_trees produces them (nleaf = 2^(gd-1));
 * slot_leaf (nleaf x T) receives the leaf of tree t placed at slot k
 * (final_tree_leaf_mapping).  When order_out and offsets_out are not NULL they
 * receive every tree's leaves in slot order (trees_leaf_first_indices_rearrange).
 * No device work.  DRPT_ERR_UNSUPPORTED when a slot finds no free leaf (the
 * reference then reads its tables at index -1). */
drpt_status drpt_locality_slots(const int32_t *order, const int32_t *offsets, int64_t n, int32_t T,
                                int32_t nleaf, int32_t *slot_leaf, int32_t *order_out,
                                int32_t *offsets_out);

/* Positional local split of every global leaf (offsets as produced above) to
 * depth ld.  final_order (T x n), final_offsets (T x (2^(gd-1+ld)+1)). */
drpt_status drpt_local_leaves(drpt_ctx *ctx, const int32_t *order, const int32_t *offsets,
                              int64_t n, int32_t T, int32_t gd, int32_t ld,
                              int32_t *final_order, int32_t *final_offsets, void *stream);

/* Exact FP32 brute force inside every final leaf: for each tree and point the
 * k nearest other members of its leaf by (distance, index).  cand_idx /
 * cand_dist are n x T x k (point-major). */
drpt_status drpt_leaf_knn(drpt_ctx *ctx, const void *X, int32_t dtype, int64_t n, int32_t d,
                          int32_t T, const int32_t *final_order, const int32_t *final_offsets,
                          int32_t n_final, int32_t k, int32_t *cand_idx, float *cand_dist,
                          void *stream);

/* Merge of the T per-tree lists of every point into its k nearest distinct
 * candidates (out_idx / out_dist n x k). */
drpt_status drpt_merge_candidates(drpt_ctx *ctx, const int32_t *cand_idx, const float *cand_dist,
                                  int64_t n, int32_t T, int32_t k, int32_t *out_idx,
                                  float *out_dist, void *stream);

/* drpt_global_trees without any device allocation.  No counterpart in the
 * reference: it is for callers that cannot call cudaMalloc -- hosts whose
 * own pool already holds the device's memory (a cudaMalloc would fail, or
 * force the pool to give memory back and synchronise the device), and
 * latency-bound loops that cannot take cudaMalloc's device-wide
 * synchronisation.  Same arguments, meaning and outputs as
 * drpt_global_trees (no context: it runs on the calling thread's current
 * device, which must be the device of P, the outputs and `stream`).
 *
 * Scratch comes from a 64 MiB array that is part of the library's device
 * image (every GPU that loads the library holds it until exit); `order` and
 * `offsets` double as one side of the level ping-pong.  A build needs about
 * 12*T*n bytes plus per-level tables; larger builds are rejected with
 * DRPT_ERR_INVALID_ARG and a message naming the bytes needed (T*n up to
 * about 5 million).  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture.  Every call shares the array: calls whose kernels overlap on the
 * GPU (other streams, other host threads) race and must be serialised. */
drpt_status drpt_global_trees_noalloc(const float *P, int64_t n, int32_t T, int32_t gd,
                                      int32_t exact, int32_t *order, int32_t *offsets,
                                      float *medians, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DRPT_GPU_H */
