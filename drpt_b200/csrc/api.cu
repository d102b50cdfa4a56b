// C ABI of libdrpt_gpu.so and the host orchestration of the k-NN-graph path
// (MDRPT::grow_trees + MDRPT::gather_nns, mdrpt.cpp:46-121, 273-291).
//
// Data layout in HBM for n points, T trees, global depth gd:
//   X            n x d row-major (f32 or u8), read by K1 and gathered by K6
//   P            (T*(gd-1)) x n column-major: the split value of every point
//                for tree t at level l is column t*(gd-1)+l (the reference
//                computes gd columns per tree and never splits on the last)
//   ord / val    T x n ping-pong: point ids grouped by node, and their values
//   off          T x (nodes+1) node starts per level
//   final_order  T x n point ids grouped by final leaf, final_off leaf starts
//   cand         n x T x nn per-tree nearest lists (dist f32 + idx i32)
//   out          n x nn merged lists
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <utility>
#include <vector>

#include "host_algo.h"
#include "kernels.cuh"

struct drpt_ctx {
  int device = 0;
  struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
  };
  std::map<std::string, Buf> bufs;
  std::map<std::pair<int64_t, int>, std::pair<std::vector<int32_t>, std::vector<int32_t>>> perms;
  cudaEvent_t ev[8] = {};
  std::vector<cudaEvent_t> tev;  // event pool of the mixed form's leaf phase
  // (start, end) indices into tev of its staging and tensor-core spans
  std::vector<std::pair<int, int>> tstage, tmma;
  int launches = 0;
  uint64_t ws_gen = 0;           // bumped whenever a workspace buffer moves
  // batches: the captured device work of the last graph-mode batch
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t gstream = nullptr;  // captures and replays (the legacy stream cannot capture)
  std::string gkey;
  uint64_t gexec_gen = 0;
  int glaunches = 0;
};

// A built mixed-form index kept for out-of-sample queries: its own copies of
// the rows, every tree's leaf order, leaf starts and node medians, and the
// split functions (the random trees' projection columns as CSC, the learned
// trees' MLPs and standardisation).  Device memory owned by the index.
struct drpt_index {
  int device = 0;
  int64_t n = 0;
  int d = 0, dtype = 0, T = 0, gd = 0, nleaf = 0, Tr = 0, Tl = 0, d_pad = 0;
  void *X = nullptr;
  int32_t *order = nullptr, *goff = nullptr;
  float *medians = nullptr;
  int32_t *csc_col = nullptr, *csc_row = nullptr;
  float *csc_val = nullptr;
  int ncols_r = 0;
  __nv_bfloat16 *w1b = nullptr;
  float *b1 = nullptr, *w2 = nullptr, *b2 = nullptr, *c = nullptr, *inv_sigma = nullptr;
  // query scratch, grown on demand
  int64_t cap = 0;
  float *Pq = nullptr;
  int32_t *leaf = nullptr, *qi = nullptr;
  float *qd = nullptr;
  void *qx = nullptr;
  __nv_bfloat16 *qxb = nullptr;
  int *err = nullptr;
};

namespace drpt {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int device_sm_count() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (dev >= 0 && dev < 64) {
    const int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
    return 148;
  if (dev >= 0 && dev < 64) cache[dev].store(sms, std::memory_order_relaxed);
  return sms;
}

namespace {

template <typename T>
drpt_status ws_get(drpt_ctx *c, const char *name, size_t count, T **out) {
  const size_t bytes = std::max<size_t>(count * sizeof(T), 256);
  drpt_ctx::Buf &b = c->bufs[name];
  if (b.bytes < bytes) {
    if (b.p) DRPT_CUDA(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
      b.p = nullptr;
      set_error("cudaMalloc(%zu) for %s: %s", bytes, name, cudaGetErrorString(e));
      return DRPT_ERR_OOM;
    }
    b.bytes = bytes;
    ++c->ws_gen;
  }
  *out = (T *)b.p;
  return DRPT_OK;
}

struct Geometry {
  int td, gd, nleaf;
};

drpt_status geometry(int64_t n, int tree_depth, double ratio, Geometry *g) {
  g->td = tree_depth > 0 ? tree_depth : (int)(std::log2((double)n) - 2);  // main.cpp:143
  g->gd = (int)(g->td * ratio);                                          // mdrpt.cpp:52
  if (g->gd <= 0 || g->gd > std::log2((double)n)) {                       // drpt_global.cpp:155-158
    set_error("global tree depth %d outside [1, log2(%lld)]", g->gd, (long long)n);
    return DRPT_ERR_DEPTH_OUT_OF_RANGE;
  }
  if (g->gd > 30) {
    set_error("global tree depth %d too large", g->gd);
    return DRPT_ERR_UNSUPPORTED;
  }
  g->nleaf = 1 << (g->gd - 1);
  return DRPT_OK;
}

// K1 with the CSC of the used columns of B built on the host.
// `tag` names the workspace buffers of the CSC ("csc": the build's own,
// which an index keeps).
drpt_status project_cols(drpt_ctx *c, const void *X, int dtype, int64_t n, int d, const float *B,
                         int L, const std::vector<int32_t> &cols, float *P, cudaStream_t s,
                         int *nnz_out = nullptr, const char *tag = "csc") {
  const int ncols = (int)cols.size();
  std::vector<int32_t> colptr(ncols + 1, 0), row;
  std::vector<float> val;
  for (int q = 0; q < ncols; ++q) {
    for (int k = 0; k < d; ++k) {
      const float b = B[(int64_t)k * L + cols[q]];
      if (b != 0.0f) {
        row.push_back(k);
        val.push_back(b);
      }
    }
    colptr[q + 1] = (int32_t)row.size();
  }
  int32_t *dcol, *drow;
  float *dval;
  const std::string t(tag);
  DRPT_TRY(ws_get(c, (t + "_colptr").c_str(), colptr.size(), &dcol));
  DRPT_TRY(ws_get(c, (t + "_row").c_str(), std::max<size_t>(row.size(), 1), &drow));
  DRPT_TRY(ws_get(c, (t + "_val").c_str(), std::max<size_t>(val.size(), 1), &dval));
  // Pageable sources: the copies complete before these calls return.
  DRPT_CUDA(cudaMemcpyAsync(dcol, colptr.data(), colptr.size() * 4, cudaMemcpyHostToDevice, s));
  if (!row.empty()) {
    DRPT_CUDA(cudaMemcpyAsync(drow, row.data(), row.size() * 4, cudaMemcpyHostToDevice, s));
    DRPT_CUDA(cudaMemcpyAsync(dval, val.data(), val.size() * 4, cudaMemcpyHostToDevice, s));
  }
  if (nnz_out) *nnz_out = (int)row.size();
  CscDev csc{dcol, drow, dval, ncols};
  DRPT_TRY(launch_project(X, dtype, n, d, csc, P, s));
  c->launches += 1;
  return DRPT_OK;
}

// The sign-matrix projection of u8 rows (K1u, a fast form): S = sign of the
// projection matrix's selected columns (the same sparsity mask), P = X.S^T
// exactly in integers on the tensor cores, at most project_i8_max_cols()
// columns per launch.  Also leaves the signs as the CSC an index keeps
// (csc_*), so that out-of-sample queries project the same way.
drpt_status project_sign(drpt_ctx *c, const void *X, int64_t n, int d, const float *B, int L,
                         const std::vector<int32_t> &cols, float *P, cudaStream_t s,
                         int *nnz_out = nullptr) {
  const int ncols = (int)cols.size();
  if (d % 16 != 0) {
    set_error("the sign-matrix projection needs d %% 16 == 0 (got %d)", d);
    return DRPT_ERR_UNSUPPORTED;
  }
  const int per = project_i8_max_cols();
  std::vector<int32_t> colptr(ncols + 1, 0), row;
  std::vector<float> val;
  const int groups = (ncols + per - 1) / per;
  std::vector<int8_t> S((size_t)groups * per * d, 0);  // per group: `per` rows of d signs
  for (int q = 0; q < ncols; ++q) {
    int8_t *srow = S.data() + ((size_t)(q / per) * per + q % per) * d;
    for (int k = 0; k < d; ++k) {
      const float b = B[(int64_t)k * L + cols[q]];
      if (b != 0.0f) {
        const int8_t sg = b > 0.0f ? 1 : -1;
        srow[k] = sg;
        row.push_back(k);
        val.push_back((float)sg);
      }
    }
    colptr[q + 1] = (int32_t)row.size();
  }
  int32_t *dcol, *drow;
  float *dval;
  int8_t *dS;
  int *err;
  DRPT_TRY(ws_get(c, "csc_colptr", colptr.size(), &dcol));
  DRPT_TRY(ws_get(c, "csc_row", std::max<size_t>(row.size(), 1), &drow));
  DRPT_TRY(ws_get(c, "csc_val", std::max<size_t>(val.size(), 1), &dval));
  DRPT_TRY(ws_get(c, "sgn_S", S.size(), &dS));
  DRPT_TRY(ws_get(c, "sgn_err", 1, &err));
  // Pageable sources: the copies complete before these calls return.
  DRPT_CUDA(cudaMemcpyAsync(dcol, colptr.data(), colptr.size() * 4, cudaMemcpyHostToDevice, s));
  if (!row.empty()) {
    DRPT_CUDA(cudaMemcpyAsync(drow, row.data(), row.size() * 4, cudaMemcpyHostToDevice, s));
    DRPT_CUDA(cudaMemcpyAsync(dval, val.data(), val.size() * 4, cudaMemcpyHostToDevice, s));
  }
  DRPT_CUDA(cudaMemcpyAsync(dS, S.data(), S.size(), cudaMemcpyHostToDevice, s));
  DRPT_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  if (nnz_out) *nnz_out = (int)row.size();
  for (int g = 0; g < groups; ++g) {
    const int nc = std::min(per, ncols - g * per);
    DRPT_TRY(launch_project_i8(static_cast<const uint8_t *>(X), n, d, dS + (size_t)g * per * d,
                               nc, P + (size_t)g * per * n, err, s));
    c->launches += 1;
  }
  return DRPT_OK;
}

// Global trees of all T trees; returns pointers to the final order/offsets
// (inside the workspace).
drpt_status global_trees(drpt_ctx *c, const float *P, int64_t n, int T, int gd, int exact,
                         float *medians, int32_t **order_out, int32_t **off_out, cudaStream_t s) {
  const int nleaf = 1 << (gd - 1);
  int32_t *ord[2], *off[2];
  float *val[2];
  DRPT_TRY(ws_get(c, "ord_a", (size_t)T * n, &ord[0]));
  DRPT_TRY(ws_get(c, "ord_b", (size_t)T * n, &ord[1]));
  DRPT_TRY(ws_get(c, "val_a", (size_t)T * n, &val[0]));
  DRPT_TRY(ws_get(c, "val_b", (size_t)T * n, &val[1]));
  DRPT_TRY(ws_get(c, "off_a", (size_t)T * (nleaf + 1), &off[0]));
  DRPT_TRY(ws_get(c, "off_b", (size_t)T * (nleaf + 1), &off[1]));
  if (gd == 1) {
    // One global leaf holding every point in index order.
    std::vector<int32_t> iota(n), o(2 * T);
    for (int64_t i = 0; i < n; ++i) iota[i] = (int32_t)i;
    for (int t = 0; t < T; ++t) {
      o[2 * t] = 0;
      o[2 * t + 1] = (int32_t)n;
      DRPT_CUDA(cudaMemcpyAsync(ord[0] + (size_t)t * n, iota.data(), n * 4, cudaMemcpyHostToDevice, s));
    }
    DRPT_CUDA(cudaMemcpyAsync(off[0], o.data(), o.size() * 4, cudaMemcpyHostToDevice, s));
    *order_out = ord[0];
    *off_out = off[0];
    return DRPT_OK;
  }
  // level scratch, sized for the deepest level
  const int last = gd - 2;
  const int64_t Gmax = (int64_t)T << last;
  const int64_t Umax = tree_level_max_units(n, T, last);
  TreeLevelArgs a{};
  DRPT_TRY(ws_get(c, "lv_node_ubase", Gmax + 1, &a.node_ubase));
  DRPT_TRY(ws_get(c, "lv_unit_node", Umax, &a.unit_node));
  DRPT_TRY(ws_get(c, "lv_unit_lo", Umax, &a.unit_lo));
  DRPT_TRY(ws_get(c, "lv_n_units", 1, &a.n_units));
  DRPT_TRY(ws_get(c, "lv_node_D", Gmax * kBins, &a.node_D));
  DRPT_TRY(ws_get(c, "lv_unit_s", 2 * Umax, &a.unit_s));
  DRPT_TRY(ws_get(c, "lv_unit_hist", Umax * kBins, &a.unit_hist));
  DRPT_TRY(ws_get(c, "lv_node_med", Gmax, &a.node_med));
  DRPT_TRY(ws_get(c, "lv_unit_left", Umax, &a.unit_left));
  DRPT_TRY(ws_get(c, "lv_unit_lbase", Umax, &a.unit_lbase));
  DRPT_TRY(ws_get(c, "lv_node_nleft", Gmax, &a.node_nleft));
  int cur = 0;
  for (int level = 0; level < gd - 1; ++level) {
    a.P = P;
    a.n = n;
    a.T = T;
    a.gd = gd;
    a.level = level;
    a.ord_in = level == 0 ? nullptr : ord[cur];
    a.val_in = level == 0 ? nullptr : val[cur];
    a.off_in = level == 0 ? nullptr : off[cur];
    a.ord_out = ord[cur ^ 1];
    a.val_out = level + 1 < gd - 1 ? val[cur ^ 1] : nullptr;
    a.off_out = off[cur ^ 1];
    a.medians = medians;
    a.exact = exact;
    DRPT_TRY(launch_tree_level(a, tree_level_max_units(n, T, level), s));
    c->launches += tree_level_kernels(exact);
    cur ^= 1;
  }
  *order_out = ord[cur];
  *off_out = off[cur];
  return DRPT_OK;
}

struct LocalPlan {
  int ld = 0;
  int64_t min_leaf = 0;
  int64_t sum_sq = 0;
  int max_leaf = 0;
};

// Host part of the local split: leaf sizes -> local depth, the reference's
// error conditions, permutation tables; then K5.
drpt_status local_phase(drpt_ctx *c, const int32_t *order, const int32_t *goff, int64_t n, int T,
                        int gd, int nn, int local_tree_offset, int forced_ld, int exact,
                        const uint32_t *local_seeds, int d, int32_t *final_order,
                        int32_t *final_off, LocalPlan *plan, cudaStream_t s) {
  const int nleaf = 1 << (gd - 1);
  std::vector<int32_t> h_off((size_t)T * (nleaf + 1));
  DRPT_CUDA(cudaMemcpyAsync(h_off.data(), goff, h_off.size() * 4, cudaMemcpyDeviceToHost, s));
  DRPT_CUDA(cudaStreamSynchronize(s));
  int64_t min_leaf = INT32_MAX;
  bool empty = false;
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < nleaf; ++j) {
      const int64_t sz = h_off[(size_t)t * (nleaf + 1) + j + 1] - h_off[(size_t)t * (nleaf + 1) + j];
      if (sz == 0) empty = true;
      else min_leaf = std::min(min_leaf, sz);
    }
  plan->min_leaf = min_leaf;
  int ld = forced_ld;
  if (ld <= 0)  // mdrpt.cpp:324
    ld = (int)(std::log2((double)(int)min_leaf) - (std::log2((double)nn) + local_tree_offset));
  plan->ld = ld;
  if (ld <= 0) {  // drpt_local.cpp:84-88
    set_error("local tree depth %d <= 0 (smallest global leaf %lld, nn %d)", ld,
              (long long)min_leaf, nn);
    return DRPT_ERR_DEPTH_OUT_OF_RANGE;
  }
  if (empty) {
    set_error("a global leaf is empty (the reference throws from DRPTLocal)");
    return DRPT_ERR_EMPTY_LEAF;
  }
  if (ld > 24 || (int64_t)nleaf << ld > INT32_MAX) {
    set_error("local tree depth %d too large", ld);
    return DRPT_ERR_UNSUPPORTED;
  }
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < nleaf; ++j) {
      const int64_t sz = h_off[(size_t)t * (nleaf + 1) + j + 1] - h_off[(size_t)t * (nleaf + 1) + j];
      if (ld > std::log2((double)sz)) {
        set_error("local tree depth %d > log2(%lld)", ld, (long long)sz);
        return DRPT_ERR_DEPTH_OUT_OF_RANGE;
      }
    }
  if (exact && local_seeds) {
    for (int t = 0; t < T; ++t)
      if (!host_local_matrix_is_zero(local_seeds[t], d, ld)) {
        set_error("local projection matrix of tree %d is not all zero", t);
        return DRPT_ERR_LOCAL_MATRIX_NONZERO;
      }
  }
  // Permutations per distinct size, appended to one pool.
  std::vector<int32_t> pool;
  std::vector<int64_t> pbase((size_t)T * nleaf), fbase((size_t)T * nleaf);
  std::map<int64_t, std::pair<int64_t, int64_t>> where;
  int64_t sum_sq = 0;
  int max_leaf = 0;
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < nleaf; ++j) {
      const int64_t sz = h_off[(size_t)t * (nleaf + 1) + j + 1] - h_off[(size_t)t * (nleaf + 1) + j];
      auto it = where.find(sz);
      if (it == where.end()) {
        auto key = std::make_pair(sz, ld);
        auto ct = c->perms.find(key);
        if (ct == c->perms.end()) {
          std::vector<int32_t> perm, first;
          host_local_permutation(sz, ld, perm, first);
          ct = c->perms.emplace(key, std::make_pair(std::move(perm), std::move(first))).first;
        }
        const int64_t pb = (int64_t)pool.size();
        pool.insert(pool.end(), ct->second.first.begin(), ct->second.first.end());
        const int64_t fb = (int64_t)pool.size();
        pool.insert(pool.end(), ct->second.second.begin(), ct->second.second.end());
        it = where.emplace(sz, std::make_pair(pb, fb)).first;
      }
      pbase[(size_t)t * nleaf + j] = it->second.first;
      fbase[(size_t)t * nleaf + j] = it->second.second;
      const int32_t *first = pool.data() + it->second.second;
      for (int l = 0; l < (1 << ld); ++l) {
        const int64_t m = first[l + 1] - first[l];
        sum_sq += m * m;
        max_leaf = std::max<int>(max_leaf, (int)m);
      }
    }
  plan->sum_sq = sum_sq;
  plan->max_leaf = max_leaf;
  int32_t *dpool;
  int64_t *dpb, *dfb;
  DRPT_TRY(ws_get(c, "perm_pool", pool.size(), &dpool));
  DRPT_TRY(ws_get(c, "perm_base", pbase.size(), &dpb));
  DRPT_TRY(ws_get(c, "first_base", fbase.size(), &dfb));
  DRPT_CUDA(cudaMemcpyAsync(dpool, pool.data(), pool.size() * 4, cudaMemcpyHostToDevice, s));
  DRPT_CUDA(cudaMemcpyAsync(dpb, pbase.data(), pbase.size() * 8, cudaMemcpyHostToDevice, s));
  DRPT_CUDA(cudaMemcpyAsync(dfb, fbase.data(), fbase.size() * 8, cudaMemcpyHostToDevice, s));
  LocalArgs la{order, goff, dpb, dfb, dpool, n, T, nleaf, ld, final_order, final_off};
  DRPT_TRY(launch_local(la, s));
  c->launches += 1;
  return DRPT_OK;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

drpt_status check_common(const drpt_build_desc *d) {
  if (!d) return DRPT_ERR_INVALID_ARG;
  if (d->n < 2 || d->n > INT32_MAX || d->d <= 0 || d->ntrees <= 0 || d->nn <= 0 ||
      (d->dtype != DRPT_DTYPE_F32 && d->dtype != DRPT_DTYPE_U8) || !(d->tree_depth_ratio > 0) ||
      (d->mode < DRPT_MODE_EXACT || d->mode > DRPT_MODE_FP32_GRAM)) {
    set_error("invalid descriptor (n=%lld d=%d ntrees=%d nn=%d dtype=%d mode=%d)",
              (long long)d->n, d->d, d->ntrees, d->nn, d->dtype, d->mode);
    return DRPT_ERR_INVALID_ARG;
  }
  if (d->nn > kMaxK) {
    set_error("nn = %d larger than %d", d->nn, kMaxK);
    return DRPT_ERR_UNSUPPORTED;
  }
  return DRPT_OK;
}

// Global depth whose 2^(gd-1) leaves hold at most about `leaf_size` points
// each (mixed and FP32-leaf modes).
drpt_status leaf_depth(int64_t n, int leaf_size_in, int *gd_out) {
  if (leaf_size_in < 0 || leaf_size_in > 4096) {
    set_error("leaf_size %d outside [0, 4096]", leaf_size_in);
    return DRPT_ERR_INVALID_ARG;
  }
  const int leaf_size = leaf_size_in > 0 ? leaf_size_in : 512;
  int gd = 1;
  while (gd < 30 && ((int64_t)1 << (gd - 1)) * leaf_size < n) ++gd;
  if (gd > std::log2((double)n)) {
    set_error("global depth %d outside [1, log2(%lld)]", gd, (long long)n);
    return DRPT_ERR_DEPTH_OUT_OF_RANGE;
  }
  *gd_out = gd;
  return DRPT_OK;
}

// Leaf phase of the mixed form over the global leaves of T trees (`order`,
// `goff`: T x n and T x (nleaf + 1)): per tree K8 centring and K10
// tensor-core brute force into the running candidate lists, then K11 re-rank
// into oi / od.  Kernel launches only (no host synchronisation), so the
// batched path can capture it in a CUDA graph; `timed` records the per-tree
// events that the stats report.  mixed_check reads the kernels' error flag.
// Candidates kept per point and tree (re-ranked at the end): the requested
// width, or 16 for nn <= 10 and 32 otherwise; -1 when the request is not
// 16 or 32 or is below nn.
int list_width_of(int req, int nn) {
  if (req == 0) return nn <= 10 ? 16 : 32;
  return (req == 16 || req == 32) && req >= nn ? req : -1;
}

// f32gram: the leaf Gram tiles in FP32 on the CUDA cores over the rows of X
// (no staging) instead of BF16 / E4M3 tiles on the tensor cores.
drpt_status mixed_leaf_phase(drpt_ctx *c, const void *X, int dtype, int64_t n, int d, int T,
                             int nn, int kp, int fp8, const int32_t *order, const int32_t *goff,
                             int nleaf, int32_t *oi, float *od, bool timed, cudaStream_t s,
                             bool f32gram = false) {
  const int d_pad = mixed_d_pad(d, fp8);
  cudaEvent_t *ev = c->ev;
  MixedTreeArgs a{};
  a.X = X;
  a.dtype = dtype;
  a.n = n;
  a.d = d;
  a.d_pad = d_pad;
  a.nleaf = nleaf;
  a.T = T;
  a.kp = kp;
  a.fp8 = fp8;
  const int Tc = f32gram ? T : mixed_stage_trees(n, d_pad, fp8, T);
  const size_t row_bytes = (size_t)d_pad * (fp8 ? 1 : 2);
  uint8_t *xb = nullptr;
  float *nrm = nullptr, *scl = nullptr;
  if (!f32gram) {
    DRPT_TRY(ws_get(c, "mx_xb", (size_t)Tc * n * row_bytes, &xb));
    DRPT_TRY(ws_get(c, "mx_nrm", (size_t)Tc * n, &nrm));
    DRPT_TRY(ws_get(c, "mx_scl", fp8 ? (size_t)Tc * n : 1, &scl));
  } else {
    DRPT_TRY(ws_get(c, "fg_nrm", (size_t)n, &nrm));  // ||x||^2, the same for every tree
  }
  LeafStageArgs st{};
  st.X = X;
  st.dtype = dtype;
  st.n = n;
  st.d = d;
  st.d_pad = d_pad;
  st.fp8 = fp8;
  st.order = order;
  st.goff = goff;
  st.nleaf = nleaf;
  st.T = T;
  if (!f32gram) {
    DRPT_TRY(ws_get(c, "mx_pos", (size_t)T * n, &st.pos));
    DRPT_TRY(ws_get(c, "mx_lf", (size_t)T * n, &st.lf));
    DRPT_TRY(ws_get(c, "mx_mu", (size_t)T * nleaf * d, &st.mu));
  }
  st.Xb = xb;
  st.nrm = nrm;
  st.scl = scl;
  const size_t tiles = (size_t)ceil_div(n, 64) + nleaf;  // the FP32 form's 64-row tiles
  DRPT_TRY(ws_get(c, "mx_tile_leaf", tiles, &a.tile_leaf));
  DRPT_TRY(ws_get(c, "mx_tile_r0", tiles, &a.tile_r0));
  DRPT_TRY(ws_get(c, "mx_n_tiles", 1, &a.n_tiles));
  DRPT_TRY(ws_get(c, "mx_err", 1, &a.err));
  DRPT_TRY(ws_get(c, "mx_run_idx", (size_t)n * kp, &a.cand_idx));
  DRPT_TRY(ws_get(c, "mx_run_dist", (size_t)n * kp, &a.cand_dist));
  DRPT_TRY(ws_get(c, "mx_tree_idx", (size_t)n * kp, &a.tree_idx));
  DRPT_TRY(ws_get(c, "mx_tree_dist", (size_t)n * kp, &a.tree_dist));
  DRPT_CUDA(cudaMemsetAsync(a.err, 0, sizeof(int), s));
  int nev = 0;
  if (timed) {
    DRPT_CUDA(cudaEventRecord(ev[3], s));
    const int need = 2 + 2 * T + 2 * T;
    while ((int)c->tev.size() < need) {
      cudaEvent_t e;
      DRPT_CUDA(cudaEventCreate(&e));
      c->tev.push_back(e);
    }
    c->tstage.clear();
    c->tmma.clear();
  }
  auto mark = [&](int *idx) -> drpt_status {
    *idx = nev++;
    DRPT_CUDA(cudaEventRecord(c->tev[*idx], s));
    return DRPT_OK;
  };
  int e0 = 0, e1 = 0;
  if (f32gram) {
    if (timed) DRPT_TRY(mark(&e0));
    DRPT_TRY(launch_row_norms(X, dtype, n, d, nrm, s));
    c->launches += 1;
    if (timed) {
      DRPT_TRY(mark(&e1));
      c->tstage.push_back({e0, e1});
    }
    a.nrm = nrm;
    for (int t = 0; t < T; ++t) {
      a.tree = t;
      a.order = order + (size_t)t * n;
      a.goff = goff + (size_t)t * (nleaf + 1);
      if (timed) DRPT_TRY(mark(&e0));
      DRPT_TRY(launch_leaf_f32(a, nrm, s));
      c->launches += t > 0 ? 3 : 2;  // tile plan, leaf kernel, fold
      if (timed) {
        DRPT_TRY(mark(&e1));
        c->tmma.push_back({e0, e1});
      }
    }
    if (timed) DRPT_CUDA(cudaEventRecord(ev[4], s));
    DRPT_TRY(launch_rerank(X, dtype, d, order + (size_t)(T - 1) * n, n, a.cand_idx, kp, nn, oi,
                           od, s));
    c->launches += 1;
    if (timed) DRPT_CUDA(cudaEventRecord(ev[5], s));
    return DRPT_OK;
  }
  if (timed) DRPT_TRY(mark(&e0));
  DRPT_TRY(launch_leaf_means(st, s));
  c->launches += 2;
  if (timed) {
    DRPT_TRY(mark(&e1));
    c->tstage.push_back({e0, e1});
  }
  for (int t0 = 0; t0 < T; t0 += Tc) {
    st.t0 = t0;
    st.tc = std::min(Tc, T - t0);
    if (timed) DRPT_TRY(mark(&e0));
    DRPT_TRY(launch_leaf_stage(st, s));
    c->launches += 1;
    if (timed) {
      DRPT_TRY(mark(&e1));
      c->tstage.push_back({e0, e1});
    }
    for (int t = t0; t < t0 + st.tc; ++t) {
      a.tree = t;
      a.order = order + (size_t)t * n;
      a.goff = goff + (size_t)t * (nleaf + 1);
      a.Xb = xb + (size_t)(t - t0) * n * row_bytes;
      a.nrm = nrm + (size_t)(t - t0) * n;
      a.scl = fp8 ? scl + (size_t)(t - t0) * n : scl;
      if (timed) DRPT_TRY(mark(&e0));
      DRPT_TRY(launch_leaf_mma(a, s));
      c->launches += t > 0 ? 3 : 2;  // tile plan, leaf kernel, fold
      if (timed) {
        DRPT_TRY(mark(&e1));
        c->tmma.push_back({e0, e1});
      }
    }
  }
  if (timed) DRPT_CUDA(cudaEventRecord(ev[4], s));
  // Re-rank in the leaf order of the last tree: a point's candidates are
  // mostly its leaf-mates there, so their rows stay in L2.
  DRPT_TRY(launch_rerank(X, dtype, d, order + (size_t)(T - 1) * n, n, a.cand_idx, kp, nn, oi,
                         od, s));
  c->launches += 1;
  if (timed) DRPT_CUDA(cudaEventRecord(ev[5], s));
  return DRPT_OK;
}

// Staging and tensor-core milliseconds of the last timed leaf phase.
void leaf_phase_ms(drpt_ctx *c, float *stage, float *mma) {
  for (const auto &p : c->tstage) *stage += elapsed(c->tev[p.first], c->tev[p.second]);
  for (const auto &p : c->tmma) *mma += elapsed(c->tev[p.first], c->tev[p.second]);
}

drpt_status mixed_check(drpt_ctx *c, cudaStream_t s) {
  int *err_d = nullptr;
  DRPT_TRY(ws_get(c, "mx_err", 1, &err_d));
  int err = 0, serr = 0;
  DRPT_CUDA(cudaMemcpyAsync(&err, err_d, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (c->bufs.count("sgn_err")) {  // the sign-matrix projection's bounded waits
    DRPT_CUDA(cudaMemcpyAsync(&serr, c->bufs["sgn_err"].p, sizeof(int), cudaMemcpyDeviceToHost, s));
  }
  DRPT_CUDA(cudaStreamSynchronize(s));
  if (serr) err |= 1;
  if (err & 2) {
    set_error("a global leaf holds more than 8192 points (the tensor-core leaf kernel's limit); "
              "use a smaller leaf_size");
    return DRPT_ERR_UNSUPPORTED;
  }
  if (err) {
    set_error("a bounded wait in the tensor-core leaf kernel gave up");
    return DRPT_ERR_TIMEOUT;
  }
  return DRPT_OK;
}

// ---------------------------------------------------------------- learned splits
// Per learned tree and level an MLP d -> 64 -> 1 (k_learned.cu).  Training
// runs level by level on a sample: the sample's 10 nearest neighbours come
// from the mixed form's own leaf brute force (the whole sample as one leaf),
// each level's MLPs of all learned trees train together with Adam, and the
// sample is then split by the level kernels on the trained outputs (the
// histogram median of every node, as the full trees split) to give the next
// level's nodes.  Inference writes every MLP's output for all n points into
// the projected-column array P, where the level kernels split on it exactly
// as on a random projection.
constexpr int kLearnIters = 10;      // default Adam steps per level
constexpr int kLearnSample = 8192;   // default sample size
constexpr int kLearnSampleMax = 1 << 20;
constexpr int kPairLeaf = 8192;      // largest leaf of the sample's neighbour search
constexpr float kLearnLr = 0.01f;
constexpr int kLearnPairs = 10;      // neighbours per sample point
constexpr int kLearnChunks = 64;     // row chunks of the backward pass

// Reverse neighbour pairs (CSR over the S sample points), each row ascending.
void pair_tables(const std::vector<int32_t> &nbr, int S, int k, std::vector<int32_t> *in_ptr,
                 std::vector<int32_t> *in_idx) {
  in_ptr->assign(S + 1, 0);
  for (int i = 0; i < S; ++i)
    for (int q = 0; q < k; ++q) {
      const int j = nbr[(size_t)i * k + q];
      if (j >= 0) ++(*in_ptr)[j + 1];
    }
  for (int i = 0; i < S; ++i) (*in_ptr)[i + 1] += (*in_ptr)[i];
  in_idx->assign((*in_ptr)[S], 0);
  std::vector<int32_t> fill(in_ptr->begin(), in_ptr->end() - 1);
  for (int i = 0; i < S; ++i)
    for (int q = 0; q < k; ++q) {
      const int j = nbr[(size_t)i * k + q];
      if (j >= 0) (*in_idx)[fill[j]++] = i;
    }
}

// Device buffers of a training run: T trees, S sample points, node tables for
// up to max_nodes nodes per tree.
drpt_status learn_buffers(drpt_ctx *c, int T, int S, int d, int k, int max_nodes, LearnArgs *a) {
  a->S = S;
  a->d = d;
  a->T = T;
  a->k = k;
  a->np = kLearnHidden * d + 2 * kLearnHidden + 1;
  a->R = kLearnChunks;
  const size_t ts = (size_t)T * S, tp = (size_t)T * a->np, tn = (size_t)T * max_nodes;
  float *Xs, *inv;
  int32_t *nbr, *in_ptr, *in_idx;
  DRPT_TRY(ws_get(c, "ln_xs", (size_t)S * d, &Xs));
  DRPT_TRY(ws_get(c, "ln_params", tp, &a->params));
  DRPT_TRY(ws_get(c, "ln_m1", tp, &a->m1));
  DRPT_TRY(ws_get(c, "ln_m2", tp, &a->m2));
  DRPT_TRY(ws_get(c, "ln_nbr", (size_t)S * k, &nbr));
  DRPT_TRY(ws_get(c, "ln_in_ptr", (size_t)S + 1, &in_ptr));
  DRPT_TRY(ws_get(c, "ln_in_idx", (size_t)S * k, &in_idx));
  DRPT_TRY(ws_get(c, "ln_inv_pairs", (size_t)T, &inv));
  DRPT_TRY(ws_get(c, "ln_A", ts * kLearnHidden, &a->A));
  DRPT_TRY(ws_get(c, "ln_f", ts, &a->f));
  DRPT_TRY(ws_get(c, "ln_g", ts, &a->g));
  DRPT_TRY(ws_get(c, "ln_sp", ts, &a->sp));
  DRPT_TRY(ws_get(c, "ln_mu", tn, &a->mu));
  DRPT_TRY(ws_get(c, "ln_var", tn, &a->var));
  DRPT_TRY(ws_get(c, "ln_sn", tn, &a->sn));
  DRPT_TRY(ws_get(c, "ln_lterm", tn, &a->lterm));
  DRPT_TRY(ws_get(c, "ln_part", (size_t)T * a->R * a->np, &a->part));
  a->Xs = Xs;
  a->nbr = nbr;
  a->in_ptr = in_ptr;
  a->in_idx = in_idx;
  a->inv_pairs = inv;
  return DRPT_OK;
}

struct LearnResult {
  float loss_start = 0.0f, loss_end = 0.0f;
};

// Trains the split MLPs of T learned trees of global depth gd and writes
// their outputs for all n points to P columns [col0, col0 + T*(gd-1)).
drpt_status learn_and_project(drpt_ctx *c, const void *X, int dtype, int64_t n, int d, int T,
                              int gd, uint32_t seed, int sample, int iters, float *P,
                              int64_t col0, LearnResult *res, cudaStream_t s) {
  const int levels = gd - 1;
  if (levels <= 0) return DRPT_OK;
  const int S = (int)std::min<int64_t>(n, sample > 0 ? sample : kLearnSample);
  if (iters <= 0) iters = kLearnIters;
  const int d_pad = (d + 63) / 64 * 64;
  // sample rows: S distinct indices, ascending
  std::mt19937 gen(seed ^ 0x5bd1e995u);
  std::vector<int32_t> ids(n);
  for (int64_t i = 0; i < n; ++i) ids[i] = (int32_t)i;
  for (int i = 0; i < S; ++i) {
    std::uniform_int_distribution<int64_t> pick(i, n - 1);
    std::swap(ids[i], ids[pick(gen)]);
  }
  ids.resize(S);
  std::sort(ids.begin(), ids.end());
  int32_t *dids;
  float *xraw, *dc, *dinv;
  double *dvar;
  DRPT_TRY(ws_get(c, "ln_ids", (size_t)S, &dids));
  DRPT_TRY(ws_get(c, "ln_xraw", (size_t)S * d, &xraw));
  DRPT_TRY(ws_get(c, "ln_c", (size_t)d, &dc));
  DRPT_TRY(ws_get(c, "ln_dvar", (size_t)d, &dvar));
  DRPT_TRY(ws_get(c, "ln_inv_sigma", 1, &dinv));
  DRPT_CUDA(cudaMemcpyAsync(dids, ids.data(), (size_t)S * 4, cudaMemcpyHostToDevice, s));
  DRPT_TRY(launch_standardise(X, dtype, S, d, d, dids, nullptr, nullptr, nullptr, xraw, s));
  DRPT_TRY(launch_sample_scale(xraw, S, d, dc, dvar, dinv, s));
  // the sample's neighbours: the mixed leaf brute force over one leaf
  int32_t *iota_t, *goff1, *nbr_d;
  float *ndist;
  const int max_nodes = 1 << (levels - 1);
  DRPT_TRY(ws_get(c, "ln_iota", (size_t)T * S, &iota_t));
  DRPT_TRY(ws_get(c, "ln_goff", (size_t)2 * T, &goff1));
  DRPT_TRY(ws_get(c, "ln_knn_idx", (size_t)S * kLearnPairs, &nbr_d));
  DRPT_TRY(ws_get(c, "ln_knn_dist", (size_t)S * kLearnPairs, &ndist));
  std::vector<int32_t> io((size_t)T * S), g2(2 * T);
  for (int t = 0; t < T; ++t) {
    for (int i = 0; i < S; ++i) io[(size_t)t * S + i] = i;
    g2[2 * t] = 0;
    g2[2 * t + 1] = S;
  }
  DRPT_CUDA(cudaMemcpyAsync(iota_t, io.data(), io.size() * 4, cudaMemcpyHostToDevice, s));
  DRPT_CUDA(cudaMemcpyAsync(goff1, g2.data(), g2.size() * 4, cudaMemcpyHostToDevice, s));
  // The brute force runs over leaves of at most kPairLeaf points (the leaf
  // kernel's limit): a larger sample is sorted along a seeded random
  // direction and cut into equal consecutive chunks, a one-level tree.
  const int chunks = (S + kPairLeaf - 1) / kPairLeaf;
  const int32_t *pord = iota_t, *poff = goff1;
  if (chunks > 1) {
    // the sample projected on the GPU onto one seeded Gaussian direction
    std::mt19937 dg(seed ^ 0x2545f491u);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    std::vector<float> w(d);
    for (int k = 0; k < d; ++k) w[k] = nd(dg);
    float *dkey;
    DRPT_TRY(ws_get(c, "ln_pair_key", (size_t)S, &dkey));
    DRPT_TRY(project_cols(c, xraw, DRPT_DTYPE_F32, S, d, w.data(), 1, std::vector<int32_t>{0},
                          dkey, s, nullptr, "ln_pair_csc"));
    std::vector<float> key(S);
    DRPT_CUDA(cudaMemcpyAsync(key.data(), dkey, (size_t)S * 4, cudaMemcpyDeviceToHost, s));
    DRPT_CUDA(cudaStreamSynchronize(s));
    std::vector<int32_t> po(S), pf(chunks + 1);
    for (int i = 0; i < S; ++i) po[i] = i;
    std::stable_sort(po.begin(), po.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
    for (int q = 0; q <= chunks; ++q) pf[q] = (int32_t)((int64_t)S * q / chunks);
    int32_t *dpo, *dpf;
    DRPT_TRY(ws_get(c, "ln_pair_order", (size_t)S, &dpo));
    DRPT_TRY(ws_get(c, "ln_pair_off", (size_t)chunks + 1, &dpf));
    DRPT_CUDA(cudaMemcpyAsync(dpo, po.data(), po.size() * 4, cudaMemcpyHostToDevice, s));
    DRPT_CUDA(cudaMemcpyAsync(dpf, pf.data(), pf.size() * 4, cudaMemcpyHostToDevice, s));
    DRPT_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
    pord = dpo;
    poff = dpf;
  }
  DRPT_TRY(mixed_leaf_phase(c, xraw, DRPT_DTYPE_F32, S, d, 1, kLearnPairs, 16, 0, pord, poff,
                            chunks, nbr_d, ndist, false, s));
  DRPT_TRY(mixed_check(c, s));
  std::vector<int32_t> nbr((size_t)S * kLearnPairs);
  DRPT_CUDA(cudaMemcpy(nbr.data(), nbr_d, nbr.size() * 4, cudaMemcpyDeviceToHost));
  // training state
  LearnArgs a{};
  DRPT_TRY(learn_buffers(c, T, S, d, kLearnPairs, max_nodes, &a));
  DRPT_TRY(launch_standardise(X, dtype, S, d, d, dids, dc, dinv, nullptr, (float *)a.Xs, s));
  DRPT_CUDA(cudaMemcpyAsync((void *)a.nbr, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, s));
  std::vector<int32_t> in_ptr, in_idx;
  pair_tables(nbr, S, kLearnPairs, &in_ptr, &in_idx);
  DRPT_CUDA(cudaMemcpyAsync((void *)a.in_ptr, in_ptr.data(), in_ptr.size() * 4,
                            cudaMemcpyHostToDevice, s));
  if (!in_idx.empty())
    DRPT_CUDA(cudaMemcpyAsync((void *)a.in_idx, in_idx.data(), in_idx.size() * 4,
                              cudaMemcpyHostToDevice, s));
  // node tables, ping-pong: level 0 is one node per tree holding the sample
  int32_t *perm[2], *noff[2], *node_of, *cnt;
  float *fp, *loss;
  DRPT_TRY(ws_get(c, "ln_perm_a", (size_t)T * S, &perm[0]));
  DRPT_TRY(ws_get(c, "ln_perm_b", (size_t)T * S, &perm[1]));
  DRPT_TRY(ws_get(c, "ln_noff_a", (size_t)T * (2 * max_nodes + 1), &noff[0]));
  DRPT_TRY(ws_get(c, "ln_noff_b", (size_t)T * (2 * max_nodes + 1), &noff[1]));
  DRPT_TRY(ws_get(c, "ln_node_of", (size_t)T * S, &node_of));
  DRPT_TRY(ws_get(c, "ln_cnt", (size_t)T, &cnt));
  DRPT_TRY(ws_get(c, "ln_fp", (size_t)T * S, &fp));
  DRPT_TRY(ws_get(c, "ln_loss", 2, &loss));
  DRPT_CUDA(cudaMemcpyAsync(perm[0], iota_t, (size_t)T * S * 4, cudaMemcpyDeviceToDevice, s));
  DRPT_CUDA(cudaMemcpyAsync(noff[0], goff1, (size_t)2 * T * 4, cudaMemcpyDeviceToDevice, s));
  DRPT_CUDA(cudaMemsetAsync(node_of, 0, (size_t)T * S * 4, s));
  DRPT_CUDA(cudaMemsetAsync(loss, 0, 2 * sizeof(float), s));
  // level-kernel scratch for the sample splits (deepest split level: levels - 2)
  TreeLevelArgs lv{};
  if (levels >= 2) {
    const int last = levels - 2;
    const int64_t Gmax = (int64_t)T << last, Umax = tree_level_max_units(S, T, last);
    DRPT_TRY(ws_get(c, "ls_node_ubase", Gmax + 1, &lv.node_ubase));
    DRPT_TRY(ws_get(c, "ls_unit_node", Umax, &lv.unit_node));
    DRPT_TRY(ws_get(c, "ls_unit_lo", Umax, &lv.unit_lo));
    DRPT_TRY(ws_get(c, "ls_n_units", 1, &lv.n_units));
    DRPT_TRY(ws_get(c, "ls_node_D", Gmax * kBins, &lv.node_D));
    DRPT_TRY(ws_get(c, "ls_unit_s", 2 * Umax, &lv.unit_s));
    DRPT_TRY(ws_get(c, "ls_unit_hist", Umax * kBins, &lv.unit_hist));
    DRPT_TRY(ws_get(c, "ls_node_med", Gmax, &lv.node_med));
    DRPT_TRY(ws_get(c, "ls_unit_left", Umax, &lv.unit_left));
    DRPT_TRY(ws_get(c, "ls_unit_lbase", Umax, &lv.unit_lbase));
    DRPT_TRY(ws_get(c, "ls_node_nleft", Gmax, &lv.node_nleft));
  }
  // stacked inference weights, MLP m = tree * levels + level
  const int M = T * levels;
  __nv_bfloat16 *wb;
  float *db1, *dw2, *db2;
  DRPT_TRY(ws_get(c, "ln_w1b", (size_t)M * kLearnHidden * d_pad, &wb));
  DRPT_TRY(ws_get(c, "ln_b1", (size_t)M * kLearnHidden, &db1));
  DRPT_TRY(ws_get(c, "ln_w2", (size_t)M * kLearnHidden, &dw2));
  DRPT_TRY(ws_get(c, "ln_b2", (size_t)M, &db2));
  DRPT_CUDA(cudaMemsetAsync(wb, 0, (size_t)M * kLearnHidden * d_pad * 2, s));
  int cur = 0;
  for (int l = 0; l < levels; ++l) {
    const int nodes = 1 << l;
    a.perm = perm[cur];
    a.noff = noff[cur];
    a.node_of = node_of;
    a.nodes = nodes;
    DRPT_TRY(launch_learn_pairs(a, cnt, s));
    DRPT_TRY(launch_learn_init(a, seed, l, s));
    DRPT_CUDA(cudaMemsetAsync(a.m1, 0, (size_t)T * a.np * 4, s));
    DRPT_CUDA(cudaMemsetAsync(a.m2, 0, (size_t)T * a.np * 4, s));
    c->launches += 3;
    for (int it = 0; it < iters; ++it) {
      const float bc1 = 1.0f - std::pow(0.9f, (float)(it + 1));
      const float bc2 = 1.0f - std::pow(0.999f, (float)(it + 1));
      DRPT_TRY(launch_learn_step(a, kLearnLr, bc1, bc2, nullptr, s));
      c->launches += learn_step_kernels();
      if (it == 0) DRPT_TRY(launch_learn_loss(a, loss, 0, s));
    }
    // the loss and outputs at the trained weights
    DRPT_TRY(launch_learn_step(a, 0.0f, 1.0f, 1.0f, nullptr, s));
    DRPT_TRY(launch_learn_loss(a, loss, 1, s));
    DRPT_TRY(launch_stack(a, d_pad, levels, l, wb, db1, dw2, db2, s));
    c->launches += learn_step_kernels() + 3;
    if (l + 1 < levels) {
      // split every node of the sample at the histogram median of f
      DRPT_TRY(launch_gather_f(a, fp, s));
      TreeLevelArgs t = lv;
      t.P = nullptr;
      t.n = S;
      t.T = T;
      t.gd = 2;
      t.level = l;
      t.p_level0 = -1;  // values come from val_in (f in node order)
      t.ord_in = perm[cur];
      t.val_in = fp;
      t.off_in = noff[cur];
      t.ord_out = perm[cur ^ 1];
      t.val_out = nullptr;
      t.off_out = noff[cur ^ 1];
      t.medians = nullptr;
      t.exact = 0;
      t.stop = nullptr;
      DRPT_TRY(launch_tree_level(t, tree_level_max_units(S, T, l), s));
      DRPT_TRY(launch_node_label(perm[cur ^ 1], noff[cur ^ 1], 2 * nodes, S, T, node_of, s));
      c->launches += tree_level_kernels(0) + 2;
      cur ^= 1;
    }
  }
  // inference over all n points
  __nv_bfloat16 *xb;
  int *err;
  DRPT_TRY(ws_get(c, "ln_xb", (size_t)n * d_pad, &xb));
  DRPT_TRY(ws_get(c, "ln_err", 1, &err));
  DRPT_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  DRPT_TRY(launch_standardise(X, dtype, n, d, d_pad, nullptr, dc, dinv, xb, nullptr, s));
  DRPT_TRY(launch_mlp_infer(xb, n, d_pad, wb, M, db1, dw2, db2, P + col0 * n, err, s));
  c->launches += 2;
  float hl[2] = {0.0f, 0.0f};
  int herr = 0;
  DRPT_CUDA(cudaMemcpyAsync(hl, loss, sizeof(hl), cudaMemcpyDeviceToHost, s));
  DRPT_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  DRPT_CUDA(cudaStreamSynchronize(s));
  if (herr) {
    set_error("a bounded wait in the split-MLP inference kernel gave up");
    return DRPT_ERR_TIMEOUT;
  }
  res->loss_start = hl[0] / ((float)T * levels);
  res->loss_end = hl[1] / ((float)T * levels);
  return DRPT_OK;
}

// Mixed-precision pipeline (DRPT_MODE_MIXED): global trees with fast
// statistics grown to leaves of about `leaf_size` points, BF16 tensor-core
// brute force of every global leaf, cross-tree merge of the approximate
// candidates, exact FP32 re-rank with the FP64 boundary check.
template <typename Tp>
drpt_status dev_copy(Tp **dst, const void *src, size_t count, cudaStream_t s) {
  const size_t bytes = std::max<size_t>(count * sizeof(Tp), 4);
  DRPT_CUDA(cudaMalloc((void **)dst, bytes));
  if (count) DRPT_CUDA(cudaMemcpyAsync(*dst, src, count * sizeof(Tp), cudaMemcpyDeviceToDevice, s));
  return DRPT_OK;
}

// check = false leaves the leaf kernel's error flag for the caller to read
// (no host synchronisation; with stats == nullptr and keep == nullptr the
// build of random trees is then fully stream-ordered).
drpt_status run_mixed(drpt_ctx *c, const drpt_build_desc *desc, const void *X, int32_t *oi,
                      float *od, drpt_stats *stats, cudaStream_t s, drpt_index *keep = nullptr,
                      bool check = true) {
  const int64_t n = desc->n;
  const int d = desc->d, T = desc->ntrees, nn = desc->nn;
  if (nn > 32) {
    set_error("mixed mode supports nn <= 32 (got %d)", nn);
    return DRPT_ERR_UNSUPPORTED;
  }
  const int kp = list_width_of(desc->list_width, nn);
  if (kp < 0) {
    set_error("list_width %d: 0, or 16 or 32 and at least nn = %d", desc->list_width, nn);
    return DRPT_ERR_INVALID_ARG;
  }
  if (desc->precision != DRPT_PRECISION_BF16 && desc->precision != DRPT_PRECISION_FP8_E4M3) {
    set_error("unknown precision %d", desc->precision);
    return DRPT_ERR_INVALID_ARG;
  }
  const bool f32gram = desc->mode == DRPT_MODE_FP32_GRAM;
  const int fp8 = !f32gram && desc->precision == DRPT_PRECISION_FP8_E4M3;
  if (d % 4 != 0 || d > 1024) {
    set_error("mixed mode supports d %% 4 == 0 and d <= 1024 (got %d)", d);
    return DRPT_ERR_UNSUPPORTED;
  }
  if (f32gram && (d % 8 != 0 || desc->learned_trees != 0)) {
    set_error("the FP32 Gram form needs d %% 8 == 0 and no learned trees (d = %d)", d);
    return DRPT_ERR_UNSUPPORTED;
  }
  const int learned = desc->learned_trees;
  if (learned < 0 || learned > T || desc->learn_sample < 0 || desc->learn_sample > kLearnSampleMax ||
      desc->learn_iters < 0) {
    set_error("learned_trees %d (of %d), learn_sample %d or learn_iters %d out of range", learned,
              T, desc->learn_sample, desc->learn_iters);
    return DRPT_ERR_INVALID_ARG;
  }
  if (learned > 0 && d > 256) {
    set_error("learned splits support d <= 256 (got %d)", d);
    return DRPT_ERR_UNSUPPORTED;
  }
  int gd = 0;
  DRPT_TRY(leaf_depth(n, desc->leaf_size, &gd));
  const int nleaf = 1 << (gd - 1);
  const int L = gd * T, Tr = T - learned;
  const float density = (float)(desc->density == 0 ? 1.0 / std::sqrt((double)d) : desc->density);
  cudaEvent_t *ev = c->ev;
  const int launches0 = c->launches;
  DRPT_CUDA(cudaEventRecord(ev[1], s));

  // trees 0 .. Tr-1 split on random projections, the learned ones on MLP values
  std::vector<float> B((size_t)d * L);
  host_projection_matrix(desc->seed, d, L, density, B.data());
  std::vector<int32_t> cols;
  for (int t = 0; t < Tr; ++t)
    for (int l = 0; l + 1 < gd; ++l) cols.push_back(t * gd + l);
  float *P = nullptr;
  DRPT_TRY(ws_get(c, "P", std::max<size_t>((size_t)T * (gd - 1), 1) * n, &P));
  int nnz = 0;
  if (desc->projection == DRPT_PROJECTION_SIGN) {
    if (desc->dtype != DRPT_DTYPE_U8) {
      set_error("the sign-matrix projection takes u8 rows");
      return DRPT_ERR_UNSUPPORTED;
    }
    if (!cols.empty()) DRPT_TRY(project_sign(c, X, n, d, B.data(), L, cols, P, s, &nnz));
  } else if (desc->projection != DRPT_PROJECTION_GAUSSIAN) {
    set_error("unknown projection %d", desc->projection);
    return DRPT_ERR_INVALID_ARG;
  } else if (!cols.empty()) {
    DRPT_TRY(project_cols(c, X, desc->dtype, n, d, B.data(), L, cols, P, s, &nnz));
  }
  LearnResult lres;
  float ms_learn = 0.0f;
  if (learned > 0) {
    const auto t0 = std::chrono::steady_clock::now();
    DRPT_TRY(learn_and_project(c, X, desc->dtype, n, d, learned, gd, desc->seed,
                               desc->learn_sample, desc->learn_iters, P, (int64_t)Tr * (gd - 1),
                               &lres, s));
    ms_learn =
        std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  int32_t *order, *goff;
  float *medians = nullptr;
  if (keep) DRPT_TRY(ws_get(c, "medians", (size_t)T * std::max(nleaf - 1, 1), &medians));
  DRPT_TRY(global_trees(c, P, n, T, gd, 0, medians, &order, &goff, s));
  DRPT_CUDA(cudaEventRecord(ev[2], s));

  DRPT_TRY(mixed_leaf_phase(c, X, desc->dtype, n, d, T, nn, kp, fp8, order, goff, nleaf, oi, od,
                            /*timed=*/true, s, f32gram));
  if (check) DRPT_TRY(mixed_check(c, s));
  if (keep) {
    // the index keeps its own copies: the workspace is reused by later calls
    keep->n = n;
    keep->d = d;
    keep->dtype = desc->dtype;
    keep->T = T;
    keep->gd = gd;
    keep->nleaf = nleaf;
    keep->Tr = Tr;
    keep->Tl = learned;
    keep->d_pad = (d + 63) / 64 * 64;
    const size_t esz = desc->dtype == DRPT_DTYPE_U8 ? 1 : 4;
    DRPT_TRY(dev_copy((uint8_t **)&keep->X, X, (size_t)n * d * esz, s));
    DRPT_TRY(dev_copy(&keep->order, order, (size_t)T * n, s));
    DRPT_TRY(dev_copy(&keep->goff, goff, (size_t)T * (nleaf + 1), s));
    DRPT_TRY(dev_copy(&keep->medians, medians, (size_t)T * std::max(nleaf - 1, 1), s));
    keep->ncols_r = (int)cols.size();
    if (!cols.empty()) {
      int32_t *dcol, *drow;
      float *dval;
      DRPT_TRY(ws_get(c, "csc_colptr", cols.size() + 1, &dcol));
      DRPT_TRY(ws_get(c, "csc_row", std::max<size_t>(nnz, 1), &drow));
      DRPT_TRY(ws_get(c, "csc_val", std::max<size_t>(nnz, 1), &dval));
      DRPT_TRY(dev_copy(&keep->csc_col, dcol, cols.size() + 1, s));
      DRPT_TRY(dev_copy(&keep->csc_row, drow, (size_t)nnz, s));
      DRPT_TRY(dev_copy(&keep->csc_val, dval, (size_t)nnz, s));
    }
    if (learned > 0) {
      const size_t M = (size_t)learned * (gd - 1);
      __nv_bfloat16 *wb;
      float *b1, *w2, *b2, *cc, *is;
      DRPT_TRY(ws_get(c, "ln_w1b", M * kLearnHidden * keep->d_pad, &wb));
      DRPT_TRY(ws_get(c, "ln_b1", M * kLearnHidden, &b1));
      DRPT_TRY(ws_get(c, "ln_w2", M * kLearnHidden, &w2));
      DRPT_TRY(ws_get(c, "ln_b2", M, &b2));
      DRPT_TRY(ws_get(c, "ln_c", (size_t)d, &cc));
      DRPT_TRY(ws_get(c, "ln_inv_sigma", 1, &is));
      DRPT_TRY(dev_copy(&keep->w1b, wb, M * kLearnHidden * keep->d_pad, s));
      DRPT_TRY(dev_copy(&keep->b1, b1, M * kLearnHidden, s));
      DRPT_TRY(dev_copy(&keep->w2, w2, M * kLearnHidden, s));
      DRPT_TRY(dev_copy(&keep->b2, b2, M, s));
      DRPT_TRY(dev_copy(&keep->c, cc, (size_t)d, s));
      DRPT_TRY(dev_copy(&keep->inv_sigma, is, 1, s));
    }
    DRPT_CUDA(cudaStreamSynchronize(s));
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->tree_depth = gd;
    stats->global_depth = gd;
    stats->local_depth = 0;
    stats->n_global_leaves = nleaf;
    stats->n_final_leaves = nleaf;
    // leaf sizes for the work figure
    std::vector<int32_t> h((size_t)T * (nleaf + 1));
    DRPT_CUDA(cudaMemcpy(h.data(), goff, h.size() * 4, cudaMemcpyDeviceToHost));
    int64_t sq = 0, mn = INT64_MAX;
    int mx = 0;
    for (int t = 0; t < T; ++t)
      for (int j = 0; j < nleaf; ++j) {
        const int64_t m = h[(size_t)t * (nleaf + 1) + j + 1] - h[(size_t)t * (nleaf + 1) + j];
        sq += m * m;
        if (m > 0) mn = std::min(mn, m);
        mx = std::max<int>(mx, (int)m);
      }
    stats->sum_leaf_sq = sq;
    int64_t padded = 0;  // 128 x 64 tiles over every leaf
    for (int t = 0; t < T; ++t)
      for (int j = 0; j < nleaf; ++j) {
        const int64_t m = h[(size_t)t * (nleaf + 1) + j + 1] - h[(size_t)t * (nleaf + 1) + j];
        padded += ceil_div(m, 128) * 128 * ceil_div(m, 64) * 64;
      }
    stats->mma_pairs_padded = padded;
    leaf_phase_ms(c, &stats->ms_leaf_stage, &stats->ms_leaf_mma);
    stats->min_global_leaf = mn;
    stats->max_final_leaf = mx;
    stats->kernels_launched = c->launches - launches0;
    stats->ms_project = elapsed(ev[0], ev[1]);  // input copy, if any
    stats->ms_global = elapsed(ev[1], ev[2]);
    stats->ms_local = elapsed(ev[2], ev[3]);
    stats->ms_leaf_knn = elapsed(ev[3], ev[4]);
    stats->ms_merge = elapsed(ev[4], ev[5]);
    stats->ms_learn = ms_learn;
    stats->learn_loss_start = lres.loss_start;
    stats->learn_loss_end = lres.loss_end;
  }
  return DRPT_OK;
}

// FP32 whole-leaf pipeline (DRPT_MODE_FP32_LEAF): the mixed form's trees,
// every global leaf brute-forced by the exact FP32 leaf kernel, cross-tree
// merge.
drpt_status run_fp32_leaf(drpt_ctx *c, const drpt_build_desc *desc, const void *X, int32_t *oi,
                          float *od, drpt_stats *stats, cudaStream_t s) {
  const int64_t n = desc->n;
  const int d = desc->d, T = desc->ntrees, nn = desc->nn;
  int gd = 0;
  DRPT_TRY(leaf_depth(n, desc->leaf_size, &gd));
  const int nleaf = 1 << (gd - 1);
  const int L = gd * T;
  const float density = (float)(desc->density == 0 ? 1.0 / std::sqrt((double)d) : desc->density);
  cudaEvent_t *ev = c->ev;
  const int launches0 = c->launches;
  DRPT_CUDA(cudaEventRecord(ev[1], s));
  std::vector<float> B((size_t)d * L);
  host_projection_matrix(desc->seed, d, L, density, B.data());
  std::vector<int32_t> cols;
  for (int t = 0; t < T; ++t)
    for (int l = 0; l + 1 < gd; ++l) cols.push_back(t * gd + l);
  float *P = nullptr;
  DRPT_TRY(ws_get(c, "P", std::max<size_t>(cols.size(), 1) * n, &P));
  if (!cols.empty()) DRPT_TRY(project_cols(c, X, desc->dtype, n, d, B.data(), L, cols, P, s));
  int32_t *order, *goff;
  DRPT_TRY(global_trees(c, P, n, T, gd, 0, nullptr, &order, &goff, s));
  DRPT_CUDA(cudaEventRecord(ev[2], s));
  DRPT_CUDA(cudaEventRecord(ev[3], s));
  int32_t *cidx;
  float *cdist;
  DRPT_TRY(ws_get(c, "cand_idx", (size_t)n * T * nn, &cidx));
  DRPT_TRY(ws_get(c, "cand_dist", (size_t)n * T * nn, &cdist));
  LeafKnnArgs ka{X, desc->dtype, n, d, T, nn, order, goff, nleaf, cidx, cdist};
  DRPT_TRY(launch_leaf_knn_exact(ka, s));
  c->launches += leaf_knn_exact_kernels();
  DRPT_CUDA(cudaEventRecord(ev[4], s));
  DRPT_TRY(launch_merge(cidx, cdist, n, T, nn, nn, oi, od, s));
  c->launches += 1;
  DRPT_CUDA(cudaEventRecord(ev[5], s));
  DRPT_CUDA(cudaStreamSynchronize(s));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->tree_depth = gd;
    stats->global_depth = gd;
    stats->n_global_leaves = nleaf;
    stats->n_final_leaves = nleaf;
    std::vector<int32_t> h((size_t)T * (nleaf + 1));
    DRPT_CUDA(cudaMemcpy(h.data(), goff, h.size() * 4, cudaMemcpyDeviceToHost));
    int64_t sq = 0, mn = INT64_MAX;
    int mx = 0;
    for (int t = 0; t < T; ++t)
      for (int j = 0; j < nleaf; ++j) {
        const int64_t m = h[(size_t)t * (nleaf + 1) + j + 1] - h[(size_t)t * (nleaf + 1) + j];
        sq += m * m;
        if (m > 0) mn = std::min(mn, m);
        mx = std::max<int>(mx, (int)m);
      }
    stats->sum_leaf_sq = sq;
    stats->min_global_leaf = mn;
    stats->max_final_leaf = mx;
    stats->kernels_launched = c->launches - launches0;
    stats->ms_global = elapsed(ev[1], ev[2]);
    stats->ms_leaf_knn = elapsed(ev[3], ev[4]);
    stats->ms_merge = elapsed(ev[4], ev[5]);
  }
  return DRPT_OK;
}


// ---------------------------------------------------------------- batches
// A batch is built as one forest.  Its first level is virtual: level l0 =
// ceil(log2(nsets)) of every tree holds the datasets as its 2^l0 root slots
// (slots past nsets are empty), the points in index order.  The level
// kernels then split every slot exactly as a build of that dataset alone
// would split its root (same node-aligned statistics, median and stable
// partition), and a dataset of global depth gd_s stops splitting after
// gd_s - 1 levels (its nodes keep all points below that).  Dataset s projects
// with the matrix its own build would draw (d x gd_s*T from the seed), so
// every dataset's trees, leaves and lists equal its single build's.
struct BatchPlan {
  int nsets = 0, l0 = 0, gdm = 0, nleaf = 0, T = 0, nn = 0, d = 0, dtype = 0, fp8 = 0, mode = 0;
  int kp = 16;                   // mixed mode: candidates kept per point and tree
  int64_t n = 0;
  int ncols = 0;                 // T * (gdm - 1) projected columns
  CscDev csc{};
  int32_t *root_off = nullptr;   // T x (2^l0 + 1)
  int8_t *stop = nullptr;        // 2^l0
  int64_t *set_off = nullptr;    // nsets + 1
  float *P = nullptr;
  int32_t *ord[2] = {}, *off[2] = {};
  float *val[2] = {};
  TreeLevelArgs lv{};
  int32_t *order = nullptr, *goff = nullptr;  // final leaves
  int32_t *cidx = nullptr;       // fp32_leaf candidates
  float *cdist = nullptr;
};

drpt_status batch_prepare(drpt_ctx *c, const drpt_batch_desc *desc, const int64_t *offs,
                          BatchPlan *bp, cudaStream_t s) {
  const int nsets = desc->nsets, T = desc->ntrees, d = desc->d;
  const int64_t n = offs[nsets];
  bp->nsets = nsets;
  bp->T = T;
  bp->nn = desc->nn;
  bp->kp = list_width_of(desc->list_width, desc->nn);
  bp->d = d;
  bp->dtype = desc->dtype;
  bp->mode = desc->mode;
  bp->fp8 = desc->precision == DRPT_PRECISION_FP8_E4M3;
  bp->n = n;
  std::vector<int> gds(nsets);
  int gdm = 2;  // at least one level runs, even if no dataset splits
  for (int i = 0; i < nsets; ++i) {
    DRPT_TRY(leaf_depth(offs[i + 1] - offs[i], desc->leaf_size, &gds[i]));
    gdm = std::max(gdm, gds[i]);
  }
  int l0 = 0;
  while ((1 << l0) < nsets) ++l0;
  bp->l0 = l0;
  bp->gdm = gdm;
  if (l0 + gdm - 1 > 24 || ((int64_t)T << (l0 + gdm - 2)) > (1 << 20)) {
    set_error("batch of %d datasets needs %d tree levels: too many nodes", nsets, l0 + gdm - 1);
    return DRPT_ERR_UNSUPPORTED;
  }
  const int nroot = 1 << l0;
  bp->nleaf = 1 << (l0 + gdm - 1);
  // projection: one column set per distinct global depth
  const int ncols = T * (gdm - 1);
  bp->ncols = ncols;
  const float density = (float)(desc->density == 0 ? 1.0 / std::sqrt((double)d) : desc->density);
  std::map<int, int> set_of_depth;
  std::vector<int32_t> colptr, row;
  std::vector<float> val;
  for (int i = 0; i < nsets; ++i) {
    if (set_of_depth.count(gds[i])) continue;
    const int g = gds[i], cs = (int)set_of_depth.size();
    set_of_depth[g] = cs;
    const int L = g * T;
    std::vector<float> B((size_t)d * L);
    host_projection_matrix(desc->seed, d, L, density, B.data());
    colptr.push_back((int32_t)row.size());
    for (int t = 0; t < T; ++t)
      for (int l = 0; l + 1 < gdm; ++l) {
        if (l + 1 < g)  // levels the dataset splits on; the others project to 0
          for (int k = 0; k < d; ++k) {
            const float b = B[(int64_t)k * L + t * g + l];
            if (b != 0.0f) {
              row.push_back(k);
              val.push_back(b);
            }
          }
        colptr.push_back((int32_t)row.size());
      }
  }
  const int pts = project_points_per_block(d);
  std::vector<int32_t> blocks;
  for (int i = 0; i < nsets; ++i)
    for (int64_t r = offs[i]; r < offs[i + 1]; r += pts) {
      blocks.push_back((int32_t)r);
      blocks.push_back((int32_t)std::min<int64_t>(pts, offs[i + 1] - r));
      blocks.push_back(set_of_depth[gds[i]]);
    }
  int32_t *dcol, *drow, *dblk;
  float *dval;
  DRPT_TRY(ws_get(c, "bt_colptr", colptr.size(), &dcol));
  DRPT_TRY(ws_get(c, "bt_row", std::max<size_t>(row.size(), 1), &drow));
  DRPT_TRY(ws_get(c, "bt_val", std::max<size_t>(val.size(), 1), &dval));
  DRPT_TRY(ws_get(c, "bt_blocks", std::max<size_t>(blocks.size(), 1), &dblk));
  // root slots, stop depths and dataset offsets
  std::vector<int32_t> ro((size_t)T * (nroot + 1));
  for (int t = 0; t < T; ++t)
    for (int j = 0; j <= nroot; ++j)
      ro[(size_t)t * (nroot + 1) + j] = (int32_t)offs[std::min(j, nsets)];
  std::vector<int8_t> stop(nroot, 0);
  for (int i = 0; i < nsets; ++i) stop[i] = (int8_t)(gds[i] - 1);
  DRPT_TRY(ws_get(c, "bt_root_off", ro.size(), &bp->root_off));
  DRPT_TRY(ws_get(c, "bt_stop", stop.size(), &bp->stop));
  DRPT_TRY(ws_get(c, "bt_set_off", (size_t)nsets + 1, &bp->set_off));
  // every other buffer of the build, sized now so that a captured run
  // allocates nothing
  DRPT_TRY(ws_get(c, "P", std::max<size_t>(ncols, 1) * n, &bp->P));
  DRPT_TRY(ws_get(c, "ord_a", (size_t)T * n, &bp->ord[0]));
  DRPT_TRY(ws_get(c, "ord_b", (size_t)T * n, &bp->ord[1]));
  DRPT_TRY(ws_get(c, "val_a", (size_t)T * n, &bp->val[0]));
  DRPT_TRY(ws_get(c, "val_b", (size_t)T * n, &bp->val[1]));
  DRPT_TRY(ws_get(c, "off_a", (size_t)T * (bp->nleaf + 1), &bp->off[0]));
  DRPT_TRY(ws_get(c, "off_b", (size_t)T * (bp->nleaf + 1), &bp->off[1]));
  const int last = l0 + gdm - 2;
  const int64_t Gmax = (int64_t)T << last;
  const int64_t Umax = tree_level_max_units(n, T, last);
  TreeLevelArgs &a = bp->lv;
  DRPT_TRY(ws_get(c, "lv_node_ubase", Gmax + 1, &a.node_ubase));
  DRPT_TRY(ws_get(c, "lv_unit_node", Umax, &a.unit_node));
  DRPT_TRY(ws_get(c, "lv_unit_lo", Umax, &a.unit_lo));
  DRPT_TRY(ws_get(c, "lv_n_units", 1, &a.n_units));
  DRPT_TRY(ws_get(c, "lv_node_D", Gmax * kBins, &a.node_D));
  DRPT_TRY(ws_get(c, "lv_unit_s", 2 * Umax, &a.unit_s));
  DRPT_TRY(ws_get(c, "lv_unit_hist", Umax * kBins, &a.unit_hist));
  DRPT_TRY(ws_get(c, "lv_node_med", Gmax, &a.node_med));
  DRPT_TRY(ws_get(c, "lv_unit_left", Umax, &a.unit_left));
  DRPT_TRY(ws_get(c, "lv_unit_lbase", Umax, &a.unit_lbase));
  DRPT_TRY(ws_get(c, "lv_node_nleft", Gmax, &a.node_nleft));
  if (bp->mode == DRPT_MODE_MIXED) {
    const int d_pad = mixed_d_pad(d, bp->fp8), kp = bp->kp;
    const size_t tiles = (size_t)ceil_div(n, 128) + bp->nleaf;
    uint8_t *u8p;
    int32_t *i32p;
    float *f32p;
    int *ip;
    const int Tc = mixed_stage_trees(n, d_pad, bp->fp8, T);
    DRPT_TRY(ws_get(c, "mx_xb", (size_t)Tc * n * d_pad * (bp->fp8 ? 1 : 2), &u8p));
    DRPT_TRY(ws_get(c, "mx_nrm", (size_t)Tc * n, &f32p));
    DRPT_TRY(ws_get(c, "mx_scl", bp->fp8 ? (size_t)Tc * n : 1, &f32p));
    DRPT_TRY(ws_get(c, "mx_pos", (size_t)T * n, &i32p));
    DRPT_TRY(ws_get(c, "mx_lf", (size_t)T * n, &i32p));
    DRPT_TRY(ws_get(c, "mx_mu", (size_t)T * bp->nleaf * d, &f32p));
    DRPT_TRY(ws_get(c, "mx_tile_leaf", tiles, &i32p));
    DRPT_TRY(ws_get(c, "mx_tile_r0", tiles, &i32p));
    DRPT_TRY(ws_get(c, "mx_n_tiles", 1, &i32p));
    DRPT_TRY(ws_get(c, "mx_err", 1, &ip));
    DRPT_TRY(ws_get(c, "mx_run_idx", (size_t)n * kp, &i32p));
    DRPT_TRY(ws_get(c, "mx_run_dist", (size_t)n * kp, &f32p));
  } else {
    DRPT_TRY(ws_get(c, "cand_idx", (size_t)n * T * bp->nn, &bp->cidx));
    DRPT_TRY(ws_get(c, "cand_dist", (size_t)n * T * bp->nn, &bp->cdist));
  }
  // uploads (pageable sources: complete before the calls return)
  DRPT_CUDA(cudaMemcpyAsync(dcol, colptr.data(), colptr.size() * 4, cudaMemcpyHostToDevice, s));
  if (!row.empty()) {
    DRPT_CUDA(cudaMemcpyAsync(drow, row.data(), row.size() * 4, cudaMemcpyHostToDevice, s));
    DRPT_CUDA(cudaMemcpyAsync(dval, val.data(), val.size() * 4, cudaMemcpyHostToDevice, s));
  }
  DRPT_CUDA(cudaMemcpyAsync(dblk, blocks.data(), blocks.size() * 4, cudaMemcpyHostToDevice, s));
  DRPT_CUDA(cudaMemcpyAsync(bp->root_off, ro.data(), ro.size() * 4, cudaMemcpyHostToDevice, s));
  DRPT_CUDA(cudaMemcpyAsync(bp->stop, stop.data(), stop.size(), cudaMemcpyHostToDevice, s));
  DRPT_CUDA(cudaMemcpyAsync(bp->set_off, offs, ((size_t)nsets + 1) * 8, cudaMemcpyHostToDevice, s));
  bp->csc = CscDev{dcol, drow, dval, ncols};
  bp->csc.blocks = dblk;
  bp->csc.nblocks = (int32_t)(blocks.size() / 3);
  // the leaf arrays the level loop ends in
  const int fin = (gdm - 1) & 1;
  bp->order = bp->ord[fin];
  bp->goff = bp->off[fin];
  return DRPT_OK;
}

// The batch's device work: kernel launches and device-side memsets only, so
// that it can be captured in a CUDA graph.
drpt_status batch_enqueue(drpt_ctx *c, const BatchPlan &bp, const void *X, int32_t *oi,
                          float *od, bool timed, cudaStream_t s) {
  const int64_t n = bp.n;
  const int T = bp.T;
  if (bp.ncols > 0) {
    DRPT_TRY(launch_project(X, bp.dtype, n, bp.d, bp.csc, bp.P, s));
    c->launches += 1;
  }
  TreeLevelArgs a = bp.lv;
  a.P = bp.P;
  a.n = n;
  a.T = T;
  a.gd = bp.gdm;
  a.p_level0 = bp.l0;
  a.stop = bp.stop;
  a.medians = nullptr;
  a.exact = 0;
  int cur = 0;
  for (int k = 0; k < bp.gdm - 1; ++k) {
    a.level = bp.l0 + k;
    a.ord_in = k == 0 ? nullptr : bp.ord[cur];  // index order at the root slots
    a.val_in = k == 0 ? nullptr : bp.val[cur];  // read from P at the root slots
    a.off_in = k == 0 ? bp.root_off : bp.off[cur];
    a.ord_out = bp.ord[cur ^ 1];
    a.val_out = k + 1 < bp.gdm - 1 ? bp.val[cur ^ 1] : nullptr;
    a.off_out = bp.off[cur ^ 1];
    DRPT_TRY(launch_tree_level(a, tree_level_max_units(n, T, a.level), s));
    c->launches += tree_level_kernels(0);
    cur ^= 1;
  }
  if (timed) DRPT_CUDA(cudaEventRecord(c->ev[2], s));
  if (bp.mode == DRPT_MODE_MIXED) {
    DRPT_TRY(mixed_leaf_phase(c, X, bp.dtype, n, bp.d, T, bp.nn, bp.kp, bp.fp8, bp.order, bp.goff,
                              bp.nleaf, oi, od, timed, s));
  } else {
    if (timed) DRPT_CUDA(cudaEventRecord(c->ev[3], s));
    LeafKnnArgs ka{X, bp.dtype, n, bp.d, T, bp.nn, bp.order, bp.goff, bp.nleaf, bp.cidx, bp.cdist};
    DRPT_TRY(launch_leaf_knn_exact(ka, s));
    c->launches += leaf_knn_exact_kernels();
    if (timed) DRPT_CUDA(cudaEventRecord(c->ev[4], s));
    DRPT_TRY(launch_merge(bp.cidx, bp.cdist, n, T, bp.nn, bp.nn, oi, od, s));
    c->launches += 1;
    if (timed) DRPT_CUDA(cudaEventRecord(c->ev[5], s));
  }
  DRPT_TRY(launch_localize(oi, n, bp.nn, bp.set_off, bp.nsets, s));
  c->launches += 1;
  return DRPT_OK;
}

std::string batch_key(const drpt_batch_desc *d, const int64_t *offs, const void *X,
                      const void *oi, const void *od) {
  std::string k;
  auto put = [&](const void *p, size_t b) { k.append(static_cast<const char *>(p), b); };
  put(d, sizeof(*d));
  put(offs, ((size_t)d->nsets + 1) * sizeof(int64_t));
  put(&X, sizeof(X));
  put(&oi, sizeof(oi));
  put(&od, sizeof(od));
  return k;
}

}  // namespace
}  // namespace drpt

using namespace drpt;

extern "C" {

const char *drpt_version(void) { return "drpt-b200 0.1.0 (sm_100a)"; }

const char *drpt_last_error(void) { return g_err; }

drpt_status drpt_ctx_create(drpt_ctx **ctx, int device) {
  if (!ctx) return DRPT_ERR_INVALID_ARG;
  *ctx = nullptr;
  int count = 0;
  DRPT_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) {
    set_error("device %d not present (%d devices)", device, count);
    return DRPT_ERR_INVALID_ARG;
  }
  DRPT_CUDA(cudaSetDevice(device));
  drpt_ctx *c = new drpt_ctx();
  c->device = device;
  for (auto &e : c->ev) {
    cudaError_t err = cudaEventCreate(&e);
    if (err != cudaSuccess) {
      set_error("cudaEventCreate: %s", cudaGetErrorString(err));
      drpt_ctx_destroy(c);
      return DRPT_ERR_CUDA;
    }
  }
  *ctx = c;
  return DRPT_OK;
}

void drpt_ctx_destroy(drpt_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  for (auto &kv : c->bufs)
    if (kv.second.p) cudaFree(kv.second.p);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : c->tev)
    if (e) cudaEventDestroy(e);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->gstream) cudaStreamDestroy(c->gstream);
  delete c;
}

drpt_status drpt_build_graph_batched(drpt_ctx *c, const drpt_batch_desc *desc,
                                     const int64_t *offsets, const void *data, int32_t *out_idx,
                                     float *out_dist, drpt_stats *stats) {
  if (!c || !desc || !offsets || !data || !out_idx) return DRPT_ERR_INVALID_ARG;
  const int nsets = desc->nsets;
  if (nsets < 1 || nsets > 65536 || desc->d <= 0 || desc->ntrees <= 0 || desc->nn <= 0 ||
      desc->nn > kMaxK || (desc->dtype != DRPT_DTYPE_F32 && desc->dtype != DRPT_DTYPE_U8) ||
      (desc->mode != DRPT_MODE_MIXED && desc->mode != DRPT_MODE_FP32_LEAF) ||
      (desc->precision != DRPT_PRECISION_BF16 && desc->precision != DRPT_PRECISION_FP8_E4M3)) {
    set_error("invalid batch descriptor");
    return DRPT_ERR_INVALID_ARG;
  }
  if (offsets[0] != 0) {
    set_error("offsets[0] must be 0");
    return DRPT_ERR_INVALID_ARG;
  }
  for (int i = 0; i < nsets; ++i)
    if (offsets[i + 1] - offsets[i] < 2) {
      set_error("dataset %d has %lld rows (at least 2 needed)", i,
                (long long)(offsets[i + 1] - offsets[i]));
      return DRPT_ERR_INVALID_ARG;
    }
  const int64_t n = offsets[nsets];
  const int d = desc->d, nn = desc->nn;
  if (n > INT32_MAX) {
    set_error("batch of %lld rows: at most 2^31 - 1", (long long)n);
    return DRPT_ERR_UNSUPPORTED;
  }
  if (desc->mode == DRPT_MODE_MIXED && (nn > 32 || d % 4 != 0 || d > 1024)) {
    set_error("mixed mode supports nn <= 32 and d %% 4 == 0, d <= 1024 (got nn %d, d %d)", nn, d);
    return DRPT_ERR_UNSUPPORTED;
  }
  if (desc->mode == DRPT_MODE_MIXED && list_width_of(desc->list_width, nn) < 0) {
    set_error("list_width %d: 0, or 16 or 32 and at least nn = %d", desc->list_width, nn);
    return DRPT_ERR_INVALID_ARG;
  }
  if (desc->use_graph && (!desc->data_on_device || !desc->out_on_device)) {
    set_error("graph mode needs device input and output pointers");
    return DRPT_ERR_INVALID_ARG;
  }
  DRPT_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = (cudaStream_t)desc->stream;
  cudaEvent_t *ev = c->ev;
  const size_t esz = desc->dtype == DRPT_DTYPE_U8 ? 1 : 4;
  const int launches0 = c->launches;

  // graph replay
  std::string key;
  if (desc->use_graph) {
    key = batch_key(desc, offsets, data, out_idx, out_dist);
    if (!c->gstream) DRPT_CUDA(cudaStreamCreateWithFlags(&c->gstream, cudaStreamNonBlocking));
    if (c->gexec && c->gkey == key && c->gexec_gen == c->ws_gen) {
      // replay on the context's stream, ordered after and before the caller's
      DRPT_CUDA(cudaEventRecord(ev[0], s));
      DRPT_CUDA(cudaStreamWaitEvent(c->gstream, ev[0], 0));
      DRPT_CUDA(cudaGraphLaunch(c->gexec, c->gstream));
      DRPT_CUDA(cudaEventRecord(ev[7], c->gstream));
      DRPT_CUDA(cudaStreamWaitEvent(s, ev[7], 0));
      DRPT_CUDA(cudaEventRecord(ev[6], s));
      if (desc->mode == DRPT_MODE_MIXED) DRPT_TRY(mixed_check(c, s));
      DRPT_CUDA(cudaEventSynchronize(ev[6]));
      c->launches += c->glaunches;
      if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->kernels_launched = c->glaunches;
        stats->ms_total = elapsed(ev[0], ev[6]);
      }
      return DRPT_OK;
    }
    if (c->gexec) {
      cudaGraphExecDestroy(c->gexec);
      c->gexec = nullptr;
    }
  }

  DRPT_CUDA(cudaEventRecord(ev[0], s));
  const void *X = data;
  if (!desc->data_on_device) {
    void *xd;
    DRPT_TRY(ws_get(c, "x", (size_t)n * d * esz, (uint8_t **)&xd));
    DRPT_CUDA(cudaMemcpyAsync(xd, data, (size_t)n * d * esz, cudaMemcpyHostToDevice, s));
    X = xd;
  }
  int32_t *oi = out_idx;
  float *od = out_dist;
  if (!desc->out_on_device) {
    DRPT_TRY(ws_get(c, "out_idx", (size_t)n * nn, &oi));
    DRPT_TRY(ws_get(c, "out_dist", (size_t)n * nn, &od));
  } else if (!od) {
    DRPT_TRY(ws_get(c, "out_dist", (size_t)n * nn, &od));
  }
  BatchPlan bp;
  DRPT_TRY(batch_prepare(c, desc, offsets, &bp, s));
  DRPT_CUDA(cudaEventRecord(ev[1], s));
  DRPT_TRY(batch_enqueue(c, bp, X, oi, od, /*timed=*/true, s));
  if (!desc->out_on_device) {
    DRPT_CUDA(cudaMemcpyAsync(out_idx, oi, (size_t)n * nn * 4, cudaMemcpyDeviceToHost, s));
    if (out_dist)
      DRPT_CUDA(cudaMemcpyAsync(out_dist, od, (size_t)n * nn * 4, cudaMemcpyDeviceToHost, s));
  }
  DRPT_CUDA(cudaEventRecord(ev[6], s));
  if (desc->mode == DRPT_MODE_MIXED) DRPT_TRY(mixed_check(c, s));
  DRPT_CUDA(cudaEventSynchronize(ev[6]));
  const int launched = c->launches - launches0;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->tree_depth = bp.l0 + bp.gdm;
    stats->global_depth = bp.gdm;
    stats->n_global_leaves = bp.nleaf;
    stats->n_final_leaves = bp.nleaf;
    stats->kernels_launched = launched;
    stats->ms_project = elapsed(ev[0], ev[1]);
    stats->ms_global = elapsed(ev[1], ev[2]);
    stats->ms_leaf_knn = elapsed(ev[3], ev[4]);
    stats->ms_merge = elapsed(ev[4], ev[5]);
    stats->ms_total = elapsed(ev[0], ev[6]);
    if (desc->mode == DRPT_MODE_MIXED) leaf_phase_ms(c, &stats->ms_leaf_stage, &stats->ms_leaf_mma);
  }
  if (desc->use_graph) {
    // capture the device work of this batch for the next calls (every
    // buffer is sized already, so the captured launches allocate nothing)
    const int l0 = c->launches;
    cudaGraph_t g = nullptr;
    DRPT_CUDA(cudaStreamBeginCapture(c->gstream, cudaStreamCaptureModeThreadLocal));
    const drpt_status st = batch_enqueue(c, bp, X, oi, od, /*timed=*/false, c->gstream);
    const cudaError_t ce = cudaStreamEndCapture(c->gstream, &g);
    if (st != DRPT_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    DRPT_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&c->gexec, g, 0);
    cudaGraphDestroy(g);
    DRPT_CUDA(ie);
    c->gkey = key;
    c->gexec_gen = c->ws_gen;
    c->glaunches = c->launches - l0;
    c->launches = l0;
  }
  return DRPT_OK;
}

drpt_status drpt_learn_gradient(drpt_ctx *c, const float *Xs, int32_t S, int32_t d,
                                const float *params, const int32_t *node, const int32_t *nbr,
                                int32_t k, float *grad, float *loss) {
  if (!c || !Xs || !params || !node || !nbr || !grad || S < 2 || d <= 0 || k <= 0)
    return DRPT_ERR_INVALID_ARG;
  int nodes = 0;
  for (int i = 0; i < S; ++i) {
    if (node[i] < 0 || node[i] >= S) return DRPT_ERR_INVALID_ARG;
    nodes = std::max(nodes, node[i] + 1);
  }
  for (int64_t e = 0; e < (int64_t)S * k; ++e)
    if (nbr[e] < -1 || nbr[e] >= S) return DRPT_ERR_INVALID_ARG;
  DRPT_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = nullptr;
  LearnArgs a{};
  DRPT_TRY(learn_buffers(c, 1, S, d, k, nodes, &a));
  int32_t *perm, *noff, *node_of, *cnt;
  float *gdev, *acc;
  DRPT_TRY(ws_get(c, "lg_perm", (size_t)S, &perm));
  DRPT_TRY(ws_get(c, "lg_noff", (size_t)nodes + 1, &noff));
  DRPT_TRY(ws_get(c, "lg_node_of", (size_t)S, &node_of));
  DRPT_TRY(ws_get(c, "lg_cnt", 1, &cnt));
  DRPT_TRY(ws_get(c, "lg_grad", (size_t)a.np, &gdev));
  DRPT_TRY(ws_get(c, "lg_loss", 2, &acc));
  std::vector<int32_t> hp(S), ho(nodes + 1, 0), nb(nbr, nbr + (size_t)S * k), in_ptr, in_idx;
  for (int i = 0; i < S; ++i) ++ho[node[i] + 1];
  for (int j = 0; j < nodes; ++j) ho[j + 1] += ho[j];
  std::vector<int32_t> fill(ho.begin(), ho.end() - 1);
  for (int i = 0; i < S; ++i) hp[fill[node[i]]++] = i;
  pair_tables(nb, S, k, &in_ptr, &in_idx);
  DRPT_CUDA(cudaMemcpy((void *)a.Xs, Xs, (size_t)S * d * 4, cudaMemcpyHostToDevice));
  DRPT_CUDA(cudaMemcpy(a.params, params, (size_t)a.np * 4, cudaMemcpyHostToDevice));
  DRPT_CUDA(cudaMemcpy(perm, hp.data(), hp.size() * 4, cudaMemcpyHostToDevice));
  DRPT_CUDA(cudaMemcpy(noff, ho.data(), ho.size() * 4, cudaMemcpyHostToDevice));
  DRPT_CUDA(cudaMemcpy(node_of, node, (size_t)S * 4, cudaMemcpyHostToDevice));
  DRPT_CUDA(cudaMemcpy((void *)a.nbr, nb.data(), nb.size() * 4, cudaMemcpyHostToDevice));
  DRPT_CUDA(cudaMemcpy((void *)a.in_ptr, in_ptr.data(), in_ptr.size() * 4, cudaMemcpyHostToDevice));
  if (!in_idx.empty())
    DRPT_CUDA(cudaMemcpy((void *)a.in_idx, in_idx.data(), in_idx.size() * 4, cudaMemcpyHostToDevice));
  a.perm = perm;
  a.noff = noff;
  a.node_of = node_of;
  a.nodes = nodes;
  DRPT_CUDA(cudaMemsetAsync(acc, 0, 2 * sizeof(float), s));
  DRPT_TRY(launch_learn_pairs(a, cnt, s));
  DRPT_TRY(launch_learn_step(a, 0.0f, 1.0f, 1.0f, gdev, s));
  DRPT_TRY(launch_learn_loss(a, acc, 0, s));
  DRPT_CUDA(cudaMemcpy(grad, gdev, (size_t)a.np * 4, cudaMemcpyDeviceToHost));
  if (loss) DRPT_CUDA(cudaMemcpy(loss, acc, sizeof(float), cudaMemcpyDeviceToHost));
  return DRPT_OK;
}

drpt_status drpt_host_projection(uint32_t seed, int32_t d, int32_t L, float density, float *B) {
  if (d <= 0 || L <= 0 || !B) return DRPT_ERR_INVALID_ARG;
  host_projection_matrix(seed, d, L, density, B);
  return DRPT_OK;
}

static drpt_status build_graph_impl(drpt_ctx *c, const drpt_build_desc *desc, const void *data,
                                    int32_t *out_idx, float *out_dist, drpt_stats *stats,
                                    drpt_index *keep) {
  if (!c || !data || !out_idx) return DRPT_ERR_INVALID_ARG;
  DRPT_TRY(check_common(desc));
  DRPT_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = (cudaStream_t)desc->stream;
  const int64_t n = desc->n;
  const int d = desc->d, T = desc->ntrees, nn = desc->nn;
  const int exact = desc->mode == DRPT_MODE_EXACT;
  Geometry g{};
  if (desc->mode == DRPT_MODE_EXACT || desc->mode == DRPT_MODE_FAST)
    DRPT_TRY(geometry(n, desc->tree_depth, desc->tree_depth_ratio, &g));
  const int L = g.gd * T;
  const float density = (float)(desc->density == 0 ? 1.0 / std::sqrt((double)d) : desc->density);
  // grow_local_trees takes the density as int (mdrpt.hpp:61-62): from 1 up the
  // local matrices are not zero and the split is no longer positional.
  if (exact && desc->density >= 1.0) {
    set_error("density %g >= 1 makes the local projection matrices non-zero; exact mode "
              "reproduces only the positional local split", desc->density);
    return DRPT_ERR_LOCAL_MATRIX_NONZERO;
  }
  const int launches0 = c->launches;
  cudaEvent_t *ev = c->ev;
  DRPT_CUDA(cudaEventRecord(ev[0], s));

  // Input rows on the device.
  const size_t esz = desc->dtype == DRPT_DTYPE_U8 ? 1 : 4;
  const void *X = data;
  if (!desc->data_on_device) {
    void *xd;
    DRPT_TRY(ws_get(c, "x", (size_t)n * d * esz, (uint8_t **)&xd));
    DRPT_CUDA(cudaMemcpyAsync(xd, data, (size_t)n * d * esz, cudaMemcpyHostToDevice, s));
    X = xd;
  }

  if (desc->projection != DRPT_PROJECTION_GAUSSIAN && desc->mode != DRPT_MODE_MIXED &&
      desc->mode != DRPT_MODE_FP32_GRAM) {
    set_error("the sign-matrix projection is an option of the mixed and FP32 Gram forms only");
    return DRPT_ERR_INVALID_ARG;
  }
  if (desc->mode == DRPT_MODE_MIXED || desc->mode == DRPT_MODE_FP32_LEAF ||
      desc->mode == DRPT_MODE_FP32_GRAM) {
    int32_t *oi = out_idx;
    float *od = out_dist;
    if (!desc->out_on_device) {
      DRPT_TRY(ws_get(c, "out_idx", (size_t)n * nn, &oi));
      DRPT_TRY(ws_get(c, "out_dist", (size_t)n * nn, &od));
    } else if (!od) {
      DRPT_TRY(ws_get(c, "out_dist", (size_t)n * nn, &od));
    }
    if (desc->mode == DRPT_MODE_MIXED || desc->mode == DRPT_MODE_FP32_GRAM)
      DRPT_TRY(run_mixed(c, desc, X, oi, od, stats, s, keep));
    else DRPT_TRY(run_fp32_leaf(c, desc, X, oi, od, stats, s));
    if (!desc->out_on_device) {
      DRPT_CUDA(cudaMemcpyAsync(out_idx, oi, (size_t)n * nn * 4, cudaMemcpyDeviceToHost, s));
      if (out_dist)
        DRPT_CUDA(cudaMemcpyAsync(out_dist, od, (size_t)n * nn * 4, cudaMemcpyDeviceToHost, s));
    }
    DRPT_CUDA(cudaEventRecord(ev[6], s));
    DRPT_CUDA(cudaEventSynchronize(ev[6]));
    if (stats) stats->ms_total = elapsed(ev[0], ev[6]);
    return DRPT_OK;
  }

  // K1: projection on the columns the global trees split on.
  std::vector<float> B((size_t)d * L);
  host_projection_matrix(desc->seed, d, L, density, B.data());
  std::vector<int32_t> cols;
  for (int t = 0; t < T; ++t)
    for (int l = 0; l + 1 < g.gd; ++l) cols.push_back(t * g.gd + l);
  float *P = nullptr;
  DRPT_TRY(ws_get(c, "P", std::max<size_t>(cols.size(), 1) * n, &P));
  if (!cols.empty()) DRPT_TRY(project_cols(c, X, desc->dtype, n, d, B.data(), L, cols, P, s));
  DRPT_CUDA(cudaEventRecord(ev[1], s));

  // K2-K4: global trees.
  int32_t *order, *goff;
  DRPT_TRY(global_trees(c, P, n, T, g.gd, exact, nullptr, &order, &goff, s));
  DRPT_CUDA(cudaEventRecord(ev[2], s));

  if (desc->locality) {
    // locality relabelling on the host: every tree's global leaves in slot order
    const size_t no = (size_t)T * n, nf = (size_t)T * (g.nleaf + 1);
    std::vector<int32_t> ho(no), hf(nf), so(no), sf(nf), slots((size_t)g.nleaf * T);
    DRPT_CUDA(cudaMemcpyAsync(ho.data(), order, no * 4, cudaMemcpyDeviceToHost, s));
    DRPT_CUDA(cudaMemcpyAsync(hf.data(), goff, nf * 4, cudaMemcpyDeviceToHost, s));
    DRPT_CUDA(cudaStreamSynchronize(s));
    DRPT_TRY(drpt_locality_slots(ho.data(), hf.data(), n, T, g.nleaf, slots.data(), so.data(),
                                 sf.data()));
    DRPT_CUDA(cudaMemcpyAsync(order, so.data(), no * 4, cudaMemcpyHostToDevice, s));
    DRPT_CUDA(cudaMemcpyAsync(goff, sf.data(), nf * 4, cudaMemcpyHostToDevice, s));
    DRPT_CUDA(cudaStreamSynchronize(s));
  }

  // K5: local split (one host round trip for the leaf sizes).
  int32_t *forder, *foff;
  DRPT_TRY(ws_get(c, "final_order", (size_t)T * n, &forder));
  LocalPlan plan;
  {
    // final_off needs the local depth; size it for the largest possible.
    int32_t *tmp;
    DRPT_TRY(ws_get(c, "final_off", (size_t)T * (n + 1), &tmp));
    foff = tmp;
  }
  DRPT_TRY(local_phase(c, order, goff, n, T, g.gd, nn, desc->local_tree_offset, 0, exact,
                       desc->local_seeds, d, forder, foff, &plan, s));
  const int n_final = g.nleaf << plan.ld;
  DRPT_CUDA(cudaEventRecord(ev[3], s));

  // K6: leaf brute force.
  int32_t *cidx;
  float *cdist;
  DRPT_TRY(ws_get(c, "cand_idx", (size_t)n * T * nn, &cidx));
  DRPT_TRY(ws_get(c, "cand_dist", (size_t)n * T * nn, &cdist));
  LeafKnnArgs ka{X, desc->dtype, n, d, T, nn, forder, foff, n_final, cidx, cdist};
  DRPT_TRY(launch_leaf_knn_exact(ka, s));
  c->launches += leaf_knn_exact_kernels();
  DRPT_CUDA(cudaEventRecord(ev[4], s));

  // K7: merge into the output.
  int32_t *oi = out_idx;
  float *od = out_dist;
  if (!desc->out_on_device) {
    DRPT_TRY(ws_get(c, "out_idx", (size_t)n * nn, &oi));
    DRPT_TRY(ws_get(c, "out_dist", (size_t)n * nn, &od));
  } else if (!od) {
    DRPT_TRY(ws_get(c, "out_dist", (size_t)n * nn, &od));
  }
  DRPT_TRY(launch_merge(cidx, cdist, n, T, nn, nn, oi, od, s));
  c->launches += 1;
  DRPT_CUDA(cudaEventRecord(ev[5], s));
  if (!desc->out_on_device) {
    DRPT_CUDA(cudaMemcpyAsync(out_idx, oi, (size_t)n * nn * 4, cudaMemcpyDeviceToHost, s));
    if (out_dist)
      DRPT_CUDA(cudaMemcpyAsync(out_dist, od, (size_t)n * nn * 4, cudaMemcpyDeviceToHost, s));
  }
  DRPT_CUDA(cudaEventRecord(ev[6], s));
  if (stats || !desc->out_on_device) DRPT_CUDA(cudaEventSynchronize(ev[6]));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->tree_depth = g.td;
    stats->global_depth = g.gd;
    stats->local_depth = plan.ld;
    stats->n_global_leaves = g.nleaf;
    stats->n_final_leaves = n_final;
    stats->max_final_leaf = plan.max_leaf;
    stats->min_global_leaf = plan.min_leaf;
    stats->sum_leaf_sq = plan.sum_sq;
    stats->kernels_launched = c->launches - launches0;
    stats->ms_project = elapsed(ev[0], ev[1]);
    stats->ms_global = elapsed(ev[1], ev[2]);
    stats->ms_local = elapsed(ev[2], ev[3]);
    stats->ms_leaf_knn = elapsed(ev[3], ev[4]);
    stats->ms_merge = elapsed(ev[4], ev[5]);
    stats->ms_total = elapsed(ev[0], ev[6]);
  }
  return DRPT_OK;
}

drpt_status drpt_build_graph(drpt_ctx *c, const drpt_build_desc *desc, const void *data,
                             int32_t *out_idx, float *out_dist, drpt_stats *stats) {
  return build_graph_impl(c, desc, data, out_idx, out_dist, stats, nullptr);
}

// Many same-shape builds from host memory, pipelined: job j's rows go to
// device buffer j % 2 on an input-copy stream, its build runs on the compute
// stream once they have landed (and once job j - 2's lists have left output
// buffer j % 2), and its lists go back on an output-copy stream.  So the
// input copy of job j + 1 and the output copy of job j - 1 overlap the build
// of job j.  The leaf kernel's error flag of every job is kept on the device
// and read once at the end.
drpt_status drpt_build_graph_stream(drpt_ctx *c, const drpt_build_desc *desc, int32_t count,
                                    const void *const *data, int32_t *const *out_idx,
                                    float *const *out_dist, drpt_stats *stats) {
  if (!c || !desc || !data || !out_idx || count < 1) {
    set_error("drpt_build_graph_stream: null argument or count < 1");
    return DRPT_ERR_INVALID_ARG;
  }
  if (desc->mode != DRPT_MODE_MIXED || desc->data_on_device || desc->out_on_device) {
    set_error("drpt_build_graph_stream: mixed mode with host inputs and outputs only");
    return DRPT_ERR_INVALID_ARG;
  }
  for (int32_t j = 0; j < count; ++j)
    if (!data[j] || !out_idx[j]) {
      set_error("drpt_build_graph_stream: job %d has a null input or output", j);
      return DRPT_ERR_INVALID_ARG;
    }
  DRPT_TRY(check_common(desc));
  DRPT_CUDA(cudaSetDevice(c->device));
  const int64_t n = desc->n;
  const int nn = desc->nn;
  const size_t in_bytes = (size_t)n * desc->d * (desc->dtype == DRPT_DTYPE_U8 ? 1 : 4);
  const size_t out_bytes = (size_t)n * nn * 4;
  uint8_t *xb[2];
  int32_t *ob_i[2];
  float *ob_d[2];
  int *errs = nullptr;
  DRPT_TRY(ws_get(c, "st_x0", in_bytes, &xb[0]));
  DRPT_TRY(ws_get(c, "st_x1", in_bytes, &xb[1]));
  DRPT_TRY(ws_get(c, "st_oi0", (size_t)n * nn, &ob_i[0]));
  DRPT_TRY(ws_get(c, "st_oi1", (size_t)n * nn, &ob_i[1]));
  DRPT_TRY(ws_get(c, "st_od0", (size_t)n * nn, &ob_d[0]));
  DRPT_TRY(ws_get(c, "st_od1", (size_t)n * nn, &ob_d[1]));
  DRPT_TRY(ws_get(c, "st_errs", (size_t)count, &errs));
  // streams and events of this call
  cudaStream_t comp = (cudaStream_t)desc->stream, sin = nullptr, sout = nullptr;
  cudaEvent_t ev_in[2] = {}, ev_comp[2] = {}, ev_out[2] = {}, t0 = nullptr, t1 = nullptr;
  drpt_status st = DRPT_OK;
  auto cu = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && st == DRPT_OK) {
      set_error("%s: %s", what, cudaGetErrorString(e));
      st = DRPT_ERR_CUDA;
    }
    return st == DRPT_OK;
  };
  cu(cudaStreamCreateWithFlags(&sin, cudaStreamNonBlocking), "cudaStreamCreate");
  cu(cudaStreamCreateWithFlags(&sout, cudaStreamNonBlocking), "cudaStreamCreate");
  for (int b = 0; b < 2; ++b) {
    cu(cudaEventCreateWithFlags(&ev_in[b], cudaEventDisableTiming), "cudaEventCreate");
    cu(cudaEventCreateWithFlags(&ev_comp[b], cudaEventDisableTiming), "cudaEventCreate");
    cu(cudaEventCreateWithFlags(&ev_out[b], cudaEventDisableTiming), "cudaEventCreate");
  }
  cu(cudaEventCreate(&t0), "cudaEventCreate");
  cu(cudaEventCreate(&t1), "cudaEventCreate");
  const int launches0 = c->launches;
  drpt_build_desc d = *desc;
  d.data_on_device = 1;
  d.out_on_device = 1;
  d.stream = comp;
  if (st == DRPT_OK) cu(cudaEventRecord(t0, sin), "cudaEventRecord");
  for (int32_t j = 0; st == DRPT_OK && j < count; ++j) {
    const int b = j & 1;
    // job j - 2's build is done with input buffer b
    if (j >= 2 && !cu(cudaStreamWaitEvent(sin, ev_comp[b], 0), "cudaStreamWaitEvent")) break;
    if (!cu(cudaMemcpyAsync(xb[b], data[j], in_bytes, cudaMemcpyHostToDevice, sin),
            "cudaMemcpyAsync")) break;
    cu(cudaEventRecord(ev_in[b], sin), "cudaEventRecord");
    cu(cudaStreamWaitEvent(comp, ev_in[b], 0), "cudaStreamWaitEvent");
    // job j - 2's lists have left output buffer b
    if (j >= 2) cu(cudaStreamWaitEvent(comp, ev_out[b], 0), "cudaStreamWaitEvent");
    if (st != DRPT_OK) break;
    st = run_mixed(c, &d, xb[b], ob_i[b], ob_d[b], nullptr, comp, nullptr, /*check=*/false);
    if (st != DRPT_OK) break;
    int *err_d = nullptr;
    st = ws_get(c, "mx_err", 1, &err_d);
    if (st != DRPT_OK) break;
    cu(cudaMemcpyAsync(errs + j, err_d, sizeof(int), cudaMemcpyDeviceToDevice, comp),
       "cudaMemcpyAsync");
    cu(cudaEventRecord(ev_comp[b], comp), "cudaEventRecord");
    cu(cudaStreamWaitEvent(sout, ev_comp[b], 0), "cudaStreamWaitEvent");
    cu(cudaMemcpyAsync(out_idx[j], ob_i[b], out_bytes, cudaMemcpyDeviceToHost, sout),
       "cudaMemcpyAsync");
    if (out_dist && out_dist[j])
      cu(cudaMemcpyAsync(out_dist[j], ob_d[b], out_bytes, cudaMemcpyDeviceToHost, sout),
         "cudaMemcpyAsync");
    cu(cudaEventRecord(ev_out[b], sout), "cudaEventRecord");
  }
  // everything issued so far is waited for, also after a failure
  if (sin) cudaStreamSynchronize(sin);
  cudaStreamSynchronize(comp);
  if (sout) {
    if (st == DRPT_OK) cu(cudaEventRecord(t1, sout), "cudaEventRecord");
    cudaStreamSynchronize(sout);
  }
  if (st == DRPT_OK) {
    std::vector<int> he((size_t)count);
    if (cu(cudaMemcpy(he.data(), errs, (size_t)count * sizeof(int), cudaMemcpyDeviceToHost),
           "cudaMemcpy")) {
      int any = 0;
      for (int e : he) any |= e;
      if (any & 2) {
        set_error("a global leaf holds more than 8192 points (the tensor-core leaf kernel's "
                  "limit); use a smaller leaf_size");
        st = DRPT_ERR_UNSUPPORTED;
      } else if (any) {
        set_error("a bounded wait in the tensor-core leaf kernel gave up");
        st = DRPT_ERR_TIMEOUT;
      }
    }
  }
  if (st == DRPT_OK && stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->kernels_launched = c->launches - launches0;
    cu(cudaEventElapsedTime(&stats->ms_total, t0, t1), "cudaEventElapsedTime");
  }
  for (int b = 0; b < 2; ++b) {
    if (ev_in[b]) cudaEventDestroy(ev_in[b]);
    if (ev_comp[b]) cudaEventDestroy(ev_comp[b]);
    if (ev_out[b]) cudaEventDestroy(ev_out[b]);
  }
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  if (sin) cudaStreamDestroy(sin);
  if (sout) cudaStreamDestroy(sout);
  return st;
}

static void index_free(drpt_index *x) {
  if (!x) return;
  cudaSetDevice(x->device);
  void *ptrs[] = {x->X, x->order, x->goff, x->medians, x->csc_col, x->csc_row, x->csc_val,
                  x->w1b, x->b1, x->w2, x->b2, x->c, x->inv_sigma, x->Pq, x->leaf, x->qi,
                  x->qd, x->qx, x->qxb, x->err};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete x;
}

drpt_status drpt_index_build(drpt_ctx *c, const drpt_build_desc *desc, const void *data,
                             int32_t *out_idx, float *out_dist, drpt_stats *stats,
                             drpt_index **index) {
  if (!c || !desc || !index) return DRPT_ERR_INVALID_ARG;
  *index = nullptr;
  if (desc->mode != DRPT_MODE_MIXED) {
    set_error("an index is built by the mixed form (mode DRPT_MODE_MIXED)");
    return DRPT_ERR_INVALID_ARG;
  }
  drpt_index *x = new drpt_index();
  x->device = c->device;
  const drpt_status st = build_graph_impl(c, desc, data, out_idx, out_dist, stats, x);
  if (st != DRPT_OK) {
    index_free(x);
    return st;
  }
  *index = x;
  return DRPT_OK;
}

void drpt_index_destroy(drpt_index *index) { index_free(index); }

drpt_status drpt_index_query(drpt_index *x, const void *queries, int64_t nq, int32_t k,
                             int32_t on_device, int32_t *out_idx, float *out_dist, void *stream) {
  if (!x || !queries || !out_idx || nq <= 0 || k <= 0) return DRPT_ERR_INVALID_ARG;
  if (k > 32) {
    set_error("queries return at most 32 neighbours (k = %d)", k);
    return DRPT_ERR_UNSUPPORTED;
  }
  DRPT_CUDA(cudaSetDevice(x->device));
  cudaStream_t s = (cudaStream_t)stream;
  const int d = x->d, T = x->T, cols = T * (x->gd - 1);
  const size_t esz = x->dtype == DRPT_DTYPE_U8 ? 1 : 4;
  if (nq > x->cap) {  // grow the query scratch
    void **bufs[] = {(void **)&x->Pq, (void **)&x->leaf, (void **)&x->qi, (void **)&x->qd,
                     (void **)&x->qx, (void **)&x->qxb, (void **)&x->err};
    for (void **b : bufs)
      if (*b) {
        cudaFree(*b);
        *b = nullptr;
      }
    x->cap = 0;
    DRPT_CUDA(cudaMalloc((void **)&x->Pq, std::max<size_t>((size_t)cols * nq, 1) * 4));
    DRPT_CUDA(cudaMalloc((void **)&x->leaf, (size_t)T * nq * 4));
    DRPT_CUDA(cudaMalloc((void **)&x->qi, (size_t)32 * nq * 4));
    DRPT_CUDA(cudaMalloc((void **)&x->qd, (size_t)32 * nq * 4));
    DRPT_CUDA(cudaMalloc(&x->qx, (size_t)nq * d * esz));
    if (x->Tl > 0) DRPT_CUDA(cudaMalloc((void **)&x->qxb, (size_t)nq * x->d_pad * 2));
    DRPT_CUDA(cudaMalloc((void **)&x->err, sizeof(int)));
    x->cap = nq;
  }
  const void *Q = queries;
  if (!on_device) {
    DRPT_CUDA(cudaMemcpyAsync(x->qx, queries, (size_t)nq * d * esz, cudaMemcpyHostToDevice, s));
    Q = x->qx;
  }
  // the queries' split values: random columns, then the learned MLP outputs
  if (x->ncols_r > 0) {
    CscDev csc{x->csc_col, x->csc_row, x->csc_val, x->ncols_r};
    DRPT_TRY(launch_project(Q, x->dtype, nq, d, csc, x->Pq, s));
  }
  if (x->Tl > 0) {
    DRPT_CUDA(cudaMemsetAsync(x->err, 0, sizeof(int), s));
    DRPT_TRY(launch_standardise(Q, x->dtype, nq, d, x->d_pad, nullptr, x->c, x->inv_sigma, x->qxb,
                                nullptr, s));
    DRPT_TRY(launch_mlp_infer(x->qxb, nq, x->d_pad, x->w1b, x->Tl * (x->gd - 1), x->b1, x->w2,
                              x->b2, x->Pq + (int64_t)x->ncols_r * nq, x->err, s));
  }
  DRPT_TRY(launch_descend(x->Pq, nq, T, x->gd, x->medians, x->leaf, s));
  int32_t *oi = on_device ? out_idx : x->qi;
  float *od = on_device ? (out_dist ? out_dist : x->qd) : x->qd;
  DRPT_TRY(launch_query(x->X, x->dtype, d, x->n, Q, nq, T, x->order, x->goff, x->nleaf, x->leaf,
                        k, oi, od, s));
  if (!on_device) {
    DRPT_CUDA(cudaMemcpyAsync(out_idx, oi, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, s));
    if (out_dist)
      DRPT_CUDA(cudaMemcpyAsync(out_dist, od, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, s));
  }
  if (x->Tl > 0) {
    int herr = 0;
    DRPT_CUDA(cudaMemcpyAsync(&herr, x->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    DRPT_CUDA(cudaStreamSynchronize(s));
    if (herr) {
      set_error("a bounded wait in the split-MLP inference kernel gave up");
      return DRPT_ERR_TIMEOUT;
    }
  }
  if (!on_device) DRPT_CUDA(cudaStreamSynchronize(s));
  return DRPT_OK;
}

drpt_status drpt_project(drpt_ctx *c, const void *X, int64_t n, int32_t d, int32_t dtype,
                         const float *B_host, int32_t L, const int32_t *cols_host, int32_t ncols,
                         float *P, void *stream) {
  if (!c || !X || !B_host || !cols_host || !P || n <= 0 || d <= 0 || L <= 0 || ncols <= 0 ||
      (dtype != DRPT_DTYPE_F32 && dtype != DRPT_DTYPE_U8))
    return DRPT_ERR_INVALID_ARG;
  for (int q = 0; q < ncols; ++q)
    if (cols_host[q] < 0 || cols_host[q] >= L) return DRPT_ERR_INVALID_ARG;
  DRPT_CUDA(cudaSetDevice(c->device));
  std::vector<int32_t> cols(cols_host, cols_host + ncols);
  return project_cols(c, X, dtype, n, d, B_host, L, cols, P, (cudaStream_t)stream);
}

drpt_status drpt_project_sign(drpt_ctx *c, const uint8_t *X, int64_t n, int32_t d,
                              const float *B_host, int32_t L, const int32_t *cols_host,
                              int32_t ncols, float *P, void *stream) {
  if (!c || !X || !B_host || !cols_host || !P || n <= 0 || d <= 0 || L <= 0 || ncols <= 0) {
    set_error("drpt_project_sign: null pointer or empty size");
    return DRPT_ERR_INVALID_ARG;
  }
  for (int q = 0; q < ncols; ++q)
    if (cols_host[q] < 0 || cols_host[q] >= L) {
      set_error("drpt_project_sign: column %d outside [0, %d)", cols_host[q], L);
      return DRPT_ERR_INVALID_ARG;
    }
  DRPT_CUDA(cudaSetDevice(c->device));
  std::vector<int32_t> cols(cols_host, cols_host + ncols);
  const cudaStream_t s = (cudaStream_t)stream;
  DRPT_TRY(project_sign(c, X, n, d, B_host, L, cols, P, s));
  int serr = 0;
  DRPT_CUDA(cudaMemcpyAsync(&serr, c->bufs["sgn_err"].p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DRPT_CUDA(cudaStreamSynchronize(s));
  if (serr) {
    set_error("a bounded wait in the sign-matrix projection gave up");
    return DRPT_ERR_TIMEOUT;
  }
  return DRPT_OK;
}

drpt_status drpt_global_trees(drpt_ctx *c, const float *P, int64_t n, int32_t T, int32_t gd,
                              int32_t exact, int32_t *order, int32_t *offsets, float *medians,
                              void *stream) {
  if (!c || !P || !order || !offsets || n < 2 || n > INT32_MAX || T <= 0 || gd <= 0 || gd > 30)
    return DRPT_ERR_INVALID_ARG;
  DRPT_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = (cudaStream_t)stream;
  int32_t *o, *f;
  DRPT_TRY(global_trees(c, P, n, T, gd, exact, medians, &o, &f, s));
  DRPT_CUDA(cudaMemcpyAsync(order, o, (size_t)T * n * 4, cudaMemcpyDeviceToDevice, s));
  DRPT_CUDA(cudaMemcpyAsync(offsets, f, (size_t)T * ((1 << (gd - 1)) + 1) * 4,
                            cudaMemcpyDeviceToDevice, s));
  return DRPT_OK;
}

drpt_status drpt_locality_slots(const int32_t *order, const int32_t *offsets, int64_t n, int32_t T,
                                int32_t nleaf, int32_t *slot_leaf, int32_t *order_out,
                                int32_t *offsets_out) {
  if (!order || !offsets || !slot_leaf || n < 1 || n > INT32_MAX || T <= 0 || nleaf <= 0 ||
      (nleaf & (nleaf - 1)) != 0 || (!order_out) != (!offsets_out)) {
    set_error("locality: invalid arguments");
    return DRPT_ERR_INVALID_ARG;
  }
  for (int t = 0; t < T; ++t) {
    const int32_t *o = offsets + (size_t)t * (nleaf + 1);
    if (o[0] != 0 || o[nleaf] != n) {
      set_error("locality: tree %d's leaf offsets do not cover the %lld points", t, (long long)n);
      return DRPT_ERR_INVALID_ARG;
    }
    for (int j = 0; j < nleaf; ++j)
      if (o[j + 1] < o[j]) {
        set_error("locality: tree %d's leaf offsets decrease", t);
        return DRPT_ERR_INVALID_ARG;
      }
  }
  for (size_t i = 0; i < (size_t)T * n; ++i)
    if (order[i] < 0 || order[i] >= n) {
      set_error("locality: point id %d out of range", order[i]);
      return DRPT_ERR_INVALID_ARG;
    }
  if (!host_locality_slots(T, nleaf, n, order, offsets, slot_leaf)) {
    set_error("locality: a slot found no free leaf (the reference reads index -1 there)");
    return DRPT_ERR_UNSUPPORTED;
  }
  if (order_out) {
    for (int t = 0; t < T; ++t) {
      const int32_t *o = offsets + (size_t)t * (nleaf + 1);
      int32_t *oo = offsets_out + (size_t)t * (nleaf + 1);
      int32_t w = 0;
      oo[0] = 0;
      for (int k = 0; k < nleaf; ++k) {
        const int leaf = slot_leaf[(size_t)k * T + t];
        for (int32_t i = o[leaf]; i < o[leaf + 1]; ++i)
          order_out[(size_t)t * n + w++] = order[(size_t)t * n + i];
        oo[k + 1] = w;
      }
    }
  }
  return DRPT_OK;
}

drpt_status drpt_local_leaves(drpt_ctx *c, const int32_t *order, const int32_t *offsets, int64_t n,
                              int32_t T, int32_t gd, int32_t ld, int32_t *final_order,
                              int32_t *final_offsets, void *stream) {
  if (!c || !order || !offsets || !final_order || !final_offsets || n < 2 || T <= 0 || gd <= 0 ||
      gd > 30 || ld <= 0)
    return DRPT_ERR_INVALID_ARG;
  DRPT_CUDA(cudaSetDevice(c->device));
  LocalPlan plan;
  return local_phase(c, order, offsets, n, T, gd, 1, 0, ld, 0, nullptr, 0, final_order,
                     final_offsets, &plan, (cudaStream_t)stream);
}

drpt_status drpt_leaf_knn(drpt_ctx *c, const void *X, int32_t dtype, int64_t n, int32_t d,
                          int32_t T, const int32_t *final_order, const int32_t *final_offsets,
                          int32_t n_final, int32_t k, int32_t *cand_idx, float *cand_dist,
                          void *stream) {
  if (!c || !X || !final_order || !final_offsets || !cand_idx || !cand_dist || n <= 0 || d <= 0 ||
      T <= 0 || n_final <= 0 || (dtype != DRPT_DTYPE_F32 && dtype != DRPT_DTYPE_U8))
    return DRPT_ERR_INVALID_ARG;
  DRPT_CUDA(cudaSetDevice(c->device));
  LeafKnnArgs ka{X, dtype, n, d, T, k, final_order, final_offsets, n_final, cand_idx, cand_dist};
  return launch_leaf_knn_exact(ka, (cudaStream_t)stream);
}

drpt_status drpt_merge_candidates(drpt_ctx *c, const int32_t *cand_idx, const float *cand_dist,
                                  int64_t n, int32_t T, int32_t k, int32_t *out_idx,
                                  float *out_dist, void *stream) {
  if (!c || !cand_idx || !cand_dist || !out_idx || !out_dist || n <= 0 || T <= 0)
    return DRPT_ERR_INVALID_ARG;
  DRPT_CUDA(cudaSetDevice(c->device));
  return launch_merge(cand_idx, cand_dist, n, T, k, k, out_idx, out_dist, (cudaStream_t)stream);
}

}  // extern "C"
