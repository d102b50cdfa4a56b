// drpt_gpu_adapter.cpp -- for the reference tree, built with -I<drpt-b200>/include
// (the binding INTEGRATION.md shows; declared in drpt_gpu_adapter.hpp).
#include "drpt_gpu_adapter.hpp"

#include <drpt_gpu.h>

#include <algorithm>
#include <stdexcept>

std::map<int, std::vector<drpt::DataPoint>>
drpt_gpu_knn_graph(const std::vector<std::vector<float>> &rows, int ntrees, int nn,
                   double tree_depth_ratio, int local_tree_offset, unsigned seed) {
  const int64_t n = rows.size();
  const int d = rows[0].size();
  std::vector<float> X(n * d);
  for (int64_t i = 0; i < n; ++i) std::copy(rows[i].begin(), rows[i].end(), &X[i * d]);
  drpt_ctx *ctx = nullptr;
  if (drpt_ctx_create(&ctx, 0)) throw std::runtime_error(drpt_last_error());
  drpt_build_desc desc{};
  desc.n = n; desc.d = d; desc.dtype = DRPT_DTYPE_F32; desc.ntrees = ntrees; desc.nn = nn;
  desc.tree_depth_ratio = tree_depth_ratio; desc.local_tree_offset = local_tree_offset;
  desc.seed = seed; desc.mode = DRPT_MODE_EXACT;
  std::vector<int32_t> idx(n * nn);
  std::vector<float> dist(n * nn);
  const drpt_status st = drpt_build_graph(ctx, &desc, X.data(), idx.data(), dist.data(), nullptr);
  drpt_ctx_destroy(ctx);
  if (st == DRPT_ERR_DEPTH_OUT_OF_RANGE) throw std::out_of_range(drpt_last_error());
  if (st != DRPT_OK) throw std::runtime_error(drpt_last_error());
  std::map<int, std::vector<drpt::DataPoint>> out;
  for (int64_t p = 0; p < n; ++p)
    for (int j = 0; j < nn && idx[p * nn + j] >= 0; ++j)
      out[p].push_back({(int)p, idx[p * nn + j], dist[p * nn + j], 0.0f, {}});
  return out;
}
