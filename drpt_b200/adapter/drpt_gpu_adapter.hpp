// The reference-side binding of libdrpt_gpu.so: one call that stands in for
// the MDRPT construction, grow_trees and gather_nns of the reference's
// main.cpp:198-217 (one rank) and returns the map its FileWriter consumes
// (main.cpp:227-228).  Compiled inside the reference tree against its
// drpt/algo/drpt_local.hpp (drpt::DataPoint) and include/drpt_gpu.h.
#pragma once

#include <map>
#include <vector>

#include "drpt/algo/drpt_local.hpp"

// rows: the reference's vector<vector<float>> of the input (n rows of d
// values).  Throws std::out_of_range where the reference does (local depth
// checks) and std::runtime_error on any other failure.
std::map<int, std::vector<drpt::DataPoint>>
drpt_gpu_knn_graph(const std::vector<std::vector<float>> &rows, int ntrees, int nn,
                   double tree_depth_ratio, int local_tree_offset, unsigned seed);
