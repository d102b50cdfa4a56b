// Driver for the reference DRPT library built from its own sources (test
// infrastructure and the timed CPU baseline; never part of the product).
//
// It follows the reference CLI (cpp/src/main.cpp:25-259) step for step:
// flags (main.cpp:43-97), validation (:99-127), default density (:129-132),
// derived tree depth (:141-145), MDRPT construction and grow_trees (:196-206),
// gather_nns (:215-217), the edge-list writer (:226-228) and the timing line
// (:235-251).  Differences, all outside the timed region:
//  * fbin input is read here (header skipped by -data-starting-index, then
//    n*d little-endian floats).  The reference's fbin reader replaces every
//    value with a fresh random number (file_reader.cpp:476-485), so it cannot
//    serve as an oracle.  ubyte input goes through the reference's own
//    ImageReader::read_ubyte (file_reader.cpp:33-87).
//  * -dump <file> writes the projection matrix, the final leaves of every
//    tree and every point's merged neighbour list in a binary layout read by
//    the Python test helpers (oracle/refdump.py); -dump-p adds P = X.B.
//  * -no-write skips the edge-list file.
//  * -median-test <in> <out> runs only MathOp::distributed_mean / _variance /
//    _median (math_operations.cpp:121-383) on the nodes stored in <in>
//    (int32 nodes, int32 sizes[nodes], float values...) and writes
//    float mean[nodes], var[nodes], median[nodes] to <out>.
// Seeds come from DRPT_REF_SEEDS (see seed_inject.cpp).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <omp.h>
#include <random>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

#include "cblas.h"
#include "mpi.h"

// The dump needs MDRPT's private leaf table (mdrpt.hpp:32-33).  Member layout
// does not depend on access specifiers in GCC, so reading it this way is
// consistent with the separately compiled mdrpt.cpp.
#define private public
#include "drpt/algo/mdrpt.hpp"
#undef private
#include "drpt/io/file_reader.hpp"
#include "drpt/io/file_writer.hpp"

using namespace std;
using namespace std::chrono;

static vector<vector<float>> read_fbin(const string &path, long n, int d, long start) {
  vector<vector<float>> out;
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) {
    fprintf(stderr, "ref_driver: cannot open %s\n", path.c_str());
    exit(1);
  }
  if (fseek(f, start, SEEK_SET) != 0) {
    fprintf(stderr, "ref_driver: seek failed\n");
    exit(1);
  }
  out.assign(n, vector<float>(d));
  for (long i = 0; i < n; ++i) {
    if (fread(out[i].data(), sizeof(float), d, f) != (size_t)d) {
      fprintf(stderr, "ref_driver: %s holds fewer than %ld points\n", path.c_str(), n);
      exit(1);
    }
  }
  fclose(f);
  return out;
}

template <typename T>
static void put(FILE *f, const T &v) {
  fwrite(&v, sizeof(T), 1, f);
}

static int median_test(const char *in_path, const char *out_path) {
  FILE *f = fopen(in_path, "rb");
  if (!f) return 1;
  int32_t nodes = 0;
  if (fread(&nodes, 4, 1, f) != 1) return 1;
  vector<int> sizes(nodes);
  if (fread(sizes.data(), 4, nodes, f) != (size_t)nodes) return 1;
  long total = 0;
  for (int s : sizes) total += s;
  vector<float> data(total);
  if (fread(data.data(), 4, total, f) != (size_t)total) return 1;
  fclose(f);
  drpt::MathOp op;
  float *mean = op.distributed_mean(data, sizes, nodes, sizes, drpt::StorageFormat::RAW, 0);
  float *var = op.distributed_variance(data, sizes, nodes, sizes, drpt::StorageFormat::RAW, 0);
  float *med = op.distributed_median(data, sizes, nodes, sizes, 7, drpt::StorageFormat::RAW, 0);
  FILE *o = fopen(out_path, "wb");
  fwrite(mean, 4, nodes, o);
  fwrite(var, 4, nodes, o);
  fwrite(med, 4, nodes, o);
  fclose(o);
  return 0;
}

int main(int argc, char *argv[]) {
  for (int p = 0; p + 2 < argc; p++)
    if (strcmp(argv[p], "-median-test") == 0) return median_test(argv[p + 1], argv[p + 2]);
  string input_path, output_path, dump_path;
  long data_set_size = 0;
  int dimension = 0, ntrees = 10, tree_depth = 0, nn = 0;
  double density = 0, tree_depth_ratio = 0.6;
  bool use_locality_optimization = true, dump_p = false, write_edges = true;
  int local_tree_offset = 2, file_format = 0, data_starting_index = 8;
  int bytes_for_data_type = 4;

  for (int p = 0; p < argc; p++) {
    auto arg = [&](const char *name) { return strcmp(argv[p], name) == 0 && p + 1 < argc; };
    if (arg("-input")) input_path = argv[p + 1];
    else if (arg("-output")) output_path = argv[p + 1];
    else if (arg("-data-set-size")) data_set_size = atol(argv[p + 1]);
    else if (arg("-dimension")) dimension = atoi(argv[p + 1]);
    else if (arg("-ntrees")) ntrees = atoi(argv[p + 1]);
    else if (arg("-tree-depth-ratio")) tree_depth_ratio = stof(argv[p + 1]);
    else if (arg("-density")) density = atoi(argv[p + 1]);
    else if (arg("-nn")) nn = atoi(argv[p + 1]);
    else if (arg("-locality")) use_locality_optimization = atoi(argv[p + 1]) == 1;
    else if (arg("-local-tree-offset")) local_tree_offset = atoi(argv[p + 1]);
    else if (arg("-data-file-format") || arg("-file_format")) file_format = atoi(argv[p + 1]);
    else if (arg("-bytes-for-data-type")) bytes_for_data_type = atoi(argv[p + 1]);
    else if (arg("-data-starting-index")) data_starting_index = atoi(argv[p + 1]);
    else if (arg("-dump")) dump_path = argv[p + 1];
    else if (strcmp(argv[p], "-dump-p") == 0) dump_p = true;
    else if (strcmp(argv[p], "-no-write") == 0) write_edges = false;
  }
  if (input_path.empty()) { printf("Valid input path needed!...\n"); exit(1); }
  if (output_path.empty()) { printf("Valid out path needed!...\n"); exit(1); }
  if (data_set_size == 0) { printf("Dataset size should be greater than 0\n"); exit(1); }
  if (dimension == 0) { printf("Dimension size should be greater than 0\n"); exit(1); }
  if (nn == 0) { printf("Nearest neighbours size should be greater than 0\n"); exit(1); }
  if (bytes_for_data_type != 4) { printf("only 4-byte fbin values are supported\n"); exit(1); }
  if (density == 0) density = 1.0 / sqrt(dimension);

  int rank, size;
  MPI_Init(&argc, &argv);
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  MPI_Comm_size(MPI_COMM_WORLD, &size);
  if (tree_depth == 0) tree_depth = static_cast<int>(log2((data_set_size / size)) - 2);

  ofstream fout(output_path + "stats.txt", std::ios_base::app);
  auto t_io0 = high_resolution_clock::now();
  vector<vector<float>> imagedatas;
  drpt::ImageReader imageReader;
  if (file_format == 0)
    imagedatas = imageReader.read_ubyte(input_path, data_set_size, dimension, rank, size);
  else if (file_format == 1)
    imagedatas = read_fbin(input_path, data_set_size, dimension, data_starting_index);
  else {
    printf("Unsupported data file format, ubyte and bin file formats are supported!...\n");
    exit(1);
  }
  auto t_io1 = high_resolution_clock::now();
  if ((long)imagedatas.size() != data_set_size) {
    fprintf(stderr, "ref_driver: read %zu points, expected %ld\n", imagedatas.size(), data_set_size);
    exit(1);
  }

  int rows = imagedatas[0].size();
  int cols = imagedatas.size();
  MPI_Barrier(MPI_COMM_WORLD);
  // grow_trees converts `imagedatas` in place into nothing, but keep a copy for
  // the optional P dump, which must see the same input.
  vector<vector<float>> data_copy;
  if (dump_p) data_copy = imagedatas;

  auto t_b0 = high_resolution_clock::now();
  drpt::MDRPT mdrpt(ntrees, tree_depth, tree_depth_ratio, local_tree_offset, data_set_size, cols,
                    rows, rank, size, input_path, output_path);
  mdrpt.grow_trees(imagedatas, density, use_locality_optimization, nn, fout);
  auto t_b1 = high_resolution_clock::now();
  auto t_q0 = high_resolution_clock::now();
  map<int, vector<drpt::DataPoint>> data_points = mdrpt.gather_nns(nn, fout);
  auto t_q1 = high_resolution_clock::now();

  auto t_w0 = high_resolution_clock::now();
  if (write_edges) {
    drpt::FileWriter<int> fileWriter;
    fileWriter.mpi_write_edge_list(data_points, output_path + "results.txt", nn - 1, rank, size,
                                   true);
  }
  auto t_w1 = high_resolution_clock::now();

  double io_ms = (duration_cast<microseconds>(t_io1 - t_io0).count() +
                  duration_cast<microseconds>(t_w1 - t_w0).count()) / 1000.0;
  double build_ms = duration_cast<microseconds>(t_b1 - t_b0).count() / 1000.0;
  double query_ms = duration_cast<microseconds>(t_q1 - t_q0).count() / 1000.0;
  cout << "IO Time (s)" << io_ms / 1000 << " Index building (s) " << build_ms / 1000
       << " Querying Time (s) " << query_ms / 1000 << endl;

  if (!dump_path.empty()) {
    int gd = (int)(tree_depth * tree_depth_ratio);
    int total_depth = mdrpt.tree_depth;  // local + global depth after grow_trees
    int ld = total_depth - gd;
    int L = gd * ntrees;
    int n_final = (int)mdrpt.trees_leaf_all[0].size();
    const char *env = getenv("DRPT_REF_SEEDS");
    unsigned seed0 = env ? (unsigned)strtoul(env, nullptr, 0) : 0u;
    drpt::MathOp mathOp;
    float *B = mathOp.build_sparse_projection_matrix(0, 1, dimension, L, (float)density, (int)seed0);
    FILE *f = fopen(dump_path.c_str(), "wb");
    fwrite("DRPTREF1", 1, 8, f);
    int32_t hdr[8] = {(int32_t)data_set_size, dimension, ntrees, nn, gd, ld, n_final, dump_p ? 1 : 0};
    fwrite(hdr, sizeof(int32_t), 8, f);
    put(f, (double)density);
    fwrite(B, sizeof(float), (size_t)dimension * L, f);
    free(B);
    if (dump_p) {
      float *X = mathOp.convert_to_row_major_format(data_copy);
      float *B2 = mathOp.build_sparse_projection_matrix(0, 1, dimension, L, (float)density, (int)seed0);
      float *P = mathOp.multiply_mat(X, B2, dimension, L, (int)data_set_size, 1.0);
      fwrite(P, sizeof(float), (size_t)data_set_size * L, f);
      free(P);
      free(B2);
      free(X);
    }
    for (int t = 0; t < ntrees; ++t)
      for (int leaf = 0; leaf < n_final; ++leaf) {
        const vector<drpt::DataPoint> &lv = mdrpt.trees_leaf_all[t][leaf];
        put(f, (int32_t)lv.size());
        for (const auto &dp : lv) put(f, (int32_t)dp.index);
      }
    put(f, (int32_t)data_points.size());
    for (const auto &kv : data_points) {
      put(f, (int32_t)kv.first);
      put(f, (int32_t)kv.second.size());
      for (const auto &dp : kv.second) {
        put(f, (int32_t)dp.index);
        put(f, (float)dp.distance);
      }
    }
    fclose(f);
  }
  MPI_Finalize();
  return 0;
}
