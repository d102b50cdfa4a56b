// Test driver of the reference-side binding: reads an fbin file (u32 n,
// u32 d, n x d float32), builds the graph through drpt_gpu_knn_graph and
// writes the edge list with the reference's own FileWriter<int>, called as
// main.cpp:227-228 calls it (nn - 1 edges, self edges filtered).
//
//   adapter_check <in.fbin> <out_dir/> <ntrees> <nn> <seed>
// Exit status 0 on success, 2 on a usage or input error, 3 when the graph
// call throws (its message on stderr).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>
#include <vector>

#include "drpt/io/file_writer.hpp"
#include "drpt_gpu_adapter.hpp"

int main(int argc, char **argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s <in.fbin> <out_dir/> <ntrees> <nn> <seed>\n", argv[0]);
    return 2;
  }
  FILE *f = std::fopen(argv[1], "rb");
  uint32_t hdr[2];
  if (!f || std::fread(hdr, 4, 2, f) != 2) {
    std::fprintf(stderr, "cannot read %s\n", argv[1]);
    return 2;
  }
  std::vector<std::vector<float>> rows(hdr[0], std::vector<float>(hdr[1]));
  for (auto &r : rows)
    if (std::fread(r.data(), 4, r.size(), f) != r.size()) {
      std::fprintf(stderr, "%s is truncated\n", argv[1]);
      return 2;
    }
  std::fclose(f);
  const int ntrees = std::atoi(argv[3]), nn = std::atoi(argv[4]);
  try {
    auto points = drpt_gpu_knn_graph(rows, ntrees, nn, 0.6, 2, (unsigned)std::strtoul(argv[5], nullptr, 10));
    drpt::FileWriter<int> writer;
    writer.mpi_write_edge_list(points, std::string(argv[2]) + "results.txt", nn - 1, 0, 1, true);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "drpt_gpu_knn_graph: %s\n", e.what());
    return 3;
  }
  return 0;
}
