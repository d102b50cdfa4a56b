// drpt -- command-line k-NN-graph builder over libdrpt_gpu.so (one B200).
//
// Accepts the reference CLI's flags with their meaning and defaults
// (cpp/src/main.cpp:27-95) and writes the same two files:
//   <output>results.txt  the edge list, "src dst\n" 1-based, the first nn-1
//                        non-self neighbours of every point in ascending
//                        source order (file_writer.cpp:36-184 as called at
//                        main.cpp:227-228);
//   <output>stats.txt    appended, one line of phase times per run.
// It prints the reference's timing line (main.cpp:247-251).
//
// Flags added here: -seed (projection seed; default drawn from
// std::random_device as the reference draws it, mdrpt.cpp:402-416, and
// printed), -mode exact|fast|mixed|fp32_leaf|fp32_gram (default exact), -leaf-size,
// -tree-depth, -device.  -locality 1 runs the reference's locality
// relabelling in the exact and fast modes (off unless given: at one rank it
// only renumbers global leaves and the graph is the same).
//
// Input formats (-data-file-format), plain or gzip-compressed:
//   0  IDX3 ubyte (file_reader.cpp:33-83): big-endian header magic 0x803,
//      count, rows, cols, then count x rows x cols bytes.  The magic is
//      checked (the reference reads any header).
//   1  raw binary (file_reader.cpp:364-497): -data-starting-index header
//      bytes, then n x dimension values of -bytes-for-data-type bytes
//      (4 = float32, 1 = uint8).  The values are read as stored (the
//      reference replaces them with random draws).  With the 8-byte fbin
//      header (u32 n, u32 d) the header is checked against -dimension and
//      -data-set-size (the reference ignores it).
// Sizes are checked against the file; a short file is an error.
//
// Further flags: -precision bf16|fp8, -projection gaussian|sign (u8 rows) and
// -learned-trees N (mixed form),
// -write-distances 1 (a third column: the neighbour's Euclidean distance).

#include <drpt_gpu.h>
#include <zlib.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace {

struct Options {
  std::string input, output;
  long long n = 0;
  int dimension = 0, ntrees = 10, nn = 0, local_tree_offset = 2, file_format = 0;
  int bytes_for_data_type = 4, data_starting_index = 8, tree_depth = 0, leaf_size = 0;
  int device = 0;
  double tree_depth_ratio = 0.6, density = 0;
  bool have_seed = false;
  uint32_t seed = 0;
  int mode = DRPT_MODE_EXACT;
  int precision = DRPT_PRECISION_BF16;
  int projection = DRPT_PROJECTION_GAUSSIAN;
  int learned_trees = 0;
  int locality = 0;
  bool write_distances = false;
};

[[noreturn]] void die(const char *msg) {
  std::printf("%s\n", msg);
  std::exit(1);
}

int parse_mode(const char *s) {
  if (!std::strcmp(s, "exact")) return DRPT_MODE_EXACT;
  if (!std::strcmp(s, "fast")) return DRPT_MODE_FAST;
  if (!std::strcmp(s, "mixed")) return DRPT_MODE_MIXED;
  if (!std::strcmp(s, "fp32_leaf")) return DRPT_MODE_FP32_LEAF;
  if (!std::strcmp(s, "fp32_gram")) return DRPT_MODE_FP32_GRAM;
  die("-mode must be exact, fast, mixed, fp32_leaf or fp32_gram");
}

Options parse(int argc, char **argv) {
  Options o;
  for (int p = 1; p + 1 < argc; ++p) {
    const char *f = argv[p], *v = argv[p + 1];
    if (!std::strcmp(f, "-input")) o.input = v;
    else if (!std::strcmp(f, "-output")) o.output = v;
    else if (!std::strcmp(f, "-data-set-size")) o.n = std::atoll(v);
    else if (!std::strcmp(f, "-dimension")) o.dimension = std::atoi(v);
    else if (!std::strcmp(f, "-ntrees")) o.ntrees = std::atoi(v);
    else if (!std::strcmp(f, "-tree-depth-ratio")) o.tree_depth_ratio = std::strtof(v, nullptr);
    else if (!std::strcmp(f, "-density")) o.density = std::strtod(v, nullptr);
    else if (!std::strcmp(f, "-nn")) o.nn = std::atoi(v);
    else if (!std::strcmp(f, "-locality")) o.locality = std::atoi(v) == 1 ? 1 : 0;
    else if (!std::strcmp(f, "-local-tree-offset")) o.local_tree_offset = std::atoi(v);
    else if (!std::strcmp(f, "-data-file-format")) o.file_format = std::atoi(v);
    else if (!std::strcmp(f, "-bytes-for-data-type")) o.bytes_for_data_type = std::atoi(v);
    else if (!std::strcmp(f, "-data-starting-index")) o.data_starting_index = std::atoi(v);
    else if (!std::strcmp(f, "-seed")) { o.seed = (uint32_t)std::strtoul(v, nullptr, 10); o.have_seed = true; }
    else if (!std::strcmp(f, "-mode")) o.mode = parse_mode(v);
    else if (!std::strcmp(f, "-leaf-size")) o.leaf_size = std::atoi(v);
    else if (!std::strcmp(f, "-tree-depth")) o.tree_depth = std::atoi(v);
    else if (!std::strcmp(f, "-device")) o.device = std::atoi(v);
    else if (!std::strcmp(f, "-precision")) {
      if (!std::strcmp(v, "bf16")) o.precision = DRPT_PRECISION_BF16;
      else if (!std::strcmp(v, "fp8")) o.precision = DRPT_PRECISION_FP8_E4M3;
      else die("-precision must be bf16 or fp8");
    } else if (!std::strcmp(f, "-projection")) {
      if (!std::strcmp(v, "gaussian")) o.projection = DRPT_PROJECTION_GAUSSIAN;
      else if (!std::strcmp(v, "sign")) o.projection = DRPT_PROJECTION_SIGN;
      else die("-projection must be gaussian or sign");
    } else if (!std::strcmp(f, "-learned-trees")) o.learned_trees = std::atoi(v);
    else if (!std::strcmp(f, "-write-distances")) o.write_distances = std::atoi(v) == 1;
  }
  // The reference's checks, in its order and with its messages (main.cpp:97-130).
  if (o.input.empty()) die("Valid input path needed!...");
  if (o.output.empty()) die("Valid out path needed!...");
  if (o.n == 0) die("Dataset size should be greater than 0");
  if (o.dimension == 0) die("Dimension size should be greater than 0");
  if (o.nn == 0) die("Nearest neighbours size should be greater than 0");
  if (o.density == 0) o.density = 1.0 / std::sqrt((double)o.dimension);
  return o;
}

uint32_t be32(const unsigned char *b) {
  return ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
}

// gzread reads plain files unchanged, so one reader serves both.
bool read_exact(gzFile f, void *dst, size_t bytes) {
  unsigned char *p = static_cast<unsigned char *>(dst);
  while (bytes > 0) {
    const unsigned chunk = (unsigned)std::min<size_t>(bytes, 1u << 30);
    const int got = gzread(f, p, chunk);
    if (got <= 0) return false;
    p += got;
    bytes -= (size_t)got;
  }
  return true;
}

uint32_t le32(const unsigned char *b) {
  return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
}

// Returns the row-major n x d values; *dtype receives their drpt_dtype.
std::vector<unsigned char> read_input(const Options &o, int *dtype) {
  gzFile f = gzopen(o.input.c_str(), "rb");
  if (!f) die("cannot open the input file");
  gzbuffer(f, 1 << 20);
  const size_t n = (size_t)o.n, d = (size_t)o.dimension;
  std::vector<unsigned char> buf;
  if (o.file_format == 0) {
    unsigned char h[16];
    if (!read_exact(f, h, 16)) die("input file shorter than an IDX3 header");
    if (be32(h) != 0x00000803u) die("not an IDX3 ubyte file (magic is not 0x00000803)");
    const uint32_t count = be32(h + 4), rows = be32(h + 8), cols = be32(h + 12);
    if ((size_t)rows * cols != d) die("IDX3 rows x cols differs from -dimension");
    if (count < n) die("IDX3 file holds fewer images than -data-set-size");
    buf.resize(n * d);
    if (!read_exact(f, buf.data(), buf.size())) die("IDX3 file shorter than its header says");
    *dtype = DRPT_DTYPE_U8;
  } else if (o.file_format == 1) {
    if (o.bytes_for_data_type != 4 && o.bytes_for_data_type != 1)
      die("-bytes-for-data-type must be 4 (float32) or 1 (uint8)");
    if (o.data_starting_index < 0) die("-data-starting-index must be >= 0");
    std::vector<unsigned char> hdr((size_t)o.data_starting_index);
    if (!hdr.empty() && !read_exact(f, hdr.data(), hdr.size()))
      die("input file shorter than its header");
    if (o.data_starting_index == 8) {  // fbin: u32 n, u32 d
      if (le32(hdr.data() + 4) != (uint32_t)o.dimension)
        die("fbin header dimension differs from -dimension");
      if (le32(hdr.data()) < (uint32_t)n) die("fbin header holds fewer points than -data-set-size");
    }
    buf.resize(n * d * (size_t)o.bytes_for_data_type);
    if (!read_exact(f, buf.data(), buf.size()))
      die("binary file holds fewer than -data-set-size x -dimension values");
    *dtype = o.bytes_for_data_type == 4 ? DRPT_DTYPE_F32 : DRPT_DTYPE_U8;
  } else {
    die("Unsupported data file format, ubyte and bin file formats are supported!...");
  }
  gzclose(f);
  return buf;
}

char *put_uint(char *p, uint32_t v) {
  char tmp[12];
  int k = 0;
  do { tmp[k++] = (char)('0' + v % 10); v /= 10; } while (v);
  while (k) *p++ = tmp[--k];
  return p;
}

// Edge list: every source in ascending order, its first `per_point` entries.
bool write_edges(const std::string &path, const std::vector<int32_t> &idx,
                 const std::vector<float> *dist, long long n, int nn, int per_point) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  std::vector<char> out;
  out.reserve(1 << 22);
  for (long long p = 0; p < n; ++p) {
    const int32_t *row = idx.data() + p * nn;
    for (int j = 0; j < per_point; ++j) {
      if (row[j] < 0) break;
      char line[64];
      char *q = put_uint(line, (uint32_t)(p + 1));
      *q++ = ' ';
      q = put_uint(q, (uint32_t)row[j] + 1);
      if (dist) q += std::snprintf(q, 20, " %.9g", (double)(*dist)[p * nn + j]);
      *q++ = '\n';
      out.insert(out.end(), line, q);
    }
    if (out.size() > (1u << 22)) {
      if (std::fwrite(out.data(), 1, out.size(), f) != out.size()) { std::fclose(f); return false; }
      out.clear();
    }
  }
  const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
  return std::fclose(f) == 0 && ok;
}

}  // namespace

int main(int argc, char **argv) {
  using clk = std::chrono::high_resolution_clock;
  const Options o = parse(argc, argv);

  const auto t_io0 = clk::now();
  int dtype = DRPT_DTYPE_F32;
  std::vector<unsigned char> data = read_input(o, &dtype);
  const auto t_io1 = clk::now();

  uint32_t seed = o.seed;
  if (!o.have_seed) seed = std::random_device{}();
  std::mt19937 seeder(seed ^ 0x9e3779b9u);
  std::vector<uint32_t> local_seeds((size_t)o.ntrees);
  for (auto &s : local_seeds) s = seeder();

  drpt_ctx *ctx = nullptr;
  if (drpt_ctx_create(&ctx, o.device) != DRPT_OK) {
    std::printf("drpt: %s\n", drpt_last_error());
    return 1;
  }
  drpt_build_desc desc;
  std::memset(&desc, 0, sizeof desc);
  desc.n = o.n;
  desc.d = o.dimension;
  desc.dtype = dtype;
  desc.ntrees = o.ntrees;
  desc.nn = o.nn;
  desc.tree_depth_ratio = o.tree_depth_ratio;
  desc.local_tree_offset = o.local_tree_offset;
  desc.tree_depth = o.tree_depth;
  desc.density = o.density;
  desc.seed = seed;
  desc.local_seeds = local_seeds.data();
  desc.mode = o.mode;
  desc.leaf_size = o.leaf_size;
  desc.precision = o.precision;
  desc.projection = o.projection;
  desc.learned_trees = o.learned_trees;
  desc.locality = o.locality;
  std::vector<int32_t> idx((size_t)o.n * o.nn);
  std::vector<float> dist(o.write_distances ? (size_t)o.n * o.nn : 0);
  drpt_stats st;
  std::memset(&st, 0, sizeof st);
  const drpt_status rc = drpt_build_graph(ctx, &desc, data.data(), idx.data(),
                                          o.write_distances ? dist.data() : nullptr, &st);
  if (rc != DRPT_OK) {
    std::printf("drpt: status %d: %s\n", (int)rc, drpt_last_error());
    drpt_ctx_destroy(ctx);
    return 1;
  }
  drpt_ctx_destroy(ctx);
  std::printf(" tree depth %d global depth %d local depth %d seed %u\n", st.tree_depth,
              st.global_depth, st.local_depth, seed);

  const auto t_w0 = clk::now();
  if (!write_edges(o.output + "results.txt", idx, o.write_distances ? &dist : nullptr, o.n, o.nn,
                   o.nn - 1)) {
    std::printf("drpt: cannot write %sresults.txt\n", o.output.c_str());
    return 1;
  }
  const auto t_w1 = clk::now();

  const double io_s = std::chrono::duration<double>((t_io1 - t_io0) + (t_w1 - t_w0)).count();
  // Index building = projection + trees (+ local split); querying = leaf
  // brute force + merge, as grow_trees / gather_nns divide the work.
  const double build_s = (st.ms_project + st.ms_global + st.ms_local) / 1e3;
  const double query_s = (st.ms_total - st.ms_project - st.ms_global - st.ms_local) / 1e3;
  std::printf("IO Time (s)%g Index building (s) %g Querying Time (s) %g\n", io_s, build_s, query_s);
  if (FILE *sf = std::fopen((o.output + "stats.txt").c_str(), "a")) {
    std::fprintf(sf, "n %lld d %d ntrees %d nn %d mode %d seed %u io_s %g build_s %g query_s %g\n",
                 o.n, o.dimension, o.ntrees, o.nn, o.mode, seed, io_s, build_s, query_s);
    std::fclose(sf);
  }
  return 0;
}
