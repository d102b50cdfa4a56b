// drpt_global_trees_noalloc: the global-tree build of drpt_global_trees for
// callers that must not allocate device memory.
//
// Who needs it: hosts that hand every byte of HBM to their own pool before
// they call into this library (a caching allocator that reserved the device
// up front, a graph service with a fixed memory budget), where a cudaMalloc
// either fails or makes the pool release memory and synchronise the device,
// and latency-bound loops that cannot take cudaMalloc/cudaFree's implicit
// device-wide synchronisation.  drpt_global_trees keeps its ping-pong and
// per-level scratch in a context workspace that grows with cudaMalloc; this
// entry point keeps that scratch in g_static_scratch below instead, and uses
// the caller's `order` and `offsets` outputs as one side of the level
// ping-pong.  It runs the same level kernels (k_tree.cu) on the same inputs,
// so its outputs are identical.
//
// The array is part of the library's device image: every GPU that loads the
// library holds kStaticScratchBytes of it until the process exits.  All calls
// on a device share it and it keeps the last call's contents; the level
// kernels write every scratch entry before they read it, so nothing has to be
// cleared between calls.  Calls whose kernels overlap on the GPU (two streams,
// two host threads) race on the array: serialise them.
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

namespace {

constexpr size_t kStaticScratchBytes = size_t(64) << 20;  // 64 MiB per device
constexpr int kMaxDevices = 64;

}  // namespace

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace drpt {
namespace {

// In host code g_static_scratch names a host-side stand-in, not device
// memory: the kernels get the address cudaGetSymbolAddress returns for the
// current device, looked up once per device.
std::mutex g_addr_mu;
unsigned char *g_addr[kMaxDevices];

drpt_status static_scratch(unsigned char **out) {
  int dev = 0;
  DRPT_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device %d outside the %d devices the static scratch tracks", dev, kMaxDevices);
    return DRPT_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_addr_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) {
      set_error("cudaGetSymbolAddress(static scratch) on device %d: %s", dev,
                cudaGetErrorString(e));
      return DRPT_ERR_CUDA;
    }
    g_addr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_addr[dev];
  return DRPT_OK;
}

// Hands out 256-byte aligned pieces of [base, base + cap); with base ==
// nullptr it only adds up the bytes.
struct Carver {
  unsigned char *base;
  size_t used = 0;
  template <typename T>
  T *take(size_t count) {
    used = (used + 255) & ~size_t(255);
    T *p = base ? reinterpret_cast<T *>(base + used) : nullptr;
    used += count * sizeof(T);
    return p;
  }
};

// Scratch of a build with global depth gd >= 2, carved from `base`.
struct Layout {
  int32_t *ord_tmp;   // T x n: the ping-pong side that is not `order`
  float *val[2];      // T x n each: split values of the next level
  int32_t *off_tmp;   // T x (nleaf + 1): the side that is not `offsets`
  TreeLevelArgs lv;   // per-level scratch, sized for the deepest level
};

size_t carve(unsigned char *base, int64_t n, int T, int gd, Layout *L) {
  Carver c{base};
  const int nleaf = 1 << (gd - 1);
  const bool deep = gd >= 3;  // two or more levels: intermediates exist
  L->ord_tmp = deep ? c.take<int32_t>((size_t)T * n) : nullptr;
  L->val[0] = deep ? c.take<float>((size_t)T * n) : nullptr;
  L->val[1] = deep ? c.take<float>((size_t)T * n) : nullptr;
  L->off_tmp = deep ? c.take<int32_t>((size_t)T * (nleaf + 1)) : nullptr;
  const int last = gd - 2;
  const int64_t G = (int64_t)T << last;
  const int64_t U = tree_level_max_units(n, T, last);
  TreeLevelArgs &a = L->lv;
  a.node_ubase = c.take<int32_t>(G + 1);
  a.unit_node = c.take<int32_t>(U);
  a.unit_lo = c.take<int32_t>(U);
  a.n_units = c.take<int32_t>(1);
  a.node_D = c.take<float>(G * kBins);
  a.unit_s = c.take<double>(2 * U);
  a.unit_hist = c.take<unsigned>(U * kBins);
  a.node_med = c.take<float>(G);
  a.unit_left = c.take<int32_t>(U);
  a.unit_lbase = c.take<int32_t>(U);
  a.node_nleft = c.take<int32_t>(G);
  return c.used;
}

// gd == 1: one global leaf per tree holding every point in index order.
__global__ void k_single_leaf(int64_t n, int T, int32_t *order, int32_t *offsets) {
  const int64_t total = (int64_t)T * n;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += stride)
    order[i] = (int32_t)(i % n);
  if (blockIdx.x == 0)
    for (int j = threadIdx.x; j < 2 * T; j += blockDim.x) offsets[j] = (j & 1) ? (int32_t)n : 0;
}

}  // namespace
}  // namespace drpt

extern "C" drpt_status drpt_global_trees_noalloc(const float *P, int64_t n, int32_t T, int32_t gd,
                                                 int32_t exact, int32_t *order, int32_t *offsets,
                                                 float *medians, void *stream) {
  using namespace drpt;
  if (!P || !order || !offsets) {
    set_error("drpt_global_trees_noalloc: P, order and offsets must be device pointers (got "
              "P=%p order=%p offsets=%p)", (const void *)P, (void *)order, (void *)offsets);
    return DRPT_ERR_INVALID_ARG;
  }
  if (n < 2 || n > INT32_MAX || T <= 0 || gd <= 0 || gd > 30) {
    set_error("drpt_global_trees_noalloc: n=%lld (2 .. 2^31-1), T=%d (>= 1) or gd=%d (1 .. 30) "
              "out of range", (long long)n, T, gd);
    return DRPT_ERR_INVALID_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (gd == 1) {
    const int64_t blocks = min64(ceil_div((int64_t)T * n, 256), (int64_t)device_sm_count() * 8);
    k_single_leaf<<<(unsigned)blocks, 256, 0, s>>>(n, T, order, offsets);
    DRPT_LAUNCH_CHECK();
    return DRPT_OK;
  }
  Layout L{};
  const size_t need = carve(nullptr, n, T, gd, &L);
  if (need > kStaticScratchBytes) {
    set_error("drpt_global_trees_noalloc: n=%lld, T=%d, gd=%d needs %zu bytes of scratch; the "
              "static scratch holds %zu (use drpt_global_trees for this size)",
              (long long)n, T, gd, need, kStaticScratchBytes);
    return DRPT_ERR_INVALID_ARG;
  }
  unsigned char *base = nullptr;
  DRPT_TRY(static_scratch(&base));
  carve(base, n, T, gd, &L);
  // The last level writes ord[cur ^ 1] with cur = (gd - 2) & 1: make that the
  // caller's arrays so the result needs no copy.
  const int fin = (gd - 1) & 1;
  int32_t *ord[2], *off[2];
  ord[fin] = order;
  ord[fin ^ 1] = L.ord_tmp;
  off[fin] = offsets;
  off[fin ^ 1] = L.off_tmp;
  TreeLevelArgs a = L.lv;
  int cur = 0;
  for (int level = 0; level < gd - 1; ++level) {
    a.P = P;
    a.n = n;
    a.T = T;
    a.gd = gd;
    a.level = level;
    a.ord_in = level == 0 ? nullptr : ord[cur];
    a.val_in = level == 0 ? nullptr : L.val[cur];
    a.off_in = level == 0 ? nullptr : off[cur];
    a.ord_out = ord[cur ^ 1];
    a.val_out = level + 1 < gd - 1 ? L.val[cur ^ 1] : nullptr;
    a.off_out = off[cur ^ 1];
    a.medians = medians;
    a.exact = exact;
    DRPT_TRY(launch_tree_level(a, tree_level_max_units(n, T, level), s));
    cur ^= 1;
  }
  return DRPT_OK;
}
