// K1u -- the sign-matrix projection of u8 rows on the tensor cores:
//   P[c][p] = sum_k X[p][k] * S[c][k],  X u8, S in {-1, 0, +1} (s8),
// computed exactly in 32-bit integers by tcgen05.mma kind::i8 (s32
// accumulators in Tensor Memory) and stored as float (exact: |P| <= 255 d).
//
// S is the sign of the reference's sparse Gaussian projection matrix with the
// same sparsity mask (math_operations.cpp:48-76 draws it; the reference's own
// projection is the FP32 product of math_operations.cpp:15-46).  It is a fast
// form of the method, not the reference's: its trees are judged by recall.
//
// Per CTA one tile of 128 rows: a TMA warp streams the rows' 128-byte K
// blocks and the matching K blocks of all nc (<= 256) sign rows into NS
// stages, an MMA warp issues four K = 32 steps per block into one
// accumulator of nc columns, and four epilogue warps read it back (thread =
// row) and write P column by column (lanes on consecutive rows).
#include "kernels.cuh"
#include "sm100.cuh"

namespace drpt {
namespace {

using namespace sm100;

constexpr int kTM = 128;        // rows per tile
constexpr int kNS = 2;          // stages
constexpr int kThreads = 192;   // 4 epilogue warps, TMA warp, MMA warp

// Instruction descriptor of kind::i8: S32 accumulator (bits [4,6) = 2),
// A unsigned 8-bit (bits [7,10) = 0), B signed 8-bit (bits [10,13) = 1),
// both K-major, N >> 3 in [17,23), M >> 4 in [24,29).
__host__ __device__ constexpr uint32_t idesc_u8s8_s32(uint32_t M, uint32_t N) {
  return (2u << 4) | (0u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__global__ void __launch_bounds__(kThreads, 1) k_project_i8(
    const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmS, int64_t n,
    int kb, int nc, int ncp, uint32_t tcols, float *__restrict__ P, int *err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const uint32_t a_bytes = kTM * 128, b_bytes = (uint32_t)ncp * 128;
  const uint32_t stage = a_bytes + ((b_bytes + 1023u) & ~1023u);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kNS * stage);
  uint64_t *full = bars, *empty = bars + kNS, *done = bars + 2 * kNS;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kNS + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r0 = (int64_t)blockIdx.x * kTM;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kNS; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 5) tmem_alloc(tmem_slot, tcols);
  if (warp == 4 && lane == 0) {
    prefetch_tmap(&tmX);
    prefetch_tmap(&tmS);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 4) {
    // ---- TMA producer: K block q of the rows and of every sign row
    if (lane == 0) {
      for (int q = 0; q < kb && !*abort_flag; ++q) {
        const int s = q % kNS;
        if (q >= kNS && !mbar_wait(empty + s, ((q / kNS) - 1) & 1)) {
          *abort_flag = 1;
          break;
        }
        uint8_t *st = smem + (size_t)s * stage;
        mbar_arrive_expect_tx(full + s, a_bytes + b_bytes);
        tma_load_2d(st, &tmX, full + s, q * 128, (int)r0);
        tma_load_2d(st + a_bytes, &tmS, full + s, q * 128, 0);
      }
    }
  } else if (warp == 5) {
    // ---- MMA issuer: four K = 32 steps per 128-byte block
    if (lane == 0) {
      const uint32_t idesc = idesc_u8s8_s32(kTM, (uint32_t)ncp);
      bool ok = true;
      for (int q = 0; ok && q < kb && !*abort_flag; ++q) {
        const int s = q % kNS;
        if (!(ok = mbar_wait(full + s, (q / kNS) & 1))) break;
        tc_fence_after();
        const uint32_t as = smem_u32(smem + (size_t)s * stage), bs = as + a_bytes;
#pragma unroll
        for (int k = 0; k < 4; ++k)
          mma_i8(tmem, desc_k_sw128(as + k * 32), desc_k_sw128(bs + k * 32), idesc,
                 (q | k) ? 1u : 0u);
        mma_commit(empty + s);
      }
      if (ok) mma_commit(done);
      else *abort_flag = 1;
    }
  } else {
    // ---- epilogue: thread = row; columns 32 at a time
    const bool ok = __all_sync(kFull, mbar_wait(done, 0));
    if (!ok) {
      *abort_flag = 1;
    } else {
      tc_fence_after();
      const int64_t row = r0 + warp * 32 + lane;
      const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
      for (int c0 = 0; c0 < nc; c0 += 32) {
        float v[32];
        tmem_ld32(lane_base + c0, v);
        if (row < n)
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (c0 + j < nc) P[(int64_t)(c0 + j) * n + row] = (float)__float_as_int(v[j]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after();
    tmem_dealloc(tmem, tcols);
  }
  if (threadIdx.x == 0 && *abort_flag) atomicOr(err, 1);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

drpt_status tmap_u8(CUtensorMap *map, const void *base, uint64_t cols, uint64_t rows,
                    uint64_t stride, uint32_t box_rows) {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available");
    return DRPT_ERR_CUDA;
  }
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {stride};
  cuuint32_t box[2] = {128, box_rows};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return DRPT_ERR_CUDA;
  }
  return DRPT_OK;
}

}  // namespace

int project_i8_max_cols() { return 256; }

drpt_status launch_project_i8(const uint8_t *X, int64_t n, int d, const int8_t *S, int nc,
                              float *P, int *err, cudaStream_t s) {
  if (d % 16 != 0 || d <= 0 || nc <= 0 || nc > project_i8_max_cols() || n <= 0) {
    set_error("sign projection: d %% 16 == 0 and 1 <= columns <= %d needed (d = %d, %d columns)",
              project_i8_max_cols(), d, nc);
    return DRPT_ERR_UNSUPPORTED;
  }
  const int ncp = (nc + 15) / 16 * 16;  // MMA N: a multiple of 16
  uint32_t tcols = 32;
  while ((int)tcols < ncp) tcols <<= 1;
  const int kb = (d + 127) / 128;
  CUtensorMap tmX, tmS;
  DRPT_TRY(tmap_u8(&tmX, X, (uint64_t)d, (uint64_t)n, (uint64_t)d, kTM));
  // S: ncp rows of d signed bytes (rows nc .. ncp - 1 zero), read as bytes
  DRPT_TRY(tmap_u8(&tmS, S, (uint64_t)d, (uint64_t)ncp, (uint64_t)d, (uint32_t)ncp));
  const uint32_t stage = kTM * 128 + ((uint32_t)ncp * 128 + 1023u) / 1024u * 1024u;
  const size_t smem = (size_t)kNS * stage + 64 + 1024;
  DRPT_CUDA(cudaFuncSetAttribute(k_project_i8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  const unsigned grid = (unsigned)ceil_div(n, kTM);
  k_project_i8<<<grid, kThreads, smem, s>>>(tmX, tmS, n, kb, nc, ncp, tcols, P, err);
  DRPT_LAUNCH_CHECK();
  return DRPT_OK;
}

}  // namespace drpt
