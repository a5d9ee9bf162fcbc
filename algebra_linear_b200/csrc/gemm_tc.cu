// Trailing update on the 5th-generation tensor cores (sm_100a, tcgen05):
//
//   C (FP32, M x N, column-major) -= A (M x K) * B (K x N)
//
// with A = L21 and B = U12 of the low-precision LU, their entries rounded to
// BF16 or TF32 and the products accumulated in FP32 in tensor memory.
//
//  1. prep kernels copy A and B into K-major operand buffers (A as M rows of
//     K entries, B as N rows of K entries) in the operand type (BF16, or FP32
//     rounded to TF32), so both MMA operands are K-major;
//  2. the GEMM kernel, persistent: each CTA takes 128 x 256 output tiles
//     tile, tile + grid, ... (the grid may be capped below the SM count so
//     that kernels of another stream find free SMs):
//       warp 0   TMA producer: 128-byte K slices of the A and B tiles into a
//                4-stage shared-memory ring (128B swizzle, no multicast),
//                running ahead across tiles;
//       warp 1   allocates 512 TMEM columns (two accumulators); one lane
//                issues tcgen05.mma (M=128, N=256, FP32 accumulator) per
//                32-byte K step into the tile's accumulator, commits each
//                stage back to the producer and the finished accumulator to
//                the epilogue;
//       8 warps  epilogue: tcgen05.ld of the accumulator (then handed back
//                to the MMA lane), C -= acc with coalesced column accesses
//                (thread = row), while the MMAs fill the other accumulator.
// Every wait on an mbarrier is bounded; on expiry the kernel raises the
// timeout flag of the status block and skips ahead.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <cstdint>
#include <algorithm>
#include <cstring>
#include <mutex>

#include "dense.cuh"

namespace alg {
namespace {

constexpr int BM = 128;
constexpr int BN = 256;
constexpr int kStages = 4;
constexpr int kSliceBytes = 128;                  // one 128B-swizzle atom along K
constexpr int kABytes = BM * kSliceBytes;         // 16 KB per stage
constexpr int kBBytes = BN * kSliceBytes;         // 32 KB per stage
constexpr int kStageBytes = kABytes + kBBytes;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;  // producer warp, MMA warp, epilogue warps
constexpr int kAccCols = BN;                    // one FP32 accumulator: 128 lanes x 256 columns
constexpr int kTmemCols = 2 * kAccCols;
constexpr size_t kSmemBytes = (size_t)kStages * kStageBytes + 1024 /*align*/ + 256 /*barriers*/;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}
// bounded wait: false after ~kWaitLimitNs
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  uint64_t t0 = 0;
  for (int it = 0;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255) == 0) {
      const uint64_t t = global_timer_ns();
      if (it == 0) t0 = t;
      else if (t - t0 > kWaitLimitNs) return false;
    }
  }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(bar) : "memory");
}

// K-major, 128B-swizzled operand tile: rows of 128 bytes, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);         // start address
  d |= (uint64_t)1 << 16;                        // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;              // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                        // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                        // layout: 128-byte swizzle
  return d;
}

// Instruction descriptor: FP32 accumulator, A/B format (1 = BF16, 2 = TF32),
// both K-major, M = 128, N = 256.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t fmt) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

template <int FMT>
__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  constexpr uint32_t idesc = instr_desc(FMT);
  if constexpr (FMT == 1) {
    asm volatile(
        "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
  } else {
    asm volatile(
        "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p; }"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
  }
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

#define TMEM_LD_X32(taddr, r)                                                                          \
  asm volatile(                                                                                        \
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15," \
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                       \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), \
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),       \
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),     \
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),     \
        "=r"(r[29]), "=r"(r[30]), "=r"(r[31])                                                          \
      : "r"(taddr))

template <int FMT>
__global__ void __launch_bounds__(kThreads, 1)
    gemm_tc_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                   int M, int N, int K, float* __restrict__ C, int ldc, DevStatus* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* stage_a = base;                                  // [kStages][kABytes]
  unsigned char* stage_b = base + (size_t)kStages * kABytes;      // [kStages][kBBytes]
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + (size_t)kStages * kStageBytes);
  // bars[0..S): stage full, [S..2S): stage empty, 2S + b: accumulator b full,
  // 2S + 2 + b: accumulator b drained, 2S + 4: every MMA done
  uint64_t* acc_full = bars + 2 * kStages;
  uint64_t* acc_empty = bars + 2 * kStages + 2;
  uint64_t* mma_done = bars + 2 * kStages + 4;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 5);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mtiles = (M + BM - 1) / BM;
  const int tiles = mtiles * ((N + BN - 1) / BN);
  const int kslice = kSliceBytes / (FMT == 1 ? 2 : 4);  // K entries per slice
  const int nslices = (K + kslice - 1) / kslice;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_addr(&bars[s]), 1);
      mbar_init(smem_addr(&bars[kStages + s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_addr(&acc_full[b]), 1);
      mbar_init(smem_addr(&acc_empty[b]), kEpiWarps);
    }
    mbar_init(smem_addr(mma_done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer: slice g of this CTA's sequence goes to stage g % S --
      uint32_t g = 0;
      for (int tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x) {
        const int m0 = (tile % mtiles) * BM, n0 = (tile / mtiles) * BN;
        for (int ks = 0; ks < nslices; ++ks, ++g) {
          const int s = g % kStages;
          if (g >= kStages && !mbar_wait_bounded(smem_addr(&bars[kStages + s]), ((g / kStages) - 1) & 1)) {
            ok = false;
            break;
          }
          const uint32_t full = smem_addr(&bars[s]);
          mbar_expect_tx(full, kStageBytes);
          tma_load_2d(smem_addr(stage_a + (size_t)s * kABytes), &map_a, ks * kslice, m0, full);
          tma_load_2d(smem_addr(stage_b + (size_t)s * kBBytes), &map_b, ks * kslice, n0, full);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer: tile i of this CTA accumulates in accumulator i & 1 --
      const int ksteps = kSliceBytes / 32;  // 32-byte K steps per slice
      uint32_t g = 0;
      int li = 0;
      for (int tile = blockIdx.x; ok && tile < tiles; tile += gridDim.x, ++li) {
        const int b = li & 1;
        // the epilogue has drained this accumulator's previous tile
        if (li >= 2 && !mbar_wait_bounded(smem_addr(&acc_empty[b]), ((li >> 1) - 1) & 1)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(b * kAccCols);
        for (int ks = 0; ks < nslices; ++ks, ++g) {
          const int s = g % kStages;
          if (!mbar_wait_bounded(smem_addr(&bars[s]), (g / kStages) & 1)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint64_t adesc = smem_desc_sw128(smem_addr(stage_a + (size_t)s * kABytes));
          const uint64_t bdesc = smem_desc_sw128(smem_addr(stage_b + (size_t)s * kBBytes));
          for (int kk = 0; kk < ksteps; ++kk) {
            // advance the start address by 32 bytes per K step inside the swizzle atom
            mma_issue<FMT>(d, adesc + (uint64_t)(2 * kk), bdesc + (uint64_t)(2 * kk), (ks | kk) != 0);
          }
          mma_commit(smem_addr(&bars[kStages + s]));  // stage free once these MMAs finish
        }
        if (!ok) break;
        mma_commit(smem_addr(&acc_full[b]));  // accumulator complete
      }
      // every MMA issued here has finished before TMEM is released
      mma_commit(smem_addr(mma_done));
      if (!mbar_wait_bounded(smem_addr(mma_done), 0)) ok = false;
    }
  } else {
    // ---- epilogue: C -= acc ----------------------------------------------------
    const int lane_base = 32 * (warp & 3);  // TMEM lanes this warp may read
    const int col_half = ((warp - 2) >> 2) * (BN / 2);
    int li = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++li) {
      const int m0 = (tile % mtiles) * BM, n0 = (tile / mtiles) * BN;
      const int b = li & 1;
      if (!mbar_wait_bounded(smem_addr(&acc_full[b]), (li >> 1) & 1)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int row = m0 + lane_base + lane;
      for (int cb = 0; cb < BN / 2; cb += 32) {
        uint32_t r[32];
        const uint32_t taddr =
            tmem + ((uint32_t)lane_base << 16) + (uint32_t)(b * kAccCols + col_half + cb);
        TMEM_LD_X32(taddr, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (cb + 32 == BN / 2) {
          // this warp's share of the accumulator is in registers: hand it back
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_addr(&acc_empty[b]));
        }
        if (row < M) {
          float cv[32];
#pragma unroll
          for (int t = 0; t < 32; ++t) {
            const int col = n0 + col_half + cb + t;
            cv[t] = col < N ? C[(size_t)row + (size_t)col * ldc] : 0.f;
          }
#pragma unroll
          for (int t = 0; t < 32; ++t) {
            const int col = n0 + col_half + cb + t;
            if (col < N) C[(size_t)row + (size_t)col * ldc] = cv[t] - __uint_as_float(r[t]);
          }
        }
      }
    }
  }
  if (!ok) atomicExch(&status->timeout, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

// ---- operand preparation ---------------------------------------------------------
// FMT 3 (TF32x3, the split-precision scheme of Ootomo and Yokota, "Recovering
// single precision accuracy from Tensor Cores while surpassing the FP32
// theoretical peak performance", IJHPCA 2022): every FP32 entry v becomes
// hi = tf32(v) and lo = tf32(v - hi) (v - hi is exact in FP32), and the
// operands are laid out along a tripled K as
//   A row: [hi | hi | lo],  B row: [hi | lo | hi]
// so one TF32 GEMM over 3K accumulates a_hi b_hi + a_hi b_lo + a_lo b_hi in
// FP32; the dropped a_lo b_lo term is below FP32 rounding of the products.
__device__ __forceinline__ void split_tf32(float v, uint32_t& hi, uint32_t& lo) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(v));
  const float r = v - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

// A (M x K, column-major) -> At (M rows of K entries, 3K for FMT 3); through a 32 x 32 tile.
template <int FMT>
__global__ void prep_a_kernel(const float* __restrict__ a, int lda, int M, int K, void* __restrict__ out) {
  __shared__ float t[32][33];
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int kk = threadIdx.y; kk < 32; kk += 8) {
    const int i = i0 + threadIdx.x, k = k0 + kk;
    t[kk][threadIdx.x] = (i < M && k < K) ? a[(size_t)i + (size_t)k * lda] : 0.f;
  }
  __syncthreads();
  for (int ii = threadIdx.y; ii < 32; ii += 8) {
    const int i = i0 + ii, k = k0 + threadIdx.x;
    if (i < M && k < K) {
      const float v = t[threadIdx.x][ii];
      if constexpr (FMT == 1) {
        reinterpret_cast<__nv_bfloat16*>(out)[(size_t)i * K + k] = __float2bfloat16_rn(v);
      } else if constexpr (FMT == 3) {
        uint32_t hi, lo;
        split_tf32(v, hi, lo);
        uint32_t* row = reinterpret_cast<uint32_t*>(out) + (size_t)i * 3 * K;
        row[k] = hi;
        row[K + k] = hi;
        row[2 * K + k] = lo;
      } else {
        uint32_t tv;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(tv) : "f"(v));
        reinterpret_cast<uint32_t*>(out)[(size_t)i * K + k] = tv;
      }
    }
  }
}

// B (K x N, column-major, K contiguous already) -> Bt (N rows of K entries, 3K for FMT 3).
template <int FMT>
__global__ void prep_b_kernel(const float* __restrict__ b, int ldb, int K, int N, void* __restrict__ out) {
  const size_t total = (size_t)K * N;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const size_t j = idx / K, k = idx % K;
    const float v = b[k + j * (size_t)ldb];
    if constexpr (FMT == 1) {
      reinterpret_cast<__nv_bfloat16*>(out)[idx] = __float2bfloat16_rn(v);
    } else if constexpr (FMT == 3) {
      uint32_t hi, lo;
      split_tf32(v, hi, lo);
      uint32_t* row = reinterpret_cast<uint32_t*>(out) + j * 3 * (size_t)K;
      row[k] = hi;
      row[K + k] = lo;
      row[2 * K + k] = hi;
    } else {
      uint32_t tv;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(tv) : "f"(v));
      reinterpret_cast<uint32_t*>(out)[idx] = tv;
    }
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link-time libcuda dependency).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// 2-D map over rows x K (K contiguous), box = 128-byte K slice x box_rows rows.
int make_map(CUtensorMap* map, const void* ptr, int fmt, int rows, int K, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (fn == nullptr) return ALG_CUDA_ERROR;
  const int esz = fmt == 1 ? 2 : 4;
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)K * esz};
  cuuint32_t box[2] = {(cuuint32_t)(kSliceBytes / esz), (cuuint32_t)box_rows};
  cuuint32_t elem_strides[2] = {1, 1};
  const CUresult r = fn(map, fmt == 1 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                        const_cast<void*>(ptr), dims, strides, box, elem_strides, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? ALG_OK : ALG_CUDA_ERROR;
}

template <int FMT>
int launch_tc(alg_ctx* ctx, int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C,
              int ldc, int ws_slot, int max_ctas) {
  const int esz = FMT == 1 ? 2 : 4;
  constexpr int KFMT = FMT == 3 ? 2 : FMT;  // the MMA's operand type (TF32x3 runs TF32 MMAs)
  // K padded to whole 128-byte slices so every TMA row stride is 16-byte aligned
  const int kslice = kSliceBytes / esz;
  if (K % kslice != 0) return ALG_BAD_SHAPE;  // K must be whole 128-byte slices (the LU's block widths are)
  const int Kp = FMT == 3 ? 3 * K : K;
  void* at = nullptr;
  void* bt = nullptr;
  ALG_TRY(ws_get(ctx, ws_slot, (size_t)esz * Kp * ((size_t)M + N) + 256, &at));
  bt = static_cast<unsigned char*>(at) + (((size_t)esz * Kp * M + 255) & ~size_t(255));
  {
    dim3 grid((M + 31) / 32, (K + 31) / 32);
    prep_a_kernel<FMT><<<grid, dim3(32, 8), 0, ctx->stream>>>(A, lda, M, K, at);
    const size_t total = (size_t)K * N;
    const int g = (int)std::min<size_t>((total + 255) / 256, (size_t)ctx->sm_count * 16);
    prep_b_kernel<FMT><<<g, 256, 0, ctx->stream>>>(B, ldb, K, N, bt);
    count_launches(2);
    ALG_CUDA_TRY(cudaGetLastError());
  }
  CUtensorMap ma, mb;
  ALG_TRY(make_map(&ma, at, KFMT, M, Kp, BM));
  ALG_TRY(make_map(&mb, bt, KFMT, N, Kp, BN));
  static const cudaError_t configured =
      cudaFuncSetAttribute(gemm_tc_kernel<KFMT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  ALG_CUDA_TRY(configured);
  // persistent CTAs, at most one per SM (the shared-memory ring and the 512
  // TMEM columns take a whole SM), fewer when the caller keeps SMs free
  const long tiles = (long)((M + BM - 1) / BM) * ((N + BN - 1) / BN);
  int ctas = max_ctas > 0 ? std::min(max_ctas, ctx->sm_count) : ctx->sm_count;
  ctas = (int)std::max<long>(1, std::min<long>(ctas, tiles));
  gemm_tc_kernel<KFMT><<<ctas, kThreads, kSmemBytes, ctx->stream>>>(ma, mb, M, N, Kp, C, ldc, ctx->d_status);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

}  // namespace

int gemm_tc_sub_dev(alg_ctx* ctx, int prec, int M, int N, int K, const float* A, int lda, const float* B,
                    int ldb, float* C, int ldc, int ws_slot, int max_ctas) {
  if (M <= 0 || N <= 0 || K <= 0) return ALG_OK;
  const int tok = prof_begin(ctx, ALG_K_GEMM_TC);
  int rc;
  if (prec == ALG_PREC_BF16) rc = launch_tc<1>(ctx, M, N, K, A, lda, B, ldb, C, ldc, ws_slot, max_ctas);
  else if (prec == ALG_PREC_TF32) rc = launch_tc<2>(ctx, M, N, K, A, lda, B, ldb, C, ldc, ws_slot, max_ctas);
  else if (prec == ALG_PREC_TF32X3) rc = launch_tc<3>(ctx, M, N, K, A, lda, B, ldb, C, ldc, ws_slot, max_ctas);
  else rc = ALG_INVALID_ARGUMENT;
  prof_end(ctx, tok, 2.0 * M * N * K, 4.0 * (2.0 * M * N + double(M) * K + double(K) * N));
  return rc;
}

}  // namespace alg

// Test hook: C -= A B through the tensor-core path on device buffers.
extern "C" int alg_gemm_tc_sub_dev(alg_ctx* ctx, int prec, int M, int N, int K, const float* A, int lda,
                                   const float* B, int ldb, float* C, int ldc) {
  if (ctx == nullptr) return ALG_INVALID_ARGUMENT;
  if (M < 0 || N < 0 || K < 0 || lda < std::max(1, M) || ldb < std::max(1, K) || ldc < std::max(1, M))
    return ALG_BAD_SHAPE;
  ALG_TRY(alg::status_reset(ctx));
  ALG_TRY(alg::gemm_tc_sub_dev(ctx, prec, M, N, K, A, lda, B, ldb, C, ldc));
  return alg::status_fetch(ctx);
}
