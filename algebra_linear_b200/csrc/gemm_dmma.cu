// FP64 C -= A B on the FP64 tensor cores (DMMA, mma.sync m8n8k4 .f64) for the
// fused (non bit-exact) forms: the FP64 LU with fused updates and the sparse
// fronts' Schur complements.
//
// CTA tile 128 x 64 (four warps in a 2 x 2 grid, two CTAs per SM), each warp
// a 64 x 32 tile = 8 x 4 m8n8 accumulators (two doubles per lane each); K in
// chunks of 16 staged in shared memory by cp.async through a three-stage
// ring: 16-byte copies of two consecutive doubles when the operands allow,
// 8-byte copies otherwise (any leading dimension and offset); out-of-range
// elements are zero-filled. The accumulators start as -C and each MMA adds
// A B (the store negates back), so every partial sum is one fused
// multiply-add chain into C, as the CUDA-core fused kernel does.
// Shared-memory rows are padded by 4 doubles so that a half-warp's fragment
// loads (4 k-rows x 4 m-columns) fall in 32 distinct banks.
#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "dense.cuh"

namespace alg {
namespace {

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 8 : 0;  // src-size 0: fill with zeros
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}

// Two consecutive doubles; src_bytes 16, 8 (the second is zero-filled) or 0.
__device__ __forceinline__ void cp_async16(double* dst, const double* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Tile shape: 128 x (32 WN) per CTA, warps in a 2 x WN grid, each warp 64 x 32
// (8 x 4 m8n8 accumulators, two doubles per lane each). K in chunks of 16
// through a STAGES-deep cp.async ring. VEC: 16-byte copies of two
// consecutive doubles (A's rows / B's k entries), when both operands and
// their leading dimensions allow it; 8-byte copies otherwise.
template <int WN, int STAGES, bool VEC>
struct DmmaCfg {
  static constexpr int kBM = 128, kBN = 32 * WN, kBK = 16, kThreads = 64 * WN;
  static constexpr int kAS = kBM + 4;  // As[k][m] row stride (doubles)
  static constexpr int kBS = kBK + 4;  // Bs[n][k] row stride
  static constexpr int kStage = kBK * kAS + kBN * kBS;
  static constexpr size_t kSmem = sizeof(double) * STAGES * kStage;
};

template <int WN, int STAGES, bool VEC>
__global__ void __launch_bounds__(64 * WN, WN == 2 ? 2 : 1)
    dmma_gemm_sub_kernel(int M, int N, int K, const double* __restrict__ A, int lda, const double* __restrict__ B,
                         int ldb, double* __restrict__ C, int ldc) {
  using Cfg = DmmaCfg<WN, STAGES, VEC>;
  constexpr int kBM = Cfg::kBM, kBN = Cfg::kBN, kBK = Cfg::kBK, kThreads = Cfg::kThreads;
  constexpr int kAS = Cfg::kAS, kBS = Cfg::kBS, kStage = Cfg::kStage;
  extern __shared__ __align__(16) double smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 1) * 64, wn = (warp >> 1) * 32;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;

  auto load_stage = [&](int stage, int k0) {
    double* As = smem + stage * kStage;
    double* Bs = As + kBK * kAS;
    if constexpr (VEC) {
#pragma unroll
      for (int r = 0; r < (kBM * kBK) / (2 * kThreads); ++r) {
        const int e = tid + r * kThreads;
        const int mm = 2 * (e % (kBM / 2)), kk = e / (kBM / 2);
        const int gm = m0 + mm, gk = k0 + kk;
        const int bytes = (gk < K && gm < M) ? (gm + 1 < M ? 16 : 8) : 0;
        cp_async16(As + kk * kAS + mm, bytes ? A + (size_t)gm + (size_t)gk * lda : A, bytes);
      }
#pragma unroll
      for (int r = 0; r < (kBN * kBK) / (2 * kThreads); ++r) {
        const int e = tid + r * kThreads;
        const int kk = 2 * (e % (kBK / 2)), nn = e / (kBK / 2);
        const int gn = n0 + nn, gk = k0 + kk;
        const int bytes = (gn < N && gk < K) ? (gk + 1 < K ? 16 : 8) : 0;
        cp_async16(Bs + nn * kBS + kk, bytes ? B + (size_t)gk + (size_t)gn * ldb : B, bytes);
      }
    } else {
#pragma unroll
      for (int r = 0; r < (kBM * kBK) / kThreads; ++r) {
        const int e = tid + r * kThreads;
        const int mm = e % kBM, kk = e / kBM;
        const int gm = m0 + mm, gk = k0 + kk;
        const bool ok = gm < M && gk < K;
        cp_async8(As + kk * kAS + mm, ok ? A + (size_t)gm + (size_t)gk * lda : A, ok);
      }
#pragma unroll
      for (int r = 0; r < (kBN * kBK) / kThreads; ++r) {
        const int e = tid + r * kThreads;
        const int kk = e % kBK, nn = e / kBK;
        const int gn = n0 + nn, gk = k0 + kk;
        const bool ok = gn < N && gk < K;
        cp_async8(Bs + nn * kBS + kk, ok ? B + (size_t)gk + (size_t)gn * ldb : B, ok);
      }
    }
  };

  const int nch = (K + kBK - 1) / kBK;
  // the ring fills while the accumulators load C
#pragma unroll
  for (int st = 0; st < STAGES - 1; ++st) {
    if (st < nch) load_stage(st, st * kBK);
    cp_async_commit();
  }

  // accumulators = -C (fragment layout: row g, columns 2t and 2t + 1 of each
  // m8n8 tile); the MMAs add A B and the store writes -acc: rounding is
  // symmetric, so -(-C + A B) equals C - A B term by term, and the operands
  // need no negation
  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gm = m0 + wm + i * 8 + g, gn = n0 + wn + j * 8 + 2 * t + h;
        acc[i][j][h] = (gm < M && gn < N) ? -C[(size_t)gm + (size_t)gn * ldc] : 0.0;
      }

  for (int ch = 0; ch < nch; ++ch) {
    cp_async_wait<STAGES - 2>();  // chunk ch has landed
    __syncthreads();              // ... for every thread; the slot refilled below is free
    const int nx = ch + STAGES - 1;
    if (nx < nch) load_stage(nx % STAGES, nx * kBK);
    cp_async_commit();
    const double* As = smem + (ch % STAGES) * kStage;
    const double* Bs = As + kBK * kAS;
#pragma unroll
    for (int k4 = 0; k4 < kBK; k4 += 4) {
      double af[8], bf[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) af[i] = As[(k4 + t) * kAS + wm + i * 8 + g];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = Bs[(wn + j * 8 + g) * kBS + k4 + t];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();

#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gm = m0 + wm + i * 8 + g, gn = n0 + wn + j * 8 + 2 * t + h;
        if (gm < M && gn < N) C[(size_t)gm + (size_t)gn * ldc] = -acc[i][j][h];
      }
}

template <int WN, int STAGES, bool VEC>
int launch_dmma(alg_ctx* ctx, int M, int N, int K, const double* A, int lda, const double* B, int ldb, double* C,
                int ldc) {
  using Cfg = DmmaCfg<WN, STAGES, VEC>;
  static const cudaError_t configured = cudaFuncSetAttribute(
      dmma_gemm_sub_kernel<WN, STAGES, VEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::kSmem);
  ALG_CUDA_TRY(configured);
  dim3 grid((M + Cfg::kBM - 1) / Cfg::kBM, (N + Cfg::kBN - 1) / Cfg::kBN);
  dmma_gemm_sub_kernel<WN, STAGES, VEC><<<grid, Cfg::kThreads, Cfg::kSmem, ctx->stream>>>(M, N, K, A, lda, B, ldb,
                                                                                          C, ldc);
  return ALG_OK;
}

// ALG_DMMA_SHAPE=1: the former shape (128 x 128 tile, 8 warps, one CTA per
// SM, two stages of 8-byte copies), for comparison.
bool dmma_old_shape() {
  static const bool v = [] {
    const char* e = std::getenv("ALG_DMMA_SHAPE");
    return e != nullptr && e[0] == '1';
  }();
  return v;
}

}  // namespace

// Default: 128 x 64 tiles of 4 warps, two CTAs per SM (one tile's C load
// and store overlap the other's MMAs), a three-stage ring; 16-byte copies
// when A, B are 16-byte aligned with even leading dimensions.
int gemm_dmma_sub_dev(alg_ctx* ctx, int M, int N, int K, const double* A, int lda, const double* B, int ldb,
                      double* C, int ldc) {
  if (M <= 0 || N <= 0 || K <= 0) return ALG_OK;
  const bool vec = ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) == 0 &&
                   (lda % 2) == 0 && (ldb % 2) == 0;
  const int tok = prof_begin(ctx, ALG_K_GEMM);
  int rc;
  if (dmma_old_shape()) rc = launch_dmma<4, 2, false>(ctx, M, N, K, A, lda, B, ldb, C, ldc);
  else if (vec) rc = launch_dmma<2, 3, true>(ctx, M, N, K, A, lda, B, ldb, C, ldc);
  else rc = launch_dmma<2, 3, false>(ctx, M, N, K, A, lda, B, ldb, C, ldc);
  count_launches();
  prof_end(ctx, tok, 2.0 * M * N * K, 8.0 * (2.0 * M * N + double(M) * K + double(K) * N));
  ALG_TRY(rc);
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

}  // namespace alg

extern "C" int alg_gemm_dmma_sub_dev(alg_ctx* ctx, int M, int N, int K, const double* A, int lda, const double* B,
                                     int ldb, double* C, int ldc) {
  if (ctx == nullptr || (M > 0 && N > 0 && K > 0 && (A == nullptr || B == nullptr || C == nullptr)))
    return ALG_INVALID_ARGUMENT;
  if (M < 0 || N < 0 || K < 0 || lda < std::max(1, M) || ldb < std::max(1, K) || ldc < std::max(1, M))
    return ALG_BAD_SHAPE;
  const int rc = alg::gemm_dmma_sub_dev(ctx, M, N, K, A, lda, B, ldb, C, ldc);
  if (rc != ALG_OK) return rc;
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return ALG_OK;
}
