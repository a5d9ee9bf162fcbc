// FP64 C -= A B on the FP64 tensor cores (DMMA, mma.sync m8n8k4 .f64) for the
// fused (non bit-exact) forms: the FP64 LU with fused updates and the sparse
// fronts' Schur complements.
//
// CTA tile 128 x 128, K in chunks of 16 staged in shared memory by cp.async
// (8-byte copies, so any leading dimension and offset works; out-of-range
// elements are zero-filled), two stages. Eight warps in a 2 x 4 grid, each
// with a 64 x 32 tile = 8 x 4 m8n8 accumulators (two doubles per lane each).
// The accumulators start as C and each MMA adds (-A) B, so every partial sum
// is one fused multiply-add chain into C, as the CUDA-core fused kernel does.
// Shared-memory rows are padded by 4 doubles so that a half-warp's fragment
// loads (4 k-rows x 4 m-columns) fall in 32 distinct banks.
#include <algorithm>

#include "dense.cuh"

namespace alg {
namespace {

constexpr int kBM = 128, kBN = 128, kBK = 16, kThreads = 256;
constexpr int kAS = kBM + 4;  // As[k][m] row stride
constexpr int kBS = kBK + 4;  // Bs[n][k] row stride
constexpr int kStageDoubles = kBK * kAS + kBN * kBS;
constexpr size_t kSmemBytes = 2 * sizeof(double) * kStageDoubles;

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 8 : 0;  // src-size 0: fill with zeros
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
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

__global__ void __launch_bounds__(kThreads, 1) dmma_gemm_sub_kernel(int M, int N, int K, const double* __restrict__ A,
                                                                     int lda, const double* __restrict__ B, int ldb,
                                                                     double* __restrict__ C, int ldc) {
  extern __shared__ __align__(16) double smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 1) * 64, wn = (warp >> 1) * 32;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;

  auto load_stage = [&](int stage, int k0) {
    double* As = smem + stage * kStageDoubles;
    double* Bs = As + kBK * kAS;
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
    cp_async_commit();
  };

  // accumulators = C (fragment layout: row g, columns 2t and 2t + 1 of each m8n8 tile)
  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gm = m0 + wm + i * 8 + g, gn = n0 + wn + j * 8 + 2 * t + h;
        acc[i][j][h] = (gm < M && gn < N) ? C[(size_t)gm + (size_t)gn * ldc] : 0.0;
      }

  const int nch = (K + kBK - 1) / kBK;
  if (nch > 0) load_stage(0, 0);
  for (int ch = 0; ch < nch; ++ch) {
    if (ch + 1 < nch) {
      load_stage((ch + 1) & 1, (ch + 1) * kBK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* As = smem + (ch & 1) * kStageDoubles;
    const double* Bs = As + kBK * kAS;
#pragma unroll
    for (int k4 = 0; k4 < kBK; k4 += 4) {
      double af[8], bf[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) af[i] = -As[(k4 + t) * kAS + wm + i * 8 + g];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = Bs[(wn + j * 8 + g) * kBS + k4 + t];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    __syncthreads();  // the stage is refilled by the next iteration's prefetch
  }

#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gm = m0 + wm + i * 8 + g, gn = n0 + wn + j * 8 + 2 * t + h;
        if (gm < M && gn < N) C[(size_t)gm + (size_t)gn * ldc] = acc[i][j][h];
      }
}

}  // namespace

int gemm_dmma_sub_dev(alg_ctx* ctx, int M, int N, int K, const double* A, int lda, const double* B, int ldb,
                      double* C, int ldc) {
  if (M <= 0 || N <= 0 || K <= 0) return ALG_OK;
  static const cudaError_t configured =
      cudaFuncSetAttribute(dmma_gemm_sub_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
  ALG_CUDA_TRY(configured);
  dim3 grid((M + kBM - 1) / kBM, (N + kBN - 1) / kBN);
  const int tok = prof_begin(ctx, ALG_K_GEMM);
  dmma_gemm_sub_kernel<<<grid, kThreads, kSmemBytes, ctx->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  count_launches();
  prof_end(ctx, tok, 2.0 * M * N * K, 8.0 * (2.0 * M * N + double(M) * K + double(K) * N));
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
