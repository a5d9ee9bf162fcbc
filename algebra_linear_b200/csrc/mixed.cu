// Mixed-precision dgesv: low-precision LU + FP64 iterative refinement.
//
// A (FP64, column-major) is cast once to an FP32 working copy and factorized
// there with the blocked LU (panel, interchanges and TRSM in FP32; trailing
// updates in FP32 on the CUDA cores, or on the tensor cores with TF32 / BF16
// inputs and FP32 accumulation). Accuracy is recovered in FP64:
//   x <- 0, r <- b
//   repeat: d = (LU)^{-1} r (FP32 solve), x += d (FP64),
//           r = b - A x (FP64, A read from the caller's FP64 matrix),
//           stop when the normwise backward error
//           ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf)
//           (src/sparse/faer/accuracy_tests.rs:61-67) is within tol,
// falling back to GMRES-IR (FP64 GMRES on A with the low-precision LU as
// preconditioner) when refinement stalls, and to a full FP64 refactorization
// when that does not converge either. A is left unchanged unless the FP64
// fallback ran (then, like dgesv, it holds the FP64 LU factors).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "dense.cuh"
#include "gmres.cuh"
#include "mixed.cuh"
#include "rbt.cuh"

namespace alg {
namespace {

constexpr int kVecThreads = 256;
// from this order on, AUTO pivoting uses tournament pivoting (below it the
// panels are short and partial pivoting's chain is cheap)
constexpr int kTournamentMinOrder = 2048;

__global__ void cast_f64_f32_kernel(const double* __restrict__ a, int lda, float* __restrict__ o, int ldo,
                                    int m, int n) {
  const size_t total = (size_t)m * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const size_t j = idx / m, i = idx % m;
    o[i + j * ldo] = __double2float_rn(a[i + j * lda]);
  }
}

// Row sums of |A| (n x n, FP64): part 1 of ||A||_inf. Grid: row blocks x column
// chunks; partial[chunk][row].
constexpr int kResRows = 256;
constexpr int kResCols = 512;
// right-hand sides from which the residual is one GEMM (the row kernel reads
// A once per right-hand side)
constexpr int kGemmResidualRhs = 4;

__global__ void abs_rowsum_kernel(const double* __restrict__ a, int lda, int n, double* __restrict__ partial) {
  const int i = blockIdx.x * kResRows + threadIdx.x;
  const int j0 = blockIdx.y * kResCols;
  const int j1 = min(n, j0 + kResCols);
  if (i >= n) return;
  double s = 0.0;
  for (int j = j0; j < j1; ++j) s += fabs(a[(size_t)i + (size_t)j * lda]);
  partial[(size_t)blockIdx.y * n + i] = s;
}

// r = b - A x for nrhs columns (FP64). Partial products per chunk of `cols`
// columns (<= kResCols), summed in a fixed order by residual_finish_kernel
// (deterministic). A thread per row streams its chunk with eight loads in
// flight.
__global__ void residual_partial_kernel(const double* __restrict__ a, int lda, int n,
                                        const double* __restrict__ x, int ldx, int nrhs, int cols,
                                        double* __restrict__ partial) {
  const int i = blockIdx.x * kResRows + threadIdx.x;
  const int j0 = blockIdx.y * cols;
  const int j1 = min(n, j0 + cols);
  const int r = blockIdx.z;
  __shared__ double xs[kResCols];
  for (int j = j0 + threadIdx.x; j < j1; j += kResRows) xs[j - j0] = x[(size_t)r * ldx + j];
  __syncthreads();
  if (i >= n) return;
  double s = 0.0;
  const double* ai = a + i;
#pragma unroll 8
  for (int j = j0; j < j1; ++j) s = __fma_rn(ai[(size_t)j * lda], xs[j - j0], s);
  partial[((size_t)r * gridDim.y + blockIdx.y) * n + i] = s;
}

// Chunk width of the residual: kResCols, narrower when the grid would give
// fewer than four CTAs per SM (the row blocks alone do not fill the GPU
// below n ~ 16k); a multiple of 32.
int res_cols(int n, int sms) {
  const long long rows = (n + kResRows - 1) / kResRows;
  int cols = kResCols;
  while (cols > 32 && rows * ((n + cols - 1) / cols) < 4LL * sms) cols /= 2;
  return cols;
}

// max that keeps a NaN (fmax would drop it and hide a diverged solve)
__device__ __forceinline__ double nanmax(double m, double v) { return (v != v || v > m) ? v : m; }

// r = b - sum(partials); also max|r| and max|x|, max|b| per RHS into stats[r*4+{0,1,2}]
// via an atomic max on the bit pattern (non-negative doubles order as integers,
// and a NaN's pattern lies above every number's).
__global__ void residual_finish_kernel(const double* __restrict__ partial, int nchunks, int n,
                                       const double* __restrict__ b, int ldb, const double* __restrict__ x,
                                       int ldx, double* __restrict__ res, int ldr, int nrhs,
                                       unsigned long long* __restrict__ stats) {
  const int r = blockIdx.y;
  double mr = 0.0, mx = 0.0, mb = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s += partial[((size_t)r * nchunks + c) * n + i];
    const double bi = b[(size_t)r * ldb + i];
    const double ri = bi - s;
    res[(size_t)r * ldr + i] = ri;
    mr = nanmax(mr, fabs(ri));
    mx = nanmax(mx, fabs(x[(size_t)r * ldx + i]));
    mb = nanmax(mb, fabs(bi));
  }
  for (int off = 16; off > 0; off >>= 1) {
    mr = nanmax(mr, __shfl_xor_sync(0xffffffffu, mr, off));
    mx = nanmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    mb = nanmax(mb, __shfl_xor_sync(0xffffffffu, mb, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&stats[r * 4 + 0], (unsigned long long)__double_as_longlong(mr));
    atomicMax(&stats[r * 4 + 1], (unsigned long long)__double_as_longlong(mx));
    atomicMax(&stats[r * 4 + 2], (unsigned long long)__double_as_longlong(mb));
  }
}

// The norms of residual_finish_kernel for a residual already formed in res.
__global__ void residual_norms_kernel(const double* __restrict__ res, int ldr, const double* __restrict__ x, int ldx,
                                      const double* __restrict__ b, int ldb, int n,
                                      unsigned long long* __restrict__ stats) {
  const int r = blockIdx.y;
  double mr = 0.0, mx = 0.0, mb = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    mr = nanmax(mr, fabs(res[(size_t)r * ldr + i]));
    mx = nanmax(mx, fabs(x[(size_t)r * ldx + i]));
    mb = nanmax(mb, fabs(b[(size_t)r * ldb + i]));
  }
  for (int off = 16; off > 0; off >>= 1) {
    mr = nanmax(mr, __shfl_xor_sync(0xffffffffu, mr, off));
    mx = nanmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    mb = nanmax(mb, __shfl_xor_sync(0xffffffffu, mb, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&stats[r * 4 + 0], (unsigned long long)__double_as_longlong(mr));
    atomicMax(&stats[r * 4 + 1], (unsigned long long)__double_as_longlong(mx));
    atomicMax(&stats[r * 4 + 2], (unsigned long long)__double_as_longlong(mb));
  }
}

__global__ void gemv_finish_kernel(const double* __restrict__ partial, int nchunks, int n, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s += partial[(size_t)c * n + i];
    y[i] = s;
  }
}

__global__ void f32_to_f64_kernel(const float* __restrict__ a, double* __restrict__ o, size_t cnt) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x)
    o[i] = (double)a[i];
}

__global__ void rowsum_finish_kernel(const double* __restrict__ partial, int nchunks, int n,
                                     unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s += partial[(size_t)c * n + i];
    m = nanmax(m, s);
  }
  for (int off = 16; off > 0; off >>= 1) m = nanmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// r32 = (float) r, for the low-precision correction solve
__global__ void f64_to_f32_kernel(const double* __restrict__ a, float* __restrict__ o, size_t cnt) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x)
    o[i] = __double2float_rn(a[i]);
}

// x += d (d in FP32)
__global__ void axpy_f32_kernel(const float* __restrict__ d, double* __restrict__ x, int n, int nrhs, int ldx) {
  const size_t cnt = (size_t)n * nrhs;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < cnt;
       idx += (size_t)gridDim.x * blockDim.x) {
    const size_t r = idx / n, i = idx % n;
    x[r * ldx + i] += (double)d[idx];
  }
}

int grid_for(size_t cnt, int sm) {
  return (int)std::max<size_t>(1, std::min<size_t>((cnt + kVecThreads - 1) / kVecThreads, (size_t)sm * 8));
}

}  // namespace

int lu_factor_lowp_dev(alg_ctx* ctx, int precision, float* a32, int n, int lda, int* ipiv, int* perm,
                       bool tournament) {
  LuPlan plan = default_plan(n, 4);
  plan.tslu = tournament ? 1 : 0;
  if (precision != ALG_PREC_FP32) {
    plan.tc_prec = precision;
    // deep blocks for the tensor-core update: K = 256 halves the update's
    // C traffic per flop and the passes of deferred interchanges
    plan.nb = n >= 8192 ? 256 : 128;
    if (const char* e = std::getenv("ALG_NB_TC")) plan.nb = std::max(32, std::atoi(e));
  }
  return lu_factor_dev<float, false>(ctx, a32, n, n, lda, ipiv, perm, plan);
}

// ---------------------------------------------------------------------------
// FP64 residual and norms
// ---------------------------------------------------------------------------
int inf_norm_dev(alg_ctx* ctx, const double* a, int n, int lda, double* out_host) {
  const int nchunks = (n + kResCols - 1) / kResCols;
  double* partial = nullptr;
  unsigned long long* st = nullptr;
  ALG_TRY(ws_get(ctx, WS_PARTIAL, sizeof(double) * (size_t)nchunks * n, reinterpret_cast<void**>(&partial)));
  ALG_TRY(ws_get(ctx, WS_MISC, 4096, reinterpret_cast<void**>(&st)));
  ALG_CUDA_TRY(cudaMemsetAsync(st, 0, 8, ctx->stream));
  const int tok = prof_begin(ctx, ALG_K_RESID);
  abs_rowsum_kernel<<<dim3((n + kResRows - 1) / kResRows, nchunks), kResRows, 0, ctx->stream>>>(a, lda, n, partial);
  rowsum_finish_kernel<<<grid_for(n, ctx->sm_count), kVecThreads, 0, ctx->stream>>>(partial, nchunks, n, st);
  count_launches(2);
  prof_end(ctx, tok, 2.0 * n * n, 8.0 * n * n);
  ALG_CUDA_TRY(cudaGetLastError());
  unsigned long long h = 0;
  ALG_CUDA_TRY(cudaMemcpyAsync(&h, st, 8, cudaMemcpyDeviceToHost, ctx->stream));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  std::memcpy(out_host, &h, 8);
  return ALG_OK;
}

int gemv_dev(alg_ctx* ctx, const double* a, int n, int lda, const double* x, double* y) {
  const int cols = res_cols(n, ctx->sm_count);
  const int nchunks = (n + cols - 1) / cols;
  double* partial = nullptr;
  ALG_TRY(ws_get(ctx, WS_PARTIAL, sizeof(double) * (size_t)nchunks * n, reinterpret_cast<void**>(&partial)));
  const int tok = prof_begin(ctx, ALG_K_RESID);
  residual_partial_kernel<<<dim3((n + kResRows - 1) / kResRows, nchunks, 1), kResRows, 0, ctx->stream>>>(
      a, lda, n, x, n, 1, cols, partial);
  gemv_finish_kernel<<<grid_for(n, ctx->sm_count), kVecThreads, 0, ctx->stream>>>(partial, nchunks, n, y);
  count_launches(2);
  prof_end(ctx, tok, 2.0 * n * n, 8.0 * n * n + 16.0 * n);
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

int residual_dev(alg_ctx* ctx, const double* a, int n, int lda, const double* x, int ldx, const double* b,
                 int ldb, double* r, int ldr, int nrhs, double* rmax, double* xmax, double* bmax) {
  const int cols = res_cols(n, ctx->sm_count);
  const int nchunks = (n + cols - 1) / cols;
  double* partial = nullptr;
  unsigned long long* st = nullptr;
  if (nrhs < kGemmResidualRhs)
    ALG_TRY(ws_get(ctx, WS_PARTIAL, sizeof(double) * (size_t)nchunks * n * nrhs, reinterpret_cast<void**>(&partial)));
  ALG_TRY(ws_get(ctx, WS_MISC, 4096 + 32 * (size_t)nrhs, reinterpret_cast<void**>(&st)));
  ALG_CUDA_TRY(cudaMemsetAsync(st, 0, 32 * (size_t)nrhs, ctx->stream));
  const dim3 fin(std::max(1, std::min(4 * ctx->sm_count, (n + 255) / 256)), nrhs);
  if (nrhs >= kGemmResidualRhs) {
    // R = B, then R -= A X as one FP64 tensor-core GEMM (A read once for
    // all right-hand sides), then the norms
    ALG_CUDA_TRY(cudaMemcpy2DAsync(r, sizeof(double) * ldr, b, sizeof(double) * ldb, sizeof(double) * n, nrhs,
                                   cudaMemcpyDeviceToDevice, ctx->stream));
    ALG_TRY(gemm_dmma_sub_dev(ctx, n, nrhs, n, a, lda, x, ldx, r, ldr));
    const int tok = prof_begin(ctx, ALG_K_RESID);
    residual_norms_kernel<<<fin, 256, 0, ctx->stream>>>(r, ldr, x, ldx, b, ldb, n, st);
    count_launches();
    prof_end(ctx, tok, 0.0, 24.0 * n * nrhs);
  } else {
    const int tok = prof_begin(ctx, ALG_K_RESID);
    residual_partial_kernel<<<dim3((n + kResRows - 1) / kResRows, nchunks, nrhs), kResRows, 0, ctx->stream>>>(
        a, lda, n, x, ldx, nrhs, cols, partial);
    residual_finish_kernel<<<fin, 256, 0, ctx->stream>>>(partial, nchunks, n, b, ldb, x, ldx, r, ldr, nrhs, st);
    count_launches(2);
    prof_end(ctx, tok, 2.0 * n * n * nrhs, 8.0 * n * n + 24.0 * n * nrhs);
  }
  ALG_CUDA_TRY(cudaGetLastError());
  std::vector<unsigned long long> h(4 * (size_t)nrhs);
  ALG_CUDA_TRY(cudaMemcpyAsync(h.data(), st, 32 * (size_t)nrhs, cudaMemcpyDeviceToHost, ctx->stream));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < nrhs; ++k) {
    std::memcpy(&rmax[k], &h[4 * k + 0], 8);
    std::memcpy(&xmax[k], &h[4 * k + 1], 8);
    std::memcpy(&bmax[k], &h[4 * k + 2], 8);
  }
  return ALG_OK;
}

// ---------------------------------------------------------------------------
// mixed dgesv on device buffers
// ---------------------------------------------------------------------------
namespace {

__global__ void iota_i32_kernel(int* v, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// Low-precision factorization and its preconditioner M^{-1} on n x k blocks.
struct LowpFactor {
  alg_ctx* ctx = nullptr;
  int n = 0;
  float* a32 = nullptr;
  int* perm = nullptr;  // row permutation (identity for the butterfly form)
  bool rbt = false;
  RbtState rs;
  double* t64 = nullptr;  // n x kmax scratch
  float* t32 = nullptr;   // n x kmax scratch
  int kmax = 0;

  // z = M^{-1} v for k columns (n x k, leading dimension n).
  int apply(const double* v, double* z, int k) {
    for (int k0 = 0; k0 < k; k0 += kmax) {
      const int kk = std::min(kmax, k - k0);
      const double* vk = v + (size_t)k0 * n;
      double* zk = z + (size_t)k0 * n;
      if (rbt) {
        for (int c = 0; c < kk; ++c) ALG_TRY(rbt_vector(ctx, rs, true, vk + (size_t)c * n, t64 + (size_t)c * n));
        vk = t64;
      }
      f64_to_f32_kernel<<<grid_for((size_t)n * kk, ctx->sm_count), kVecThreads, 0, ctx->stream>>>(vk, t32,
                                                                                                 (size_t)n * kk);
      count_launches();
      ALG_TRY((lu_solve_dev<float, false>(ctx, a32, n, n, perm, t32, kk, n)));
      double* dst = rbt ? t64 : zk;
      f32_to_f64_kernel<<<grid_for((size_t)n * kk, ctx->sm_count), kVecThreads, 0, ctx->stream>>>(t32, dst,
                                                                                                 (size_t)n * kk);
      count_launches();
      if (rbt)
        for (int c = 0; c < kk; ++c) ALG_TRY(rbt_vector(ctx, rs, false, t64 + (size_t)c * n, zk + (size_t)c * n));
      ALG_CUDA_TRY(cudaGetLastError());
    }
    return ALG_OK;
  }
};

// x += d
__global__ void axpy_f64_kernel(const double* __restrict__ d, double* __restrict__ x, size_t cnt) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (size_t)gridDim.x * blockDim.x)
    x[i] += d[i];
}

}  // namespace

int dgesv_mixed_dev(alg_ctx* ctx, const alg_mixed_opts& o, double* d_a, int n, int lda, double* d_b, int nrhs,
                    int ldb, alg_mixed_report* rep) {
  alg_mixed_report local{};
  alg_mixed_report& R = rep ? *rep : local;
  std::memset(&R, 0, sizeof(R));
  R.precision = o.precision;
  if (n == 0 || nrhs == 0) return ALG_OK;
  const double tol = o.tol > 0 ? o.tol : 10.0 * n * std::ldexp(1.0, -53);
  const int max_ir = o.max_ir > 0 ? o.max_ir : 30;
  // right-hand sides per preconditioner application: all of them up to 256
  // (from 16 the FP32 solve is blocked, GEMM-rich)
  const int kmax = std::min(nrhs, 256);

  LowpFactor F;
  F.ctx = ctx;
  F.n = n;
  F.kmax = kmax;
  double* x = nullptr;
  int* ipiv = nullptr;
  ALG_TRY(ws_get(ctx, WS_A32, sizeof(float) * (size_t)n * n, reinterpret_cast<void**>(&F.a32)));
  ALG_TRY(ws_get(ctx, WS_R,
                 sizeof(double) * (size_t)n * nrhs * 3 + sizeof(double) * (size_t)n * kmax +
                     sizeof(float) * (size_t)n * kmax + 64,
                 reinterpret_cast<void**>(&x)));
  double* r = x + (size_t)n * nrhs;
  double* dlt = r + (size_t)n * nrhs;
  F.t64 = dlt + (size_t)n * nrhs;
  F.t32 = reinterpret_cast<float*>(F.t64 + (size_t)n * kmax);
  ALG_TRY(ws_get(ctx, WS_IPIV, sizeof(int) * n, reinterpret_cast<void**>(&ipiv)));

  // ---- factorize in low precision --------------------------------------
  // AUTO pivots (tournament pivoting from kTournamentMinOrder on): on
  // matrices that are already random (the dense workloads here) LU without
  // pivoting has large growth even after the butterflies, so the butterfly
  // form is an explicit choice.
  bool use_rbt = o.pivoting == ALG_PIVOT_RBT;
  if (o.pivoting == ALG_PIVOT_RBT && n % 4 != 0) return ALG_BAD_SHAPE;
  bool lowp_singular = false;
  if (use_rbt) {
    ALG_TRY(ws_get(ctx, WS_IDENT, sizeof(int) * n, reinterpret_cast<void**>(&F.perm)));
    iota_i32_kernel<<<grid_for(n, ctx->sm_count), kVecThreads, 0, ctx->stream>>>(F.perm, n);
    count_launches();
    ALG_TRY(rbt_prepare(ctx, n, 0x5eed0f1eULL ^ (uint64_t)n, &F.rs));
    ALG_TRY(status_reset(ctx));
    ALG_TRY(rbt_transform(ctx, F.rs, d_a, lda, F.a32, n));
    ALG_TRY(genp_factor(ctx, o.precision, F.a32, n, n, 128));
    ALG_TRY(status_fetch(ctx));
    if (ctx->h_status->singular_col != INT_MAX) use_rbt = false;  // a zero pivot: pivot after all
    F.rbt = use_rbt;
    R.reserved[0] = use_rbt ? 1.0 : 0.0;
  }
  if (!use_rbt) {
    ALG_TRY(ws_get(ctx, WS_PERM, sizeof(int) * n, reinterpret_cast<void**>(&F.perm)));
    ALG_TRY(status_reset(ctx));
    {
      const int tok = prof_begin(ctx, ALG_K_CAST);
      cast_f64_f32_kernel<<<grid_for((size_t)n * n, ctx->sm_count), kVecThreads, 0, ctx->stream>>>(d_a, lda, F.a32,
                                                                                                   n, n, n);
      count_launches();
      prof_end(ctx, tok, 0.0, 12.0 * n * n);
      ALG_CUDA_TRY(cudaGetLastError());
    }
    const bool tournament =
        o.pivoting == ALG_PIVOT_TOURNAMENT || (o.pivoting == ALG_PIVOT_AUTO && n >= kTournamentMinOrder);
    R.reserved[1] = tournament ? 1.0 : 0.0;
    ALG_TRY(lu_factor_lowp_dev(ctx, o.precision, F.a32, n, n, ipiv, F.perm, tournament));
    ALG_TRY(status_fetch(ctx));
    lowp_singular = ctx->h_status->singular_col != INT_MAX;
  }

  double anorm = 0.0;
  ALG_TRY(inf_norm_dev(ctx, d_a, n, lda, &anorm));
  ALG_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * (size_t)n * nrhs, ctx->stream));
  ALG_CUDA_TRY(cudaMemcpy2DAsync(r, sizeof(double) * n, d_b, sizeof(double) * ldb, sizeof(double) * n, nrhs,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
  std::vector<double> rmax(nrhs), xmax(nrhs), bmax(nrhs), eta(nrhs, INFINITY);
  bool converged = false;
  if (!lowp_singular) {
    // ---- plain refinement: x += M^{-1} r, r = b - A x -------------------
    double prev = INFINITY;
    int stall = 0;
    for (int it = 0; it < max_ir; ++it) {
      ALG_TRY(F.apply(r, dlt, nrhs));
      axpy_f64_kernel<<<grid_for((size_t)n * nrhs, ctx->sm_count), kVecThreads, 0, ctx->stream>>>(
          dlt, x, (size_t)n * nrhs);
      count_launches();
      ALG_CUDA_TRY(cudaGetLastError());
      ALG_TRY(residual_dev(ctx, d_a, n, lda, x, n, d_b, ldb, r, n, nrhs, rmax.data(), xmax.data(), bmax.data()));
      double worst = 0.0;
      for (int k = 0; k < nrhs; ++k) {
        const double den = anorm * xmax[k] + bmax[k];
        eta[k] = den == 0.0 ? rmax[k] : rmax[k] / den;
        worst = std::max(worst, eta[k]);
      }
      R.ir_iterations = it + 1;
      R.backward_error = worst;
      if (!(worst == worst) || std::isinf(worst)) break;  // diverged
      if (worst <= tol) {
        converged = true;
        break;
      }
      if (worst > 0.5 * prev) {  // stalled: less than a halving, twice in a row
        if (++stall >= 2) break;
      } else {
        stall = 0;
      }
      prev = worst;
    }
    if (!converged && !o.no_gmres) {
      // ---- GMRES-IR: FP64 GMRES preconditioned by the low-precision LU ----
      Precond M = [&](alg_ctx*, const double* v, double* z) -> int { return F.apply(v, z, 1); };
      GmresOpts go;
      go.tol = tol;
      if (o.gmres_restart > 0) go.restart = o.gmres_restart;
      bool all = true;
      double worst = 0.0;
      for (int k = 0; k < nrhs && all; ++k) {
        double* xk = x + (size_t)k * n;
        if (!(eta[k] == eta[k]) || eta[k] > 1.0) ALG_CUDA_TRY(cudaMemsetAsync(xk, 0, sizeof(double) * n, ctx->stream));
        GmresResult gr;
        const int rc = gmres_ir_dev(ctx, d_a, n, lda, d_b + (size_t)k * ldb, xk, anorm, M, go, &gr);
        R.gmres_iterations += gr.inner;
        worst = std::max(worst, gr.backward_error);
        if (rc != ALG_OK || !gr.converged) all = false;
      }
      if (all) {
        converged = true;
        R.backward_error = worst;
        R.path = ALG_MIXED_PATH_GMRES;
      }
    }
  }
  if (converged) {
    ALG_CUDA_TRY(cudaMemcpy2DAsync(d_b, sizeof(double) * ldb, x, sizeof(double) * n, sizeof(double) * n, nrhs,
                                   cudaMemcpyDeviceToDevice, ctx->stream));
    ALG_TRY(status_fetch(ctx));  // synchronises; a timed-out sweep of the refinement is an error
    if (R.path != ALG_MIXED_PATH_GMRES) R.path = ALG_MIXED_PATH_IR;
    return ALG_OK;
  }
  if (o.no_fallback) return ALG_CONVERGENCE;
  // ---- FP64 refactorization (A becomes its FP64 LU, like dgesv) ---------
  R.path = ALG_MIXED_PATH_FP64;
  int* perm = nullptr;
  ALG_TRY(ws_get(ctx, WS_PERM, sizeof(int) * n, reinterpret_cast<void**>(&perm)));
  ALG_TRY(status_reset(ctx));
  ALG_TRY((lu_factor_dev<double, false>(ctx, d_a, n, n, lda, ipiv, perm, default_plan(n, 8))));
  ALG_TRY(status_fetch(ctx));
  if (ctx->h_status->singular_col != INT_MAX) return ALG_SINGULAR;
  ALG_TRY((lu_solve_dev<double, false>(ctx, d_a, n, lda, perm, d_b, nrhs, ldb)));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  R.backward_error = -1.0;  // not measured on this path (A was overwritten)
  return ALG_OK;
}

}  // namespace alg

// ===========================================================================
// C entry points
// ===========================================================================
extern "C" {

void alg_mixed_opts_default(alg_mixed_opts* o) {
  if (o == nullptr) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = ALG_PREC_FP32;
  o->tol = 0.0;
  o->max_ir = 30;
  o->no_fallback = 0;
  o->no_gmres = 0;
  o->gmres_restart = 30;
  o->pivoting = ALG_PIVOT_AUTO;
}

int alg_dgesv_mixed_dev(alg_ctx* ctx, const alg_mixed_opts* opts, double* d_a, int n, int lda, double* d_b,
                        int nrhs, int ldb, alg_mixed_report* report) {
  if (ctx == nullptr) return ALG_INVALID_ARGUMENT;
  if (n < 0 || nrhs < 0 || lda < std::max(1, n) || ldb < std::max(1, n)) return ALG_BAD_SHAPE;
  alg_mixed_opts o;
  alg_mixed_opts_default(&o);
  if (opts) o = *opts;
  if (o.precision != ALG_PREC_FP32 && o.precision != ALG_PREC_TF32 && o.precision != ALG_PREC_BF16 &&
      o.precision != ALG_PREC_TF32X3)
    return ALG_INVALID_ARGUMENT;
  if (o.pivoting < ALG_PIVOT_AUTO || o.pivoting > ALG_PIVOT_TOURNAMENT) return ALG_INVALID_ARGUMENT;
  return alg::dgesv_mixed_dev(ctx, o, d_a, n, lda, d_b, nrhs, ldb, report);
}

int alg_dgesv_mixed(const alg_mixed_opts* opts, double* a, double* b, size_t n, size_t nrhs,
                    alg_mixed_report* report) {
  if (n == 0 || nrhs == 0) return ALG_OK;
  if (a == nullptr || b == nullptr) return ALG_INVALID_ARGUMENT;
  if (n > (size_t)INT_MAX / 2 || nrhs > 65535) return ALG_BAD_SHAPE;
  alg_ctx* ctx = nullptr;
  ALG_TRY(alg::default_ctx(&ctx));
  std::lock_guard<std::mutex> g(ctx->mu);
  double* d_a = nullptr;
  double* d_b = nullptr;
  ALG_TRY(alg::ws_get(ctx, alg::WS_A, sizeof(double) * n * n, reinterpret_cast<void**>(&d_a)));
  ALG_TRY(alg::ws_get(ctx, alg::WS_B, sizeof(double) * n * nrhs, reinterpret_cast<void**>(&d_b)));
  ALG_CUDA_TRY(cudaMemcpyAsync(d_a, a, sizeof(double) * n * n, cudaMemcpyHostToDevice, ctx->stream));
  ALG_CUDA_TRY(cudaMemcpyAsync(d_b, b, sizeof(double) * n * nrhs, cudaMemcpyHostToDevice, ctx->stream));
  alg_mixed_opts o;
  alg_mixed_opts_default(&o);
  if (opts) o = *opts;
  alg_mixed_report rep{};
  const int rc = alg::dgesv_mixed_dev(ctx, o, d_a, (int)n, (int)n, d_b, (int)nrhs, (int)n, &rep);
  if (rc == ALG_OK) {
    ALG_CUDA_TRY(cudaMemcpyAsync(b, d_b, sizeof(double) * n * nrhs, cudaMemcpyDeviceToHost, ctx->stream));
    if (rep.path == ALG_MIXED_PATH_FP64)
      ALG_CUDA_TRY(cudaMemcpyAsync(a, d_a, sizeof(double) * n * n, cudaMemcpyDeviceToHost, ctx->stream));
    ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  if (report) *report = rep;
  return rc;
}

}  // extern "C"
