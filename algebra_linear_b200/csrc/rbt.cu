// Random butterfly transformation (RBT) + LU without pivoting, the
// low-precision factorization of the mixed-precision solve.
//
// Method (Parker 1995; Baboulin, Dongarra, Herrmann, Tomov, "Accelerating
// linear system solutions using randomization techniques", ACM TOMS 2013):
// with U, V random recursive butterflies of depth 2, A_r = U^T A V can be
// factorized without pivoting with growth comparable to partial pivoting, and
// A x = b becomes A_r y = U^T b, x = V y. Here A_r is formed in FP64 and
// stored in FP32, factorized without pivoting (diagonal blocks in shared
// memory, the block columns by row-parallel triangular solves, the trailing
// updates on the tensor cores), and used as the preconditioner
// M^{-1} = V (L U)^{-1} U^T of the FP64 refinement. No pivot search means no
// column-by-column cross-CTA exchange on the critical path.
//
// A depth-2 butterfly W = diag(B1, B2) B of order n (n divisible by 4), with
// B = [R S; R -S] / sqrt(2) and B1, B2 of order n/2 built the same way, mixes
// only the four indices {i, i + n/4, i + n/2, i + 3n/4} of each orbit
// i < n/4, so U^T A V is computed orbit block by orbit block (16 entries in,
// 16 out). Diagonal entries are exp(rho / 10), rho uniform in [-1/2, 1/2]
// (Parker's choice), from a fixed-seed generator.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "dense.cuh"
#include "rbt.cuh"

namespace alg {
namespace {

constexpr double kInvSqrt2 = 0.70710678118654752440;

// 8 coefficient arrays of length n/4 per butterfly:
//   ra = R[i], sa = S[i], rb = R[i + n/4], sb = S[i + n/4] (first level),
//   r1, s1 (B1), r2, s2 (B2) at orbit index i.
struct Coef {
  const double* c;  // [8][q]
  int q;
  __device__ __forceinline__ double get(int k, int i) const { return c[(size_t)k * q + i]; }
};

// z = W x on one orbit: x0..x3 at i, i+q, i+2q, i+3q.
__device__ __forceinline__ void butterfly_apply(const Coef& w, int i, const double x[4], double z[4]) {
  const double ra = w.get(0, i), sa = w.get(1, i), rb = w.get(2, i), sb = w.get(3, i);
  const double r1 = w.get(4, i), s1 = w.get(5, i), r2 = w.get(6, i), s2 = w.get(7, i);
  const double y0 = (ra * x[0] + sa * x[2]) * kInvSqrt2;
  const double y2 = (ra * x[0] - sa * x[2]) * kInvSqrt2;
  const double y1 = (rb * x[1] + sb * x[3]) * kInvSqrt2;
  const double y3 = (rb * x[1] - sb * x[3]) * kInvSqrt2;
  z[0] = (r1 * y0 + s1 * y1) * kInvSqrt2;
  z[1] = (r1 * y0 - s1 * y1) * kInvSqrt2;
  z[2] = (r2 * y2 + s2 * y3) * kInvSqrt2;
  z[3] = (r2 * y2 - s2 * y3) * kInvSqrt2;
}

// z = W^T x on one orbit (the transpose of the two stages, in reverse order).
__device__ __forceinline__ void butterfly_apply_t(const Coef& w, int i, const double x[4], double z[4]) {
  const double ra = w.get(0, i), sa = w.get(1, i), rb = w.get(2, i), sb = w.get(3, i);
  const double r1 = w.get(4, i), s1 = w.get(5, i), r2 = w.get(6, i), s2 = w.get(7, i);
  // diag(B1, B2)^T
  const double y0 = r1 * (x[0] + x[1]) * kInvSqrt2;
  const double y1 = s1 * (x[0] - x[1]) * kInvSqrt2;
  const double y2 = r2 * (x[2] + x[3]) * kInvSqrt2;
  const double y3 = s2 * (x[2] - x[3]) * kInvSqrt2;
  // B^T
  z[0] = ra * (y0 + y2) * kInvSqrt2;
  z[2] = sa * (y0 - y2) * kInvSqrt2;
  z[1] = rb * (y1 + y3) * kInvSqrt2;
  z[3] = sb * (y1 - y3) * kInvSqrt2;
}

// A_r = U^T A V for every orbit pair (i0, j0); FP64 in, FP32 out.
__global__ void rbt_transform_kernel(const double* __restrict__ a, int lda, int n, Coef u, Coef v,
                                     float* __restrict__ ar, int ldr) {
  const int q = n / 4;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = blockIdx.y;
  if (i0 >= q) return;
  double blk[4][4];  // blk[t][s] = A[i0 + t q][j0 + s q]
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int t = 0; t < 4; ++t) blk[t][s] = a[(size_t)(i0 + t * q) + (size_t)(j0 + s * q) * lda];
  // left: columns of the block get U^T
  double tmp[4][4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    double x[4] = {blk[0][s], blk[1][s], blk[2][s], blk[3][s]}, z[4];
    butterfly_apply_t(u, i0, x, z);
#pragma unroll
    for (int t = 0; t < 4; ++t) tmp[t][s] = z[t];
  }
  // right: rows of the block get V (row vector times V = (V^T row^T)^T)
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    double x[4] = {tmp[t][0], tmp[t][1], tmp[t][2], tmp[t][3]}, z[4];
    butterfly_apply_t(v, j0, x, z);
#pragma unroll
    for (int s = 0; s < 4; ++s) ar[(size_t)(i0 + t * q) + (size_t)(j0 + s * q) * ldr] = (float)z[s];
  }
}

// z = U^T x (transpose = 1) or z = V x (transpose = 0) on a length-n vector.
__global__ void rbt_vector_kernel(const double* __restrict__ x, double* __restrict__ z, int n, Coef w,
                                  int transpose) {
  const int q = n / 4;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < q; i += gridDim.x * blockDim.x) {
    double xi[4] = {x[i], x[i + q], x[i + 2 * q], x[i + 3 * q]}, zi[4];
    if (transpose) butterfly_apply_t(w, i, xi, zi);
    else butterfly_apply(w, i, xi, zi);
    z[i] = zi[0];
    z[i + q] = zi[1];
    z[i + 2 * q] = zi[2];
    z[i + 3 * q] = zi[3];
  }
}

// ---- LU without pivoting --------------------------------------------------
constexpr int kDiagThreads = 512;

// Diagonal block (kb x kb, kb <= 128): LU in place without pivoting, then
// U11^{-1} into inv (kb x kb column-major, upper). Thread (g, i) owns row i
// and every fourth column of the update.
__global__ void __launch_bounds__(kDiagThreads) genp_diag_kernel(float* a, int lda, int k0, int kb, float* inv,
                                                                 DevStatus* st) {
  extern __shared__ float dsm[];
  const int ld = kb + 1;
  float* t = dsm;  // kb x ld, column-major
  for (int idx = threadIdx.x; idx < kb * kb; idx += kDiagThreads) {
    const int i = idx % kb, j = idx / kb;
    t[i + j * ld] = a[(size_t)(k0 + i) + (size_t)(k0 + j) * lda];
  }
  __syncthreads();
  const int i = threadIdx.x % 128, g = threadIdx.x / 128;
  for (int k = 0; k < kb; ++k) {
    const float d = t[k + k * ld];
    if (threadIdx.x == 0 && !(fabsf(d) > 0.f)) atomicMin(&st->singular_col, k0 + k);
    if (g == 0 && i > k && i < kb) t[i + k * ld] = __fdiv_rn(t[i + k * ld], d);
    __syncthreads();
    if (i > k && i < kb) {
      const float l = t[i + k * ld];
      for (int j = k + 1 + g; j < kb; j += 4) t[i + j * ld] = __fmaf_rn(-l, t[k + j * ld], t[i + j * ld]);
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < kb * kb; idx += kDiagThreads) {
    const int r = idx % kb, c = idx / kb;
    a[(size_t)(k0 + r) + (size_t)(k0 + c) * lda] = t[r + c * ld];
  }
  // U11^{-1}: column c solves U x = e_c by back substitution (thread per column)
  if (threadIdx.x < kb) {
    const int c = threadIdx.x;
    float* x = inv + (size_t)c * kb;
    for (int r = kb - 1; r > c; --r) x[r] = 0.f;
    x[c] = __frcp_rn(t[c + c * ld]);
    for (int r = c - 1; r >= 0; --r) {
      float s = 0.f;
      for (int k = r + 1; k <= c; ++k) s = __fmaf_rn(t[r + k * ld], x[k], s);
      x[r] = -__fdiv_rn(s, t[r + r * ld]);
    }
  }
}

// L21 = A21 U11^{-1} in place for rows [r0, m): a CTA takes 64 rows, stages
// them and U11^{-1} in shared memory and forms the product.
constexpr int kL21Rows = 64;
constexpr int kL21Threads = 256;
__global__ void __launch_bounds__(kL21Threads) genp_l21_kernel(float* a, int lda, int m, int k0, int kb, int r0,
                                                               const float* __restrict__ inv) {
  extern __shared__ float lsm[];
  float* iv = lsm;                       // kb x kb
  float* blk = lsm + kb * kb;            // kL21Rows x kb, [col][row]
  const int row0 = r0 + blockIdx.x * kL21Rows;
  const int rows = min(kL21Rows, m - row0);
  for (int idx = threadIdx.x; idx < kb * kb; idx += kL21Threads) iv[idx] = inv[idx];
  for (int idx = threadIdx.x; idx < kL21Rows * kb; idx += kL21Threads) {
    const int r = idx % kL21Rows, c = idx / kL21Rows;
    blk[idx] = r < rows ? a[(size_t)(row0 + r) + (size_t)(k0 + c) * lda] : 0.f;
  }
  __syncthreads();
  // thread (r, cg): row r, columns cg, cg+4, ...
  const int r = threadIdx.x % kL21Rows, cg = threadIdx.x / kL21Rows;
  if (r < rows) {
    for (int c = cg; c < kb; c += kL21Threads / kL21Rows) {
      float s = 0.f;
      for (int k = 0; k <= c; ++k) s = __fmaf_rn(blk[k * kL21Rows + r], iv[k + c * kb], s);
      a[(size_t)(row0 + r) + (size_t)(k0 + c) * lda] = s;
    }
  }
}

uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

int rbt_prepare(alg_ctx* ctx, int n, uint64_t seed, RbtState* st) {
  if (n % 4 != 0 || n < 4) return ALG_BAD_SHAPE;
  const int q = n / 4;
  std::vector<double> h((size_t)16 * q);
  uint64_t s = seed;
  for (auto& v : h) {
    const double rho = (double)(splitmix64(s) >> 11) * 0x1p-53 - 0.5;
    v = std::exp(rho / 10.0);
  }
  double* d = nullptr;
  ALG_TRY(ws_get(ctx, WS_RBT, sizeof(double) * h.size(), reinterpret_cast<void**>(&d)));
  ALG_CUDA_TRY(cudaMemcpyAsync(d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, ctx->stream));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // h is a host temporary
  st->n = n;
  st->u = d;
  st->v = d + (size_t)8 * q;
  return ALG_OK;
}

int rbt_transform(alg_ctx* ctx, const RbtState& st, const double* a, int lda, float* ar, int ldr) {
  const int q = st.n / 4;
  const int tok = prof_begin(ctx, ALG_K_CAST);
  rbt_transform_kernel<<<dim3((q + 127) / 128, q), 128, 0, ctx->stream>>>(a, lda, st.n, Coef{st.u, q},
                                                                           Coef{st.v, q}, ar, ldr);
  count_launches();
  prof_end(ctx, tok, 0.0, 12.0 * st.n * st.n);
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

int rbt_vector(alg_ctx* ctx, const RbtState& st, bool transpose_u, const double* x, double* z) {
  const int q = st.n / 4;
  const int g = std::max(1, std::min((q + 255) / 256, ctx->sm_count * 4));
  rbt_vector_kernel<<<g, 256, 0, ctx->stream>>>(x, z, st.n, Coef{transpose_u ? st.u : st.v, q},
                                                 transpose_u ? 1 : 0);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

int genp_factor(alg_ctx* ctx, int prec, float* a, int n, int lda, int nb) {
  nb = std::min(nb, 128);
  float* inv = nullptr;
  ALG_TRY(ws_get(ctx, WS_PRECOND, sizeof(float) * 128 * 128 + sizeof(float) * (size_t)n,
                 reinterpret_cast<void**>(&inv)));
  inv += n;  // the first n floats are the preconditioner's FP32 vector
  static const cudaError_t configured = [] {
    const cudaError_t e = cudaFuncSetAttribute(genp_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 80 * 1024);
    return e != cudaSuccess ? e
                            : cudaFuncSetAttribute(genp_l21_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   120 * 1024);
  }();
  ALG_CUDA_TRY(configured);
  for (int k0 = 0; k0 < n; k0 += nb) {
    const int kb = std::min(nb, n - k0);
    const int kr = k0 + kb;
    int tok = prof_begin(ctx, ALG_K_PANEL);
    genp_diag_kernel<<<1, kDiagThreads, sizeof(float) * kb * (kb + 1), ctx->stream>>>(a, lda, k0, kb, inv,
                                                                                      ctx->d_status);
    count_launches();
    if (kr < n) {
      genp_l21_kernel<<<(n - kr + kL21Rows - 1) / kL21Rows, kL21Threads,
                        sizeof(float) * (kb * kb + kL21Rows * kb), ctx->stream>>>(a, lda, n, k0, kb, kr, inv);
      count_launches();
    }
    prof_end(ctx, tok, 2.0 / 3.0 * kb * kb * kb + double(n - kr) * kb * kb, 0.0);
    ALG_CUDA_TRY(cudaGetLastError());
    if (kr < n) {
      ALG_TRY(trsm_lower_unit_f32(ctx, a, lda, k0, kb, kr, n));
      if (prec == ALG_PREC_FP32) {
        ALG_TRY((gemm_sub_dev<float, false>(ctx, n - kr, n - kr, kb, a + (size_t)kr + (size_t)k0 * lda, lda,
                                            a + (size_t)k0 + (size_t)kr * lda, lda, a + (size_t)kr + (size_t)kr * lda,
                                            lda)));
      } else {
        ALG_TRY(gemm_tc_sub_dev(ctx, prec, n - kr, n - kr, kb, a + (size_t)kr + (size_t)k0 * lda, lda,
                                a + (size_t)k0 + (size_t)kr * lda, lda, a + (size_t)kr + (size_t)kr * lda, lda));
      }
    }
  }
  return ALG_OK;
}

}  // namespace alg
