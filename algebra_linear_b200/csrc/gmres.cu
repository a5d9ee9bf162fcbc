// GMRES-based iterative refinement (GMRES-IR) in FP64 with a low-precision
// LU as preconditioner, for the mixed-precision solve when plain refinement
// stalls (the low-precision LU's error times the condition number is too
// large for refinement to contract).
//
// Outer loop (FP64): r = b - A x; stop when the normwise backward error is
// within tol; otherwise solve A d = r approximately with GMRES(m) on the
// left-preconditioned operator M^{-1} A (M^{-1} = the low-precision LU solve),
// then x += d. Inner GMRES: Arnoldi with classical Gram-Schmidt applied twice
// (CGS2) for the basis, Givens rotations on the host for the small
// Hessenberg least-squares problem. Every reduction (dot products, norms) is
// summed in a fixed order, so a run is deterministic.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gmres.cuh"
#include "mixed.cuh"

namespace alg {
namespace {

constexpr int kG = 256;   // threads per block
constexpr int kChunk = 2048;  // vector entries per reduction block

// partial[v * nchunks + chunk] = sum over the chunk of V[:, v] . w
__global__ void basis_dot_kernel(const double* __restrict__ V, int ldv, const double* __restrict__ w, int n,
                                 double* __restrict__ partial, int nchunks) {
  const int v = blockIdx.y, chunk = blockIdx.x;
  const int i0 = chunk * kChunk, i1 = min(n, i0 + kChunk);
  double s = 0.0;
  for (int i = i0 + threadIdx.x; i < i1; i += kG) s = __fma_rn(V[(size_t)v * ldv + i], w[i], s);
  __shared__ double red[kG / 32];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < kG / 32; ++k) t += red[k];
    partial[(size_t)v * nchunks + chunk] = t;
  }
}

// w -= V[:, 0:k] h
__global__ void basis_update_kernel(const double* __restrict__ V, int ldv, const double* __restrict__ h, int k,
                                    double* __restrict__ w, int n) {
  for (int i = blockIdx.x * kG + threadIdx.x; i < n; i += gridDim.x * kG) {
    double s = 0.0;
    for (int v = 0; v < k; ++v) s = __fma_rn(V[(size_t)v * ldv + i], h[v], s);
    w[i] -= s;
  }
}

// d += V[:, 0:k] y
__global__ void basis_combine_kernel(const double* __restrict__ V, int ldv, const double* __restrict__ y, int k,
                                     double* __restrict__ d, int n) {
  for (int i = blockIdx.x * kG + threadIdx.x; i < n; i += gridDim.x * kG) {
    double s = 0.0;
    for (int v = 0; v < k; ++v) s = __fma_rn(V[(size_t)v * ldv + i], y[v], s);
    d[i] += s;
  }
}

__global__ void scale_copy_kernel(const double* __restrict__ a, double alpha, double* __restrict__ o, int n) {
  for (int i = blockIdx.x * kG + threadIdx.x; i < n; i += gridDim.x * kG) o[i] = a[i] * alpha;
}

int grid_n(alg_ctx* ctx, int n) { return std::max(1, std::min((n + kG - 1) / kG, ctx->sm_count * 4)); }

// host-side fixed-order sums of the per-chunk partials
int dots(alg_ctx* ctx, const double* V, int ldv, int k, const double* w, int n, double* partial, double* h_out) {
  const int nchunks = (n + kChunk - 1) / kChunk;
  basis_dot_kernel<<<dim3(nchunks, k), kG, 0, ctx->stream>>>(V, ldv, w, n, partial, nchunks);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  std::vector<double> hp((size_t)nchunks * k);
  ALG_CUDA_TRY(cudaMemcpyAsync(hp.data(), partial, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, ctx->stream));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int v = 0; v < k; ++v) {
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s += hp[(size_t)v * nchunks + c];
    h_out[v] = s;
  }
  return ALG_OK;
}

}  // namespace

int gmres_ir_dev(alg_ctx* ctx, const double* a, int n, int lda, const double* b, double* x, double anorm,
                 const Precond& M, const GmresOpts& go, GmresResult* res) {
  const int m = std::max(2, go.restart);
  double* V = nullptr;  // n x (m+1) basis, then w, r, d, scratch
  ALG_TRY(ws_get(ctx, WS_GMRES, sizeof(double) * (size_t)n * (m + 6) + sizeof(double) * 4096,
                 reinterpret_cast<void**>(&V)));
  double* w = V + (size_t)n * (m + 1);
  double* r = w + n;
  double* d = r + n;
  double* t = d + n;
  double* partial = t + n;  // reduction scratch (<= 4096 doubles)
  double* hdev = partial + 2048;
  const int nchunks = (n + kChunk - 1) / kChunk;
  if ((size_t)nchunks * (m + 1) > 2048) return ALG_BAD_SHAPE;
  double rmax = 0, xmax = 0, bmax = 0;
  res->outer = res->inner = 0;
  double prev_eta = INFINITY;
  int stalled = 0;
  for (int outer = 0; outer < go.max_outer; ++outer) {
    ALG_TRY(residual_dev(ctx, a, n, lda, x, n, b, n, r, n, 1, &rmax, &xmax, &bmax));
    const double den = anorm * xmax + bmax;
    res->backward_error = den == 0.0 ? rmax : rmax / den;
    if (!(res->backward_error == res->backward_error)) return ALG_CONVERGENCE;
    if (res->backward_error <= go.tol) {
      res->converged = true;
      return ALG_OK;
    }
    // two restart cycles in a row that do not halve the backward error: the
    // preconditioner is too weak for this matrix; give up (the caller falls
    // back to the FP64 LU) instead of running out the cycle limit
    if (res->backward_error > 0.5 * prev_eta) {
      if (++stalled >= 2) return ALG_CONVERGENCE;
    } else {
      stalled = 0;
    }
    prev_eta = res->backward_error;
    // z0 = M^{-1} r, beta = ||z0||
    ALG_TRY(M(ctx, r, t));
    double beta = 0.0;
    ALG_TRY(dots(ctx, t, n, 1, t, n, partial, &beta));
    beta = std::sqrt(beta);
    if (!(beta > 0.0)) return ALG_CONVERGENCE;
    scale_copy_kernel<<<grid_n(ctx, n), kG, 0, ctx->stream>>>(t, 1.0 / beta, V, n);
    count_launches();
    std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1, 0.0), h(m + 1);
    g[0] = beta;
    int k = 0;
    for (; k < m; ++k) {
      // w = M^{-1} A v_k
      ALG_TRY(gemv_dev(ctx, a, n, lda, V + (size_t)k * n, t));
      ALG_TRY(M(ctx, t, w));
      // CGS2: h = V^T w; w -= V h; twice
      std::vector<double> hsum(k + 1, 0.0);
      for (int pass = 0; pass < 2; ++pass) {
        ALG_TRY(dots(ctx, V, n, k + 1, w, n, partial, h.data()));
        ALG_CUDA_TRY(cudaMemcpyAsync(hdev, h.data(), sizeof(double) * (k + 1), cudaMemcpyHostToDevice, ctx->stream));
        basis_update_kernel<<<grid_n(ctx, n), kG, 0, ctx->stream>>>(V, n, hdev, k + 1, w, n);
        count_launches();
        for (int v = 0; v <= k; ++v) hsum[v] += h[v];
      }
      double hn = 0.0;
      ALG_TRY(dots(ctx, w, n, 1, w, n, partial, &hn));
      hn = std::sqrt(hn);
      for (int v = 0; v <= k; ++v) H[(size_t)k * (m + 1) + v] = hsum[v];
      H[(size_t)k * (m + 1) + k + 1] = hn;
      // apply the previous rotations, then a new one that zeroes H[k+1][k]
      double* col = &H[(size_t)k * (m + 1)];
      for (int v = 0; v < k; ++v) {
        const double t0 = cs[v] * col[v] + sn[v] * col[v + 1];
        col[v + 1] = -sn[v] * col[v] + cs[v] * col[v + 1];
        col[v] = t0;
      }
      const double rr = std::hypot(col[k], col[k + 1]);
      cs[k] = rr == 0.0 ? 1.0 : col[k] / rr;
      sn[k] = rr == 0.0 ? 0.0 : col[k + 1] / rr;
      col[k] = rr;
      col[k + 1] = 0.0;
      g[k + 1] = -sn[k] * g[k];
      g[k] = cs[k] * g[k];
      res->inner += 1;
      if (hn > 0.0) {
        scale_copy_kernel<<<grid_n(ctx, n), kG, 0, ctx->stream>>>(w, 1.0 / hn, V + (size_t)(k + 1) * n, n);
        count_launches();
      }
      if (std::fabs(g[k + 1]) <= go.inner_tol * beta || hn == 0.0) {
        ++k;
        break;
      }
    }
    // y = R^{-1} g (back substitution on the rotated Hessenberg), d = V y, x += d
    std::vector<double> y(k, 0.0);
    for (int i = k - 1; i >= 0; --i) {
      double s = g[i];
      for (int j = i + 1; j < k; ++j) s -= H[(size_t)j * (m + 1) + i] * y[j];
      y[i] = s / H[(size_t)i * (m + 1) + i];
    }
    ALG_CUDA_TRY(cudaMemcpyAsync(hdev, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, ctx->stream));
    basis_combine_kernel<<<grid_n(ctx, n), kG, 0, ctx->stream>>>(V, n, hdev, k, x, n);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
    res->outer = outer + 1;
  }
  ALG_TRY(residual_dev(ctx, a, n, lda, x, n, b, n, r, n, 1, &rmax, &xmax, &bmax));
  const double den = anorm * xmax + bmax;
  res->backward_error = den == 0.0 ? rmax : rmax / den;
  res->converged = res->backward_error <= go.tol;
  return res->converged ? ALG_OK : ALG_CONVERGENCE;
}

}  // namespace alg
