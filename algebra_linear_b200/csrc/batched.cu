// Batched dgesv for many independent dense systems of uneven order, in one
// persistent launch per size bucket (capturable in a CUDA graph).
//
// Each system is the reference's dgesv (src/lapack/mod.rs:309-354): LU with
// partial pivoting (first index of max |a_ik|, NaN rule as the reference),
// multipliers by division, then the forward/back sweeps. A CTA pulls systems
// from a queue ordered by decreasing order n (largest first, for balance) and
// factorizes each one in place in its global buffer with a right-looking
// blocked schedule: a 16- or 32-column panel factored in shared memory, its row
// interchanges applied to the other columns by one gather, U12 by a
// row-block triangular solve, and the trailing update in 64 x 64 tiles (U12
// staged in shared memory, a register micro-tile per thread). The mixed form factorizes an FP32 copy and refines
// x in FP64 against the FP64 matrix until the system's normwise backward
// error is within tol.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <math_constants.h>

#include "batched.cuh"

namespace alg {
namespace {

constexpr int kMaxN = 512;    // largest order a CTA handles
constexpr int kT = 64;        // trailing-update tile
constexpr int kTR = 4;        // rows of a thread's micro-tile in the trailing update

template <typename T>
__device__ __forceinline__ T fma_t(T a, T b, T c);
template <>
__device__ __forceinline__ double fma_t<double>(double a, double b, double c) { return __fma_rn(a, b, c); }
template <>
__device__ __forceinline__ float fma_t<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }

__device__ __forceinline__ double pkey(double v, bool diag) {
  const double a = fabs(v);
  if (isnan(a)) return diag ? CUDART_INF : -CUDART_INF;
  return a;
}

// Block-wide first-index argmax of keys (largest key, lowest index among
// equals); returns the winning index to all threads. One barrier: each warp
// posts its best in a mailbox slot double-buffered by `par` (the caller
// alternates it per call, and its other barriers separate two calls with the
// same parity), and every warp reduces the mailboxes itself.
__device__ int block_argmax(double key, int idx, double* red_k, int* red_i, int par) {
  for (int off = 16; off > 0; off >>= 1) {
    const double ok = __shfl_down_sync(0xffffffffu, key, off);
    const int oi = __shfl_down_sync(0xffffffffu, idx, off);
    if (ok > key || (ok == key && oi < idx)) { key = ok; idx = oi; }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { red_k[16 * par + warp] = key; red_i[16 * par + warp] = idx; }
  __syncthreads();
  const int nw = (int)(blockDim.x >> 5);
  double k = lane < nw ? red_k[16 * par + lane] : -CUDART_INF;
  int i = lane < nw ? red_i[16 * par + lane] : INT_MAX;
  for (int off = 16; off > 0; off >>= 1) {
    const double ok = __shfl_xor_sync(0xffffffffu, k, off);
    const int oi = __shfl_xor_sync(0xffffffffu, i, off);
    if (ok > k || (ok == k && oi < i)) { k = ok; i = oi; }
  }
  return i;
}

// LU with partial pivoting of the n x n matrix a (global, leading dim n),
// in place; ipiv (global, n ints); returns 0 or 1 + the first singular column.
// Shared memory of cta_getrf for panels of up to `cap` rows.
template <typename T>
__host__ __device__ constexpr size_t getrf_smem(int cap, int pb) {
  return sizeof(T) * ((size_t)cap * pb + 2 * pb * kT) + 32 * 8 + 32 * 4 + (4 * pb + 4) * 4;
}

// NT: threads of the CTA; kPB: panel width (16 or 32, the autotuner's choice).
template <typename T, int NT, int kPB>
__device__ int cta_getrf(T* a, int n, int* ipiv, unsigned char* smem, int cap) {
  const int kMaxN = cap;                                   // panel stride (rows)
  T* panel = reinterpret_cast<T*>(smem);                   // cap x kPB, [col][row]
  T* ut = panel + (size_t)cap * kPB;                       // kPB x kT (U12 tile), [col][row]
  T* ct = ut + kPB * kT;                                   // staging (row labels)
  double* red_k = reinterpret_cast<double*>(ct + kT * kPB);
  int* red_i = reinterpret_cast<int*>(red_k + 32);
  int* mv = red_i + 32;        // row moves of the panel: dst [2*kPB], src [2*kPB]
  int* cnt = mv + 4 * kPB;
  int* info_s = cnt + 1;
  if (threadIdx.x == 0) *info_s = 0;
  __syncthreads();
  for (int k0 = 0; k0 < n; k0 += kPB) {
    const int w = min(kPB, n - k0);
    const int m = n - k0;  // panel rows
    // ---- panel into shared memory --------------------------------------
    for (int c = 0; c < w; ++c)
      for (int r = threadIdx.x; r < m; r += blockDim.x) panel[c * kMaxN + r] = a[(size_t)(k0 + r) + (size_t)(k0 + c) * n];
    // row labels for the interchanges of this panel
    int* lab = reinterpret_cast<int*>(ct);  // m ints (ct is free during the panel)
    for (int r = threadIdx.x; r < m; r += blockDim.x) lab[r] = r;
    __syncthreads();
    for (int j = 0; j < w; ++j) {
      double key = -CUDART_INF;
      int idx = INT_MAX;
      for (int r = j + threadIdx.x; r < m; r += blockDim.x) {
        const double kk = pkey((double)panel[j * kMaxN + r], r == j);
        if (kk > key) { key = kk; idx = r; }
      }
      const int p = block_argmax(key, idx, red_k, red_i, j & 1);
      const T d = panel[j * kMaxN + p];
      if (threadIdx.x == 0) {
        ipiv[k0 + j] = k0 + p;
        if (fabs((double)d) <= 0.0 && *info_s == 0) *info_s = k0 + j + 1;
      }
      if (p != j) {
        for (int c = threadIdx.x; c < w; c += blockDim.x) {
          const T t = panel[c * kMaxN + j];
          panel[c * kMaxN + j] = panel[c * kMaxN + p];
          panel[c * kMaxN + p] = t;
        }
        if (threadIdx.x == 0) {
          const int t = lab[j];
          lab[j] = lab[p];
          lab[p] = t;
        }
      }
      __syncthreads();
      // each row's multiplier and its rank-1 update by the same thread (the
      // pivot row, read here, is not written in this phase: no barrier between)
      for (int r = j + 1 + threadIdx.x; r < m; r += blockDim.x) {
        const T l = panel[j * kMaxN + r] / d;
        panel[j * kMaxN + r] = l;
        for (int c = j + 1; c < w; ++c) panel[c * kMaxN + r] = fma_t<T>(-l, panel[c * kMaxN + j], panel[c * kMaxN + r]);
      }
      __syncthreads();
    }
    for (int c = 0; c < w; ++c)
      for (int r = threadIdx.x; r < m; r += blockDim.x) a[(size_t)(k0 + r) + (size_t)(k0 + c) * n] = panel[c * kMaxN + r];
    // ---- the panel's interchanges on the other columns: one gather ----------
    if (threadIdx.x == 0) *cnt = 0;
    __syncthreads();
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      if (lab[r] != r) {
        const int s = atomicAdd(cnt, 1);
        if (s < 2 * kPB) { mv[s] = r; mv[2 * kPB + s] = lab[r]; }
      }
    }
    __syncthreads();
    const int moves = min(*cnt, 2 * kPB);
    // stage the moved rows 64 columns at a time in shared memory (ut and ct,
    // contiguous, hold 2 * kPB * kT entries): all reads of a chunk, then all writes
    T* stage = ut;
    for (int cb = 0; cb < n; cb += kT) {
      const int cw = min(kT, n - cb);
      for (int e = threadIdx.x; e < moves * cw; e += blockDim.x) {
        const int sidx = e / cw, c = cb + e % cw;
        if (c < k0 || c >= k0 + w) stage[e] = a[(size_t)(k0 + mv[2 * kPB + sidx]) + (size_t)c * n];
      }
      __syncthreads();
      for (int e = threadIdx.x; e < moves * cw; e += blockDim.x) {
        const int sidx = e / cw, c = cb + e % cw;
        if (c < k0 || c >= k0 + w) a[(size_t)(k0 + mv[sidx]) + (size_t)c * n] = stage[e];
      }
      __syncthreads();
    }
    const int kr = k0 + w;
    if (kr < n) {
      // ---- U12 = L11^{-1} A12, 64 columns at a time through shared memory ---
      for (int cb = kr; cb < n; cb += kT) {
        const int cw = min(kT, n - cb);
        for (int e = threadIdx.x; e < w * cw; e += blockDim.x) {
          const int i = e % w, c = e / w;
          stage[c * kPB + i] = a[(size_t)(k0 + i) + (size_t)(cb + c) * n];
        }
        __syncthreads();
        if (threadIdx.x < cw) {
          T* x = stage + threadIdx.x * kPB;
          for (int i = 1; i < w; ++i) {
            T acc = x[i];
            for (int kk = 0; kk < i; ++kk) acc = fma_t<T>(-panel[kk * kMaxN + i], x[kk], acc);
            x[i] = acc;
          }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < w * cw; e += blockDim.x) {
          const int i = e % w, c = e / w;
          a[(size_t)(k0 + i) + (size_t)(cb + c) * n] = stage[c * kPB + i];
        }
        __syncthreads();
      }
      // ---- A22 -= L21 U12 in 64 x 64 tiles ----------------------------------
      const int mt = n - kr;
      const int tiles = (mt + kT - 1) / kT;
      for (int tj = 0; tj < tiles; ++tj) {
        const int c0 = kr + tj * kT, cw = min(kT, n - c0);
        for (int idx2 = threadIdx.x; idx2 < w * kT; idx2 += blockDim.x) {
          const int kk = idx2 % kPB, c = idx2 / kPB;
          if (kk < w) ut[c * kPB + kk] = c < cw ? a[(size_t)(k0 + kk) + (size_t)(c0 + c) * n] : T(0);
        }
        __syncthreads();
        // register micro-tile per thread: kTR rows (tr + 16 i) x kTC columns
        // (tc + kCG j) of the 64 x 64 tile; each entry's terms are still
        // accumulated in increasing kk, one fused multiply-add each
        constexpr int kRG = kT / kTR, kCG = NT / kRG, kTC = kT / kCG;
        static_assert(kRG * kCG == NT && kCG * kTC == kT, "micro-tile covers the tile");
        const int tr = threadIdx.x % kRG, tc = threadIdx.x / kRG;
        for (int ti = 0; ti < tiles; ++ti) {
          const int r0 = kr + ti * kT, rw = min(kT, n - r0);
          T acc[kTR][kTC];
#pragma unroll
          for (int i = 0; i < kTR; ++i)
#pragma unroll
            for (int j = 0; j < kTC; ++j) {
              const int r = tr + kRG * i, c = tc + kCG * j;
              acc[i][j] = (r < rw && c < cw) ? a[(size_t)(r0 + r) + (size_t)(c0 + c) * n] : T(0);
            }
          const T* lcol = panel + (r0 - k0);
          for (int kk = 0; kk < w; ++kk) {
            T l[kTR], u[kTC];
#pragma unroll
            for (int i = 0; i < kTR; ++i) {
              const int r = tr + kRG * i;
              l[i] = r < rw ? lcol[kk * kMaxN + r] : T(0);
            }
#pragma unroll
            for (int j = 0; j < kTC; ++j) u[j] = ut[(tc + kCG * j) * kPB + kk];
#pragma unroll
            for (int i = 0; i < kTR; ++i)
#pragma unroll
              for (int j = 0; j < kTC; ++j) acc[i][j] = fma_t<T>(-l[i], u[j], acc[i][j]);
          }
#pragma unroll
          for (int i = 0; i < kTR; ++i)
#pragma unroll
            for (int j = 0; j < kTC; ++j) {
              const int r = tr + kRG * i, c = tc + kCG * j;
              if (r < rw && c < cw) a[(size_t)(r0 + r) + (size_t)(c0 + c) * n] = acc[i][j];
            }
        }
        __syncthreads();
      }
    }
    __syncthreads();
  }
  const int info = *info_s;
  __syncthreads();
  return info;
}

// x <- (LU)^{-1} P x for one vector (global), LU n x n in global, x staged in shared memory.
template <typename T, typename V>
__device__ void cta_getrs(const T* lu, int n, const int* ipiv, V* x, V* xs) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = x[i];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < n; ++k) {
      const int p = ipiv[k];
      if (p != k) { const V t = xs[k]; xs[k] = xs[p]; xs[p] = t; }
    }
  __syncthreads();
  // forward (unit lower), column sweep
  for (int j = 0; j < n; ++j) {
    const V xj = xs[j];
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) xs[i] -= (V)lu[(size_t)i + (size_t)j * n] * xj;
    __syncthreads();
  }
  // backward (upper), column sweep
  for (int j = n - 1; j >= 0; --j) {
    if (threadIdx.x == 0) xs[j] = xs[j] / (V)lu[(size_t)j + (size_t)j * n];
    __syncthreads();
    const V xj = xs[j];
    for (int i = threadIdx.x; i < j; i += blockDim.x) xs[i] -= (V)lu[(size_t)i + (size_t)j * n] * xj;
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = xs[i];
  __syncthreads();
}

// Normwise backward error of x for A x = b (FP64, A n x n in global).
__device__ double cta_backward_error(const double* a, int n, const double* x, const double* b, double* rs,
                                     double* red) {
  double rmax = 0.0, amax = 0.0, xmax = 0.0, bmax = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double s = 0.0, ra = 0.0;
    for (int j = 0; j < n; ++j) {
      const double aij = a[(size_t)i + (size_t)j * n];
      s = __fma_rn(aij, x[j], s);
      ra += fabs(aij);
    }
    rs[i] = b[i] - s;
    rmax = fmax(rmax, fabs(rs[i]));
    amax = fmax(amax, ra);
    xmax = fmax(xmax, fabs(x[i]));
    bmax = fmax(bmax, fabs(b[i]));
  }
  for (int off = 16; off > 0; off >>= 1) {
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, off));
    amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, off));
    xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, off));
    bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, off));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[4 * warp + 0] = rmax;
    red[4 * warp + 1] = amax;
    red[4 * warp + 2] = xmax;
    red[4 * warp + 3] = bmax;
  }
  __syncthreads();
  double R = 0, A = 0, X = 0, B = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    R = fmax(R, red[4 * w + 0]);
    A = fmax(A, red[4 * w + 1]);
    X = fmax(X, red[4 * w + 2]);
    B = fmax(B, red[4 * w + 3]);
  }
  __syncthreads();
  const double den = A * X + B;
  return den == 0.0 ? R : R / den;
}

struct BatchArgs {
  int count;
  const int* order;        // systems of this bucket, largest first
  const int* n;
  const long long* a_off;  // offsets (entries) of A in a
  const long long* b_off;  // offsets of b in b
  double* a;               // FP64 matrices (overwritten by the LU in the FP64 form)
  double* b;               // right-hand sides -> solutions
  float* a32;              // FP32 working copies (mixed form), same offsets as a
  int* ipiv;               // same offsets as b
  double* work;            // same offsets as b: residual / correction
  int* info;               // per system: 0, 1 + singular column, or -(iterations+1) without convergence
  double* eta;             // per system backward error (mixed form)
  int* queue;              // work counter
  int cap;                 // largest order in the bucket
  int mixed;               // 0: FP64 LU; 1: FP32 LU + FP64 refinement
  int max_ir;
  double tol_scale;        // tol = tol_scale * n * 2^-53
};

template <int NT, int PB>
__global__ void __launch_bounds__(NT) batched_gesv_kernel(BatchArgs p) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int next;
  __shared__ double red[4 * (NT / 32)];
  double* vs = reinterpret_cast<double*>(smem);   // cap doubles for vectors
  unsigned char* lus = smem + sizeof(double) * p.cap;
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(p.queue, 1);
    __syncthreads();
    const int q = next;
    __syncthreads();
    if (q >= p.count) return;
    const int s = p.order[q];
    const int n = p.n[s];
    double* a = p.a + p.a_off[s];
    double* b = p.b + p.b_off[s];
    int* ipiv = p.ipiv + p.b_off[s];
    if (!p.mixed) {
      const int info = cta_getrf<double, NT, PB>(a, n, ipiv, lus, p.cap);
      if (threadIdx.x == 0) p.info[s] = info;
      if (info == 0) cta_getrs<double, double>(a, n, ipiv, b, vs);
      continue;
    }
    // ---- mixed: FP32 LU, FP64 refinement against the FP64 matrix ------------
    float* a32 = p.a32 + p.a_off[s];
    for (size_t e = threadIdx.x; e < (size_t)n * n; e += NT) a32[e] = __double2float_rn(a[e]);
    __syncthreads();
    const int info = cta_getrf<float, NT, PB>(a32, n, ipiv, lus, p.cap);
    if (info != 0) {
      if (threadIdx.x == 0) p.info[s] = info;
      continue;
    }
    double* x = p.work + p.b_off[s];               // correction / residual (global)
    double* sol = vs;                              // solution (shared)
    double* r = reinterpret_cast<double*>(lus);    // solve staging (the panel area is free now)
    for (int i = threadIdx.x; i < n; i += NT) x[i] = b[i];
    __syncthreads();
    cta_getrs<float, double>(a32, n, ipiv, x, r);
    for (int i = threadIdx.x; i < n; i += NT) sol[i] = x[i];
    __syncthreads();
    const double tol = p.tol_scale * n * 0x1p-53;
    int it = 0;
    double e = 0.0;
    for (;;) {
      e = cta_backward_error(a, n, sol, b, x, red);  // also x = b - A sol
      if (e <= tol || it >= p.max_ir || !(e == e)) break;
      cta_getrs<float, double>(a32, n, ipiv, x, r);
      for (int i = threadIdx.x; i < n; i += NT) sol[i] += x[i];
      __syncthreads();
      ++it;
    }
    for (int i = threadIdx.x; i < n; i += NT) b[i] = sol[i];
    if (threadIdx.x == 0) {
      p.info[s] = (e <= tol) ? 0 : -(it + 1);
      p.eta[s] = e;
    }
    __syncthreads();
  }
}

size_t kernel_smem(int cap, bool mixed, int pb) {
  const size_t g = mixed ? getrf_smem<float>(cap, pb) : getrf_smem<double>(cap, pb);
  return sizeof(double) * (size_t)cap + std::max(g, sizeof(double) * (size_t)cap) + 64;
}
// one limit for every bucket sharing an instantiation: the largest any asks for
size_t kernel_smem_max() {
  return std::max(kernel_smem(kMaxN, false, 32), kernel_smem(kMaxN, true, 32));
}

// Host-side configuration (not stream work, so never inside a graph capture).
template <int NT, int PB>
int configure_bucket(alg_ctx* ctx, int cap, bool mixed, int count, int* grid) {
  const size_t smem = kernel_smem(cap, mixed, PB);
  ALG_CUDA_TRY(cudaFuncSetAttribute(batched_gesv_kernel<NT, PB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kernel_smem_max()));
  int per_sm = 0;
  ALG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_gesv_kernel<NT, PB>, NT, smem));
  *grid = std::max(1, std::min(std::max(1, per_sm) * ctx->sm_count, count));
  return ALG_OK;
}

template <int NT, int PB>
int launch_bucket(alg_ctx* ctx, const BatchArgs& p, int grid) {
  const size_t smem = kernel_smem(p.cap, p.mixed != 0, PB);
  batched_gesv_kernel<NT, PB><<<grid, NT, smem, ctx->stream>>>(p);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

}  // namespace

int batch_launch_bucket(alg_ctx* ctx, const BatchSpec& sp, const BucketLaunch& bl) {
  BatchArgs p;
  p.count = bl.count;
  p.order = bl.d_order;
  p.n = sp.d_n;
  p.a_off = sp.d_a_off;
  p.b_off = sp.d_b_off;
  p.a = sp.d_a;
  p.b = sp.d_b;
  p.a32 = sp.d_a32;
  p.ipiv = sp.d_ipiv;
  p.work = sp.d_work;
  p.info = sp.d_info;
  p.eta = sp.d_eta;
  p.queue = bl.d_queue;
  p.cap = bl.cap;
  p.mixed = sp.mixed;
  p.max_ir = sp.max_ir > 0 ? sp.max_ir : 10;
  p.tol_scale = sp.tol_scale > 0 ? sp.tol_scale : 10.0;
  ALG_CUDA_TRY(cudaMemsetAsync(bl.d_queue, 0, sizeof(int), ctx->stream));
  const bool narrow = bl.panel == 16;
  switch (bl.threads) {
    case 128: return narrow ? launch_bucket<128, 16>(ctx, p, bl.grid) : launch_bucket<128, 32>(ctx, p, bl.grid);
    case 512: return narrow ? launch_bucket<512, 16>(ctx, p, bl.grid) : launch_bucket<512, 32>(ctx, p, bl.grid);
    default: return narrow ? launch_bucket<256, 16>(ctx, p, bl.grid) : launch_bucket<256, 32>(ctx, p, bl.grid);
  }
}

int batch_configure_bucket(alg_ctx* ctx, bool mixed, BucketLaunch* bl) {
  if (bl->panel != 16) bl->panel = 32;
  const bool narrow = bl->panel == 16;
  switch (bl->threads) {
    case 128:
      return narrow ? configure_bucket<128, 16>(ctx, bl->cap, mixed, bl->count, &bl->grid)
                    : configure_bucket<128, 32>(ctx, bl->cap, mixed, bl->count, &bl->grid);
    case 512:
      return narrow ? configure_bucket<512, 16>(ctx, bl->cap, mixed, bl->count, &bl->grid)
                    : configure_bucket<512, 32>(ctx, bl->cap, mixed, bl->count, &bl->grid);
    default:
      bl->threads = 256;
      return narrow ? configure_bucket<256, 16>(ctx, bl->cap, mixed, bl->count, &bl->grid)
                    : configure_bucket<256, 32>(ctx, bl->cap, mixed, bl->count, &bl->grid);
  }
}

int batch_max_order() { return kMaxN; }

}  // namespace alg

// ===========================================================================
// Plans and C entry points
// ===========================================================================
struct alg_batch {
  alg_ctx* ctx = nullptr;
  int count = 0;
  int mixed = 0;
  std::vector<int> n;
  std::vector<long long> a_off, b_off;
  long long a_total = 0, b_total = 0;
  double flops = 0.0;
  // device
  int* d_n = nullptr;
  long long* d_a_off = nullptr;
  long long* d_b_off = nullptr;
  int* d_order = nullptr;
  int* d_queues = nullptr;
  int* d_ipiv = nullptr;
  double* d_work = nullptr;
  double* d_eta = nullptr;
  float* d_a32 = nullptr;
  std::vector<alg::BucketLaunch> buckets;
  // captured graph of the launch sequence (for fixed buffers)
  cudaGraphExec_t graph = nullptr;
  cudaStream_t cap_stream = nullptr;  // capture stream (the context's may be the legacy stream)
  double* g_a = nullptr;
  double* g_b = nullptr;
  int* g_info = nullptr;
};

namespace {

// Size buckets (orders): the shared-memory panel of a CTA is sized for the
// largest order of its bucket, so small systems keep many CTAs per SM.
const int kBucketCaps[] = {32, 64, 128, 256, 512};

void free_batch(alg_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  for (void* p : {(void*)b->d_n, (void*)b->d_a_off, (void*)b->d_b_off, (void*)b->d_order, (void*)b->d_queues,
                  (void*)b->d_ipiv, (void*)b->d_work, (void*)b->d_eta, (void*)b->d_a32})
    if (p) cudaFree(p);
}

int issue(alg_batch* b, double* d_a, double* d_b, int* d_info) {
  alg::BatchSpec sp;
  sp.count = b->count;
  sp.d_n = b->d_n;
  sp.d_a_off = b->d_a_off;
  sp.d_b_off = b->d_b_off;
  sp.d_a = d_a;
  sp.d_b = d_b;
  sp.d_a32 = b->d_a32;
  sp.d_ipiv = b->d_ipiv;
  sp.d_work = b->d_work;
  sp.d_info = d_info;
  sp.d_eta = b->d_eta;
  sp.mixed = b->mixed;
  sp.flops = b->flops;
  const int tok = alg::prof_begin(b->ctx, ALG_K_BATCH);
  for (const auto& bl : b->buckets) ALG_TRY(alg::batch_launch_bucket(b->ctx, sp, bl));
  alg::prof_end(b->ctx, tok, b->flops, 8.0 * (double)b->a_total);
  return ALG_OK;
}

}  // namespace

extern "C" {

int alg_batch_create(alg_ctx* ctx, int count, const int* n_host, int mixed, alg_batch** out) {
  if (ctx == nullptr || out == nullptr || count < 0 || (count > 0 && n_host == nullptr)) return ALG_INVALID_ARGUMENT;
  for (int i = 0; i < count; ++i)
    if (n_host[i] < 1 || n_host[i] > alg::batch_max_order()) return ALG_BAD_SHAPE;
  auto* b = new alg_batch();
  b->ctx = ctx;
  b->count = count;
  b->mixed = mixed ? 1 : 0;
  b->n.assign(n_host, n_host + count);
  b->a_off.resize(count);
  b->b_off.resize(count);
  for (int i = 0; i < count; ++i) {
    b->a_off[i] = b->a_total;
    b->b_off[i] = b->b_total;
    b->a_total += (long long)b->n[i] * b->n[i];
    b->b_total += b->n[i];
    const double nn = b->n[i];
    b->flops += 2.0 / 3.0 * nn * nn * nn + 2.0 * nn * nn;
  }
  // order: bucket by cap, largest orders first inside each bucket
  std::vector<int> idx(count);
  for (int i = 0; i < count; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return b->n[x] > b->n[y]; });
  auto fail = [&](int rc) {
    free_batch(b);
    delete b;
    *out = nullptr;
    return rc;
  };
  auto dmalloc = [&](void** p, size_t bytes) { return cudaMalloc(p, std::max<size_t>(bytes, 16)); };
  if (dmalloc((void**)&b->d_n, sizeof(int) * count) || dmalloc((void**)&b->d_a_off, 8 * (size_t)count) ||
      dmalloc((void**)&b->d_b_off, 8 * (size_t)count) || dmalloc((void**)&b->d_order, sizeof(int) * count) ||
      dmalloc((void**)&b->d_queues, sizeof(int) * 16) || dmalloc((void**)&b->d_ipiv, sizeof(int) * b->b_total) ||
      dmalloc((void**)&b->d_work, sizeof(double) * b->b_total) || dmalloc((void**)&b->d_eta, sizeof(double) * count))
    return fail(ALG_OUT_OF_DEVICE_MEMORY);
  if (b->mixed && dmalloc((void**)&b->d_a32, sizeof(float) * b->a_total)) return fail(ALG_OUT_OF_DEVICE_MEMORY);
  cudaMemcpyAsync(b->d_n, b->n.data(), sizeof(int) * count, cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(b->d_a_off, b->a_off.data(), 8 * (size_t)count, cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(b->d_b_off, b->b_off.data(), 8 * (size_t)count, cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(b->d_order, idx.data(), sizeof(int) * count, cudaMemcpyHostToDevice, ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail(ALG_CUDA_ERROR);
  int pos = 0, qi = 0;
  for (int bi = (int)(sizeof(kBucketCaps) / sizeof(int)) - 1; bi >= 0 && pos < count; --bi) {
    const int lo = bi > 0 ? kBucketCaps[bi - 1] : 0;
    int end = pos;
    while (end < count && b->n[idx[end]] > lo) ++end;
    if (end > pos) {
      alg::BucketLaunch bl;
      bl.count = end - pos;
      bl.cap = kBucketCaps[bi];
      bl.threads = kBucketCaps[bi] >= 256 ? 512 : (kBucketCaps[bi] >= 64 ? 256 : 128);
      bl.d_order = b->d_order + pos;
      bl.d_queue = b->d_queues + qi++;
      const int rc = alg::batch_configure_bucket(ctx, b->mixed != 0, &bl);
      if (rc != ALG_OK) return fail(rc);
      b->buckets.push_back(bl);
    }
    pos = end;
  }
  *out = b;
  return ALG_OK;
}

int alg_batch_offsets(const alg_batch* b, int64_t* a_off, int64_t* b_off) {
  if (b == nullptr) return ALG_INVALID_ARGUMENT;
  for (int i = 0; i < b->count; ++i) {
    if (a_off) a_off[i] = b->a_off[i];
    if (b_off) b_off[i] = b->b_off[i];
  }
  return ALG_OK;
}

int alg_batch_solve(alg_batch* b, double* d_a, double* d_b, int* d_info) {
  if (b == nullptr || (b->count > 0 && (d_a == nullptr || d_b == nullptr || d_info == nullptr)))
    return ALG_INVALID_ARGUMENT;
  return issue(b, d_a, d_b, d_info);
}

int alg_batch_solve_graph(alg_batch* b, double* d_a, double* d_b, int* d_info) {
  if (b == nullptr || (b->count > 0 && (d_a == nullptr || d_b == nullptr || d_info == nullptr)))
    return ALG_INVALID_ARGUMENT;
  alg_ctx* ctx = b->ctx;
  if (b->graph == nullptr || b->g_a != d_a || b->g_b != d_b || b->g_info != d_info) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    // configure the kernels outside the capture (attributes are not stream work)
    ALG_TRY(issue(b, d_a, d_b, d_info));
    ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (b->cap_stream == nullptr) ALG_CUDA_TRY(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    // capture on the plan's own stream, issuing through the context meanwhile
    cudaStream_t saved = ctx->stream;
    ctx->stream = b->cap_stream;
    const bool prof = ctx->prof_on;
    ctx->prof_on = false;
    cudaError_t e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
    int rc = e == cudaSuccess ? issue(b, d_a, d_b, d_info) : ALG_CUDA_ERROR;
    if (e == cudaSuccess) e = cudaStreamEndCapture(b->cap_stream, &g);
    ctx->prof_on = prof;
    ctx->stream = saved;
    if (rc != ALG_OK) return rc;
    ALG_CUDA_TRY(e);
    ALG_CUDA_TRY(cudaGraphInstantiate(&b->graph, g, 0));
    cudaGraphDestroy(g);
    b->g_a = d_a;
    b->g_b = d_b;
    b->g_info = d_info;
    return ALG_OK;  // the warm-up issue above already solved this batch
  }
  const int tok = alg::prof_begin(ctx, ALG_K_BATCH);
  ALG_CUDA_TRY(cudaGraphLaunch(b->graph, ctx->stream));
  alg::count_launches(b->buckets.size());
  alg::prof_end(ctx, tok, b->flops, 8.0 * (double)b->a_total);
  return ALG_OK;
}

// Tries every launch shape for each bucket on the given batch (which it
// solves several times: pass scratch copies) and keeps the fastest: 128 / 256
// / 512 threads per CTA (with the trailing update's micro-tile 4 x 8, 4 x 4
// or 4 x 2 per thread) times a 16- or 32-column panel (the split between the
// column-serial panel and the register-tiled update).
int alg_batch_autotune(alg_batch* b, double* d_a, double* d_b, int* d_info, const double* d_a_src,
                       const double* d_b_src, int* threads_out) {
  if (b == nullptr) return ALG_INVALID_ARGUMENT;
  alg_ctx* ctx = b->ctx;
  cudaEvent_t e0, e1;
  ALG_CUDA_TRY(cudaEventCreate(&e0));
  ALG_CUDA_TRY(cudaEventCreate(&e1));
  alg::BatchSpec sp;
  sp.count = b->count;
  sp.d_n = b->d_n;
  sp.d_a_off = b->d_a_off;
  sp.d_b_off = b->d_b_off;
  sp.d_a = d_a;
  sp.d_b = d_b;
  sp.d_a32 = b->d_a32;
  sp.d_ipiv = b->d_ipiv;
  sp.d_work = b->d_work;
  sp.d_info = d_info;
  sp.d_eta = b->d_eta;
  sp.mixed = b->mixed;
  for (size_t k = 0; k < b->buckets.size(); ++k) {
    auto& bl = b->buckets[k];
    float best = 1e30f;
    int best_t = bl.threads, best_p = bl.panel;
    for (int cfg = 0; cfg < 6; ++cfg) {
      const int t = 128 << (cfg >> 1), pb = (cfg & 1) ? 32 : 16;
      alg::BucketLaunch trial = bl;
      trial.threads = t;
      trial.panel = pb;
      ALG_TRY(alg::batch_configure_bucket(ctx, b->mixed != 0, &trial));
      for (int rep = 0; rep < 2; ++rep) {
        ALG_CUDA_TRY(cudaMemcpyAsync(d_a, d_a_src, 8 * (size_t)b->a_total, cudaMemcpyDeviceToDevice, ctx->stream));
        ALG_CUDA_TRY(cudaMemcpyAsync(d_b, d_b_src, 8 * (size_t)b->b_total, cudaMemcpyDeviceToDevice, ctx->stream));
        ALG_CUDA_TRY(cudaEventRecord(e0, ctx->stream));
        ALG_TRY(alg::batch_launch_bucket(ctx, sp, trial));
        ALG_CUDA_TRY(cudaEventRecord(e1, ctx->stream));
        ALG_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        ALG_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (rep == 1 && ms < best) {
          best = ms;
          best_t = t;
          best_p = pb;
        }
      }
    }
    bl.threads = best_t;
    bl.panel = best_p;
    ALG_TRY(alg::batch_configure_bucket(ctx, b->mixed != 0, &bl));
    if (threads_out) threads_out[k] = best_t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return ALG_OK;
}

int alg_batch_info(const alg_batch* b, int* n_buckets, int* caps, int* threads, int* counts, double* flops) {
  if (b == nullptr) return ALG_INVALID_ARGUMENT;
  if (n_buckets) *n_buckets = (int)b->buckets.size();
  for (size_t k = 0; k < b->buckets.size(); ++k) {
    if (caps) caps[k] = b->buckets[k].cap;
    if (threads) threads[k] = b->buckets[k].threads;
    if (counts) counts[k] = b->buckets[k].count;
  }
  if (flops) *flops = b->flops;
  return ALG_OK;
}

int alg_batch_panels(const alg_batch* b, int* panels) {
  if (b == nullptr || panels == nullptr) return ALG_INVALID_ARGUMENT;
  for (size_t k = 0; k < b->buckets.size(); ++k) panels[k] = b->buckets[k].panel;
  return ALG_OK;
}

int alg_batch_set_config(alg_batch* b, int bucket, int threads, int panel) {
  if (b == nullptr || bucket < 0 || bucket >= (int)b->buckets.size()) return ALG_INVALID_ARGUMENT;
  if ((threads != 128 && threads != 256 && threads != 512) || (panel != 16 && panel != 32))
    return ALG_INVALID_ARGUMENT;
  alg::BucketLaunch& bl = b->buckets[bucket];
  bl.threads = threads;
  bl.panel = panel;
  ALG_TRY(alg::batch_configure_bucket(b->ctx, b->mixed != 0, &bl));
  if (b->graph) {  // the captured launches used the old shape
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return ALG_OK;
}

int alg_batch_eta(const alg_batch* b, double* eta_host) {
  if (b == nullptr || eta_host == nullptr) return ALG_INVALID_ARGUMENT;
  ALG_CUDA_TRY(cudaMemcpy(eta_host, b->d_eta, sizeof(double) * b->count, cudaMemcpyDeviceToHost));
  return ALG_OK;
}

int alg_batch_ipiv(const alg_batch* b, int* ipiv_host) {
  if (b == nullptr || ipiv_host == nullptr) return ALG_INVALID_ARGUMENT;
  if (b->b_total == 0) return ALG_OK;
  ALG_CUDA_TRY(cudaMemcpy(ipiv_host, b->d_ipiv, sizeof(int) * b->b_total, cudaMemcpyDeviceToHost));
  return ALG_OK;
}

// Frees the plan's device buffers (cudaFree waits for work that uses them).
// Does not touch the context, which the caller may already have destroyed.
void alg_batch_destroy(alg_batch* b) {
  if (b == nullptr) return;
  free_batch(b);
  delete b;
}

}  // extern "C"

// ===========================================================================
// Allocation-free solve of one small system (no counterpart in the reference)
// ===========================================================================
// Some callers cannot call cudaMalloc: code running inside another library's
// memory pool that owns the device's free memory, serving loops where the
// implicit device-wide synchronisation of cudaMalloc/cudaFree would stall
// unrelated streams, and callers that must never fail with out-of-memory after
// start-up. alg_dgesv_mixed_noalloc serves them: it runs the mixed form of the
// batched kernel above (FP32 LU with partial pivoting, FP64 refinement) on
// one system, and takes its working memory (the FP32 copy of A, the residual
// vector, the work counter) from the file-scope array below instead of from
// an allocation. Set-up per device (the array's address, the kernels' load
// and the shared-memory limit) is host-side work done by the first call in
// each CUDA context; a call with n = 0 does only the set-up. Every call on a
// device shares the one array, so calls that overlap on the GPU (different
// streams, or different host threads) race on it; calls on one stream are
// ordered and safe.
namespace alg {
namespace {

constexpr int kNoAllocMaxN = 512;
// Layout: FP32 copy of A (max order squared), residual (max order doubles),
// pivots (max order ints), then a 256-byte header of per-call fields.
constexpr size_t kNoAllocA32 = sizeof(float) * (size_t)kNoAllocMaxN * kNoAllocMaxN;
constexpr size_t kNoAllocWork = sizeof(double) * kNoAllocMaxN;
constexpr size_t kNoAllocIpiv = sizeof(int) * kNoAllocMaxN;
constexpr size_t kNoAllocHeader = 256;
constexpr size_t kNoAllocBytes = kNoAllocA32 + kNoAllocWork + kNoAllocIpiv + kNoAllocHeader;
static_assert(kNoAllocBytes == 1054976, "scratch size is part of the C interface");

struct NoAllocHeader {
  long long a_off;  // offset of the system in A, b, pivots and the FP32 copy (always 0)
  long long b_off;
  int queue;        // work counter of the persistent kernel: must be 0 when it starts
  int order;        // queue position -> system (always 0)
  int n;            // the system's order
  int info;         // spare slot (the caller's info pointer is required)
  double eta;       // used when the caller passes no backward-error pointer
};
static_assert(sizeof(NoAllocHeader) <= kNoAllocHeader, "header fits its slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Writes the per-call header, in stream order before the solve kernel; this
// is what resets the work counter to 0 for each call.
__global__ void noalloc_header_kernel(NoAllocHeader* h, int n) {
  h->a_off = 0;
  h->b_off = 0;
  h->queue = 0;
  h->order = 0;
  h->n = n;
  h->info = 0;
  h->eta = 0.0;
}

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
// Per device: the array's address and the unique id (cuCtxGetId) of the CUDA
// context it was looked up in. A __device__ symbol's address belongs to one
// context; after cudaDeviceReset, or when the caller makes another context
// current, the id differs and the set-up runs again.
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};
unsigned long long g_noalloc_ctx[kNoAllocMaxDevices] = {};

// The two driver calls are reached through the runtime's entry-point table,
// so the library does not link libcuda (it stays loadable on hosts without
// a driver, where every call reports ALG_NO_DEVICE).
int current_context_id(unsigned long long* id) {
  static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
  static PFN_cuCtxGetId_v12000 get_id = nullptr;
  if (get_current == nullptr || get_id == nullptr) {
    cudaDriverEntryPointQueryResult q1, q2;
    void* f1 = nullptr;
    void* f2 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
      cudaGetLastError();
      return ALG_CUDA_ERROR;
    }
    get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f1);
    get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f2);
  }
  CUcontext c = nullptr;
  if (get_current(&c) != CUDA_SUCCESS || c == nullptr) return ALG_CUDA_ERROR;
  if (get_id(c, id) != CUDA_SUCCESS) return ALG_CUDA_ERROR;
  return ALG_OK;
}

// Set-up (host side, not stream work), with `dev` current. cudaGetSymbolAddress
// loads this file's module if lazy loading (the CUDA 12 default) has not
// yet, which is when the static array comes into being on the device; the
// kernels are loaded here too (cudaFuncGetAttributes / cudaFuncSetAttribute),
// so no later call loads code or data.
int noalloc_setup(int dev, unsigned char** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  unsigned long long id = 0;
  if (g_noalloc_ptr[dev] == nullptr || current_context_id(&id) != ALG_OK || id != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    ALG_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));  // also makes the primary context current
    ALG_TRY(current_context_id(&id));
    cudaFuncAttributes fa;
    ALG_CUDA_TRY(cudaFuncGetAttributes(&fa, noalloc_header_kernel));
    const int smem_max = (int)kernel_smem_max();
    ALG_CUDA_TRY(cudaFuncSetAttribute(batched_gesv_kernel<128, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem_max));
    ALG_CUDA_TRY(cudaFuncSetAttribute(batched_gesv_kernel<256, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem_max));
    ALG_CUDA_TRY(cudaFuncSetAttribute(batched_gesv_kernel<512, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem_max));
    g_noalloc_ptr[dev] = p;
    g_noalloc_ctx[dev] = id;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
  return ALG_OK;
}

template <int NT>
int noalloc_launch(cudaStream_t s, const BatchArgs& p) {
  batched_gesv_kernel<NT, 32><<<1, NT, kernel_smem(p.cap, true, 32), s>>>(p);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

}  // namespace
}  // namespace alg

extern "C" int alg_dgesv_mixed_noalloc(void* stream, const double* d_a, double* d_b, int n, int* d_ipiv,
                                       int* d_info, double* d_eta) {
  using namespace alg;
  if (n < 0 || n > kNoAllocMaxN) {
    if (std::getenv("ALG_VERBOSE"))
      std::fprintf(stderr, "alg_dgesv_mixed_noalloc: order %d outside 0..%d (the size of its static scratch)\n", n,
                   kNoAllocMaxN);
    return ALG_BAD_SHAPE;
  }
  if (n > 0 && (d_a == nullptr || d_b == nullptr || d_info == nullptr)) return ALG_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return ALG_NO_DEVICE;
  }
  int dev = 0;
  ALG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return ALG_INVALID_ARGUMENT;
  unsigned char* base = nullptr;
  ALG_TRY(noalloc_setup(dev, &base));
  if (n == 0) return ALG_OK;  // the set-up call: nothing is queued
  auto* hdr = reinterpret_cast<NoAllocHeader*>(base + kNoAllocA32 + kNoAllocWork + kNoAllocIpiv);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the size bucket and CTA size a one-system plan of this order uses
  int cap = 32;
  while (cap < n) cap *= 2;
  const int threads = cap >= 256 ? 512 : (cap >= 64 ? 256 : 128);
  BatchArgs p;
  p.count = 1;
  p.order = &hdr->order;
  p.n = &hdr->n;
  p.a_off = &hdr->a_off;
  p.b_off = &hdr->b_off;
  p.a = const_cast<double*>(d_a);  // the mixed form only reads A
  p.b = d_b;
  p.a32 = reinterpret_cast<float*>(base);
  p.ipiv = d_ipiv ? d_ipiv : reinterpret_cast<int*>(base + kNoAllocA32 + kNoAllocWork);
  p.work = reinterpret_cast<double*>(base + kNoAllocA32);
  p.info = d_info;
  p.eta = d_eta ? d_eta : &hdr->eta;
  p.queue = &hdr->queue;
  p.cap = cap;
  p.mixed = 1;
  p.max_ir = 10;
  p.tol_scale = 10.0;
  noalloc_header_kernel<<<1, 1, 0, s>>>(hdr, n);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  switch (threads) {
    case 128: return noalloc_launch<128>(s, p);
    case 512: return noalloc_launch<512>(s, p);
    default: return noalloc_launch<256>(s, p);
  }
}
