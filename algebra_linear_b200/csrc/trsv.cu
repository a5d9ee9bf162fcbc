// Triangular solves with the packed LU factors in one launch (dataflow).
//
// Forward (unit lower L) and backward (upper U) sweeps over column-major
// factors, nrhs right-hand sides. The rows are cut into blocks of kTB; CTA c
// of a cooperative grid owns block rows c, c+G, c+2G, ... in sweep order. For
// its block row i it subtracts L_ij x_j for every earlier block j as soon as
// block j's ready flag is set (acquire load, bounded spin), solves the
// diagonal block, stores x_i and releases its own flag. Block 0 needs
// nothing, and a CTA only waits on blocks that come earlier in the sweep, each
// owned by a co-resident CTA that reaches it before any later block of its
// own, so the chain always progresses.
//
// EXACT: each entry takes its terms in increasing column order with rounded
// products and differences — the row-dot order of the reference's forward
// sweep (src/lapack/mod.rs:341-347), bit for bit. Otherwise a block's 64
// terms are split over four threads and their partial sums are combined in a
// fixed order (deterministic, not the reference's rounding).
#include <algorithm>
#include <climits>

#include "dense.cuh"

namespace alg {
namespace {

constexpr int kTB = 64;         // block rows
constexpr int kTThreads = 256;  // 64 rows x 4 column quarters
constexpr int kMaxRhs = 4;      // right-hand sides handled per pass
template <typename T>
constexpr size_t kTSmem = 4 * kTB * kTB * sizeof(T);  // two factor tiles, the diagonal block, its inverse

__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void cp_async_elem(void* dst, const void* src, int bytes) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Tile (rows x cols) of the factor at (i0, j0) into smem [col][row], asynchronously.
template <typename T>
__device__ __forceinline__ void prefetch_tile(T* tile, const T* lu, int lda, int i0, int j0, int rows, int cols) {
  for (int idx = threadIdx.x; idx < kTB * kTB; idx += kTThreads) {
    const int rr = idx % kTB, cc = idx / kTB;
    if (rr < rows && cc < cols)
      cp_async_elem(&tile[cc * kTB + rr], lu + (size_t)(i0 + rr) + (size_t)(j0 + cc) * lda, (int)sizeof(T));
  }
}

// Thread 0's bounded wait for a block's ready flag: 1 when it is set, 0 when
// another CTA aborted or the limit ran out (then this CTA raises the abort
// flag and the status block's timeout, so every CTA of the launch returns).
__device__ __forceinline__ int wait_ready(const int* flag, int* abort_flag, DevStatus* status, uint64_t limit_ns) {
  uint64_t t0 = 0;
  for (int it = 0;; ++it) {
    if (ld_acquire(flag) != 0) return 1;
    if (ld_acquire(abort_flag) != 0) return 0;
    if ((it & 255) == 0) {
      const uint64_t now = global_timer_ns();
      if (it == 0) {
        t0 = now;
      } else if (now - t0 > limit_ns) {
        atomicExch(abort_flag, 1);
        atomicExch(&status->timeout, 1);
        return 0;
      }
    }
  }
}

// stuck_wait != 0: the CTA of the sweep's first block waits on flags[nb], a
// slot cleared before the launch that nothing sets, so the wait runs out
// (the timeout path, exercised by tests without any fault).
template <typename T, bool EXACT, bool UPPER>
__global__ void __launch_bounds__(kTThreads) trsv_dataflow_kernel(const T* __restrict__ lu, int lda, int n, T* x,
                                                                  int ldx, int nrhs, int* flags, int* abort_flag,
                                                                  DevStatus* status, uint64_t wait_limit_ns,
                                                                  int stuck_wait) {
  extern __shared__ __align__(16) unsigned char tsm[];
  T* tiles = reinterpret_cast<T*>(tsm);                 // [2][kTB*kTB] factor tiles, [col][row]
  T* dtile = tiles + 2 * kTB * kTB;                      // diagonal block, [col][row]
  T* dinv = tiles + 3 * kTB * kTB;                       // its inverse (non-EXACT), [col][row]
  __shared__ T xs[kTB][kMaxRhs];       // x of the block being consumed
  __shared__ T part[4][kTB][kMaxRhs];  // partial sums of the four column quarters
  __shared__ T acc_s[kTB][kMaxRhs];
  __shared__ int stop;
  const int nb = (n + kTB - 1) / kTB;
  const int r = threadIdx.x & (kTB - 1);  // row within the block
  const int qt = threadIdx.x >> 6;        // column quarter
  if (stuck_wait && blockIdx.x == 0) {
    if (threadIdx.x == 0) stop = !wait_ready(&flags[nb], abort_flag, status, wait_limit_ns);
    __syncthreads();
    if (stop) return;
  }
  for (int s = blockIdx.x; s < nb; s += gridDim.x) {
    // sweep position s -> block index (forward: ascending, backward: descending)
    const int bi = UPPER ? nb - 1 - s : s;
    const int i0 = bi * kTB;
    const int rows = min(kTB, n - i0);
    if (qt == 0 && r < rows)
      for (int k = 0; k < nrhs; ++k) acc_s[r][k] = x[(size_t)k * ldx + i0 + r];
    // the diagonal block and the first off-diagonal tile start loading now
    prefetch_tile<T>(dtile, lu, lda, i0, i0, rows, rows);
    cp_async_commit();
    if (s > 0) {
      const int bj = UPPER ? nb - 1 : 0;
      prefetch_tile<T>(tiles, lu, lda, i0, bj * kTB, rows, min(kTB, n - bj * kTB));
    }
    cp_async_commit();
    if constexpr (!EXACT) {
      // Invert the diagonal block now, while earlier blocks are still being
      // solved: the critical path then only pays a matrix-vector product.
      cp_async_wait<1>();  // the diagonal block (first group) has landed
      __syncthreads();
      if (threadIdx.x < rows) {
        const int c = threadIdx.x;
        T* xcol = dinv + c * kTB;
        if constexpr (!UPPER) {  // unit lower: x = L^{-1} e_c
          for (int rr = 0; rr < c; ++rr) xcol[rr] = T(0);
          xcol[c] = T(1);
          for (int rr = c + 1; rr < rows; ++rr) {
            T acc = T(0);
            for (int k = c; k < rr; ++k) acc = fma_rn(dtile[k * kTB + rr], xcol[k], acc);
            xcol[rr] = -acc;
          }
        } else {  // upper: x = U^{-1} e_c
          for (int rr = c + 1; rr < rows; ++rr) xcol[rr] = T(0);
          xcol[c] = div_rn(T(1), dtile[c * kTB + c]);
          for (int rr = c - 1; rr >= 0; --rr) {
            T acc = T(0);
            for (int k = rr + 1; k <= c; ++k) acc = fma_rn(dtile[k * kTB + rr], xcol[k], acc);
            xcol[rr] = -div_rn(acc, dtile[rr * kTB + rr]);
          }
        }
      }
    }
    __syncthreads();
    for (int t = 0; t < s; ++t) {
      const int bj = UPPER ? nb - 1 - t : t;
      const int j0 = bj * kTB;
      const int cols = min(kTB, n - j0);
      const T* tile = tiles + (size_t)(t & 1) * kTB * kTB;
      // next tile in flight while this one is consumed
      if (t + 1 < s) {
        const int bn = UPPER ? nb - 2 - t : t + 1;
        prefetch_tile<T>(tiles + (size_t)((t + 1) & 1) * kTB * kTB, lu, lda, i0, bn * kTB, rows,
                         min(kTB, n - bn * kTB));
      }
      cp_async_commit();
      // wait for block bj (bounded); a failure anywhere stops every CTA
      if (threadIdx.x == 0) stop = !wait_ready(&flags[bj], abort_flag, status, wait_limit_ns);
      __syncthreads();
      if (stop) {
        cp_async_wait<0>();
        return;
      }
      for (int idx = threadIdx.x; idx < cols * nrhs; idx += kTThreads) {
        const int c = idx % cols, k = idx / cols;
        xs[c][k] = __ldcg(&x[(size_t)k * ldx + j0 + c]);
      }
      cp_async_wait<1>();  // tile t has landed (tile t+1 may still be in flight)
      __syncthreads();
      if (r < rows) {
        if constexpr (EXACT) {
          if (qt == 0) {
            for (int k = 0; k < nrhs; ++k) {
              T a = acc_s[r][k];
#pragma unroll 8
              for (int c = 0; c < cols; ++c) a = msub<true>(a, tile[c * kTB + r], xs[c][k]);
              acc_s[r][k] = a;
            }
          }
        } else {
          const int c0 = qt * (kTB / 4), c1 = min(cols, c0 + kTB / 4);
          for (int k = 0; k < nrhs; ++k) {
            T p = T(0);
#pragma unroll 4
            for (int c = c0; c < c1; ++c) p = fma_rn(tile[c * kTB + r], xs[c][k], p);
            part[qt][r][k] = p;
          }
        }
      }
      __syncthreads();
      if constexpr (!EXACT) {
        if (qt == 0 && r < rows)
          for (int k = 0; k < nrhs; ++k)
            acc_s[r][k] = acc_s[r][k] - ((part[0][r][k] + part[1][r][k]) + (part[2][r][k] + part[3][r][k]));
        __syncthreads();
      }
    }
    cp_async_wait<0>();
    __syncthreads();
    if constexpr (!EXACT) {
      // x_i = inv(D_ii) y_i: four column quarters per row, fixed-order combine
      if (r < rows) {
        const int c0 = qt * (kTB / 4), c1 = min(rows, c0 + kTB / 4);
        for (int k = 0; k < nrhs; ++k) {
          T p = T(0);
          for (int c = c0; c < c1; ++c) p = fma_rn(dinv[c * kTB + r], acc_s[c][k], p);
          part[qt][r][k] = p;
        }
      }
      __syncthreads();
      if (qt == 0 && r < rows)
        for (int k = 0; k < nrhs; ++k)
          acc_s[r][k] = (part[0][r][k] + part[1][r][k]) + (part[2][r][k] + part[3][r][k]);
    } else if (threadIdx.x < 32) {
      for (int k = 0; k < nrhs; ++k) {
        if constexpr (!UPPER) {
          for (int c = 0; c + 1 < rows; ++c) {
            const T u = acc_s[c][k];
            for (int ii = c + 1 + threadIdx.x; ii < rows; ii += 32)
              acc_s[ii][k] = msub<EXACT>(acc_s[ii][k], dtile[c * kTB + ii], u);
            __syncwarp();
          }
        } else {
          for (int c = rows - 1; c >= 0; --c) {
            if (threadIdx.x == 0) acc_s[c][k] = div_rn(acc_s[c][k], dtile[c * kTB + c]);
            __syncwarp();
            const T u = acc_s[c][k];
            for (int ii = threadIdx.x; ii < c; ii += 32) acc_s[ii][k] = msub<EXACT>(acc_s[ii][k], dtile[c * kTB + ii], u);
            __syncwarp();
          }
        }
      }
    }
    __syncthreads();
    if (qt == 0 && r < rows)
      for (int k = 0; k < nrhs; ++k) x[(size_t)k * ldx + i0 + r] = acc_s[r][k];
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();  // cumulative: the block's stores, ordered by the barrier, before the flag
      st_release(&flags[bi], 1);
    }
  }
}

template <typename T, bool EXACT, bool UPPER>
int launch_trsv(alg_ctx* ctx, const T* lu, int lda, int n, T* x, int ldx, int nrhs, int* flags, int* abort_flag) {
  const int nb = (n + kTB - 1) / kTB;
  static int max_blocks = 0;
  if (max_blocks == 0) {
    int per_sm = 0;
    ALG_CUDA_TRY(cudaFuncSetAttribute(trsv_dataflow_kernel<T, EXACT, UPPER>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTSmem<T>));
    ALG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsv_dataflow_kernel<T, EXACT, UPPER>,
                                                               kTThreads, kTSmem<T>));
    max_blocks = std::max(1, per_sm) * ctx->sm_count;
  }
  int grid = std::min(nb, max_blocks);
  ALG_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int) * (nb + 1), ctx->stream));
  uint64_t limit = ctx->wait_limit_ns ? ctx->wait_limit_ns : kWaitLimitNs;
  int stuck = 0;
  if (ctx->stuck_waits > 0) {
    --ctx->stuck_waits;
    stuck = 1;
  }
  void* args[] = {(void*)&lu, (void*)&lda, (void*)&n, (void*)&x, (void*)&ldx, (void*)&nrhs,
                  (void*)&flags, (void*)&abort_flag, (void*)&ctx->d_status, (void*)&limit, (void*)&stuck};
  ALG_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)trsv_dataflow_kernel<T, EXACT, UPPER>, dim3(grid),
                                           dim3(kTThreads), args, kTSmem<T>, ctx->stream));
  count_launches();
  return ALG_OK;
}

__global__ void gather_rows_kernel_d(const double* __restrict__ b, int ldb, const int* __restrict__ perm, int n,
                                     int nrhs, double* __restrict__ x, int ldx) {
  const size_t cnt = (size_t)n * nrhs;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < cnt; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t k = idx / n, i = idx % n;
    x[k * ldx + i] = b[k * ldb + perm[i]];
  }
}
__global__ void gather_rows_kernel_f(const float* __restrict__ b, int ldb, const int* __restrict__ perm, int n,
                                     int nrhs, float* __restrict__ x, int ldx) {
  const size_t cnt = (size_t)n * nrhs;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < cnt; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t k = idx / n, i = idx % n;
    x[k * ldx + i] = b[k * ldb + perm[i]];
  }
}

template <typename T>
void gather_rows(alg_ctx* ctx, const T* b, int ldb, const int* perm, int n, int nrhs, T* x, int ldx) {
  const size_t cnt = (size_t)n * nrhs;
  const int g = (int)std::max<size_t>(1, std::min<size_t>((cnt + 255) / 256, (size_t)ctx->sm_count * 8));
  if constexpr (sizeof(T) == 8) gather_rows_kernel_d<<<g, 256, 0, ctx->stream>>>(b, ldb, perm, n, nrhs, x, ldx);
  else gather_rows_kernel_f<<<g, 256, 0, ctx->stream>>>(b, ldb, perm, n, nrhs, x, ldx);
  count_launches();
}

}  // namespace

// b (n x nrhs, ldb) <- (LU)^{-1} P b, one gather + two dataflow launches per
// group of up to kMaxRhs right-hand sides.
template <typename T, bool EXACT>
int lu_solve_dataflow_dev(alg_ctx* ctx, const T* lu, int n, int lda, const int* perm, T* b, int nrhs, int ldb) {
  if (n == 0 || nrhs == 0) return ALG_OK;
  const int nb = (n + kTB - 1) / kTB;
  T* x = nullptr;
  int* flags = nullptr;
  ALG_TRY(ws_get(ctx, WS_X, sizeof(T) * (size_t)n * nrhs, reinterpret_cast<void**>(&x)));
  ALG_TRY(ws_get(ctx, WS_LAB, sizeof(int) * (size_t)(2 * nb + 4) + sizeof(int) * n,
                 reinterpret_cast<void**>(&flags)));
  int* abort_flag = flags + 2 * nb + 2;
  const int tok = prof_begin(ctx, ALG_K_SOLVE);
  gather_rows<T>(ctx, b, ldb, perm, n, nrhs, x, n);
  ALG_CUDA_TRY(cudaMemsetAsync(abort_flag, 0, sizeof(int), ctx->stream));
  for (int k0 = 0; k0 < nrhs; k0 += kMaxRhs) {
    const int kr = std::min(kMaxRhs, nrhs - k0);
    T* xk = x + (size_t)k0 * n;
    ALG_TRY((launch_trsv<T, EXACT, false>(ctx, lu, lda, n, xk, n, kr, flags, abort_flag)));
    ALG_TRY((launch_trsv<T, EXACT, true>(ctx, lu, lda, n, xk, n, kr, flags + nb + 1, abort_flag)));
  }
  ALG_CUDA_TRY(cudaMemcpy2DAsync(b, sizeof(T) * (size_t)ldb, x, sizeof(T) * (size_t)n, sizeof(T) * (size_t)n, nrhs,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
  prof_end(ctx, tok, 2.0 * n * n * nrhs, sizeof(T) * (double(n) * n + 4.0 * n * nrhs));
  return ALG_OK;
}

// One triangular sweep (non-exact arithmetic) over the leading n x n block
// of column-major factors: unit-lower (upper = false) or upper. flags holds
// n / 64 + 1 ints (cleared here); abort_flag must be zero.
template <typename T>
int tri_solve_dev(alg_ctx* ctx, const T* lu, int lda, int n, T* x, bool upper, int* flags, int* abort_flag) {
  if (n <= 0) return ALG_OK;
  if (upper) return launch_trsv<T, false, true>(ctx, lu, lda, n, x, n, 1, flags, abort_flag);
  return launch_trsv<T, false, false>(ctx, lu, lda, n, x, n, 1, flags, abort_flag);
}

template int tri_solve_dev<double>(alg_ctx*, const double*, int, int, double*, bool, int*, int*);
template int tri_solve_dev<float>(alg_ctx*, const float*, int, int, float*, bool, int*, int*);
template int lu_solve_dataflow_dev<double, true>(alg_ctx*, const double*, int, int, const int*, double*, int, int);
template int lu_solve_dataflow_dev<double, false>(alg_ctx*, const double*, int, int, const int*, double*, int, int);
template int lu_solve_dataflow_dev<float, false>(alg_ctx*, const float*, int, int, const int*, float*, int, int);
template int lu_solve_dataflow_dev<float, true>(alg_ctx*, const float*, int, int, const int*, float*, int, int);

}  // namespace alg
