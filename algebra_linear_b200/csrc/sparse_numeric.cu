// Numeric multifrontal factorization and solve of the sparse LU on the GPU,
// over the static front plan (sparse.cuh).
//
// Factorization. Small fronts (few rows, all-small subtrees) are factored by
// one persistent launch per tree level, one CTA per front: assemble (entering
// rows of A plus the children's contribution blocks), partial-pivoting LU of
// the front's own columns over all its rows with the interchanges spanning
// the whole front, and the Schur complement left in place as the front's
// contribution block. Large fronts are factored one after another in
// postorder by the blocked dense LU (cluster panel kernel, block TRSM,
// trailing GEMM) on a front buffer; their contribution blocks live on a
// stack. The L panel, the U12 panel and the row of every slot are kept.
//
// Solve (supernodal, level by level): y = P b; for each front from the
// leaves up, y_s = L11^-1 y_s and y[rows below] -= L21 y_s; then from the
// root down, x_s = U11^-1 (x_s - U12 x[Struct(s)]); b = Q x.
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "dense.cuh"
#include "sparse_numeric.cuh"

namespace alg {
namespace sp {
namespace {

constexpr int kSmallThreads = 256;

struct SmallArgs {
  const FrontDesc* fronts;
  const int32_t* level_fronts;
  const int32_t* child_idx;
  const int32_t* child_slot;
  const int32_t* cb_colmap;
  const int64_t* anew_q;
  const int32_t* anew_slot;
  const int32_t* anew_col;
  const int32_t* new_rows;
  const double* values;
  double* block;
  double* L;
  double* U;
  int32_t* rowid;
  int* singular;
};

// First index of the largest key over the block (ties to the lower index).
__device__ int block_first_max(double key, int idx, double* rk, int* ri) {
  for (int off = 16; off > 0; off >>= 1) {
    const double ok = __shfl_down_sync(0xffffffffu, key, off);
    const int oi = __shfl_down_sync(0xffffffffu, idx, off);
    if (ok > key || (ok == key && oi < idx)) {
      key = ok;
      idx = oi;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    rk[warp] = key;
    ri[warp] = idx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double k = rk[0];
    int i = ri[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (rk[w] > k || (rk[w] == k && ri[w] < i)) {
        k = rk[w];
        i = ri[w];
      }
    rk[0] = k;
    ri[0] = i;
  }
  __syncthreads();
  const int r = ri[0];
  __syncthreads();
  return r;
}

// C (mr x nc) -= A (mr x kd) B (kd x nc), all inside one front (column-major,
// leading dimension ld), by one CTA of kSmallThreads: 64 x 64 tiles, each
// thread a 4 x 4 register block, K staged through shared memory 16 at a time.
__device__ void cta_gemm_sub(double* C, const double* A, const double* B, int ld, int mr, int nc, int kd,
                             double* As, double* Bs) {
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  for (int i0 = 0; i0 < mr; i0 += 64)
    for (int j0 = 0; j0 < nc; j0 += 64) {
      double acc[4][4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
      for (int k0 = 0; k0 < kd; k0 += 16) {
        __syncthreads();
        for (int e = tid; e < 64 * 16; e += kSmallThreads) {
          const int r = e & 63, k = e >> 6;  // A tile, rows contiguous
          As[k * 64 + r] = (i0 + r < mr && k0 + k < kd) ? A[(i0 + r) + (int64_t)(k0 + k) * ld] : 0.0;
          const int kk = e & 15, c = e >> 4;  // B tile, k contiguous
          Bs[kk * 64 + c] = (j0 + c < nc && k0 + kk < kd) ? B[(k0 + kk) + (int64_t)(j0 + c) * ld] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < 16; ++k) {
          double av[4], bv[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) av[r] = As[k * 64 + tx * 4 + r];
#pragma unroll
          for (int c = 0; c < 4; ++c) bv[c] = Bs[k * 64 + ty * 4 + c];
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
        }
      }
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int i = i0 + tx * 4 + r, j = j0 + ty * 4 + c;
          if (i < mr && j < nc) C[i + (int64_t)j * ld] -= acc[r][c];
        }
    }
  __syncthreads();
}

__global__ void __launch_bounds__(kSmallThreads) small_front_kernel(SmallArgs a) {
  __shared__ double rk[kSmallThreads / 32];
  __shared__ int ri[kSmallThreads / 32];
  __shared__ double piv_s;
  const int s = a.level_fronts[blockIdx.x];
  const FrontDesc d = a.fronts[s];
  const int rows = d.rows, size = d.size, cols = d.size + d.ncb;
  double* f = a.block + d.block_off;
  int32_t* rid = a.rowid + d.rowid_off;
  const int tid = threadIdx.x;
  const int64_t total = (int64_t)rows * cols;
  for (int64_t e = tid; e < total; e += kSmallThreads) f[e] = 0.0;
  // slots: the children's unpivoted rows, then the rows entering here
  for (int k = d.child_begin; k < d.child_end; ++k) {
    const FrontDesc c = a.fronts[a.child_idx[k]];
    const int slot0 = a.child_slot[k];
    for (int i = tid; i < c.rows - c.size; i += kSmallThreads) rid[slot0 + i] = a.rowid[c.rowid_off + c.size + i];
  }
  {
    const int slot0 = rows - (d.new_end - d.new_begin);
    for (int i = tid; i < d.new_end - d.new_begin; i += kSmallThreads) rid[slot0 + i] = a.new_rows[d.new_begin + i];
  }
  __syncthreads();
  for (int q = d.anew_begin + tid; q < d.anew_end; q += kSmallThreads)
    f[a.anew_slot[q] + (int64_t)a.anew_col[q] * rows] = a.values[a.anew_q[q]];
  for (int k = d.child_begin; k < d.child_end; ++k) {
    const FrontDesc c = a.fronts[a.child_idx[k]];
    const int slot0 = a.child_slot[k];
    const int crows = c.rows - c.size;
    const double* cb = a.block + c.cb_off;
    const int64_t ce = (int64_t)crows * c.ncb;
    for (int64_t e = tid; e < ce; e += kSmallThreads) {
      const int i = (int)(e % crows), t = (int)(e / crows);
      f[(slot0 + i) + (int64_t)a.cb_colmap[c.struct_begin + t] * rows] = cb[i + (int64_t)t * c.cb_ld];
    }
  }
  __syncthreads();
  for (int k = 0; k < size; ++k) {
    double key = -1.0;
    int idx = INT_MAX;
    for (int i = k + tid; i < rows; i += kSmallThreads) {
      const double v = fabs(f[i + (int64_t)k * rows]);
      if (v > key) {
        key = v;
        idx = i;
      }
    }
    const int p = block_first_max(key, idx, rk, ri);
    if (tid == 0) piv_s = f[p + (int64_t)k * rows];
    __syncthreads();
    const double pv = piv_s;
    if (!(fabs(pv) > 0.0)) {
      if (tid == 0) atomicExch(a.singular, 1);
      return;  // uniform: every thread read the same pivot
    }
    if (p != k) {
      for (int j = tid; j < cols; j += kSmallThreads) {
        const double t = f[k + (int64_t)j * rows];
        f[k + (int64_t)j * rows] = f[p + (int64_t)j * rows];
        f[p + (int64_t)j * rows] = t;
      }
      if (tid == 0) {
        const int32_t t = rid[k];
        rid[k] = rid[p];
        rid[p] = t;
      }
    }
    __syncthreads();
    const double inv = 1.0 / pv;
    for (int i = k + 1 + tid; i < rows; i += kSmallThreads) f[i + (int64_t)k * rows] *= inv;
    __syncthreads();
    // rank-1 update of the front's own columns only
    const int mr = rows - k - 1, mc = size - k - 1;
    const int64_t upd = (int64_t)mr * mc;
    for (int64_t e = tid; e < upd; e += kSmallThreads) {
      const int i = k + 1 + (int)(e % mr), j = k + 1 + (int)(e / mr);
      f[i + (int64_t)j * rows] = fma(-f[k + (int64_t)j * rows], f[i + (int64_t)k * rows], f[i + (int64_t)j * rows]);
    }
    __syncthreads();
  }
  __shared__ double As[64 * 16], Bs[16 * 64];
  // U12 = L11^-1 A12 in 16-row blocks: forward substitution within the block
  // (a thread per column), then the rows below by the tiled update
  for (int kb = 0; kb < size; kb += 16) {
    const int ke = min(size, kb + 16);
    for (int c = size + tid; c < cols; c += kSmallThreads) {
      double* col = f + (int64_t)c * rows;
      for (int k = kb; k < ke; ++k) {
        const double uk = col[k];
        for (int i = k + 1; i < ke; ++i) col[i] = fma(-f[i + (int64_t)k * rows], uk, col[i]);
      }
    }
    __syncthreads();
    if (ke < size)
      cta_gemm_sub(f + ke + (int64_t)size * rows, f + ke + (int64_t)kb * rows, f + kb + (int64_t)size * rows, rows,
                   size - ke, d.ncb, ke - kb, As, Bs);
  }
  // contribution block: CB -= L21 U12 (register-tiled)
  cta_gemm_sub(f + size + (int64_t)size * rows, f + size, f + (int64_t)size * rows, rows, rows - size, d.ncb, size,
               As, Bs);
  double* lp = a.L + d.l_off;
  for (int64_t e = tid; e < (int64_t)rows * size; e += kSmallThreads) lp[e] = f[e];
  double* up = a.U + d.u_off;
  for (int64_t e = tid; e < (int64_t)size * d.ncb; e += kSmallThreads) {
    const int kk = (int)(e % size), t = (int)(e / size);
    up[e] = f[kk + (int64_t)(size + t) * rows];
  }
}

// ---- large fronts ----------------------------------------------------------
struct BigArgs {
  FrontDesc d;
  const FrontDesc* fronts;
  const int32_t* child_idx;
  const int32_t* child_slot;
  const int32_t* cb_colmap;
  const int64_t* anew_q;
  const int32_t* anew_slot;
  const int32_t* anew_col;
  const int32_t* new_rows;
  const double* values;
  const double* block;  // small children's contribution blocks
  const double* stack;  // large children's contribution blocks
  double* front;        // rows x (size + ncb), ld = rows (zeroed before)
  const int32_t* rowid;
  int32_t* rowtmp;      // the front's slots before pivoting
};

__global__ void big_assemble_kernel(BigArgs a) {
  const FrontDesc& d = a.d;
  const int rows = d.rows;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  {
    const int slotn = rows - (d.new_end - d.new_begin);
    for (int64_t i = tid; i < d.new_end - d.new_begin; i += nth) a.rowtmp[slotn + i] = a.new_rows[d.new_begin + i];
  }
  for (int64_t q = d.anew_begin + tid; q < d.anew_end; q += nth)
    a.front[a.anew_slot[q] + (int64_t)a.anew_col[q] * rows] = a.values[a.anew_q[q]];
  for (int k = d.child_begin; k < d.child_end; ++k) {
    const FrontDesc c = a.fronts[a.child_idx[k]];
    const int slot0 = a.child_slot[k];
    const int crows = c.rows - c.size;
    for (int64_t i = tid; i < crows; i += nth) a.rowtmp[slot0 + i] = a.rowid[c.rowid_off + c.size + i];
    const double* cb = (c.small ? a.block : a.stack) + c.cb_off;
    const int64_t ce = (int64_t)crows * c.ncb;
    for (int64_t e = tid; e < ce; e += nth) {
      const int i = (int)(e % crows), t = (int)(e / crows);
      a.front[(slot0 + i) + (int64_t)a.cb_colmap[c.struct_begin + t] * rows] = cb[i + (int64_t)t * c.cb_ld];
    }
  }
}

// After the partial LU: rows of the slots, U12, and the contribution block.
__global__ void big_finalize_kernel(FrontDesc d, const double* front, const int* perm, const int32_t* rowtmp,
                                    int32_t* rowid, double* U, double* stack) {
  const int rows = d.rows, size = d.size;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = tid; i < rows; i += nth) rowid[d.rowid_off + i] = rowtmp[perm[i]];
  double* up = U + d.u_off;
  for (int64_t e = tid; e < (int64_t)size * d.ncb; e += nth) {
    const int kk = (int)(e % size), t = (int)(e / size);
    up[e] = front[kk + (int64_t)(size + t) * rows];
  }
  const int crows = rows - size;
  if (crows > 0) {
    double* cb = stack + d.cb_off;
    for (int64_t e = tid; e < (int64_t)crows * d.ncb; e += nth) {
      const int i = (int)(e % crows), t = (int)(e / crows);
      cb[i + (int64_t)t * d.cb_ld] = front[(size + i) + (int64_t)(size + t) * rows];
    }
  }
}

// ---- after the factorization -----------------------------------------------
// Final position of every row, the row permutation, and the nonzero counts
// of each column of L and U (exact zeros are not stored, as in the reference).
__global__ void positions_counts_kernel(const FrontDesc* fronts, int ns, const int32_t* rowid, const double* L,
                                        const double* U, const int32_t* struct_cols, int32_t* pos_of_row,
                                        int32_t* row_perm, int32_t* lcount, unsigned* ucount) {
  const int s = blockIdx.x;
  if (s >= ns) return;
  const FrontDesc d = fronts[s];
  const int rows = d.rows, size = d.size;
  for (int k = threadIdx.x; k < size; k += blockDim.x) {
    const int32_t r = rowid[d.rowid_off + k];
    pos_of_row[r] = d.begin + k;
    row_perm[d.begin + k] = r;
  }
  const double* lp = L + d.l_off;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int jj = warp; jj < size; jj += nw) {
    int cl = 0, cu = 0;
    for (int i = lane; i < rows; i += 32) {
      const double v = lp[i + (int64_t)jj * rows];
      if (i > jj) cl += v != 0.0;
      if (i < jj) cu += v != 0.0;
    }
    for (int off = 16; off > 0; off >>= 1) {
      cl += __shfl_xor_sync(0xffffffffu, cl, off);
      cu += __shfl_xor_sync(0xffffffffu, cu, off);
    }
    if (lane == 0) {
      lcount[d.begin + jj] = cl + 1;
      atomicAdd(&ucount[d.begin + jj], (unsigned)(cu + 1));
    }
  }
  const double* up = U + d.u_off;
  for (int t = warp; t < d.ncb; t += nw) {
    int cu = 0;
    for (int kk = lane; kk < size; kk += 32) cu += up[kk + (int64_t)t * size] != 0.0;
    for (int off = 16; off > 0; off >>= 1) cu += __shfl_xor_sync(0xffffffffu, cu, off);
    if (lane == 0 && cu) atomicAdd(&ucount[struct_cols[d.struct_begin + t]], (unsigned)cu);
  }
}

// ---- solve ------------------------------------------------------------------
constexpr int kSolveThreads = 256;

__global__ void gather_rows_kernel(const double* b, const int32_t* row_perm, double* y, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = b[row_perm[i]];
}

__global__ void scatter_cols_kernel(const double* x, const int32_t* col_perm, double* b, int n) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) b[col_perm[j]] = x[j];
}

constexpr int kRowChunk = 256;   // rows of L21 / U12 per CTA
constexpr int kColChunk = 1024;  // columns of U12 per CTA

// Forward, diagonal block of each front of a level (one CTA per front):
// unit-lower solve in 32-column blocks, a warp for the block, all threads
// for the rows below it.
__global__ void __launch_bounds__(kSolveThreads) fwd_diag_kernel(const FrontDesc* fronts, const int32_t* level,
                                                                 const double* L, double* y) {
  const FrontDesc d = fronts[level[blockIdx.x]];
  const int rows = d.rows, m = d.size;
  const double* lp = L + d.l_off;
  double* ys = y + d.begin;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int kb = 0; kb < m; kb += 32) {
    const int w = min(32, m - kb);
    if (warp == 0) {
      double v = lane < w ? ys[kb + lane] : 0.0;
      for (int k = 0; k < w; ++k) {
        const double yk = __shfl_sync(0xffffffffu, v, k);
        if (lane > k && lane < w) v -= lp[(kb + lane) + (int64_t)(kb + k) * rows] * yk;
      }
      if (lane < w) ys[kb + lane] = v;
    }
    __syncthreads();
    for (int i = kb + w + threadIdx.x; i < m; i += kSolveThreads) {
      double acc = 0.0;
      for (int k = 0; k < w; ++k) acc = fma(lp[i + (int64_t)(kb + k) * rows], ys[kb + k], acc);
      ys[i] -= acc;
    }
    __syncthreads();
  }
}

// Forward, rows below the diagonal block: y[pos(row)] -= L21 y_s, a CTA per
// chunk of rows (rows of different fronts of one level are distinct).
__global__ void __launch_bounds__(kSolveThreads) fwd_l21_kernel(const FrontDesc* fronts, const SolveItem* items,
                                                                const double* L, const int32_t* rowid,
                                                                const int32_t* pos_of_row, double* y) {
  const SolveItem it = items[blockIdx.x];
  const FrontDesc d = fronts[it.front];
  const int i = d.size + it.chunk * kRowChunk + threadIdx.x;
  if (i >= d.rows) return;
  const double* lp = L + d.l_off;
  const double* ys = y + d.begin;
  double acc = 0.0;
  for (int k = 0; k < d.size; ++k) acc = fma(lp[i + (int64_t)k * d.rows], ys[k], acc);
  y[pos_of_row[rowid[d.rowid_off + i]]] -= acc;
}

// Backward, U12 x[Struct(s)] in partial sums over column chunks (summed in a
// fixed order by the diagonal kernel, so a solve is deterministic).
__global__ void __launch_bounds__(kSolveThreads) bwd_u12_kernel(const FrontDesc* fronts, const SolveItem* items,
                                                                const double* U, const int32_t* struct_cols,
                                                                const int64_t* part_off, const double* x,
                                                                double* partial) {
  const SolveItem it = items[blockIdx.x];
  const FrontDesc d = fronts[it.front];
  const int kk = it.chunk * kRowChunk + threadIdx.x;
  if (kk >= d.size) return;
  const double* up = U + d.u_off;
  const int32_t* st = struct_cols + d.struct_begin;
  const int t0 = it.tchunk * kColChunk, t1 = min(d.ncb, t0 + kColChunk);
  double acc = 0.0;
  for (int t = t0; t < t1; ++t) acc = fma(up[kk + (int64_t)t * d.size], x[st[t]], acc);
  partial[part_off[it.front] + (int64_t)it.tchunk * d.size + kk] = acc;
}

// Backward, diagonal block (one CTA per front): subtract the U12 partial sums,
// then the upper solve in 32-column blocks from the last, x_j times the
// reciprocal of its diagonal as in the reference's upper sweep.
__global__ void __launch_bounds__(kSolveThreads) bwd_diag_kernel(const FrontDesc* fronts, const int32_t* level,
                                                                 const double* L, const int64_t* part_off,
                                                                 const double* partial, double* x) {
  const int s = level[blockIdx.x];
  const FrontDesc d = fronts[s];
  const int rows = d.rows, m = d.size;
  const double* lp = L + d.l_off;
  double* xs = x + d.begin;
  const int ntc = (d.ncb + kColChunk - 1) / kColChunk;
  for (int kk = threadIdx.x; kk < m; kk += kSolveThreads) {
    double acc = 0.0;
    for (int tc = 0; tc < ntc; ++tc) acc += partial[part_off[s] + (int64_t)tc * m + kk];
    xs[kk] -= acc;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int jb = m; jb > 0; jb -= 32) {
    const int j0 = max(0, jb - 32), w = jb - j0;
    if (warp == 0) {
      double v = lane < w ? xs[j0 + lane] : 0.0;
      for (int j = w - 1; j >= 0; --j) {
        if (lane == j) v = v * (1.0 / lp[(j0 + j) + (int64_t)(j0 + j) * rows]);
        const double xj = __shfl_sync(0xffffffffu, v, j);
        if (lane < j) v -= lp[(j0 + lane) + (int64_t)(j0 + j) * rows] * xj;
      }
      if (lane < w) xs[j0 + lane] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < j0; i += kSolveThreads) {
      double acc = 0.0;
      for (int l = 0; l < w; ++l) acc = fma(lp[i + (int64_t)(j0 + l) * rows], xs[j0 + l], acc);
      xs[i] -= acc;
    }
    __syncthreads();
  }
}

template <typename T>
int upload(const std::vector<T>& h, T** d) {
  const size_t bytes = std::max<size_t>(sizeof(T) * h.size(), 16);
  ALG_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(d), bytes));
  if (!h.empty()) ALG_CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return ALG_OK;
}

int dmalloc(void** p, size_t bytes) {
  ALG_CUDA_TRY(cudaMalloc(p, std::max<size_t>(bytes, 16)));
  return ALG_OK;
}

int grid_for(alg_ctx* ctx, int64_t work, int threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((work + threads - 1) / threads, 8LL * ctx->sm_count));
}

}  // namespace

// ---------------------------------------------------------------------------
int DeviceLu::init(alg_ctx* c, const FrontPlan* p) {
  ctx = c;
  plan = p;
  const FrontPlan& F = *p;
  ALG_TRY(upload(F.fronts, &d_fronts));
  ALG_TRY(upload(F.child_idx, &d_child_idx));
  ALG_TRY(upload(F.child_slot, &d_child_slot));
  ALG_TRY(upload(F.struct_cols, &d_struct_cols));
  ALG_TRY(upload(F.cb_colmap, &d_cb_colmap));
  ALG_TRY(upload(F.anew_q, &d_anew_q));
  ALG_TRY(upload(F.anew_slot, &d_anew_slot));
  ALG_TRY(upload(F.anew_col, &d_anew_col));
  ALG_TRY(upload(F.new_rows, &d_new_rows));
  ALG_TRY(upload(F.small_level_fronts, &d_small_levels));
  ALG_TRY(upload(F.solve_level_fronts, &d_solve_levels));
  ALG_TRY(upload(F.col_perm, &d_col_perm));
  const size_t n = (size_t)std::max<idx>(F.n, 1);
  ALG_TRY(dmalloc((void**)&d_values, sizeof(double) * std::max<idx>(F.nnz, 1)));
  ALG_TRY(dmalloc((void**)&d_block, sizeof(double) * F.block_total));
  ALG_TRY(dmalloc((void**)&d_stack, sizeof(double) * F.stack_total));
  ALG_TRY(dmalloc((void**)&d_front, sizeof(double) * F.front_buf));
  int64_t max_rows = 1;
  for (const auto& d : F.fronts) max_rows = std::max<int64_t>(max_rows, d.rows);
  ALG_TRY(dmalloc((void**)&d_ipiv, sizeof(int) * max_rows));
  ALG_TRY(dmalloc((void**)&d_perm, sizeof(int) * max_rows));
  ALG_TRY(dmalloc((void**)&d_rowtmp, sizeof(int32_t) * max_rows));
  ALG_TRY(dmalloc((void**)&d_flag, sizeof(int) * 4));
  ALG_TRY(dmalloc((void**)&d_y, sizeof(double) * n));
  ALG_TRY(dmalloc((void**)&d_rhs, sizeof(double) * n));
  {
    // solve work items per level and the U12 partial-sum offsets
    std::vector<SolveItem> fwd, bwd;
    std::vector<int64_t> poff(std::max<idx>(F.ns, 1), 0);
    int64_t ptot = 0;
    for (idx s = 0; s < F.ns; ++s) {
      const FrontDesc& d = F.fronts[s];
      poff[s] = ptot;
      ptot += (int64_t)((d.ncb + kColChunk - 1) / kColChunk) * d.size;
    }
    const int nl = (int)F.solve_level_ptr.size() - 1;
    fwd_item_ptr.assign(std::max(nl, 0) + 1, 0);
    bwd_item_ptr.assign(std::max(nl, 0) + 1, 0);
    for (int h = 0; h < nl; ++h) {
      for (int t = F.solve_level_ptr[h]; t < F.solve_level_ptr[h + 1]; ++t) {
        const int s = F.solve_level_fronts[t];
        const FrontDesc& d = F.fronts[s];
        for (int c = 0; c * kRowChunk < d.rows - d.size; ++c) fwd.push_back(SolveItem{s, c, 0, 0});
        for (int c = 0; c * kRowChunk < d.size; ++c)
          for (int tc = 0; tc * kColChunk < d.ncb; ++tc) bwd.push_back(SolveItem{s, c, tc, 0});
      }
      fwd_item_ptr[h + 1] = (int)fwd.size();
      bwd_item_ptr[h + 1] = (int)bwd.size();
    }
    ALG_TRY(upload(fwd, &d_fwd_items));
    ALG_TRY(upload(bwd, &d_bwd_items));
    ALG_TRY(upload(poff, &d_part_off));
    ALG_TRY(dmalloc((void**)&d_partial, sizeof(double) * std::max<int64_t>(ptot, 1)));
  }
  for (int b = 0; b < 2; ++b) {
    ALG_TRY(dmalloc((void**)&fac[b].L, sizeof(double) * F.l_total));
    ALG_TRY(dmalloc((void**)&fac[b].U, sizeof(double) * F.u_total));
    ALG_TRY(dmalloc((void**)&fac[b].rowid, sizeof(int32_t) * F.rowid_total));
    ALG_TRY(dmalloc((void**)&fac[b].pos_of_row, sizeof(int32_t) * n));
    ALG_TRY(dmalloc((void**)&fac[b].row_perm, sizeof(int32_t) * n));
    ALG_TRY(dmalloc((void**)&fac[b].lcount, sizeof(int32_t) * n));
    ALG_TRY(dmalloc((void**)&fac[b].ucount, sizeof(unsigned) * n));
  }
  return ALG_OK;
}

void DeviceLu::release() {
  for (void* q : {(void*)d_fronts, (void*)d_child_idx, (void*)d_child_slot, (void*)d_struct_cols,
                  (void*)d_cb_colmap, (void*)d_anew_q, (void*)d_anew_slot, (void*)d_anew_col, (void*)d_new_rows,
                  (void*)d_small_levels, (void*)d_solve_levels, (void*)d_col_perm, (void*)d_values,
                  (void*)d_block, (void*)d_stack, (void*)d_front, (void*)d_ipiv, (void*)d_perm, (void*)d_rowtmp,
                  (void*)d_flag, (void*)d_y, (void*)d_rhs, (void*)d_fwd_items, (void*)d_bwd_items,
                  (void*)d_part_off, (void*)d_partial})
    if (q) cudaFree(q);
  for (auto& f : fac)
    for (void* q : {(void*)f.L, (void*)f.U, (void*)f.rowid, (void*)f.pos_of_row, (void*)f.row_perm,
                    (void*)f.lcount, (void*)f.ucount})
      if (q) cudaFree(q);
  *this = DeviceLu();
}

// Factors the values in d_values into factor set `b`. Stream-ordered; the
// singular flag and the dense status block are read by the caller.
int DeviceLu::factor(int b) {
  const FrontPlan& F = *plan;
  Factors& out = fac[b];
  cudaStream_t st = ctx->stream;
  const int tok = prof_begin(ctx, ALG_K_SPARSE);
  ALG_CUDA_TRY(cudaMemsetAsync(d_flag, 0, sizeof(int) * 4, st));
  ALG_TRY(status_reset(ctx));
  // small fronts, one launch per level
  SmallArgs sa;
  sa.fronts = d_fronts;
  sa.child_idx = d_child_idx;
  sa.child_slot = d_child_slot;
  sa.cb_colmap = d_cb_colmap;
  sa.anew_q = d_anew_q;
  sa.anew_slot = d_anew_slot;
  sa.anew_col = d_anew_col;
  sa.new_rows = d_new_rows;
  sa.values = d_values;
  sa.block = d_block;
  sa.L = out.L;
  sa.U = out.U;
  sa.rowid = out.rowid;
  sa.singular = d_flag;
  const int tok_small = prof_begin(ctx, ALG_K_BATCH);
  for (size_t h = 0; h + 1 < F.small_level_ptr.size(); ++h) {
    const int cnt = F.small_level_ptr[h + 1] - F.small_level_ptr[h];
    if (cnt == 0) continue;
    sa.level_fronts = d_small_levels + F.small_level_ptr[h];
    small_front_kernel<<<cnt, kSmallThreads, 0, st>>>(sa);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
  }
  prof_end(ctx, tok_small, 0.0, 0.0);
  // large fronts in postorder
  LuPlan lp;
  lp.nb = 64;
  lp.nbl = 16;
  for (int32_t s : F.big_order) {
    const FrontDesc& d = F.fronts[s];
    const int cols = d.size + d.ncb;
    ALG_CUDA_TRY(cudaMemsetAsync(d_front, 0, sizeof(double) * (size_t)d.rows * cols, st));
    BigArgs ba;
    ba.d = d;
    ba.fronts = d_fronts;
    ba.child_idx = d_child_idx;
    ba.child_slot = d_child_slot;
    ba.cb_colmap = d_cb_colmap;
    ba.anew_q = d_anew_q;
    ba.anew_slot = d_anew_slot;
    ba.anew_col = d_anew_col;
    ba.new_rows = d_new_rows;
    ba.values = d_values;
    ba.block = d_block;
    ba.stack = d_stack;
    ba.front = d_front;
    ba.rowid = out.rowid;
    ba.rowtmp = d_rowtmp;
    int64_t work = (int64_t)(d.anew_end - d.anew_begin) + d.rows;
    for (int k = d.child_begin; k < d.child_end; ++k) {
      const FrontDesc& c = F.fronts[F.child_idx[k]];
      work = std::max<int64_t>(work, (int64_t)(c.rows - c.size) * c.ncb);
    }
    big_assemble_kernel<<<grid_for(ctx, work, 256), 256, 0, st>>>(ba);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
    ALG_TRY((lu_factor_partial_dev<double, false>(ctx, d_front, d.rows, d.size, cols, d.rows, d_ipiv, d_perm, lp)));
    ALG_CUDA_TRY(cudaMemcpyAsync(out.L + d.l_off, d_front, sizeof(double) * (size_t)d.rows * d.size,
                                 cudaMemcpyDeviceToDevice, st));
    const int64_t fw = std::max<int64_t>((int64_t)d.rows, (int64_t)d.rows * d.ncb);
    big_finalize_kernel<<<grid_for(ctx, fw, 256), 256, 0, st>>>(d, d_front, d_perm, d_rowtmp, out.rowid, out.U,
                                                                 d_stack);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
  }
  ALG_CUDA_TRY(cudaMemsetAsync(out.ucount, 0, sizeof(unsigned) * std::max<idx>(F.n, 1), st));
  if (F.ns > 0) {
    positions_counts_kernel<<<(int)F.ns, 256, 0, st>>>(d_fronts, (int)F.ns, out.rowid, out.L, out.U,
                                                        d_struct_cols, out.pos_of_row, out.row_perm, out.lcount,
                                                        out.ucount);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
  }
  prof_end(ctx, tok, F.flops, 0.0);
  return ALG_OK;
}

// Reads the factorization's outcome (synchronises): SP_OK or SP_SINGULAR.
int DeviceLu::finish(int b, Stats* stats) {
  const FrontPlan& F = *plan;
  int h_flag[4] = {0, 0, 0, 0};
  ALG_CUDA_TRY(cudaMemcpyAsync(h_flag, d_flag, sizeof(h_flag), cudaMemcpyDeviceToHost, ctx->stream));
  ALG_TRY(status_fetch(ctx));
  if (h_flag[0] != 0 || ctx->h_status->singular_col != INT_MAX) return SP_SINGULAR;
  if (ctx->h_status->timeout) return ALG_TIMEOUT;
  if (stats) {
    const size_t n = (size_t)F.n;
    std::vector<int32_t> lc(n);
    std::vector<unsigned> uc(n);
    if (n) {
      ALG_CUDA_TRY(cudaMemcpy(lc.data(), fac[b].lcount, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
      ALG_CUDA_TRY(cudaMemcpy(uc.data(), fac[b].ucount, sizeof(unsigned) * n, cudaMemcpyDeviceToHost));
    }
    uint64_t nl = 0, nu = 0, fl = 0;
    for (size_t j = 0; j < n; ++j) {
      nl += (uint64_t)lc[j];
      nu += uc[j];
      fl += (uint64_t)lc[j] * uc[j];
    }
    stats->nnz_l = nl;
    stats->nnz_u = nu;
    stats->flops_estimate = fl;
  }
  return SP_OK;
}

// x = A^-1 b for the factors of set `b`, with b (n) already on the device in
// d_rhs; the result lands in d_rhs. Stream-ordered.
int DeviceLu::solve(int b) {
  const FrontPlan& F = *plan;
  const Factors& f = fac[b];
  cudaStream_t st = ctx->stream;
  const int n = (int)F.n;
  if (n == 0) return ALG_OK;
  const int tok = prof_begin(ctx, ALG_K_SOLVE);
  gather_rows_kernel<<<grid_for(ctx, n, 256), 256, 0, st>>>(d_rhs, f.row_perm, d_y, n);
  count_launches();
  const int nl = (int)F.solve_level_ptr.size() - 1;
  for (int h = 0; h < nl; ++h) {
    const int cnt = F.solve_level_ptr[h + 1] - F.solve_level_ptr[h];
    if (cnt == 0) continue;
    fwd_diag_kernel<<<cnt, kSolveThreads, 0, st>>>(d_fronts, d_solve_levels + F.solve_level_ptr[h], f.L, d_y);
    count_launches();
    const int ni = fwd_item_ptr[h + 1] - fwd_item_ptr[h];
    if (ni > 0) {
      fwd_l21_kernel<<<ni, kSolveThreads, 0, st>>>(d_fronts, d_fwd_items + fwd_item_ptr[h], f.L, f.rowid,
                                                   f.pos_of_row, d_y);
      count_launches();
    }
  }
  for (int h = nl - 1; h >= 0; --h) {
    const int cnt = F.solve_level_ptr[h + 1] - F.solve_level_ptr[h];
    if (cnt == 0) continue;
    const int ni = bwd_item_ptr[h + 1] - bwd_item_ptr[h];
    if (ni > 0) {
      bwd_u12_kernel<<<ni, kSolveThreads, 0, st>>>(d_fronts, d_bwd_items + bwd_item_ptr[h], f.U, d_struct_cols,
                                                   d_part_off, d_y, d_partial);
      count_launches();
    }
    bwd_diag_kernel<<<cnt, kSolveThreads, 0, st>>>(d_fronts, d_solve_levels + F.solve_level_ptr[h], f.L,
                                                    d_part_off, d_partial, d_y);
    count_launches();
  }
  scatter_cols_kernel<<<grid_for(ctx, n, 256), 256, 0, st>>>(d_y, d_col_perm, d_rhs, n);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  prof_end(ctx, tok, 4.0 * (double)(F.l_total + F.u_total), 8.0 * (double)(F.l_total + F.u_total));
  return ALG_OK;
}

}  // namespace sp
}  // namespace alg
