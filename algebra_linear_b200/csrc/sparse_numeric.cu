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
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "dense.cuh"
#include "sparse_numeric.cuh"

namespace alg {
namespace sp {
namespace {

constexpr int kSmallThreads = 256;

template <typename T>
__device__ __forceinline__ T fma_t(T a, T b, T c);
template <>
__device__ __forceinline__ double fma_t<double>(double a, double b, double c) { return __fma_rn(a, b, c); }
template <>
__device__ __forceinline__ float fma_t<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// The scalar of SparseLu<Complex64> (num_complex::Complex<f64>; lu.rs:61-82),
// stored interleaved (re, im) as the host's arrays: num-complex's product
// (ac - bd) + i(ad + bc), the pivot measure Complex::norm = hypot(re, im) and
// the reciprocal Complex::inv = (re / |z|^2, -im / |z|^2). The factors equal
// the reference's to rounding (the products may be fused here).
struct zc {
  double re, im;
  zc() = default;
  __host__ __device__ constexpr zc(double r, double i = 0.0) : re(r), im(i) {}
};
__device__ __forceinline__ zc operator+(zc a, zc b) { return zc(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ zc operator-(zc a, zc b) { return zc(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ zc operator-(zc a) { return zc(-a.re, -a.im); }
__device__ __forceinline__ zc operator*(zc a, zc b) {
  return zc(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__device__ __forceinline__ zc& operator+=(zc& a, zc b) { return a = a + b; }
__device__ __forceinline__ zc& operator-=(zc& a, zc b) { return a = a - b; }
__device__ __forceinline__ zc& operator*=(zc& a, zc b) { return a = a * b; }
__device__ __forceinline__ bool operator!=(zc a, zc b) { return a.re != b.re || a.im != b.im; }
template <>
__device__ __forceinline__ zc fma_t<zc>(zc a, zc b, zc c) {
  return zc(__fma_rn(a.re, b.re, __fma_rn(-a.im, b.im, c.re)), __fma_rn(a.re, b.im, __fma_rn(a.im, b.re, c.im)));
}

// |x| as the pivot search compares it (SparseScalar::abs)
template <typename T>
__device__ __forceinline__ double pivot_key(T v) { return fabs((double)v); }
template <>
__device__ __forceinline__ double pivot_key<zc>(zc v) { return hypot(v.re, v.im); }

// 1 / x (SparseScalar::recip)
template <typename T>
__device__ __forceinline__ T recip_t(T v) { return T(1) / v; }
template <>
__device__ __forceinline__ zc recip_t<zc>(zc v) {
  const double ns = v.re * v.re + v.im * v.im;
  return zc(v.re / ns, -v.im / ns);
}

template <typename T>
__device__ __forceinline__ T shfl_t(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <>
__device__ __forceinline__ zc shfl_t<zc>(zc v, int src) {
  return zc(__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src));
}

// entry q of a host-layout value array (doubles; complex: interleaved pairs)
template <typename T>
__device__ __forceinline__ T load_value(const double* v, int64_t q) { return (T)v[q]; }
template <>
__device__ __forceinline__ zc load_value<zc>(const double* v, int64_t q) { return zc(v[2 * q], v[2 * q + 1]); }
template <typename T>
__device__ __forceinline__ void store_value(double* v, int64_t q, T x) { v[q] = (double)x; }
template <>
__device__ __forceinline__ void store_value<zc>(double* v, int64_t q, zc x) {
  v[2 * q] = x.re;
  v[2 * q + 1] = x.im;
}

template <typename T>
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
  T* block;
  T* L;
  T* U;
  int32_t* rowid;
  int* singular;
};

// The 64 x 64 tile at (i0, j0) of C (mr x nc) -= A (mr x kd) B (kd x nc),
// all inside one front (column-major, leading dimension ld), by one CTA of
// kSmallThreads: each thread a 4 x 4 register block, K staged through shared
// memory 16 at a time.
template <typename T>
__device__ __forceinline__ void cta_gemm_tile(T* C, const T* A, const T* B, int ld, int mr, int nc, int kd, int i0,
                                              int j0, T* As, T* Bs) {
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = T(0);
  for (int k0 = 0; k0 < kd; k0 += 16) {
    __syncthreads();
    for (int e = tid; e < 64 * 16; e += kSmallThreads) {
      const int r = e & 63, k = e >> 6;  // A tile, rows contiguous
      As[k * 64 + r] = (i0 + r < mr && k0 + k < kd) ? A[(i0 + r) + (int64_t)(k0 + k) * ld] : T(0);
      const int kk = e & 15, c = e >> 4;  // B tile, k contiguous
      Bs[kk * 64 + c] = (j0 + c < nc && k0 + kk < kd) ? B[(k0 + kk) + (int64_t)(j0 + c) * ld] : T(0);
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < 16; ++k) {
      T av[4], bv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) av[r] = As[k * 64 + tx * 4 + r];
#pragma unroll
      for (int c = 0; c < 4; ++c) bv[c] = Bs[k * 64 + ty * 4 + c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = fma_t(av[r], bv[c], acc[r][c]);
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

// All tiles of it, by one CTA.
template <typename T>
__device__ void cta_gemm_sub(T* C, const T* A, const T* B, int ld, int mr, int nc, int kd, T* As, T* Bs) {
  for (int i0 = 0; i0 < mr; i0 += 64)
    for (int j0 = 0; j0 < nc; j0 += 64) cta_gemm_tile(C, A, B, ld, mr, nc, kd, i0, j0, As, Bs);
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kSmallThreads) small_front_kernel(SmallArgs<T> a) {
  const int s = a.level_fronts[blockIdx.x];
  const FrontDesc d = a.fronts[s];
  const int rows = d.rows, size = d.size, cols = d.size + d.ncb;
  T* f = a.block + d.block_off;
  int32_t* rid = a.rowid + d.rowid_off;
  const int tid = threadIdx.x;
  const int64_t total = (int64_t)rows * cols;
  for (int64_t e = tid; e < total; e += kSmallThreads) f[e] = T(0);
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
    f[a.anew_slot[q] + (int64_t)a.anew_col[q] * rows] = load_value<T>(a.values, a.anew_q[q]);
  for (int k = d.child_begin; k < d.child_end; ++k) {
    const FrontDesc c = a.fronts[a.child_idx[k]];
    const int slot0 = a.child_slot[k];
    const int crows = c.rows - c.size;
    const T* cb = a.block + c.cb_off;
    for (int t = 0; t < c.ncb; ++t) {
      T* dst = f + slot0 + a.cb_colmap[c.struct_begin + t] * rows;
      const T* src = cb + t * c.cb_ld;
      for (int i = tid; i < crows; i += kSmallThreads) dst[i] = src[i];
    }
  }
  __syncthreads();
  // Three barriers per column: (1) the previous column's multipliers are
  // scaled and this column's pivot is searched, each warp posting its
  // candidate in a mailbox double-buffered by column parity that every
  // thread then reduces itself; (2) the row interchange (the pivot is read
  // from row k only after it); (3) the rank-1 update, which forms each
  // multiplier a_ik * (1 / pivot) itself, exactly as it is stored (so the
  // arithmetic is that of scale-then-update).
  __shared__ double mk[2][kSmallThreads / 32];
  __shared__ int mi[2][kSmallThreads / 32];
  const int lane = tid & 31, warp = tid >> 5;
  T inv_prev = T(0);
  for (int k = 0; k < size; ++k) {
    if (k > 0)
      for (int i = k + tid; i < rows; i += kSmallThreads) f[i + (k - 1) * rows] *= inv_prev;
    double key = -1.0;
    int idx = INT_MAX;
    for (int i = k + tid; i < rows; i += kSmallThreads) {
      const double v = pivot_key(f[i + (int64_t)k * rows]);
      if (v > key) {
        key = v;
        idx = i;
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double ok = __shfl_down_sync(0xffffffffu, key, off);
      const int oi = __shfl_down_sync(0xffffffffu, idx, off);
      if (ok > key || (ok == key && oi < idx)) {
        key = ok;
        idx = oi;
      }
    }
    const int par = k & 1;
    if (lane == 0) {
      mk[par][warp] = key;
      mi[par][warp] = idx;
    }
    __syncthreads();
    double bk = mk[par][0];
    int p = mi[par][0];
    for (int w = 1; w < kSmallThreads / 32; ++w)
      if (mk[par][w] > bk || (mk[par][w] == bk && mi[par][w] < p)) {
        bk = mk[par][w];
        p = mi[par][w];
      }
    if (!(bk > 0.0)) {  // bk = |pivot|
      if (tid == 0) atomicExch(a.singular, 1);
      return;  // uniform: every thread reduced the same mailboxes
    }
    if (p != k) {
      for (int j = tid; j < cols; j += kSmallThreads) {
        const T t = f[k + (int64_t)j * rows];
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
    const T inv = recip_t(f[k + (int64_t)k * rows]);  // the pivot, swapped into row k
    // rank-1 update of the front's own columns, spread over all threads
    const int mr = rows - k - 1, mc = size - k - 1;
    for (int e = tid; e < mr * mc; e += kSmallThreads) {
      const int i = k + 1 + e % mr, j = k + 1 + e / mr;
      f[i + j * rows] = fma_t(-f[k + j * rows], f[i + k * rows] * inv, f[i + j * rows]);
    }
    inv_prev = inv;
    __syncthreads();
  }
  if (size > 0) {
    for (int i = size + tid; i < rows; i += kSmallThreads) f[i + (size - 1) * rows] *= inv_prev;
    __syncthreads();
  }
  __shared__ T As[64 * 16], Bs[16 * 64];
  // U12 = L11^-1 A12 in 16-row blocks: forward substitution within the block
  // (a thread per column), then the rows below by the tiled update
  for (int kb = 0; kb < size; kb += 16) {
    const int ke = min(size, kb + 16);
    for (int c = size + tid; c < cols; c += kSmallThreads) {
      T* col = f + (int64_t)c * rows;
      for (int k = kb; k < ke; ++k) {
        const T uk = col[k];
        for (int i = k + 1; i < ke; ++i) col[i] = fma_t(-f[i + (int64_t)k * rows], uk, col[i]);
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
  T* lp = a.L + d.l_off;
  for (int e = tid; e < rows * size; e += kSmallThreads) lp[e] = f[e];
  T* up = a.U + d.u_off;
  for (int t = 0; t < d.ncb; ++t)
    for (int kk = tid; kk < size; kk += kSmallThreads) up[kk + t * size] = f[kk + (size + t) * rows];
}

// ---- large fronts ----------------------------------------------------------
template <typename T>
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
  const T* block;  // small children's contribution blocks
  const T* stack;  // large children's contribution blocks
  T* front;        // rows x (size + ncb), ld = rows (zeroed before)
  const int32_t* rowid;
  int32_t* rowtmp;      // the front's slots before pivoting
};

template <typename T>
__global__ void big_assemble_kernel(BigArgs<T> a) {
  const FrontDesc& d = a.d;
  const int rows = d.rows;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  {
    const int slotn = rows - (d.new_end - d.new_begin);
    for (int64_t i = tid; i < d.new_end - d.new_begin; i += nth) a.rowtmp[slotn + i] = a.new_rows[d.new_begin + i];
  }
  for (int64_t q = d.anew_begin + tid; q < d.anew_end; q += nth)
    a.front[a.anew_slot[q] + (int64_t)a.anew_col[q] * rows] = load_value<T>(a.values, a.anew_q[q]);
  for (int k = d.child_begin; k < d.child_end; ++k) {
    const FrontDesc c = a.fronts[a.child_idx[k]];
    const int slot0 = a.child_slot[k];
    const int crows = c.rows - c.size;
    for (int64_t i = tid; i < crows; i += nth) a.rowtmp[slot0 + i] = a.rowid[c.rowid_off + c.size + i];
    const T* cb = (c.small ? a.block : a.stack) + c.cb_off;
    const int64_t ce = (int64_t)crows * c.ncb;
    for (int64_t e = tid; e < ce; e += nth) {
      const int i = (int)(e % crows), t = (int)(e / crows);
      a.front[(slot0 + i) + (int64_t)a.cb_colmap[c.struct_begin + t] * rows] = cb[i + (int64_t)t * c.cb_ld];
    }
  }
}

// After the partial LU: rows of the slots, U12, and the contribution block.
template <typename T>
__global__ void big_finalize_kernel(FrontDesc d, const T* front, const int* perm, const int32_t* rowtmp,
                                    int32_t* rowid, T* U, T* stack) {
  const int rows = d.rows, size = d.size;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = tid; i < rows; i += nth) rowid[d.rowid_off + i] = rowtmp[perm[i]];
  T* up = U + d.u_off;
  for (int64_t e = tid; e < (int64_t)size * d.ncb; e += nth) {
    const int kk = (int)(e % size), t = (int)(e / size);
    up[e] = front[kk + (int64_t)(size + t) * rows];
  }
  const int crows = rows - size;
  if (crows > 0) {
    T* cb = stack + d.cb_off;
    for (int64_t e = tid; e < (int64_t)crows * d.ncb; e += nth) {
      const int i = (int)(e % crows), t = (int)(e / crows);
      cb[i + (int64_t)t * d.cb_ld] = front[(size + i) + (int64_t)(size + t) * rows];
    }
  }
}

// ---- large complex fronts ----------------------------------------------------
// The partial LU of a complex front (the contract of lu_factor_partial_dev:
// the first `size` columns over all rows, interchanges across every column,
// U12 and the Schur complement), blocked by kZnb columns, five launches per
// block: the block's columns over all rows by one CTA (the reference's pivot
// rule, lu_front supernodal_lu.rs:490-533: the first row of largest modulus,
// multipliers by the reciprocal, the rank-1 updates inside the block); its
// interchanges on the other columns; its rows of U12 by a unit-lower solve;
// the trailing block as one real FP64 tensor-core GEMM (below).
constexpr int kZnb = 32;
constexpr int kZPanelThreads = 1024;

__device__ __forceinline__ bool front_stopped(const DevStatus* st) {
  return *reinterpret_cast<const volatile int*>(&st->singular_col) != INT_MAX;
}

__global__ void __launch_bounds__(kZPanelThreads) zfront_panel_kernel(zc* f, int rows, int k0, int k1, int* ipiv,
                                                                      int* perm, DevStatus* st) {
  __shared__ double mk[2][kZPanelThreads / 32];
  __shared__ int mi[2][kZPanelThreads / 32];
  if (front_stopped(st)) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (k0 == 0) {
    for (int i = tid; i < rows; i += kZPanelThreads) perm[i] = i;
    __syncthreads();
  }
  zc inv_prev(0.0);
  for (int k = k0; k < k1; ++k) {
    if (k > k0)
      for (int i = k + tid; i < rows; i += kZPanelThreads) f[i + (int64_t)(k - 1) * rows] *= inv_prev;
    double key = -1.0;
    int idx = INT_MAX;
    for (int i = k + tid; i < rows; i += kZPanelThreads) {
      const double v = pivot_key(f[i + (int64_t)k * rows]);
      if (v > key) {
        key = v;
        idx = i;
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double ok = __shfl_down_sync(0xffffffffu, key, off);
      const int oi = __shfl_down_sync(0xffffffffu, idx, off);
      if (ok > key || (ok == key && oi < idx)) {
        key = ok;
        idx = oi;
      }
    }
    const int par = k & 1;
    if (lane == 0) {
      mk[par][warp] = key;
      mi[par][warp] = idx;
    }
    __syncthreads();
    double bk = mk[par][0];
    int p = mi[par][0];
    for (int w = 1; w < kZPanelThreads / 32; ++w)
      if (mk[par][w] > bk || (mk[par][w] == bk && mi[par][w] < p)) {
        bk = mk[par][w];
        p = mi[par][w];
      }
    if (!(bk > 0.0)) {
      if (tid == 0) atomicMin(&st->singular_col, k);
      return;  // uniform: every thread reduced the same mailboxes
    }
    if (p != k) {
      for (int j = k0 + tid; j < k1; j += kZPanelThreads) {
        const zc t = f[k + (int64_t)j * rows];
        f[k + (int64_t)j * rows] = f[p + (int64_t)j * rows];
        f[p + (int64_t)j * rows] = t;
      }
      if (tid == 0) {
        const int t = perm[k];
        perm[k] = perm[p];
        perm[p] = t;
      }
    }
    if (tid == 0) ipiv[k] = p;
    __syncthreads();
    const zc inv = recip_t(f[k + (int64_t)k * rows]);
    const int mr = rows - k - 1, mc = k1 - k - 1;
    for (int e = tid; e < mr * mc; e += kZPanelThreads) {
      const int i = k + 1 + e % mr, j = k + 1 + e / mr;
      f[i + (int64_t)j * rows] = fma_t(-f[k + (int64_t)j * rows], f[i + (int64_t)k * rows] * inv,
                                       f[i + (int64_t)j * rows]);
    }
    inv_prev = inv;
    __syncthreads();
  }
  for (int i = k1 + tid; i < rows; i += kZPanelThreads) f[i + (int64_t)(k1 - 1) * rows] *= inv_prev;
}

// The block's interchanges, in order, on every column outside it (a thread per column).
__global__ void zfront_swap_kernel(zc* f, int rows, int cols, int k0, int k1, const int* ipiv, const DevStatus* st) {
  if (front_stopped(st)) return;
  const int w = k1 - k0, other = cols - w;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < other; t += gridDim.x * blockDim.x) {
    zc* col = f + (int64_t)(t < k0 ? t : t + w) * rows;
    for (int k = k0; k < k1; ++k) {
      const int p = ipiv[k];
      if (p != k) {
        const zc v = col[k];
        col[k] = col[p];
        col[p] = v;
      }
    }
  }
}

// U12 rows [k0, k1): x <- L11^-1 x for every column right of the block (a
// thread per column; the unit-lower block in shared memory).
__global__ void __launch_bounds__(256) zfront_trsm_kernel(zc* f, int rows, int cols, int k0, int k1,
                                                          const DevStatus* st) {
  __shared__ zc l11[kZnb][kZnb + 1];
  if (front_stopped(st)) return;
  const int w = k1 - k0;
  for (int e = threadIdx.x; e < kZnb * kZnb; e += blockDim.x) {
    const int r = e % kZnb, c = e / kZnb;
    l11[c][r] = (r < w && c < w && r > c) ? f[(k0 + r) + (int64_t)(k0 + c) * rows] : zc(0.0);
  }
  __syncthreads();
  for (int j = k1 + blockIdx.x * blockDim.x + threadIdx.x; j < cols; j += gridDim.x * blockDim.x) {
    zc* col = f + k0 + (int64_t)j * rows;
    zc x[kZnb];
#pragma unroll
    for (int r = 0; r < kZnb; ++r) x[r] = r < w ? col[r] : zc(0.0);
#pragma unroll
    for (int k = 0; k < kZnb; ++k)
#pragma unroll
      for (int i = k + 1; i < kZnb; ++i) x[i] = fma_t(-l11[k][i], x[k], x[i]);  // zero outside the block
#pragma unroll
    for (int r = 0; r < kZnb; ++r)
      if (r < w) col[r] = x[r];
  }
}

// L21 of a block (mr x w complex, rows k1.. of columns k0..k1) written as the
// real 2mr x 2w matrix whose complex entry a occupies the 2 x 2 block
// [re -im; im re]: then, with B and C viewed as real matrices of twice the
// rows (the interleaved (re, im) layout), C -= L21 U12 is one real GEMM
// (the FP64 tensor cores), the complex products' four real terms summed in
// another order than num-complex's (values to rounding, as the real path).
__global__ void zblock_expand_kernel(const zc* __restrict__ f, int rows, int k0, int w, int k1, int mr,
                                     double* __restrict__ ah, const DevStatus* st) {
  if (front_stopped(st)) return;
  const int ld = 2 * mr;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)mr * w;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % mr), l = (int)(e / mr);
    const zc a = f[(k1 + i) + (int64_t)(k0 + l) * rows];
    double* c0 = ah + (int64_t)(2 * l) * ld + 2 * i;
    double* c1 = c0 + ld;
    c0[0] = a.re;
    c0[1] = a.im;
    c1[0] = -a.im;
    c1[1] = a.re;
  }
}

// ---- after the factorization -----------------------------------------------
// Final position of every row, the row permutation, and the nonzero counts
// of each column of L and U (exact zeros are not stored, as in the reference).
// Grid: fronts x kCountSplit; CTA (s, y) takes every kCountSplit-th group of
// a front's columns, a warp per column.
constexpr int kCountSplit = 16;

template <typename T>
__global__ void positions_counts_kernel(const FrontDesc* fronts, int ns, const int32_t* rowid, const T* L,
                                        const T* U, const int32_t* struct_cols, int32_t* pos_of_row,
                                        int32_t* row_perm, int32_t* lcount, unsigned* ucount) {
  const int s = blockIdx.x;
  if (s >= ns) return;
  const FrontDesc d = fronts[s];
  const int rows = d.rows, size = d.size;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int warp = (threadIdx.x >> 5) + (int)blockIdx.y * nw, nwt = nw * (int)gridDim.y;
  if ((int)blockIdx.y * nw >= max(size, d.ncb)) return;  // no column for this CTA
  if (blockIdx.y == 0)
    for (int k = threadIdx.x; k < size; k += blockDim.x) {
      const int32_t r = rowid[d.rowid_off + k];
      pos_of_row[r] = d.begin + k;
      row_perm[d.begin + k] = r;
    }
  const T* lp = L + d.l_off;
  for (int jj = warp; jj < size; jj += nwt) {
    int cl = 0, cu = 0;
    for (int i = lane; i < rows; i += 32) {
      const T v = lp[i + (int64_t)jj * rows];
      if (i > jj) cl += v != T(0);
      if (i < jj) cu += v != T(0);
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
  const T* up = U + d.u_off;
  for (int t = warp; t < d.ncb; t += nwt) {
    int cu = 0;
    for (int kk = lane; kk < size; kk += 32) cu += up[kk + (int64_t)t * size] != T(0);
    for (int off = 16; off > 0; off >>= 1) cu += __shfl_xor_sync(0xffffffffu, cu, off);
    if (lane == 0 && cu) atomicAdd(&ucount[struct_cols[d.struct_begin + t]], (unsigned)cu);
  }
}

// ---- solve ------------------------------------------------------------------
constexpr int kSolveThreads = 256;

template <typename T>
__global__ void gather_rows_kernel(const double* b, const int32_t* row_perm, T* y, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = load_value<T>(b, row_perm[i]);
}

template <typename T>
__global__ void scatter_cols_kernel(const T* x, const int32_t* col_perm, double* b, int n) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) store_value(b, col_perm[j], x[j]);
}

constexpr int kRowChunk = 256;  // rows of L21 / U12 per CTA (one per thread)
constexpr int kKChunk = 256;    // columns of L21 / U12 per CTA
constexpr int kSolveBigSize = 512;  // larger diagonal blocks take the multi-CTA triangular sweep

// Forward, diagonal block of each front of a level (one CTA per front, for
// fronts of at most kSolveBigSize columns by default): unit-lower solve in 32-column
// blocks; the block's 32 x 32 triangle is staged in shared memory so the
// warp's 32 dependent steps read no global memory, and the rows below it in
// the diagonal block take the block's 32 terms with independent loads.
template <typename T>
__global__ void __launch_bounds__(kSolveThreads) fwd_diag_kernel(const FrontDesc* fronts, const int32_t* level,
                                                                 const T* L, T* y) {
  __shared__ T tri[32][33];
  __shared__ T yb[32];
  const FrontDesc d = fronts[level[blockIdx.x]];
  const int rows = d.rows, m = d.size;
  const T* lp = L + d.l_off;
  T* ys = y + d.begin;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int kb = 0; kb < m; kb += 32) {
    const int w = min(32, m - kb);
    for (int e = threadIdx.x; e < 32 * 32; e += kSolveThreads) {
      const int r = e & 31, c = e >> 5;
      tri[c][r] = (r < w && c < w && r > c) ? lp[(kb + r) + (int64_t)(kb + c) * rows] : T(0);
    }
    __syncthreads();
    if (warp == 0) {
      T v = lane < w ? ys[kb + lane] : T(0);
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const T yk = shfl_t(v, k);
        v -= tri[k][lane] * yk;  // zero on and above the diagonal and outside the block
      }
      if (lane < w) ys[kb + lane] = v;
      yb[lane] = lane < w ? v : T(0);
    }
    __syncthreads();
    for (int i = kb + w + threadIdx.x; i < m; i += kSolveThreads) {
      const T* row = lp + i + (int64_t)kb * rows;
      T acc = T(0);
      if (w == 32) {
#pragma unroll
        for (int k = 0; k < 32; ++k) acc = fma_t(row[(int64_t)k * rows], yb[k], acc);
      } else {
        for (int k = 0; k < w; ++k) acc = fma_t(row[(int64_t)k * rows], yb[k], acc);
      }
      ys[i] -= acc;
    }
    __syncthreads();
  }
}

// Forward, rows below the diagonal block: y[pos(row)] -= L21 y_s. A CTA per
// (chunk of rows, chunk of columns); a front with one column chunk subtracts
// directly (rows of different fronts of one level are distinct), otherwise
// the chunks' partial sums are combined in a fixed order by fwd_finish_kernel.
template <typename T>
__global__ void __launch_bounds__(kSolveThreads) fwd_l21_kernel(const FrontDesc* fronts, const SolveItem* items,
                                                                const T* L, const int32_t* rowid,
                                                                const int32_t* pos_of_row, const int64_t* fpart_off,
                                                                T* fpartial, T* y) {
  const SolveItem it = items[blockIdx.x];
  const FrontDesc d = fronts[it.front];
  const int i = d.size + it.chunk * kRowChunk + threadIdx.x;
  if (i >= d.rows) return;
  const int k0 = it.tchunk * kKChunk, k1 = min(d.size, k0 + kKChunk);
  const T* row = L + d.l_off + i;
  const T* ys = y + d.begin;
  T acc = T(0);
  int k = k0;
  for (; k + 8 <= k1; k += 8) {
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = row[(int64_t)(k + u) * d.rows];
#pragma unroll
    for (int u = 0; u < 8; ++u) acc = fma_t(v[u], ys[k + u], acc);
  }
  for (; k < k1; ++k) acc = fma_t(row[(int64_t)k * d.rows], ys[k], acc);
  if (d.size <= kKChunk)
    y[pos_of_row[rowid[d.rowid_off + i]]] -= acc;
  else
    fpartial[fpart_off[it.front] + (int64_t)it.tchunk * (d.rows - d.size) + (i - d.size)] = acc;
}

template <typename T>
__global__ void __launch_bounds__(kSolveThreads) fwd_finish_kernel(const FrontDesc* fronts, const SolveItem* items,
                                                                   const int32_t* rowid, const int32_t* pos_of_row,
                                                                   const int64_t* fpart_off, const T* fpartial,
                                                                   T* y) {
  const SolveItem it = items[blockIdx.x];
  const FrontDesc d = fronts[it.front];
  const int i = d.size + it.chunk * kRowChunk + threadIdx.x;
  if (i >= d.rows) return;
  const int nk = (d.size + kKChunk - 1) / kKChunk;
  const int64_t below = d.rows - d.size;
  T acc = T(0);
  for (int c = 0; c < nk; ++c) acc += fpartial[fpart_off[it.front] + c * below + (i - d.size)];
  y[pos_of_row[rowid[d.rowid_off + i]]] -= acc;
}

// Backward, U12 x[Struct(s)] in partial sums over column chunks (summed in a
// fixed order afterwards, so a solve is deterministic).
template <typename T>
__global__ void __launch_bounds__(kSolveThreads) bwd_u12_kernel(const FrontDesc* fronts, const SolveItem* items,
                                                                const T* U, const int32_t* struct_cols,
                                                                const int64_t* part_off, const T* x,
                                                                T* partial) {
  const SolveItem it = items[blockIdx.x];
  const FrontDesc d = fronts[it.front];
  const int kk = it.chunk * kRowChunk + threadIdx.x;
  if (kk >= d.size) return;
  const T* up = U + d.u_off + kk;
  const int32_t* st = struct_cols + d.struct_begin;
  const int t0 = it.tchunk * kKChunk, t1 = min(d.ncb, t0 + kKChunk);
  T acc = T(0);
  int t = t0;
  for (; t + 8 <= t1; t += 8) {
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = up[(int64_t)(t + u) * d.size];
#pragma unroll
    for (int u = 0; u < 8; ++u) acc = fma_t(v[u], x[st[t + u]], acc);
  }
  for (; t < t1; ++t) acc = fma_t(up[(int64_t)t * d.size], x[st[t]], acc);
  partial[part_off[it.front] + (int64_t)it.tchunk * d.size + kk] = acc;
}

// x_s -= (the U12 partial sums of front s), in chunk order
template <typename T>
__device__ __forceinline__ void subtract_partials(const FrontDesc& d, int64_t poff, const T* partial, T* xs) {
  const int ntc = (d.ncb + kKChunk - 1) / kKChunk;
  for (int kk = threadIdx.x; kk < d.size; kk += blockDim.x) {
    T acc = T(0);
    for (int tc = 0; tc < ntc; ++tc) acc += partial[poff + (int64_t)tc * d.size + kk];
    xs[kk] -= acc;
  }
}

// Backward, diagonal block (one CTA per front of at most kSolveBigSize
// columns): subtract the U12 partial sums, then the upper solve in 32-column
// blocks from the last, x_j times the reciprocal of its diagonal as in the
// reference's upper sweep; the block's triangle is staged in shared memory.
template <typename T>
__global__ void __launch_bounds__(kSolveThreads) bwd_diag_kernel(const FrontDesc* fronts, const int32_t* level,
                                                                 const T* L, const int64_t* part_off,
                                                                 const T* partial, T* x) {
  __shared__ T tri[32][33];
  __shared__ T xb[32];
  const int s = level[blockIdx.x];
  const FrontDesc d = fronts[s];
  const int rows = d.rows, m = d.size;
  const T* lp = L + d.l_off;
  T* xs = x + d.begin;
  subtract_partials(d, part_off[s], partial, xs);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int jb = m; jb > 0; jb -= 32) {
    const int j0 = max(0, jb - 32), w = jb - j0;
    for (int e = threadIdx.x; e < 32 * 32; e += kSolveThreads) {
      const int r = e & 31, c = e >> 5;
      tri[c][r] = (r < w && c < w && r <= c) ? lp[(j0 + r) + (int64_t)(j0 + c) * rows] : T(0);
    }
    __syncthreads();
    if (warp == 0) {
      T v = lane < w ? xs[j0 + lane] : T(0);
      for (int j = w - 1; j >= 0; --j) {
        if (lane == j) v = v * recip_t(tri[j][j]);
        const T xj = shfl_t(v, j);
        if (lane < j) v -= tri[j][lane] * xj;
      }
      if (lane < w) xs[j0 + lane] = v;
      xb[lane] = lane < w ? v : T(0);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < j0; i += kSolveThreads) {
      const T* row = lp + i + (int64_t)j0 * rows;
      T acc = T(0);
      if (w == 32) {
#pragma unroll
        for (int l = 0; l < 32; ++l) acc = fma_t(row[(int64_t)l * rows], xb[l], acc);
      } else {
        for (int l = 0; l < w; ++l) acc = fma_t(row[(int64_t)l * rows], xb[l], acc);
      }
      xs[i] -= acc;
    }
    __syncthreads();
  }
}

// Backward, the U12 partial sums of one large front (its diagonal block is
// then solved by the multi-CTA triangular solve).
template <typename T>
__global__ void __launch_bounds__(kSolveThreads) bwd_partials_kernel(const FrontDesc* fronts, int s,
                                                                     const int64_t* part_off, const T* partial,
                                                                     T* x) {
  const FrontDesc d = fronts[s];
  const int ntc = (d.ncb + kKChunk - 1) / kKChunk;
  const int kk = blockIdx.x * kSolveThreads + threadIdx.x;
  if (kk >= d.size) return;
  T acc = T(0);
  for (int tc = 0; tc < ntc; ++tc) acc += partial[part_off[s] + (int64_t)tc * d.size + kk];
  x[d.begin + kk] -= acc;
}

// ---- the mixed form's refinement ---------------------------------------------
// max that keeps a NaN (a diverged solve must not look converged)
__device__ __forceinline__ double nanmax(double m, double v) { return (v != v || v > m) ? v : m; }

// r = b - A x in FP64 (row by row, entries in column order) and the maxima
// of |r|, |x| and |b| into norms[0..2] (atomic max on the bit patterns:
// non-negative doubles order as integers and a NaN lies above all numbers)
__global__ void residual_csr_kernel(int n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ col,
                                    const int64_t* __restrict__ map, const double* __restrict__ values,
                                    const double* __restrict__ x, const double* __restrict__ b,
                                    double* __restrict__ r, unsigned long long* norms) {
  double mr = 0.0, mx = 0.0, mb = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int64_t q = ptr[i]; q < ptr[i + 1]; ++q) acc = __fma_rn(values[map[q]], x[col[q]], acc);
    const double ri = b[i] - acc;
    r[i] = ri;
    mr = nanmax(mr, fabs(ri));
    mx = nanmax(mx, fabs(x[i]));
    mb = nanmax(mb, fabs(b[i]));
  }
  for (int off = 16; off > 0; off >>= 1) {
    mr = nanmax(mr, __shfl_xor_sync(0xffffffffu, mr, off));
    mx = nanmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    mb = nanmax(mb, __shfl_xor_sync(0xffffffffu, mb, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&norms[0], (unsigned long long)__double_as_longlong(mr));
    atomicMax(&norms[1], (unsigned long long)__double_as_longlong(mx));
    atomicMax(&norms[2], (unsigned long long)__double_as_longlong(mb));
  }
}

// ||A||_inf into norms[3]
__global__ void row_abs_sum_kernel(int n, const int64_t* __restrict__ ptr, const int64_t* __restrict__ map,
                                   const double* __restrict__ values, unsigned long long* norms) {
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int64_t q = ptr[i]; q < ptr[i + 1]; ++q) acc += fabs(values[map[q]]);
    m = nanmax(m, acc);
  }
  for (int off = 16; off > 0; off >>= 1) m = nanmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(&norms[3], (unsigned long long)__double_as_longlong(m));
}

__global__ void axpy_kernel(const double* __restrict__ d, double* __restrict__ x, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += d[i];
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

// The complex front's partial LU (kernels above) on lane context lc.
// Stream-ordered; a zero pivot lands in lc's status (singular_col).
int zfront_lu(alg_ctx* lc, zc* f, int rows, int size, int cols, int* ipiv, int* perm, double* ah) {
  cudaStream_t st = lc->stream;
  for (int k0 = 0; k0 < size; k0 += kZnb) {
    const int k1 = std::min(size, k0 + kZnb);
    zfront_panel_kernel<<<1, kZPanelThreads, 0, st>>>(f, rows, k0, k1, ipiv, perm, lc->d_status);
    count_launches();
    if (cols > k1 - k0) {
      zfront_swap_kernel<<<grid_for(lc, cols - (k1 - k0), 256), 256, 0, st>>>(f, rows, cols, k0, k1, ipiv,
                                                                                 lc->d_status);
      count_launches();
    }
    if (cols > k1) {
      zfront_trsm_kernel<<<grid_for(lc, cols - k1, 256), 256, 0, st>>>(f, rows, cols, k0, k1, lc->d_status);
      count_launches();
      if (rows > k1) {
        // trailing block: C -= L21 U12 as one real FP64 tensor-core GEMM of
        // the 2 x 2 real form of L21 and the real views of U12 and C
        const int mr = rows - k1, w = k1 - k0;
        zblock_expand_kernel<<<grid_for(lc, (int64_t)mr * w, 256), 256, 0, st>>>(f, rows, k0, w, k1, mr, ah,
                                                                                  lc->d_status);
        count_launches();
        ALG_TRY(gemm_dmma_sub_dev(lc, 2 * mr, cols - k1, 2 * w, ah, 2 * mr,
                                  reinterpret_cast<const double*>(f + k0 + (int64_t)k1 * rows), 2 * rows,
                                  reinterpret_cast<double*>(f + k1 + (int64_t)k1 * rows), 2 * rows));
      }
    }
    ALG_CUDA_TRY(cudaGetLastError());
  }
  return ALG_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
int DeviceLu::init(alg_ctx* c, const FrontPlan* p, int w) {
  ctx = c;
  plan = p;
  words = w;
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
  ALG_TRY(upload(F.col_perm, &d_col_perm));
  const size_t n = (size_t)std::max<idx>(F.n, 1);
  ALG_TRY(dmalloc((void**)&d_values, sizeof(double) * words * std::max<idx>(F.nnz, 1)));
  ALG_TRY(dmalloc((void**)&d_block, sizeof(double) * words * F.block_total));
  ALG_TRY(dmalloc((void**)&d_stack, sizeof(double) * words * F.stack_total));
  n_lanes = std::max(1, std::min(F.n_lanes, kMaxLanes));
  lane_ctx[0] = ctx;
  int64_t max_rows = 1;
  for (const auto& d : F.fronts) max_rows = std::max<int64_t>(max_rows, d.rows);
  for (int k = 0; k < n_lanes; ++k) {
    if (k > 0) {
      ALG_TRY(alg_ctx_create(nullptr, &lane_ctx[k]));
      lane_ctx[k]->prof_parent = ctx;  // the lanes' launches show in the handle's profile
      ALG_CUDA_TRY(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
    }
    const int64_t fb = k < (int)F.lane_front_buf.size() ? F.lane_front_buf[k] : F.front_buf;
    ALG_TRY(dmalloc((void**)&d_front[k], sizeof(double) * words * std::max<int64_t>(fb, 1)));
    ALG_TRY(dmalloc((void**)&d_ipiv[k], sizeof(int) * max_rows));
    ALG_TRY(dmalloc((void**)&d_perm[k], sizeof(int) * max_rows));
    ALG_TRY(dmalloc((void**)&d_rowtmp[k], sizeof(int32_t) * max_rows));
    if (words == 2)  // 2 rows x 2 kZnb columns of doubles per complex row
      ALG_TRY(dmalloc((void**)&d_zblock[k], sizeof(double) * 4 * kZnb * max_rows));
  }
  ALG_CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
  ALG_TRY(dmalloc((void**)&d_flag, sizeof(int) * 4));
  ALG_TRY(dmalloc((void**)&d_y, sizeof(double) * words * n));
  ALG_TRY(dmalloc((void**)&d_rhs, sizeof(double) * words * n));
  {
    // solve schedule and the partial-sum offsets of the column chunks
    std::vector<SolveItem> fwd, fin, bwd;
    std::vector<int32_t> small_list;
    std::vector<int64_t> poff(std::max<idx>(F.ns, 1), 0), fpoff(std::max<idx>(F.ns, 1), 0);
    int64_t ptot = 0, fptot = 0;
    int max_big = 0;
    // fronts with more columns than this take the multi-CTA sweeps
    // (ALG_SPLU_SOLVE_BIG overrides, for tests of that path on small grids)
    int big_size = kSolveBigSize;
    if (const char* e = std::getenv("ALG_SPLU_SOLVE_BIG")) big_size = std::max(32, std::atoi(e));
    if (words == 2) big_size = INT_MAX;  // complex: every diagonal block by the one-CTA kernels
    for (idx s = 0; s < F.ns; ++s) {
      const FrontDesc& d = F.fronts[s];
      poff[s] = ptot;
      ptot += (int64_t)((d.ncb + kKChunk - 1) / kKChunk) * d.size;
      fpoff[s] = fptot;
      if (d.size > kKChunk) fptot += (int64_t)((d.size + kKChunk - 1) / kKChunk) * (d.rows - d.size);
    }
    const int nl = (int)F.solve_level_ptr.size() - 1;
    fwd_item_ptr.assign(std::max(nl, 0) + 1, 0);
    fin_item_ptr.assign(std::max(nl, 0) + 1, 0);
    bwd_item_ptr.assign(std::max(nl, 0) + 1, 0);
    solve_small_ptr.assign(std::max(nl, 0) + 1, 0);
    solve_big.assign(std::max(nl, 0), {});
    for (int h = 0; h < nl; ++h) {
      for (int t = F.solve_level_ptr[h]; t < F.solve_level_ptr[h + 1]; ++t) {
        const int s = F.solve_level_fronts[t];
        const FrontDesc& d = F.fronts[s];
        if (d.size > big_size) {
          solve_big[h].push_back(s);
          max_big = std::max(max_big, (int)d.size);
        } else {
          small_list.push_back(s);
        }
        const int nk = (d.size + kKChunk - 1) / kKChunk;
        for (int c = 0; c * kRowChunk < d.rows - d.size; ++c) {
          for (int kc = 0; kc < nk; ++kc) fwd.push_back(SolveItem{s, c, kc, 0});
          if (nk > 1) fin.push_back(SolveItem{s, c, 0, 0});
        }
        for (int c = 0; c * kRowChunk < d.size; ++c)
          for (int tc = 0; tc * kKChunk < d.ncb; ++tc) bwd.push_back(SolveItem{s, c, tc, 0});
      }
      solve_small_ptr[h + 1] = (int)small_list.size();
      fwd_item_ptr[h + 1] = (int)fwd.size();
      fin_item_ptr[h + 1] = (int)fin.size();
      bwd_item_ptr[h + 1] = (int)bwd.size();
    }
    ALG_TRY(upload(small_list, &d_solve_small));
    ALG_TRY(upload(fwd, &d_fwd_items));
    ALG_TRY(upload(fin, &d_fin_items));
    ALG_TRY(upload(bwd, &d_bwd_items));
    ALG_TRY(upload(poff, &d_part_off));
    ALG_TRY(upload(fpoff, &d_fpart_off));
    ALG_TRY(dmalloc((void**)&d_partial, sizeof(double) * words * std::max<int64_t>(ptot, 1)));
    ALG_TRY(dmalloc((void**)&d_fpartial, sizeof(double) * words * std::max<int64_t>(fptot, 1)));
    tflag_count = max_big / 64 + 2;
    ALG_TRY(dmalloc((void**)&d_tflags, sizeof(int) * (tflag_count + 1)));
  }
  for (int b = 0; b < 2; ++b) {
    ALG_TRY(dmalloc((void**)&fac[b].L, sizeof(double) * words * F.l_total));
    ALG_TRY(dmalloc((void**)&fac[b].U, sizeof(double) * words * F.u_total));
    ALG_TRY(dmalloc((void**)&fac[b].rowid, sizeof(int32_t) * F.rowid_total));
    ALG_TRY(dmalloc((void**)&fac[b].pos_of_row, sizeof(int32_t) * n));
    ALG_TRY(dmalloc((void**)&fac[b].row_perm, sizeof(int32_t) * n));
    ALG_TRY(dmalloc((void**)&fac[b].lcount, sizeof(int32_t) * n));
    ALG_TRY(dmalloc((void**)&fac[b].ucount, sizeof(unsigned) * n));
  }
  return ALG_OK;
}

int DeviceLu::ensure_refine_buffers() {
  if (d_csr_ptr != nullptr) return ALG_OK;
  const FrontPlan& F = *plan;
  const size_t n = (size_t)std::max<idx>(F.n, 1);
  ALG_TRY(upload(F.csr_ptr, &d_csr_ptr));
  ALG_TRY(upload(F.csr_col, &d_csr_col));
  ALG_TRY(upload(F.csr_map, &d_csr_map));
  ALG_TRY(dmalloc((void**)&d_b0, sizeof(double) * n));
  ALG_TRY(dmalloc((void**)&d_x, sizeof(double) * n));
  ALG_TRY(dmalloc((void**)&d_norms, sizeof(unsigned long long) * 4));
  for (auto& f : fac) ALG_TRY(dmalloc((void**)&f.values, sizeof(double) * std::max<idx>(F.nnz, 1)));
  return ALG_OK;
}

void DeviceLu::release() {
  for (int k = 0; k < kMaxLanes; ++k) {
    for (void* q : {(void*)d_front[k], (void*)d_ipiv[k], (void*)d_perm[k], (void*)d_rowtmp[k], (void*)d_zblock[k]})
      if (q) cudaFree(q);
    if (k > 0 && lane_ctx[k]) alg_ctx_destroy(lane_ctx[k]);
    if (ev_join[k]) cudaEventDestroy(ev_join[k]);
  }
  if (ev_fork) cudaEventDestroy(ev_fork);
  for (void* q : {(void*)d_fronts, (void*)d_child_idx, (void*)d_child_slot, (void*)d_struct_cols,
                  (void*)d_cb_colmap, (void*)d_anew_q, (void*)d_anew_slot, (void*)d_anew_col, (void*)d_new_rows,
                  (void*)d_small_levels, (void*)d_col_perm, (void*)d_values, (void*)d_block, (void*)d_stack,
                  (void*)d_flag, (void*)d_y,
                  (void*)d_rhs, (void*)d_solve_small, (void*)d_fwd_items, (void*)d_fin_items, (void*)d_bwd_items,
                  (void*)d_part_off, (void*)d_fpart_off, (void*)d_partial, (void*)d_fpartial, (void*)d_tflags,
                  (void*)d_csr_ptr, (void*)d_csr_col, (void*)d_csr_map, (void*)d_b0, (void*)d_x, (void*)d_norms})
    if (q) cudaFree(q);
  for (auto& f : fac)
    for (void* q : {(void*)f.values, (void*)f.L, (void*)f.U, (void*)f.rowid, (void*)f.pos_of_row,
                    (void*)f.row_perm, (void*)f.lcount, (void*)f.ucount})
      if (q) cudaFree(q);
  *this = DeviceLu();
}

int DeviceLu::factor(int b) {
  if (words == 2) return factor_t<zc>(b, d_values, -1);  // complex: FP64 only
  if (prec < 0) return factor_t<double>(b, d_values, -1);
  ALG_TRY(ensure_refine_buffers());
  const FrontPlan& F = *plan;
  cudaStream_t st = ctx->stream;
  // the refinement's A and its norm belong to the factor set
  ALG_CUDA_TRY(cudaMemcpyAsync(fac[b].values, d_values, sizeof(double) * std::max<idx>(F.nnz, 1),
                               cudaMemcpyDeviceToDevice, st));
  ALG_CUDA_TRY(cudaMemsetAsync(d_norms + 3, 0, sizeof(unsigned long long), st));
  row_abs_sum_kernel<<<grid_for(ctx, F.n, 256), 256, 0, st>>>((int)F.n, d_csr_ptr, d_csr_map, fac[b].values,
                                                               d_norms);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  return factor_t<float>(b, d_values, prec == ALG_PREC_FP32 ? -1 : prec);
}

// Factors `values` into factor set `b` in precision T. Stream-ordered; the
// singular flag and the dense status block are read by finish().
template <typename T>
int DeviceLu::factor_t(int b, const double* values, int tc_prec) {
  const FrontPlan& F = *plan;
  Factors& out = fac[b];
  out.prec = std::is_same<T, float>::value ? (tc_prec < 0 ? ALG_PREC_FP32 : tc_prec) : -1;
  cudaStream_t st = ctx->stream;
  T* block = reinterpret_cast<T*>(d_block);
  T* L = reinterpret_cast<T*>(out.L);
  T* U = reinterpret_cast<T*>(out.U);
  const int tok = prof_begin(ctx, ALG_K_SPARSE);
  ALG_CUDA_TRY(cudaMemsetAsync(d_flag, 0, sizeof(int) * 4, st));
  ALG_TRY(status_reset(ctx));
  // small fronts, one launch per level
  SmallArgs<T> sa;
  sa.fronts = d_fronts;
  sa.child_idx = d_child_idx;
  sa.child_slot = d_child_slot;
  sa.cb_colmap = d_cb_colmap;
  sa.anew_q = d_anew_q;
  sa.anew_slot = d_anew_slot;
  sa.anew_col = d_anew_col;
  sa.new_rows = d_new_rows;
  sa.values = values;
  sa.block = block;
  sa.L = L;
  sa.U = U;
  sa.rowid = out.rowid;
  sa.singular = d_flag;
  const int tok_small = prof_begin(ctx, ALG_K_BATCH);
  for (size_t h = 0; h + 1 < F.small_level_ptr.size(); ++h) {
    const int cnt = F.small_level_ptr[h + 1] - F.small_level_ptr[h];
    if (cnt == 0) continue;
    sa.level_fronts = d_small_levels + F.small_level_ptr[h];
    small_front_kernel<T><<<cnt, kSmallThreads, 0, st>>>(sa);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
  }
  prof_end(ctx, tok_small, 0.0, 0.0);
  // large fronts: the lanes' subtrees concurrently (issued front by front in
  // turn), then the fronts above them on the handle's stream
  if (n_lanes > 1) {
    ALG_CUDA_TRY(cudaEventRecord(ev_fork, st));
    for (int k = 1; k < n_lanes; ++k) {
      ALG_CUDA_TRY(cudaStreamWaitEvent(lane_ctx[k]->stream, ev_fork, 0));
      ALG_TRY(status_reset(lane_ctx[k]));
    }
  }
  std::vector<int> next(n_lanes);
  for (int k = 0; k < n_lanes; ++k) next[k] = F.lane_ptr[k];
  for (bool more = true; more;) {
    more = false;
    for (int k = 0; k < n_lanes; ++k) {
      if (next[k] >= F.lane_ptr[k + 1]) continue;
      ALG_TRY(factor_big<T>(b, F.lane_fronts[next[k]++], k, values, tc_prec));
      more = true;
    }
  }
  for (int k = 1; k < n_lanes; ++k) {
    ALG_CUDA_TRY(cudaEventRecord(ev_join[k], lane_ctx[k]->stream));
    ALG_CUDA_TRY(cudaStreamWaitEvent(st, ev_join[k], 0));
  }
  for (int32_t s : F.top_fronts) ALG_TRY(factor_big<T>(b, s, 0, values, tc_prec));
  ALG_CUDA_TRY(cudaMemsetAsync(out.ucount, 0, sizeof(unsigned) * std::max<idx>(F.n, 1), st));
  if (F.ns > 0) {
    positions_counts_kernel<T><<<dim3((unsigned)F.ns, kCountSplit), 256, 0, st>>>(
        d_fronts, (int)F.ns, out.rowid, L, U, d_struct_cols, out.pos_of_row, out.row_perm, out.lcount, out.ucount);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
  }
  prof_end(ctx, tok, F.flops, 0.0);
  return ALG_OK;
}

// One large front on lane `lane`: assemble, blocked partial-pivoting LU of
// its columns over all its rows, then its rows, U12 and contribution block.
template <typename T>
int DeviceLu::factor_big(int b, int32_t s, int lane, const double* values, int tc_prec) {
  const FrontPlan& F = *plan;
  Factors& out = fac[b];
  alg_ctx* lc = lane_ctx[lane];
  cudaStream_t st = lc->stream;
  T* front = reinterpret_cast<T*>(d_front[lane]);
  const FrontDesc& d = F.fronts[s];
  const int cols = d.size + d.ncb;
  ALG_CUDA_TRY(cudaMemsetAsync(front, 0, sizeof(T) * (size_t)d.rows * cols, st));
  BigArgs<T> ba;
  ba.d = d;
  ba.fronts = d_fronts;
  ba.child_idx = d_child_idx;
  ba.child_slot = d_child_slot;
  ba.cb_colmap = d_cb_colmap;
  ba.anew_q = d_anew_q;
  ba.anew_slot = d_anew_slot;
  ba.anew_col = d_anew_col;
  ba.new_rows = d_new_rows;
  ba.values = values;
  ba.block = reinterpret_cast<T*>(d_block);
  ba.stack = reinterpret_cast<T*>(d_stack);
  ba.front = front;
  ba.rowid = out.rowid;
  ba.rowtmp = d_rowtmp[lane];
  int64_t work = (int64_t)(d.anew_end - d.anew_begin) + d.rows;
  for (int k = d.child_begin; k < d.child_end; ++k) {
    const FrontDesc& c = F.fronts[F.child_idx[k]];
    work = std::max<int64_t>(work, (int64_t)(c.rows - c.size) * c.ncb);
  }
  big_assemble_kernel<T><<<grid_for(lc, work, 256), 256, 0, st>>>(ba);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  if constexpr (std::is_same<T, zc>::value) {
    ALG_TRY(zfront_lu(lc, front, d.rows, d.size, cols, d_ipiv[lane], d_perm[lane], d_zblock[lane]));
  } else {
    LuPlan lp;
    // block width of a large front's LU (ALG_SPLU_NB: measurement switch)
    static const int splu_nb = [] {
      const char* e = std::getenv("ALG_SPLU_NB");
      return e ? std::max(16, std::atoi(e)) : 64;
    }();
    // leaf-panel width (ALG_SPLU_NBL: measurement switch)
    static const int splu_nbl = [] {
      const char* e = std::getenv("ALG_SPLU_NBL");
      return e ? std::max(1, std::min(32, std::atoi(e))) : 16;
    }();
    lp.nb = splu_nb;
    lp.nbl = splu_nbl;
    lp.tc_prec = tc_prec;
    if constexpr (std::is_same<T, float>::value) {
      // the mixed form's FP32 fronts pivot by tournament (refinement restores
      // the FP64 backward error); the FP64 form keeps the reference's pivots
      lp.tslu = 1;
      lp.nbl = 32;
    }
    ALG_TRY((lu_factor_partial_dev<T, false>(lc, front, d.rows, d.size, cols, d.rows, d_ipiv[lane], d_perm[lane],
                                             lp)));
  }
  T* L = reinterpret_cast<T*>(out.L);
  T* U = reinterpret_cast<T*>(out.U);
  ALG_CUDA_TRY(cudaMemcpyAsync(L + d.l_off, front, sizeof(T) * (size_t)d.rows * d.size, cudaMemcpyDeviceToDevice, st));
  const int64_t fw = std::max<int64_t>((int64_t)d.rows, (int64_t)d.rows * d.ncb);
  big_finalize_kernel<T><<<grid_for(lc, fw, 256), 256, 0, st>>>(d, front, d_perm[lane], d_rowtmp[lane], out.rowid, U,
                                                                 reinterpret_cast<T*>(d_stack));
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

// Reads the factorization's outcome (synchronises): SP_OK or SP_SINGULAR.
// The mixed form refactors in FP64 when its FP32 factorization met a zero
// pivot (an FP32 underflow need not be a singular A).
int DeviceLu::finish(int b, Stats* stats) {
  const FrontPlan& F = *plan;
  int h_flag[4] = {0, 0, 0, 0};
  ALG_CUDA_TRY(cudaMemcpyAsync(h_flag, d_flag, sizeof(h_flag), cudaMemcpyDeviceToHost, ctx->stream));
  ALG_TRY(status_fetch(ctx));
  bool timeout = ctx->h_status->timeout != 0, singular = ctx->h_status->singular_col != INT_MAX;
  for (int k = 1; k < n_lanes; ++k) {
    ALG_TRY(status_fetch(lane_ctx[k]));
    timeout = timeout || lane_ctx[k]->h_status->timeout != 0;
    singular = singular || lane_ctx[k]->h_status->singular_col != INT_MAX;
  }
  if (timeout) return ALG_TIMEOUT;
  if (h_flag[0] != 0 || singular) {
    if (fac[b].prec < 0) return SP_SINGULAR;
    ALG_TRY(refactor_fp64(b));
    return finish(b, stats);
  }
  if (fac[b].prec >= 0) {
    unsigned long long bits = 0;
    ALG_CUDA_TRY(cudaMemcpy(&bits, d_norms + 3, sizeof(bits), cudaMemcpyDeviceToHost));
    std::memcpy(&fac[b].anorm, &bits, sizeof(double));
  }
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

// The set's own values in FP64 (the mixed form's last resort).
int DeviceLu::refactor_fp64(int b) {
  return factor_t<double>(b, fac[b].values, -1);
}

// d_rhs <- (the set's LU)^-1 d_rhs in the set's precision. Stream-ordered.
template <typename T>
int DeviceLu::sweep_t(int b) {
  const FrontPlan& F = *plan;
  const Factors& f = fac[b];
  const T* L = reinterpret_cast<const T*>(f.L);
  const T* U = reinterpret_cast<const T*>(f.U);
  T* y = reinterpret_cast<T*>(d_y);
  T* partial = reinterpret_cast<T*>(d_partial);
  T* fpartial = reinterpret_cast<T*>(d_fpartial);
  int* abort_flag = d_tflags + tflag_count;
  cudaStream_t st = ctx->stream;
  const int n = (int)F.n;
  const int tok = prof_begin(ctx, ALG_K_SOLVE);
  gather_rows_kernel<T><<<grid_for(ctx, n, 256), 256, 0, st>>>(d_rhs, f.row_perm, y, n);
  count_launches();
  ALG_CUDA_TRY(cudaMemsetAsync(abort_flag, 0, sizeof(int), st));
  const int nl = (int)F.solve_level_ptr.size() - 1;
  for (int h = 0; h < nl; ++h) {
    const int cnt = solve_small_ptr[h + 1] - solve_small_ptr[h];
    if (cnt > 0) {
      fwd_diag_kernel<T><<<cnt, kSolveThreads, 0, st>>>(d_fronts, d_solve_small + solve_small_ptr[h], L, y);
      count_launches();
    }
    if constexpr (!std::is_same<T, zc>::value) {  // (none for complex factors)
      for (int32_t s : solve_big[h]) {
        const FrontDesc& d = F.fronts[s];
        ALG_TRY(tri_solve_dev<T>(ctx, L + d.l_off, d.rows, d.size, y + d.begin, false, d_tflags, abort_flag));
      }
    }
    const int ni = fwd_item_ptr[h + 1] - fwd_item_ptr[h];
    if (ni > 0) {
      fwd_l21_kernel<T><<<ni, kSolveThreads, 0, st>>>(d_fronts, d_fwd_items + fwd_item_ptr[h], L, f.rowid,
                                                      f.pos_of_row, d_fpart_off, fpartial, y);
      count_launches();
    }
    const int nf = fin_item_ptr[h + 1] - fin_item_ptr[h];
    if (nf > 0) {
      fwd_finish_kernel<T><<<nf, kSolveThreads, 0, st>>>(d_fronts, d_fin_items + fin_item_ptr[h], f.rowid,
                                                         f.pos_of_row, d_fpart_off, fpartial, y);
      count_launches();
    }
  }
  for (int h = nl - 1; h >= 0; --h) {
    const int ni = bwd_item_ptr[h + 1] - bwd_item_ptr[h];
    if (ni > 0) {
      bwd_u12_kernel<T><<<ni, kSolveThreads, 0, st>>>(d_fronts, d_bwd_items + bwd_item_ptr[h], U, d_struct_cols,
                                                      d_part_off, y, partial);
      count_launches();
    }
    const int cnt = solve_small_ptr[h + 1] - solve_small_ptr[h];
    if (cnt > 0) {
      bwd_diag_kernel<T><<<cnt, kSolveThreads, 0, st>>>(d_fronts, d_solve_small + solve_small_ptr[h], L,
                                                        d_part_off, partial, y);
      count_launches();
    }
    if constexpr (!std::is_same<T, zc>::value) {
      for (int32_t s : solve_big[h]) {
        const FrontDesc& d = F.fronts[s];
        if (d.ncb > 0) {
          bwd_partials_kernel<T><<<(d.size + kSolveThreads - 1) / kSolveThreads, kSolveThreads, 0, st>>>(
              d_fronts, s, d_part_off, partial, y);
          count_launches();
        }
        ALG_TRY(tri_solve_dev<T>(ctx, L + d.l_off, d.rows, d.size, y + d.begin, true, d_tflags, abort_flag));
      }
    }
  }
  scatter_cols_kernel<T><<<grid_for(ctx, n, 256), 256, 0, st>>>(y, d_col_perm, d_rhs, n);
  count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  prof_end(ctx, tok, 4.0 * (double)(F.l_total + F.u_total), sizeof(T) * (double)(F.l_total + F.u_total));
  return ALG_OK;
}

// x = A^-1 b for the factors of set `b`, with b (n) already on the device in
// d_rhs; the result lands in d_rhs.
int DeviceLu::solve(int b) {
  const FrontPlan& F = *plan;
  if (F.n == 0) return ALG_OK;
  last = RefineReport();
  last.precision = fac[b].prec;
  if (words == 2) return sweep_t<zc>(b);
  if (fac[b].prec < 0) return sweep_t<double>(b);
  return refine(b);
}

// The mixed form: x_0 = 0, r_0 = b; x += LU32^-1 r, r = b - A x (FP64)
// until ||r||_inf <= tol (||A||_inf ||x||_inf + ||b||_inf); a stall (less
// than a halving twice running), divergence or max_ir steps refactor the set
// in FP64 and solve directly.
int DeviceLu::refine(int b) {
  const FrontPlan& F = *plan;
  const int n = (int)F.n;
  cudaStream_t st = ctx->stream;
  const double target = tol > 0 ? tol : 10.0 * (double)n * std::ldexp(1.0, -53);
  const int steps = max_ir > 0 ? max_ir : 10;
  const int g = grid_for(ctx, n, 256);
  ALG_CUDA_TRY(cudaMemcpyAsync(d_b0, d_rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  ALG_CUDA_TRY(cudaMemsetAsync(d_x, 0, sizeof(double) * n, st));
  double prev = INFINITY;
  int stall = 0;
  for (int it = 0; it < steps; ++it) {
    ALG_TRY(sweep_t<float>(b));  // d_rhs: r -> the correction
    axpy_kernel<<<g, 256, 0, st>>>(d_rhs, d_x, n);
    count_launches();
    ALG_CUDA_TRY(cudaMemsetAsync(d_norms, 0, sizeof(unsigned long long) * 3, st));
    residual_csr_kernel<<<g, 256, 0, st>>>(n, d_csr_ptr, d_csr_col, d_csr_map, fac[b].values, d_x, d_b0, d_rhs,
                                           d_norms);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
    unsigned long long bits[3];
    ALG_CUDA_TRY(cudaMemcpyAsync(bits, d_norms, sizeof(bits), cudaMemcpyDeviceToHost, st));
    ALG_CUDA_TRY(cudaStreamSynchronize(st));
    double nr, nx, nb;
    std::memcpy(&nr, &bits[0], sizeof(double));
    std::memcpy(&nx, &bits[1], sizeof(double));
    std::memcpy(&nb, &bits[2], sizeof(double));
    const double den = fac[b].anorm * nx + nb;
    const double eta = den == 0.0 ? nr : nr / den;
    last.iterations = it + 1;
    last.backward_error = eta;
    if (!(eta == eta) || std::isinf(eta)) break;
    if (eta <= target) {
      ALG_CUDA_TRY(cudaMemcpyAsync(d_rhs, d_x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      return ALG_OK;
    }
    if (eta > 0.5 * prev) {
      if (++stall >= 2) break;
    } else {
      stall = 0;
    }
    prev = eta;
  }
  // FP64 refactorization of this set's values, then a direct solve
  ALG_TRY(refactor_fp64(b));
  const int rc = finish(b, nullptr);
  if (rc != SP_OK) return rc;
  last.fell_back = 1;
  last.precision = -1;
  last.backward_error = -1.0;
  ALG_CUDA_TRY(cudaMemcpyAsync(d_rhs, d_b0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  return sweep_t<double>(b);
}

}  // namespace sp
}  // namespace alg
