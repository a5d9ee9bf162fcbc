// Complex twins of the dense LU (src/lapack/complex.rs): zgetrf, zgetrf_rect,
// zgesv and zgetri on the GPU, bit-identical to the reference.
//
// The reference's Complex64 is num_complex::Complex<f64> (num-complex 0.4),
// whose operators are
//   (a + ib)(c + id) = (ac - bd) + i(ad + bc)
//   (a + ib)/(c + id) = ((ac + bd) + i(bc - ad)) / (cc + dd)
//   (a + ib) - (c + id) = (a - c) + i(b - d)
// each product, sum and quotient rounded on its own (rustc contracts
// nothing); the kernels below spell every operation with the _rn intrinsics
// so that nvcc cannot fuse them. The pivot measure is |Re| + |Im|.
//
// Layout: a complex entry is a double2 (re, im), the interleaved layout of
// the host's complex arrays; matrices column-major, a[i + j * lda].
//
// Factorization (complex.rs:67-124 zgetf2, 169-208 zgetrf_rect): blocked by
// 16 columns (zpanel_kernel, zswap_trsm_kernel, zgemm_exact_kernel below),
// every entry still taking its terms in increasing column order with each
// operation rounded on its own, so the factors are the reference's bit for
// bit. The pivot is the first row with the largest |Re| + |Im| at or below
// the diagonal (the reference's strict-greater scan, NaN included); a zero
// pivot stops the factorization with exactly the steps before it applied,
// as the reference's early return leaves the matrix. The unblocked form
// (zpivot_kernel + zupdate_kernel, one step per column) stays as a
// measurement switch.
//
// Solve (complex.rs:279-312): the interchanges applied to b in order; the
// unit-lower sweep as a column pipeline (one CTA; row i takes its term for
// b_j, j = 0, 1, ..., as each b_j becomes final); the upper sweep row
// by row from the bottom: the products u_ij b_j of a row in parallel, then
// subtracted from b_i in increasing j by one thread (the reference's order)
// and divided by u_ii.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstddef>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "dense.cuh"

namespace alg {
namespace {

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 zsub(double2 a, double2 b) {
  return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
__device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
  const double norm_sqr = __dadd_rn(__dmul_rn(b.x, b.x), __dmul_rn(b.y, b.y));
  const double re = __dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
  const double im = __dsub_rn(__dmul_rn(a.y, b.x), __dmul_rn(a.x, b.y));
  return make_double2(__ddiv_rn(re, norm_sqr), __ddiv_rn(im, norm_sqr));
}
__device__ __forceinline__ double2 zadd(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double zabs1(double2 z) { return __dadd_rn(fabs(z.x), fabs(z.y)); }

__device__ __forceinline__ bool stopped(const DevStatus* st) {
  return *reinterpret_cast<const volatile int*>(&st->singular_col) != INT_MAX;
}

constexpr int kPivThreads = 1024;

// The pivot row of column j (rows j..m-1) by the reference's scan, computed
// by every thread of the CTA: the diagonal comes first, a row below replaces
// it only when strictly greater in |Re| + |Im| (a NaN never is), and among
// equal rows the first. ipiv[j] is written; a zero (or empty) pivot is
// recorded in the status block and -1 returned instead. sb and si hold one
// entry per warp.
__device__ int zpick_pivot(const double2* __restrict__ col, int m, int j, int* __restrict__ ipiv, DevStatus* st,
                           double* sb, int* si, int* piv_s) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nt = blockDim.x;
  // the diagonal's measure, loaded early by the thread that decides
  const double vj = t == 0 ? zabs1(col[j]) : 0.0;
  // first maximum over this thread's rows below the diagonal; -1 means none
  double best = -1.0;
  int bi = INT_MAX;
  for (int i = j + 1 + t; i < m; i += nt) {
    const double c = zabs1(col[i]);
    if (c > best) {
      best = c;
      bi = i;
    }
  }
  // larger value wins, the lower row among equals
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_down_sync(0xffffffffu, best, off);
    const int oi = __shfl_down_sync(0xffffffffu, bi, off);
    if (ob > best || (ob == best && oi < bi)) {
      best = ob;
      bi = oi;
    }
  }
  if (lane == 0) {
    sb[warp] = best;
    si[warp] = bi;
  }
  __syncthreads();
  if (t == 0) {
    double gb = sb[0];
    int gi = si[0];
    for (int w = 1; w < nt / 32; ++w)
      if (sb[w] > gb || (sb[w] == gb && si[w] < gi)) {
        gb = sb[w];
        gi = si[w];
      }
    int jp = j;
    double pbest = vj;
    if (gi != INT_MAX && gb > vj) {
      jp = gi;
      pbest = gb;
    }
    if (pbest <= 0.0) {  // ZERO_DETERMINANT = 0.0
      atomicMin(&st->singular_col, j);
      jp = -1;
    } else {
      ipiv[j] = jp;
    }
    *piv_s = jp;
  }
  __syncthreads();
  return *piv_s;
}

// Step j of the factorization of an m x nc matrix (m >= nc): pivot, swap of
// the whole rows (all nc columns), scaling of column j below the diagonal.
__global__ void __launch_bounds__(kPivThreads) zpivot_kernel(double2* __restrict__ a, int lda, int m, int nc, int j,
                                                             int* __restrict__ ipiv, DevStatus* st) {
  __shared__ double sb[kPivThreads / 32];
  __shared__ int si[kPivThreads / 32];
  __shared__ int piv_s;
  if (stopped(st)) return;
  const int t = threadIdx.x;
  double2* col = a + (size_t)j * lda;
  const int jp = zpick_pivot(col, m, j, ipiv, st, sb, si, &piv_s);
  if (jp < 0) return;
  if (jp != j) {
    for (int k = t; k < nc; k += kPivThreads) {
      double2* c = a + (size_t)k * lda;
      const double2 x = c[j];
      c[j] = c[jp];
      c[jp] = x;
    }
  }
  __syncthreads();
  const double2 d = col[j];
  for (int i = j + 1 + t; i < m; i += kPivThreads) col[i] = zdiv(col[i], d);
}

// Step j's rank-1 update: a[i, k] -= a[i, j] * a[j, k] for i in (j, m),
// k in (j, nc); a thread per row, a CTA row per column (grid-strided).
__global__ void __launch_bounds__(256) zupdate_kernel(double2* __restrict__ a, int lda, int m, int nc, int j,
                                                      const DevStatus* st) {
  if (stopped(st)) return;
  const int i = j + 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double2 l = a[i + (size_t)j * lda];
  for (int k = j + 1 + blockIdx.y; k < nc; k += gridDim.y) {
    double2* c = a + (size_t)k * lda;
    c[i] = zsub(c[i], zmul(l, c[j]));
  }
}

// ---- Blocked form: the same operations on every entry, in the same order ----
//
// Columns are taken kZpw at a time. For the block [k0, k0 + w):
//   zpanel_kernel      one CTA runs the reference's steps k0..k0+w-1 on the
//                      block's own columns over all rows (pivot, swap within
//                      the block, division, rank-1 updates of the block's
//                      later columns);
//   zswap_trsm_kernel  a thread per column outside the block applies the
//                      block's interchanges in order; right of the block it
//                      then forms the block's rows of U by the unit-lower
//                      solve, row r taking l_rk u_k for k = k0, k0 + 1, ...;
//   zgemm_exact_kernel the trailing block a_ic -= l_ik u_kc, k increasing
//                      over the block, a CTA per 64 x 64 tile.
// Every entry right of the block therefore receives the terms of steps
// k0, k0 + 1, ... in that order, each product and difference rounded on its
// own, as in the reference's loop, and the interchanges move whole rows
// (factors and all) before any of the block's terms reach them, which is
// where the reference's row swap leaves them. A zero pivot at column s of
// the block stops the panel there; the other two kernels then apply only
// the steps k0..s-1 (the valid width), which is the state the reference's
// loop leaves on its early return.
constexpr int kZpw = 16;
constexpr int kZpanelThreads = 384;
constexpr int kZtile = 64;

// Steps of the block [k0, k0 + w) that ran: w, fewer when the panel stopped
// at a zero pivot inside the block, 0 or less after one before it.
__device__ __forceinline__ int valid_width(const DevStatus* st, int k0, int w) {
  const int s = *reinterpret_cast<const volatile int*>(&st->singular_col);
  return s == INT_MAX ? w : min(w, s - k0);
}

// The panel runs in sub-panels of kZsub columns, so that each step's rank-1
// update touches at most kZsub - 1 columns: after a sub-panel's steps, the
// block's columns right of it take that sub-panel's terms at once (its rows
// of U by a unit-lower solve, a thread per column; the rows below by a rank
// kZsub update, a thread per row, each entry's terms in increasing k), which
// reads and writes the block about a third as often as a rank-1 update per
// step. A zero pivot inside a sub-panel still lets the steps before it reach
// the columns right of it, as the reference's loop has applied them.
constexpr int kZsub = 4;

// A shared-memory load the compiler keeps where it is written: the rank
// update reads the same kZsub x 12 values of U for every row, and hoisted
// out of the row loop they would not fit in registers.
__device__ __forceinline__ double2 lds_f64x2(const double2* p) {
  double2 r;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
               : "=d"(r.x), "=d"(r.y)
               : "r"(static_cast<unsigned>(__cvta_generic_to_shared(p))));
  return r;
}

__global__ void __launch_bounds__(kZpanelThreads) zpanel_kernel(double2* __restrict__ a, int lda, int m, int k0, int w,
                                                                int* __restrict__ ipiv, DevStatus* st) {
  __shared__ double sb[kZpanelThreads / 32];
  __shared__ int si[kZpanelThreads / 32];
  __shared__ int piv_s;
  __shared__ double2 urow[kZpw];
  __shared__ double2 usub[kZsub][kZpw];  // the sub-panel's rows of U right of it
  if (stopped(st)) return;
  const int t = threadIdx.x, kend = k0 + w;
  for (int s0 = k0; s0 < kend; s0 += kZsub) {
    const int s1 = min(s0 + kZsub, kend);
    int jv = s1 - s0;  // the sub-panel's steps that ran
#pragma unroll 1
    for (int j = s0; j < s1; ++j) {
      double2* col = a + (size_t)j * lda;
      const int jp = zpick_pivot(col, m, j, ipiv, st, sb, si, &piv_s);
      if (jp < 0) {  // the same for every thread (read from shared memory)
        jv = j - s0;
        break;
      }
      // the interchange within the block's columns; row j (the pivot row
      // after it) kept for the updates
      if (t < w) {
        double2* c = a + (size_t)(k0 + t) * lda;
        const double2 x = c[j];
        if (jp != j) {
          const double2 y = c[jp];
          c[j] = y;
          c[jp] = x;
          urow[t] = y;
        } else {
          urow[t] = x;
        }
      }
      __syncthreads();
      const int jj = j - s0;
      const double2 d = urow[j - k0];
#pragma unroll 1
      for (int i = j + 1 + t; i < m; i += kZpanelThreads) {
        // the row's entries in the sub-panel's later columns loaded together
        // with the one below the pivot, before any store
        double2* row = a + i + (size_t)s0 * lda;
        const double2 x = col[i];
        double2 v[kZsub];
#pragma unroll
        for (int c = 1; c < kZsub; ++c)
          if (c > jj && s0 + c < s1) v[c] = row[(size_t)c * lda];
        const double2 l = zdiv(x, d);
        col[i] = l;
#pragma unroll
        for (int c = 1; c < kZsub; ++c)
          if (c > jj && s0 + c < s1) row[(size_t)c * lda] = zsub(v[c], zmul(l, urow[s0 - k0 + c]));
      }
      __syncthreads();  // column j + 1 is final below row j before its pivot search
    }
    const int nr = kend - s1;  // the block's columns right of the sub-panel
    if (nr > 0 && jv > 0) {
      if (t < nr) {
        double2* c = a + (size_t)(s1 + t) * lda;
        double2 v[kZsub];
#pragma unroll
        for (int r = 0; r < kZsub; ++r)
          if (s0 + r < s1) v[r] = c[s0 + r];
#pragma unroll
        for (int r = 1; r < kZsub; ++r)
#pragma unroll
          for (int k = 0; k < kZsub - 1; ++k)
            if (s0 + r < s1 && k < r && k < jv) v[r] = zsub(v[r], zmul(a[s0 + r + (size_t)(s0 + k) * lda], v[k]));
#pragma unroll
        for (int r = 0; r < kZsub; ++r)
          if (s0 + r < s1) {
            if (r > 0) c[s0 + r] = v[r];
            usub[r][t] = v[r];
          }
      }
      __syncthreads();
#pragma unroll 1
      for (int i = s1 + t; i < m; i += kZpanelThreads) {
        double2 l[kZsub];
#pragma unroll
        for (int k = 0; k < kZsub; ++k)
          if (k < jv) l[k] = a[i + (size_t)(s0 + k) * lda];
        double2* row = a + i + (size_t)s1 * lda;
        double2 v[kZpw - kZsub];
#pragma unroll
        for (int c = 0; c < kZpw - kZsub; ++c)
          if (c < nr) v[c] = row[(size_t)c * lda];
#pragma unroll
        for (int c = 0; c < kZpw - kZsub; ++c)
          if (c < nr) {
#pragma unroll
            for (int k = 0; k < kZsub; ++k)
              if (k < jv) v[c] = zsub(v[c], zmul(l[k], lds_f64x2(&usub[k][c])));
            row[(size_t)c * lda] = v[c];
          }
      }
      __syncthreads();
    }
    if (jv < s1 - s0) return;  // stopped at a zero pivot
  }
}

// A thread per column outside the block (nc - w of them): the block's valid
// interchanges; right of the block, then the block's rows of U:
// u_r = a_r - sum over k < r of l_rk u_k, the terms in increasing k, with
// the block's unit-lower factor staged in shared memory. The interchanges
// (row j with row ipiv[j], j = k0, k0 + 1, ... in order) are composed once
// per CTA into a gather over the rows they touch: the block's own rows
// first, then the rows below the block that a pivot came from, at most
// 2 kZpw in all. Each thread then loads those entries of its column together
// and stores them permuted: the same final rows as the swaps one by one.
constexpr int kZswapThreads = 128;

__global__ void __launch_bounds__(kZswapThreads) zswap_trsm_kernel(double2* __restrict__ a, int lda, int nc, int k0, int w,
                                                         const int* __restrict__ ipiv, const DevStatus* st) {
  constexpr int kRows = 2 * kZpw;
  __shared__ double2 Ls[kZpw * kZpw];  // Ls[r + k * kZpw] = l(k0 + r, k0 + k)
  __shared__ int pos_s[kRows];         // the touched rows
  __shared__ int src_s[kRows];         // the row whose entry ends at pos_s[q]
  __shared__ int ns_s;
  const int wv = valid_width(st, k0, w);
  if (wv <= 0) return;
  for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
    const int r = e % w, k = e / w;
    Ls[r + k * kZpw] = a[k0 + r + (size_t)(k0 + k) * lda];
  }
  __shared__ int piv_s[kZpw];
  if (threadIdx.x < wv) piv_s[threadIdx.x] = ipiv[k0 + threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    int ns = w;
    for (int q = 0; q < w; ++q) pos_s[q] = src_s[q] = k0 + q;
    for (int j = k0; j < k0 + wv; ++j) {
      const int jp = piv_s[j - k0];  // jp >= j
      if (jp == j) continue;
      int qb = jp - k0;
      if (jp >= k0 + w) {
        qb = w;
        while (qb < ns && pos_s[qb] != jp) ++qb;
        if (qb == ns) {
          pos_s[ns] = src_s[ns] = jp;
          ++ns;
        }
      }
      const int qa = j - k0, x = src_s[qa];
      src_s[qa] = src_s[qb];
      src_s[qb] = x;
    }
    ns_s = ns;
  }
  __syncthreads();
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc - w) return;
  const bool right = c >= k0;
  if (right) c += w;  // past the block's own columns
  double2* col = a + (size_t)c * lda;
  const int ns = ns_s;
  double2 v[kRows];
#pragma unroll
  for (int q = 0; q < kRows; ++q)
    if (q < ns) v[q] = col[src_s[q]];
  if (right) {
#pragma unroll
    for (int r = 1; r < kZpw; ++r) {
      const int kend = min(r, wv);
#pragma unroll
      for (int k = 0; k < kZpw - 1; ++k)
        if (r < w && k < kend) v[r] = zsub(v[r], zmul(Ls[r + k * kZpw], v[k]));
    }
  }
#pragma unroll
  for (int q = 0; q < kRows; ++q)
    if (q < ns && (src_s[q] != pos_s[q] || (right && q > 0 && q < w))) col[pos_s[q]] = v[q];
}

// The trailing block, rows and columns from k0 + w: a CTA per 64 x 64 tile,
// 256 threads with 4 x 4 entries each (rows tx + 16 i, columns ty + 16 j);
// the block's 64 x wv slice of L and wv x 64 slice of U staged in shared
// memory, each entry's terms taken in increasing k.
__global__ void __launch_bounds__(256) zgemm_exact_kernel(double2* __restrict__ a, int lda, int m, int nc, int k0,
                                                          int w, const DevStatus* st) {
  __shared__ double2 As[kZpw][kZtile];  // As[k][r] = l(r0 + r, k0 + k)
  __shared__ double2 Bs[kZpw][kZtile];  // Bs[k][c] = u(k0 + k, c0 + c)
  const int wv = valid_width(st, k0, w);
  if (wv <= 0) return;
  const int r0 = k0 + w + blockIdx.x * kZtile, c0 = k0 + w + blockIdx.y * kZtile;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const double2 zero = make_double2(0.0, 0.0);
  for (int e = t; e < wv * kZtile; e += blockDim.x) {
    const int r = e % kZtile, k = e / kZtile;  // rows fastest: contiguous in a column
    As[k][r] = r0 + r < m ? a[r0 + r + (size_t)(k0 + k) * lda] : zero;
  }
  for (int e = t; e < wv * kZtile; e += blockDim.x) {
    const int k = e % wv, cc = e / wv;  // the block's rows fastest: contiguous in a column
    Bs[k][cc] = c0 + cc < nc ? a[k0 + k + (size_t)(c0 + cc) * lda] : zero;
  }
  __syncthreads();
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = r0 + tx + 16 * i, cc = c0 + ty + 16 * j;
      acc[i][j] = (r < m && cc < nc) ? a[r + (size_t)cc * lda] : zero;
    }
  for (int k = 0; k < wv; ++k) {
    double2 l[4], u[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) l[i] = As[k][tx + 16 * i];
#pragma unroll
    for (int j = 0; j < 4; ++j) u[j] = Bs[k][ty + 16 * j];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = zsub(acc[i][j], zmul(l[i], u[j]));
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = r0 + tx + 16 * i, cc = c0 + ty + 16 * j;
      if (r < m && cc < nc) a[r + (size_t)cc * lda] = acc[i][j];
    }
}

constexpr int kSolveThreads = 1024;
constexpr int kFoldChunk = 2048;  // products per chunk of the upper sweep (32 KB of shared memory)

// zgesv's interchanges and unit-lower sweep (complex.rs:287-301), one CTA:
// at step j every row below j takes its term l_ij b_j, so each row's terms
// arrive in increasing j and b_j is final when step j starts.
__global__ void __launch_bounds__(kSolveThreads) zforward_kernel(const double2* __restrict__ lu, int lda, int n,
                                                                 const int* __restrict__ ipiv, double2* b) {
  const int t = threadIdx.x;
  if (t == 0)
    for (int k = 0; k < n; ++k) {
      const int p = ipiv[k];
      const double2 x = b[k];
      b[k] = b[p];
      b[p] = x;
    }
  for (int j = 0; j + 1 < n; ++j) {
    __syncthreads();  // step j - 1's updates (b_j's last term among them) are in place
    const double2 bj = b[j];
    const double2* lcol = lu + (size_t)j * lda;
    for (int i = j + 1 + t; i < n; i += kSolveThreads) b[i] = zsub(b[i], zmul(lcol[i], bj));
  }
}

// zgesv's upper sweep (complex.rs:304-311), one CTA: row i's products in
// parallel (by chunks), folded into b_i in increasing j by thread 0.
__global__ void __launch_bounds__(kSolveThreads) zbackward_kernel(const double2* __restrict__ lu, int lda, int n,
                                                                  double2* b) {
  __shared__ double2 p[kFoldChunk];
  __shared__ double2 sum_s;
  const int t = threadIdx.x;
  for (int i = n - 1; i >= 0; --i) {
    if (t == 0) sum_s = b[i];
    for (int j0 = i + 1; j0 < n; j0 += kFoldChunk) {
      const int j1 = min(n, j0 + kFoldChunk);
      for (int j = j0 + t; j < j1; j += kSolveThreads) p[j - j0] = zmul(lu[i + (size_t)j * lda], b[j]);
      __syncthreads();
      if (t == 0) {
        double2 s = sum_s;
        for (int j = j0; j < j1; ++j) s = zsub(s, p[j - j0]);
        sum_s = s;
      }
      __syncthreads();
    }
    if (t == 0) b[i] = zdiv(sum_s, lu[i + (size_t)i * lda]);
    __syncthreads();
  }
}

// zgetri (complex.rs:130-158 ztrti2 'Upper' 'Non-unit', then 217-271), in
// three parts. U is inverted in place in one CTA, column after column: the
// diagonal becomes 1/u_jj, and row i < j of the column becomes
// -(1/u_jj) * (sum over k = i..j-1 of a_ik a_kj, summed from zero in
// increasing k) with a_ik already inverted; x holds the sums so that no
// entry of the column is overwritten before every row has read it. A zero
// u_jj stops with the columns before it inverted, as in the reference.
__global__ void __launch_bounds__(kSolveThreads) ztrti2_kernel(double2* __restrict__ a, int lda, int n,
                                                              double2* __restrict__ x, DevStatus* st) {
  const int t = threadIdx.x;
  for (int j = 0; j < n; ++j) {
    const double2 ujj = a[j + (size_t)j * lda];  // columns before j never write it
    if (ujj.x == 0.0 && ujj.y == 0.0) {
      if (t == 0) atomicMin(&st->singular_col, j);
      return;
    }
    const double2 inv = zdiv(make_double2(1.0, 0.0), ujj);
    const double2 ajj = make_double2(-inv.x, -inv.y);
    for (int i = t; i < j; i += kSolveThreads) {
      double2 sum = make_double2(0.0, 0.0);
      for (int k = i; k < j; ++k) sum = zadd(sum, zmul(a[i + (size_t)k * lda], a[k + (size_t)j * lda]));
      x[i] = sum;
    }
    __syncthreads();  // every row has read column j
    if (t == 0) a[j + (size_t)j * lda] = inv;
    for (int i = t; i < j; i += kSolveThreads) a[i + (size_t)j * lda] = zmul(ajj, x[i]);
    __syncthreads();  // column j is final before column j + 1 reads it
  }
}

// Column j of inv(A) L = inv(U) (columns right of j already final): the L
// entries below the diagonal move to work and become zero ...
__global__ void __launch_bounds__(256) zgetri_work_kernel(double2* __restrict__ a, int lda, int n, int j,
                                                          double2* __restrict__ work) {
  for (int i = j + 1 + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double2* e = a + i + (size_t)j * lda;
    work[i] = *e;
    *e = make_double2(0.0, 0.0);
  }
}

// ... then a_ij -= sum over k > j of a_ik work_k (from zero, increasing k), a
// thread per row.
__global__ void __launch_bounds__(256) zgetri_col_kernel(double2* __restrict__ a, int lda, int n, int j,
                                                         const double2* __restrict__ work) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double2 sum = make_double2(0.0, 0.0);
  for (int k = j + 1; k < n; ++k) sum = zadd(sum, zmul(a[i + (size_t)k * lda], work[k]));
  double2* e = a + i + (size_t)j * lda;
  *e = zsub(*e, sum);
}

// The interchanges undone as column swaps, from the second-to-last pivot
// down; a thread per row.
__global__ void __launch_bounds__(256) zgetri_swap_kernel(double2* __restrict__ a, int lda, int n,
                                                          const int* __restrict__ ipiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = n - 2; j >= 0; --j) {
    const int jp = ipiv[j];
    if (jp != j) {
      const double2 v = a[i + (size_t)j * lda];
      a[i + (size_t)j * lda] = a[i + (size_t)jp * lda];
      a[i + (size_t)jp * lda] = v;
    }
  }
}

// Factorization of the m x nc device matrix (m >= nc), stream-ordered; a zero
// pivot lands in the status block's singular_col.
int zlu_factor_dev(alg_ctx* ctx, double2* d_a, int m, int nc, int lda, int* d_ipiv) {
  // ALG_ZLU_UNBLOCKED=1 (measurement switch): one pivot and one rank-1
  // launch per column instead of the blocked form; both give the same bits
  static const bool unblocked = std::getenv("ALG_ZLU_UNBLOCKED") != nullptr;
  if (!unblocked) {
    for (int k0 = 0; k0 < nc; k0 += kZpw) {
      const int w = std::min(kZpw, nc - k0);
      zpanel_kernel<<<1, kZpanelThreads, 0, ctx->stream>>>(d_a, lda, m, k0, w, d_ipiv, ctx->d_status);
      int launches = 1;
      if (nc > w) {
        zswap_trsm_kernel<<<(nc - w + kZswapThreads - 1) / kZswapThreads, kZswapThreads, 0, ctx->stream>>>(d_a, lda, nc, k0, w, d_ipiv, ctx->d_status);
        ++launches;
      }
      const int rows = m - k0 - w, cols = nc - k0 - w;
      if (rows > 0 && cols > 0) {
        dim3 grid((rows + kZtile - 1) / kZtile, (cols + kZtile - 1) / kZtile);
        zgemm_exact_kernel<<<grid, 256, 0, ctx->stream>>>(d_a, lda, m, nc, k0, w, ctx->d_status);
        ++launches;
      }
      count_launches(launches);
    }
    ALG_CUDA_TRY(cudaGetLastError());
    return ALG_OK;
  }
  for (int j = 0; j < nc; ++j) {
    zpivot_kernel<<<1, kPivThreads, 0, ctx->stream>>>(d_a, lda, m, nc, j, d_ipiv, ctx->d_status);
    const int rows = m - j - 1, cols = nc - j - 1;
    int launches = 1;
    if (rows > 0 && cols > 0) {
      dim3 grid((rows + 255) / 256, std::min(cols, 65535));
      zupdate_kernel<<<grid, 256, 0, ctx->stream>>>(d_a, lda, m, nc, j, ctx->d_status);
      ++launches;
    }
    count_launches(launches);
  }
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

bool zsize_ok(size_t n) { return n <= (size_t)INT_MAX / 4; }

struct ZCtxLock {
  alg_ctx* ctx = nullptr;
  std::unique_lock<std::mutex> lk;
  int rc = ALG_OK;
  ZCtxLock() {
    rc = default_ctx(&ctx);
    if (rc == ALG_OK) lk = std::unique_lock<std::mutex>(ctx->mu);
  }
};

// Host drop-in core: a (m x nc complex, interleaved) and b (m complex, or
// null) copied in, factored (and solved), copied back.
int host_zlu(double* a, size_t m, size_t nc, size_t* ipiv, double* b) {
  if (!zsize_ok(m) || !zsize_ok(nc)) return ALG_BAD_SHAPE;
  ZCtxLock L;
  if (L.rc != ALG_OK) return L.rc;
  alg_ctx* ctx = L.ctx;
  const int M = (int)m, N = (int)nc;
  const size_t abytes = 2 * sizeof(double) * m * nc;
  double2* d_a = nullptr;
  double2* d_b = nullptr;
  int* d_ipiv = nullptr;
  ALG_TRY(ws_get(ctx, WS_A, abytes, reinterpret_cast<void**>(&d_a)));
  ALG_TRY(ws_get(ctx, WS_IPIV, sizeof(int) * std::max<size_t>(nc, 1), reinterpret_cast<void**>(&d_ipiv)));
  if (b != nullptr) ALG_TRY(ws_get(ctx, WS_B, 2 * sizeof(double) * m, reinterpret_cast<void**>(&d_b)));
  ALG_CUDA_TRY(cudaMemcpyAsync(d_a, a, abytes, cudaMemcpyHostToDevice, ctx->stream));
  if (d_b) ALG_CUDA_TRY(cudaMemcpyAsync(d_b, b, 2 * sizeof(double) * m, cudaMemcpyHostToDevice, ctx->stream));
  ALG_TRY(status_reset(ctx));
  ALG_TRY(zlu_factor_dev(ctx, d_a, M, N, M, d_ipiv));
  ALG_TRY(status_fetch(ctx));
  const bool singular = ctx->h_status->singular_col != INT_MAX;
  if (!singular && d_b) {
    zforward_kernel<<<1, kSolveThreads, 0, ctx->stream>>>(d_a, M, M, d_ipiv, d_b);
    zbackward_kernel<<<1, kSolveThreads, 0, ctx->stream>>>(d_a, M, M, d_b);
    count_launches(2);
    ALG_CUDA_TRY(cudaGetLastError());
    ALG_CUDA_TRY(cudaMemcpyAsync(b, d_b, 2 * sizeof(double) * m, cudaMemcpyDeviceToHost, ctx->stream));
  }
  ALG_CUDA_TRY(cudaMemcpyAsync(a, d_a, abytes, cudaMemcpyDeviceToHost, ctx->stream));
  std::vector<int> h_ipiv(std::max<size_t>(nc, 1));
  ALG_CUDA_TRY(cudaMemcpyAsync(h_ipiv.data(), d_ipiv, sizeof(int) * nc, cudaMemcpyDeviceToHost, ctx->stream));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (singular) return ALG_SINGULAR;
  if (ipiv)
    for (size_t k = 0; k < nc; ++k) ipiv[k] = (size_t)h_ipiv[k];
  return ALG_OK;
}

// Host drop-in core of zgetri: the factors copied in, inverted, copied back
// (also on ALG_SINGULAR, with the reference's partial state).
int host_zgetri(double* lu, size_t n, const size_t* ipiv) {
  if (!zsize_ok(n)) return ALG_BAD_SHAPE;
  std::vector<int> h_ipiv(n);
  for (size_t k = 0; k < n; ++k) {
    if (ipiv[k] >= n) return ALG_BAD_SHAPE;
    h_ipiv[k] = (int)ipiv[k];
  }
  ZCtxLock L;
  if (L.rc != ALG_OK) return L.rc;
  alg_ctx* ctx = L.ctx;
  const int N = (int)n;
  const size_t abytes = 2 * sizeof(double) * n * n;
  double2* d_a = nullptr;
  double2* d_x = nullptr;
  int* d_ipiv = nullptr;
  ALG_TRY(ws_get(ctx, WS_A, abytes, reinterpret_cast<void**>(&d_a)));
  ALG_TRY(ws_get(ctx, WS_X, 2 * sizeof(double) * n, reinterpret_cast<void**>(&d_x)));
  ALG_TRY(ws_get(ctx, WS_IPIV, sizeof(int) * n, reinterpret_cast<void**>(&d_ipiv)));
  ALG_CUDA_TRY(cudaMemcpyAsync(d_a, lu, abytes, cudaMemcpyHostToDevice, ctx->stream));
  ALG_CUDA_TRY(cudaMemcpyAsync(d_ipiv, h_ipiv.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
  ALG_TRY(status_reset(ctx));
  ztrti2_kernel<<<1, kSolveThreads, 0, ctx->stream>>>(d_a, N, N, d_x, ctx->d_status);
  count_launches();
  ALG_TRY(status_fetch(ctx));
  const bool singular = ctx->h_status->singular_col != INT_MAX;
  if (!singular) {
    const int grid = (N + 255) / 256;
    for (int j = N - 2; j >= 0; --j) {
      zgetri_work_kernel<<<std::max(1, (N - j - 1 + 255) / 256), 256, 0, ctx->stream>>>(d_a, N, N, j, d_x);
      zgetri_col_kernel<<<grid, 256, 0, ctx->stream>>>(d_a, N, N, j, d_x);
      count_launches(2);
    }
    zgetri_swap_kernel<<<grid, 256, 0, ctx->stream>>>(d_a, N, N, d_ipiv);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
  }
  ALG_CUDA_TRY(cudaMemcpyAsync(lu, d_a, abytes, cudaMemcpyDeviceToHost, ctx->stream));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return singular ? ALG_SINGULAR : ALG_OK;
}

}  // namespace
}  // namespace alg

// complex.rs:217 zgetri(lu, n, ipiv)
extern "C" int alg_zgetri(double* lu, size_t n, const size_t* ipiv) {
  if (n == 0) return ALG_OK;
  if (lu == nullptr || ipiv == nullptr) return ALG_INVALID_ARGUMENT;
  return alg::host_zgetri(lu, n, ipiv);
}

// complex.rs:67 zgetrf(a, n) -> ipiv
extern "C" int alg_zgetrf(double* a, size_t n, size_t* ipiv) {
  if (n == 0) return ALG_OK;
  if (a == nullptr || ipiv == nullptr) return ALG_INVALID_ARGUMENT;
  return alg::host_zlu(a, n, n, ipiv, nullptr);
}

// complex.rs:169 zgetrf_rect(a, nrows, ncols, ipiv)
extern "C" int alg_zgetrf_rect(double* a, size_t nrows, size_t ncols, size_t* ipiv) {
  if (nrows < ncols) return ALG_BAD_SHAPE;
  if (ncols == 0) return ALG_OK;
  if (a == nullptr || ipiv == nullptr) return ALG_INVALID_ARGUMENT;
  return alg::host_zlu(a, nrows, ncols, ipiv, nullptr);
}

// complex.rs:279 zgesv(a, b)
extern "C" int alg_zgesv(double* a, double* b, size_t n) {
  if (n == 0) return ALG_OK;
  if (a == nullptr || b == nullptr) return ALG_INVALID_ARGUMENT;
  std::vector<size_t> ipiv(n);
  return alg::host_zlu(a, n, n, ipiv.data(), b);
}
