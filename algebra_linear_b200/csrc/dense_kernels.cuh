// Kernels of the blocked right-looking LU with partial pivoting.
//
// Reference algorithm: lapack::dgetrf_with_pivots (src/lapack/mod.rs:112-163),
// an unblocked kij loop. The blocked schedule below gives every matrix entry
// exactly the same sequence of operations as that loop — the rank-1 terms
// `a_ij -= l_ik * u_kj` in increasing k, multipliers by true division, rows
// swapped before they are used — so with EXACT = true the factors are
// bit-identical to the reference; only the order in which *different* entries
// are processed changes.
//
// Layout: column-major, leading dimension lda, as the reference stores it.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math_constants.h>

#include "common.cuh"

namespace alg {
namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------
// K1: leaf panel LU on one thread-block cluster.
//
// Factors the n_rows x w leaf panel whose top-left entry is (c0, c0). The
// rows are split into C contiguous slabs, one per CTA of the cluster, each
// held in shared memory for the whole panel. Per column j:
//   1. every CTA finds its slab's candidate (first index of max |a_ij|; the
//      row-j entry counts a NaN as the maximum, other rows never pick a NaN —
//      the exact semantics of the strict '>' scan seeded with |a_jj|,
//      mod.rs:123-134) and publishes it with a copy of the row;
//   2. one cluster barrier;
//   3. every CTA reads the C candidates over DSMEM, takes the same winner,
//      swaps rows j and p inside the slabs that own them, and applies the
//      rank-1 update to its own rows (mod.rs:141-159).
// Publication buffers are double-buffered by column parity, so a column costs
// one barrier. Rows carry two labels through the swaps: the original row
// index within the current block-panel (for the deferred interchange of the
// other columns) and within this leaf (for the block-panel's other columns,
// which this kernel swaps itself at the end).
// ---------------------------------------------------------------------------
template <typename T>
struct PanelArgs {
  T* a;
  int lda;
  int n;           // rows of the matrix
  int c0;          // first row and column of the leaf
  int w;           // leaf width
  int kb0, kb1;    // columns of the enclosing block-panel
  int* ipiv;       // global interchanges (0-based global rows)
  int* lab;        // cumulative source labels of rows [kb0, n)
  int first_leaf;  // labels start as the identity
  DevStatus* status;
};

constexpr int kPanelThreads = 256;
constexpr int kPanelMaxW = 32;

template <typename T>
__host__ __device__ inline size_t panel_smem_bytes(int rows_per_cta, int w) {
  size_t b = 0;
  b += sizeof(T) * (size_t)rows_per_cta * (w + 1);   // tile
  b += sizeof(T) * 6 * (size_t)kPanelMaxW;            // pub_row[2], pub_diag[2], u_s, spare
  b += sizeof(int) * 2 * (size_t)rows_per_cta;        // cumulative + leaf labels
  b += 64 * sizeof(double);                           // keys, indices, labels, reductions
  b += 2 * kPanelMaxW * (kPanelMaxW + 2) * sizeof(T); // gathered rows for the side swap
  b += 4 * kPanelMaxW * sizeof(int);                  // side-swap bookkeeping
  return (b + 255) & ~size_t(255);
}

struct KeyIdx {
  double key;
  int idx;
};

__device__ __forceinline__ void keyidx_combine(double& k, int& i, double ok, int oi) {
  if (ok > k || (ok == k && oi < i)) {
    k = ok;
    i = oi;
  }
}

template <typename T, bool EXACT>
__global__ void __launch_bounds__(kPanelThreads, 1) panel_cluster_kernel(PanelArgs<T> p) {
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks();
  const int q = (int)cl.block_rank();
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int m = p.n - p.c0;
  const int R = (m + C - 1) / C;
  const int rb = q * R;
  const int re = min(m, rb + R);
  const int nr = max(0, re - rb);
  const int w = p.w;
  const int ld = w + 1;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);
  T* pub_row = tile + (size_t)R * ld;        // [2][kPanelMaxW]
  T* pub_diag = pub_row + 2 * kPanelMaxW;    // [2][kPanelMaxW]
  T* u_s = pub_diag + 2 * kPanelMaxW;        // [kPanelMaxW]
  int* lab_s = reinterpret_cast<int*>(u_s + 2 * kPanelMaxW);  // [R]
  int* loc_s = lab_s + R;                                      // [R]
  double* misc = reinterpret_cast<double*>(
      (reinterpret_cast<uintptr_t>(loc_s + R) + 15) & ~uintptr_t(15));
  double* pub_key = misc;                                  // [2]
  double* red_key = misc + 2;                              // [8]
  int* pub_idx = reinterpret_cast<int*>(misc + 10);        // [2]
  int* pub_rlab = pub_idx + 2;                             // [2][2] candidate row labels
  int* pub_dlab = pub_rlab + 4;                            // [2][2] diagonal row labels
  int* red_idx = pub_dlab + 4;                             // [8]
  int* win = red_idx + 8;                                  // [4]
  T* side_vals = reinterpret_cast<T*>(misc + 64);          // [2*kPanelMaxW][kPanelMaxW+2]
  int* side_rows = reinterpret_cast<int*>(side_vals + 2 * kPanelMaxW * (kPanelMaxW + 2));
  int* side_cnt = side_rows + 2 * kPanelMaxW;

  // ---- load the slab ------------------------------------------------------
  for (int idx = tid; idx < nr * w; idx += kPanelThreads) {
    const int r = idx % nr, c = idx / nr;
    tile[r * ld + c] = p.a[(size_t)(p.c0 + rb + r) + (size_t)(p.c0 + c) * p.lda];
  }
  for (int r = tid; r < nr; r += kPanelThreads) {
    const int g = p.c0 + rb + r;
    lab_s[r] = p.first_leaf ? g : p.lab[g];
    loc_s[r] = g;
  }
  __syncthreads();

  for (int j = 0; j < w; ++j) {
    const int par = j & 1;
    // ---- 1. slab candidate -------------------------------------------------
    double bk = -CUDART_INF;
    int bi = INT_MAX;
    for (int r = tid; r < nr; r += kPanelThreads) {
      const int gr = rb + r;
      if (gr < j) continue;
      const double v = fabs(static_cast<double>(tile[r * ld + j]));
      double key;
      if (gr == j) key = isnan(v) ? CUDART_INF : v;
      else key = isnan(v) ? -CUDART_INF : v;
      if (key > bk) { bk = key; bi = gr; }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ok = __shfl_down_sync(0xffffffffu, bk, off);
      const int oi = __shfl_down_sync(0xffffffffu, bi, off);
      keyidx_combine(bk, bi, ok, oi);
    }
    if (lane == 0) { red_key[warp] = bk; red_idx[warp] = bi; }
    __syncthreads();
    if (tid == 0) {
      for (int w2 = 1; w2 < kPanelThreads / 32; ++w2) keyidx_combine(bk, bi, red_key[w2], red_idx[w2]);
      pub_key[par] = bk;
      pub_idx[par] = bi;
      win[3] = bi;
      if (bi != INT_MAX) {
        pub_rlab[par * 2 + 0] = lab_s[bi - rb];
        pub_rlab[par * 2 + 1] = loc_s[bi - rb];
      }
      if (j >= rb && j < re) {
        pub_dlab[par * 2 + 0] = lab_s[j - rb];
        pub_dlab[par * 2 + 1] = loc_s[j - rb];
      }
    }
    __syncthreads();
    {
      const int mine = win[3];
      if (mine != INT_MAX && tid < w) pub_row[par * kPanelMaxW + tid] = tile[(mine - rb) * ld + tid];
      if (j >= rb && j < re && tid >= 64 && tid < 64 + w)
        pub_diag[par * kPanelMaxW + (tid - 64)] = tile[(j - rb) * ld + (tid - 64)];
    }
    // ---- 2. cluster barrier (release/acquire at cluster scope) -------------
    cl.sync();
    // ---- 3. winner, swap, update ------------------------------------------
    if (warp == 0) {
      double k = -CUDART_INF;
      int i = INT_MAX;
      if (lane < C) {
        k = *cl.map_shared_rank(&pub_key[par], lane);
        i = *cl.map_shared_rank(&pub_idx[par], lane);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ok = __shfl_down_sync(0xffffffffu, k, off);
        const int oi = __shfl_down_sync(0xffffffffu, i, off);
        keyidx_combine(k, i, ok, oi);
      }
      if (lane == 0) win[0] = i;
    }
    __syncthreads();
    const int pr = win[0];          // winning panel row (>= j)
    const int po = pr / R;          // its owner
    const int jo = j / R;           // owner of row j
    if (tid < w) u_s[tid] = *cl.map_shared_rank(&pub_row[par * kPanelMaxW + tid], po);
    if (q == po && pr != j && tid >= 64 && tid < 64 + w) {
      tile[(pr - rb) * ld + (tid - 64)] = *cl.map_shared_rank(&pub_diag[par * kPanelMaxW + (tid - 64)], jo);
    }
    if (tid == 128) {
      if (q == jo) {
        lab_s[j - rb] = *cl.map_shared_rank(&pub_rlab[par * 2 + 0], po);
        loc_s[j - rb] = *cl.map_shared_rank(&pub_rlab[par * 2 + 1], po);
      }
      if (q == po && pr != j) {
        lab_s[pr - rb] = *cl.map_shared_rank(&pub_dlab[par * 2 + 0], jo);
        loc_s[pr - rb] = *cl.map_shared_rank(&pub_dlab[par * 2 + 1], jo);
      }
    }
    __syncthreads();
    if (q == jo && tid < w) tile[(j - rb) * ld + tid] = u_s[tid];
    const T d = u_s[j];
    if (q == 0 && tid == 0) {
      p.ipiv[p.c0 + j] = p.c0 + pr;
      if (fabs(static_cast<double>(d)) <= 0.0) atomicMin(&p.status->singular_col, p.c0 + j);
    }
    __syncthreads();
    // multipliers (true division, mod.rs:154)
    for (int r = tid; r < nr; r += kPanelThreads) {
      if (rb + r > j) tile[r * ld + j] = div_rn(tile[r * ld + j], d);
    }
    __syncthreads();
    const int wr = w - j - 1;
    if (wr > 0) {
      const int r_first = max(0, j + 1 - rb);
      const int cnt = (nr - r_first) * wr;
      for (int idx = tid; idx < cnt; idx += kPanelThreads) {
        const int r = r_first + idx / wr;
        const int c = j + 1 + idx % wr;
        tile[r * ld + c] = msub<EXACT>(tile[r * ld + c], tile[r * ld + j], u_s[c]);
      }
    }
    __syncthreads();
  }

  // ---- swap the block-panel's other columns by this leaf's interchanges -----
  // Rows whose leaf label moved receive the old content of the labelled row.
  // All reads happen before the cluster barrier, all writes after it.
  if (tid == 0) side_cnt[0] = 0;
  __syncthreads();
  for (int r = tid; r < nr; r += kPanelThreads) {
    if (loc_s[r] != p.c0 + rb + r) {
      const int s = atomicAdd(side_cnt, 1);
      if (s < 2 * kPanelMaxW) side_rows[s] = r;
    }
  }
  __syncthreads();
  const int n_side = min(side_cnt[0], 2 * kPanelMaxW);
  const int side_w = (p.kb1 - p.kb0) - w;  // other columns of the block-panel
  const int sw = min(side_w, kPanelMaxW + 2);
  // other columns are processed in chunks of (kPanelMaxW + 2) columns
  for (int cbase = 0; cbase < side_w; cbase += sw) {
    const int ncol = min(sw, side_w - cbase);
    for (int idx = tid; idx < n_side * ncol; idx += kPanelThreads) {
      const int s = idx / ncol, cc = idx % ncol;
      int col = p.kb0 + cbase + cc;
      if (col >= p.c0) col += w;  // skip the leaf's own columns
      const int src = loc_s[side_rows[s]];
      side_vals[s * (kPanelMaxW + 2) + cc] = p.a[(size_t)src + (size_t)col * p.lda];
    }
    cl.sync();
    for (int idx = tid; idx < n_side * ncol; idx += kPanelThreads) {
      const int s = idx / ncol, cc = idx % ncol;
      int col = p.kb0 + cbase + cc;
      if (col >= p.c0) col += w;
      const int dst = p.c0 + rb + side_rows[s];
      p.a[(size_t)dst + (size_t)col * p.lda] = side_vals[s * (kPanelMaxW + 2) + cc];
    }
    cl.sync();
  }
  if (side_w <= 0) cl.sync();  // no DSMEM reader may outlive an owner

  // ---- write the slab back ------------------------------------------------
  for (int idx = tid; idx < nr * w; idx += kPanelThreads) {
    const int r = idx % nr, c = idx / nr;
    p.a[(size_t)(p.c0 + rb + r) + (size_t)(p.c0 + c) * p.lda] = tile[r * ld + c];
  }
  for (int r = tid; r < nr; r += kPanelThreads) p.lab[p.c0 + rb + r] = lab_s[r];
}

// ---------------------------------------------------------------------------
// K2: deferred row interchange of the columns outside a block-panel.
// Row r (r in [k0, n)) of every such column takes the old content of row
// lab[r]; the rows that move are compacted once per CTA, and one warp owns a
// column (all loads of a column precede its stores).
// The net permutation `perm` is carried the same way (CTA 0, one extra pass).
// ---------------------------------------------------------------------------
constexpr int kSwapThreads = 256;
constexpr int kSwapMaxMoves = 512;

template <typename T>
__global__ void __launch_bounds__(kSwapThreads) laswp_outside_kernel(
    T* a, int lda, int n, int ncols, int k0, int kb, const int* lab, int* perm, int* perm_tmp) {
  __shared__ int mv_dst[kSwapMaxMoves];
  __shared__ int mv_src[kSwapMaxMoves];
  __shared__ int mv_cnt;
  if (threadIdx.x == 0) mv_cnt = 0;
  __syncthreads();
  for (int r = k0 + threadIdx.x; r < n; r += kSwapThreads) {
    const int s = lab[r];
    if (s != r) {
      const int slot = atomicAdd(&mv_cnt, 1);
      if (slot < kSwapMaxMoves) { mv_dst[slot] = r; mv_src[slot] = s; }
    }
  }
  __syncthreads();
  const int moves = min(mv_cnt, kSwapMaxMoves);
  const int lane = threadIdx.x & 31;
  const int warps_total = gridDim.x * (kSwapThreads / 32);
  const int gwarp = blockIdx.x * (kSwapThreads / 32) + (threadIdx.x >> 5);
  const int n_out = k0 + (ncols - k0 - kb);  // columns [0,k0) and [k0+kb, ncols)
  constexpr int kPer = kSwapMaxMoves / 32;
  for (int cidx = gwarp; cidx < n_out; cidx += warps_total) {
    const int col = cidx < k0 ? cidx : cidx + kb;
    T* colp = a + (size_t)col * lda;
    T vals[kPer];
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const int s = lane + 32 * t;
      if (s < moves) vals[t] = colp[mv_src[s]];
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const int s = lane + 32 * t;
      if (s < moves) colp[mv_dst[s]] = vals[t];
    }
  }
  if (perm != nullptr && blockIdx.x == 0) {
    // perm_new[r] = perm_old[lab[r]] over the moved rows
    for (int s = threadIdx.x; s < moves; s += kSwapThreads) perm_tmp[s] = perm[mv_src[s]];
    __syncthreads();
    for (int s = threadIdx.x; s < moves; s += kSwapThreads) perm[mv_dst[s]] = perm_tmp[s];
  }
}

__global__ void iota_kernel(int* v, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// ---------------------------------------------------------------------------
// K3: U12 = L11^{-1} A12 for rows [r0, r0+kb) of columns [cb, ce), unit lower
// L11 = a[r0:r0+kb, r0:r0+kb]. Entry (i, c) receives `-= l_ik * u_kc` for
// k = r0 .. i-1 in that order, the reference's order for those entries.
// One CTA owns 32 columns; a step k updates every row below k in parallel.
// ---------------------------------------------------------------------------
constexpr int kTrsmThreads = 256;
constexpr int kTrsmCols = 32;

template <typename T, bool EXACT>
__global__ void __launch_bounds__(kTrsmThreads) trsm_lower_unit_kernel(
    T* a, int lda, int r0, int kb, int cb, int ce) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* L = reinterpret_cast<T*>(smem_raw);     // kb x kb, column-major
  T* X = L + (size_t)kb * kb;                 // kb x kTrsmCols, row-major
  const int c_first = cb + blockIdx.x * kTrsmCols;
  const int ncol = min(kTrsmCols, ce - c_first);
  if (ncol <= 0) return;
  for (int idx = threadIdx.x; idx < kb * kb; idx += kTrsmThreads) {
    const int i = idx % kb, k = idx / kb;
    L[idx] = a[(size_t)(r0 + i) + (size_t)(r0 + k) * lda];
  }
  for (int idx = threadIdx.x; idx < kb * kTrsmCols; idx += kTrsmThreads) {
    const int i = idx % kb, c = idx / kb;
    X[i * kTrsmCols + c] = c < ncol ? a[(size_t)(r0 + i) + (size_t)(c_first + c) * lda] : T(0);
  }
  __syncthreads();
  const int c = threadIdx.x % kTrsmCols;
  const int g = threadIdx.x / kTrsmCols;
  constexpr int G = kTrsmThreads / kTrsmCols;
  for (int k = 0; k + 1 < kb; ++k) {
    const T u = X[k * kTrsmCols + c];
    for (int i = k + 1 + g; i < kb; i += G) {
      X[i * kTrsmCols + c] = msub<EXACT>(X[i * kTrsmCols + c], L[i + (size_t)k * kb], u);
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < kb * kTrsmCols; idx += kTrsmThreads) {
    const int i = idx % kb, cc = idx / kb;
    if (cc < ncol) a[(size_t)(r0 + i) + (size_t)(c_first + cc) * lda] = X[i * kTrsmCols + cc];
  }
}

// ---------------------------------------------------------------------------
// K4 (CUDA-core form): C -= A * B with C M x N, A M x K, B K x N, all
// column-major. Each thread owns an 8 x 8 block of C in registers, loads it
// once, applies the K terms in increasing k (EXACT: rounded product then
// rounded difference, the reference's per-entry sequence), and stores it once.
// 128 x 128 CTA tile, K staged through shared memory 8 at a time with
// register double buffering. Out-of-range A rows / B columns / k are zero,
// which leaves every in-range entry unchanged bit for bit (x - 0*0 = x).
// ---------------------------------------------------------------------------
constexpr int kGemmBM = 128, kGemmBN = 128, kGemmBK = 8, kGemmThreads = 256;

template <typename T, bool EXACT>
__global__ void __launch_bounds__(kGemmThreads, 1) gemm_sub_kernel(
    int M, int N, int K, const T* __restrict__ A, int lda, const T* __restrict__ B, int ldb,
    T* __restrict__ Cm, int ldc) {
  __shared__ __align__(16) T As[2][kGemmBK][kGemmBM];
  __shared__ __align__(16) T Bs[2][kGemmBK][kGemmBN + 2];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * kGemmBN;

  T acc[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int mi = m0 + (r >> 2) * 64 + tx * 4 + (r & 3);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int nj = n0 + (c >> 2) * 64 + ty * 4 + (c & 3);
      acc[r][c] = (mi < M && nj < N) ? Cm[(size_t)mi + (size_t)nj * ldc] : T(0);
    }
  }

  // loader mapping: A chunk is kGemmBK x 128 (k-major in smem): 4 per thread
  // B chunk is kGemmBK x 128: 4 per thread
  T ra[4], rb[4];
  auto load_chunk = [&](int k0) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int idx = tid + t * kGemmThreads;
      const int mm = idx & 127, kk = idx >> 7;
      const int gm = m0 + mm, gk = k0 + kk;
      ra[t] = (gm < M && gk < K) ? A[(size_t)gm + (size_t)gk * lda] : T(0);
      const int bk = idx & 7, bn = idx >> 3;
      const int gn = n0 + bn, gk2 = k0 + bk;
      rb[t] = (gn < N && gk2 < K) ? B[(size_t)gk2 + (size_t)gn * ldb] : T(0);
    }
  };
  auto store_chunk = [&](int buf) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int idx = tid + t * kGemmThreads;
      As[buf][idx >> 7][idx & 127] = ra[t];
      Bs[buf][idx & 7][idx >> 3] = rb[t];
    }
  };

  const int nchunks = (K + kGemmBK - 1) / kGemmBK;
  if (nchunks > 0) {
    load_chunk(0);
    store_chunk(0);
  }
  __syncthreads();
  for (int ch = 0; ch < nchunks; ++ch) {
    const int buf = ch & 1;
    if (ch + 1 < nchunks) load_chunk((ch + 1) * kGemmBK);
#pragma unroll
    for (int kk = 0; kk < kGemmBK; ++kk) {
      T af[8], bf[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) af[r] = As[buf][kk][(r >> 2) * 64 + tx * 4 + (r & 3)];
#pragma unroll
      for (int c = 0; c < 8; ++c) bf[c] = Bs[buf][kk][(c >> 2) * 64 + ty * 4 + (c & 3)];
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = msub<EXACT>(acc[r][c], af[r], bf[c]);
    }
    if (ch + 1 < nchunks) store_chunk(buf ^ 1);
    __syncthreads();
  }

#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int mi = m0 + (r >> 2) * 64 + tx * 4 + (r & 3);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int nj = n0 + (c >> 2) * 64 + ty * 4 + (c & 3);
      if (mi < M && nj < N) Cm[(size_t)mi + (size_t)nj * ldc] = acc[r][c];
    }
  }
}

// ---------------------------------------------------------------------------
// K5: triangular solves with the packed factors (getrs), blocked by kSolveB
// rows. The forward sweep gives x_i the terms l_ij x_j in increasing j with
// rounded product and difference — the reference's row-dot sequence
// (mod.rs:341-347) — so it is bit-identical; the backward sweep applies the
// terms of each block as soon as the block is solved (a different order from
// the reference's row-dot, mod.rs:348-353, which no parallel schedule can keep).
//
// Launch b of a sweep updates every remaining row with block b's solved
// unknowns; CTA 0 owns the rows of the next block and, after updating them,
// solves that block's triangle so the next launch can use it.
// ---------------------------------------------------------------------------
constexpr int kSolveB = 64;
constexpr int kSolveThreads = 256;

// x = b[perm] for every right-hand side, then solve block 0's triangle.
template <typename T>
__global__ void __launch_bounds__(kSolveThreads) solve_gather_kernel(
    const T* __restrict__ lu, int lda, int n, const int* __restrict__ perm,
    const T* __restrict__ b, int ldb, T* __restrict__ x, int ldx) {
  const int rhs = blockIdx.y;
  const T* bc = b + (size_t)rhs * ldb;
  T* xc = x + (size_t)rhs * ldx;
  for (int i = blockIdx.x * kSolveThreads + threadIdx.x; i < n; i += gridDim.x * kSolveThreads) {
    xc[i] = bc[perm[i]];
  }
}

template <typename T, bool EXACT>
__device__ void solve_diag_block_lower(const T* lu, int lda, T* xc, int j0, int bs, T* xs) {
  // unit lower triangle of rows/cols [j0, j0+bs); xs is shared scratch [bs]
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xs[i] = xc[j0 + i];
  __syncthreads();
  for (int k = 0; k + 1 < bs; ++k) {
    const T u = xs[k];
    for (int i = k + 1 + threadIdx.x; i < bs; i += blockDim.x)
      xs[i] = msub<EXACT>(xs[i], lu[(size_t)(j0 + i) + (size_t)(j0 + k) * lda], u);
    __syncthreads();
  }
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xc[j0 + i] = xs[i];
}

template <typename T, bool EXACT>
__device__ void solve_diag_block_upper(const T* lu, int lda, T* xc, int j0, int bs, T* xs) {
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xs[i] = xc[j0 + i];
  __syncthreads();
  for (int k = bs - 1; k >= 0; --k) {
    if (threadIdx.x == 0) xs[k] = div_rn(xs[k], lu[(size_t)(j0 + k) + (size_t)(j0 + k) * lda]);
    __syncthreads();
    const T u = xs[k];
    for (int i = threadIdx.x; i < k; i += blockDim.x)
      xs[i] = msub<EXACT>(xs[i], lu[(size_t)(j0 + i) + (size_t)(j0 + k) * lda], u);
    __syncthreads();
  }
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xc[j0 + i] = xs[i];
}

// Forward: rows [j0+bs, n) take block [j0, j0+bs)'s terms. CTA 0 owns the next
// block's rows and then solves its triangle. j0 = -bs means "only solve block 0".
template <typename T, bool EXACT>
__global__ void __launch_bounds__(kSolveThreads) solve_fwd_kernel(
    const T* __restrict__ lu, int lda, int n, T* __restrict__ x, int ldx, int j0, int bs) {
  __shared__ T xb[kSolveB];
  __shared__ T xs[kSolveB];
  const int rhs = blockIdx.y;
  T* xc = x + (size_t)rhs * ldx;
  const int j1 = j0 + bs;                // first row below the block
  const int nb1 = min(kSolveB, n - j1);  // rows in the next block
  if (j0 >= 0) {
    for (int k = threadIdx.x; k < bs; k += kSolveThreads) xb[k] = xc[j0 + k];
    __syncthreads();
    int i_begin, i_end;
    if (blockIdx.x == 0) { i_begin = j1; i_end = j1 + nb1; }
    else {
      i_begin = j1 + nb1 + (blockIdx.x - 1) * kSolveThreads;
      i_end = min(n, i_begin + kSolveThreads);
    }
    const int i = i_begin + threadIdx.x;
    if (i < i_end) {
      T acc = xc[i];
      for (int k = 0; k < bs; ++k) acc = msub<EXACT>(acc, lu[(size_t)i + (size_t)(j0 + k) * lda], xb[k]);
      xc[i] = acc;
    }
  }
  if (blockIdx.x == 0 && nb1 > 0) {
    __syncthreads();
    solve_diag_block_lower<T, EXACT>(lu, lda, xc, j1, nb1, xs);
  }
}

// Backward: rows [0, j0) take block [j0, j0+bs)'s terms. CTA 0 owns the
// previous block's rows [j0-bp, j0) and then solves its triangle.
// j0 = n means "only solve the last block" (bs is then that block's size).
template <typename T, bool EXACT>
__global__ void __launch_bounds__(kSolveThreads) solve_bwd_kernel(
    const T* __restrict__ lu, int lda, int n, T* __restrict__ x, int ldx, int j0, int bs,
    int bp) {
  __shared__ T xb[kSolveB];
  __shared__ T xs[kSolveB];
  const int rhs = blockIdx.y;
  T* xc = x + (size_t)rhs * ldx;
  const int jp = j0 - bp;  // first row of the previous block
  if (j0 < n) {
    for (int k = threadIdx.x; k < bs; k += kSolveThreads) xb[k] = xc[j0 + k];
    __syncthreads();
    int i_begin, i_end;
    if (blockIdx.x == 0) { i_begin = jp; i_end = j0; }
    else {
      i_begin = (blockIdx.x - 1) * kSolveThreads;
      i_end = min(jp, i_begin + kSolveThreads);
    }
    const int i = i_begin + threadIdx.x;
    if (i < i_end) {
      T acc = xc[i];
      for (int k = 0; k < bs; ++k) acc = msub<EXACT>(acc, lu[(size_t)i + (size_t)(j0 + k) * lda], xb[k]);
      xc[i] = acc;
    }
  }
  if (blockIdx.x == 0 && bp > 0) {
    __syncthreads();
    solve_diag_block_upper<T, EXACT>(lu, lda, xc, jp, bp, xs);
  }
}

}  // namespace alg
