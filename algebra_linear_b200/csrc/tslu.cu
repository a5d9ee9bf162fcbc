// Tournament pivoting for the leaf panels of the low-precision LU (the
// mixed-precision form only; the FP64 drop-in keeps partial pivoting).
//
// Partial pivoting needs one reduction over all rows per column, and that
// chain is the critical path of the look-ahead LU. Tournament pivoting
// (TSLU: Grigori, Demmel, Xiang, "CALU: a communication optimal LU
// factorization algorithm", SIAM J. Matrix Anal. Appl. 32, 2011) chooses the
// panel's w pivot rows first and factors afterwards:
//   1. select: each CTA runs partial-pivoting LU on its own chunk of 256 rows
//      (one row per thread, the chunk in shared memory) and proposes the w
//      rows it pivoted on, with their original values;
//   2. merge: a CTA runs the same LU on the up to 8 x w rows its 8 children
//      proposed (original values), level after level, until one CTA holds
//      the panel's w pivots in order and, as its LU's leading rows,
//      L11 \ U11 of the winners;
//   3. apply: the interchanges (LAPACK sequential form, as the partial-
//      pivoting panel records them) move the winners to the top, every other
//      row gets its multipliers l = a U11^-1, the labels of the moved rows
//      and the block panel's other columns follow the interchanges, and the
//      top rows of the block panel's trailing columns become U12.
// The factorization differs from partial pivoting's (other pivots); the
// mixed form's refinement in FP64 then brings the solution to the FP64
// backward error, which is its contract. In the single-launch form every CTA
// waits (bounded) for the root's release; the multi-launch form has no waits.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstddef>
#include <cstdlib>

#include "dense.cuh"

namespace alg {
namespace {

constexpr int kW = 32;            // widest leaf
constexpr int kRows = 256;        // rows per CTA (one per thread)
constexpr int kFan = 8;           // children merged by one CTA (8 x 32 = 256 rows)
constexpr int kMaxGroups = 1024;  // CTAs of the first level: up to 262 144 panel rows
constexpr int kMaxMoves = 2 * kW;

constexpr int kMaxLevels = 4;        // merge levels: 1024 -> 128 -> 16 -> 2 -> 1
constexpr int kFusedMaxGroups = 32;  // panels of up to 8192 rows take the single launch

struct TsluScratch {
  // single-launch form: arrivals per parent and level (the last arrival merges
  // and resets the count) and the root's release flag (the launch's epoch)
  int counter[kMaxLevels][kMaxGroups / kFan];
  unsigned ready;
  int cand_rows[2][kMaxGroups][kW];        // proposals of each CTA of a level, in step order
  int cand_cnt[2][kMaxGroups];
  float cand_vals[2][kMaxGroups][kW * kW];  // their original values, [col][k]
  int win[kW];                              // the panel's pivot rows in order
  int nmoves;
  int move_pos[kMaxMoves];                  // a position whose row changed
  int move_src[kMaxMoves];                  // the position that row came from (at the leaf's start)
  int move_lab[kMaxMoves];                  // its new label
  float top_lu[kW * kW];                    // L11 \ U11 of the winners ([col][k], stride kW)
  float top_orig[kW * kW];                  // original values of the rows at the top positions
};

constexpr int kWarps = kRows / 32;

// Partial-pivoting LU of the first w columns of nr <= 256 rows, row t in
// thread t's registers v[], rows left in place, blocked by kSub columns:
// inside a sub-block each column costs one barrier — every warp publishes its
// best candidate (key, index and the row's kSub sub-block entries) in a
// mailbox double-buffered by column parity and every warp reduces the
// mailboxes itself — and only the sub-block's columns are updated; after the
// sub-block its pivot rows' entries right of it become U12 by a forward
// substitution in shared memory and every other row takes the rank-kSub
// update at once. Returns the step at which this thread's row was chosen
// (-1: not chosen); the chosen row's v[] then holds its multipliers (columns
// before its step) and its U entries (from its step on). zero_col: first
// column whose pivot was zero.
constexpr int kSub = 8;

// Pivot keys as ordered integers: |v|'s bit pattern + 1 (bit patterns of
// non-negative floats order like the values), 0 for a row that is out of the
// running, so one warp-wide integer max (redux) and a ballot for its first
// lane find the largest |v| and, among equals, the lowest row.
__device__ __forceinline__ unsigned pivot_key(float v, bool live) { return live ? __float_as_uint(fabsf(v)) + 1u : 0u; }

struct GeppShared {
  float row[2][kWarps][kSub];  // mailboxes: each warp's best row, sub-block entries
  unsigned key[2][kWarps];
  int idx[2][kWarps];
  float prow[kSub][kW];        // the sub-block's pivot rows (then U12 right of the sub-block)
};

template <int W>
__device__ __forceinline__ int block_gepp(float (&v)[W], int nr, int w, GeppShared& sh, int* zero_col) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  int chosen = -1;
  bool done = false;
  // both loops unroll completely, so every column index below is a
  // compile-time constant (the row stays in registers, no selects)
#pragma unroll
  for (int jb = 0; jb < W; jb += kSub) {
    if (done || jb >= w) break;
    const int nsub = min(kSub, w - jb);
#pragma unroll
    for (int jj = 0; jj < kSub; ++jj) {
      if (jj >= nsub) break;
      const int j = jb + jj, par = j & 1;
      const float vj = v[j];
      const unsigned key = pivot_key(vj, t < nr && chosen < 0);
      const unsigned wmax = __reduce_max_sync(0xffffffffu, key);
      if (wmax == 0u) {
        if (lane == 0) {
          sh.key[par][warp] = 0u;
          sh.idx[par][warp] = INT_MAX;
        }
      } else if (lane == __ffs(__ballot_sync(0xffffffffu, key == wmax)) - 1) {
        sh.key[par][warp] = wmax;
        sh.idx[par][warp] = t;
#pragma unroll
        for (int cc = jj; cc < kSub; ++cc) sh.row[par][warp][cc] = v[jb + cc];
      }
      __syncthreads();
      // every warp reduces the mailboxes itself (warps in row order, so the
      // first warp holding the maximum holds its lowest row)
      const unsigned mk = lane < kWarps ? sh.key[par][lane] : 0u;
      const unsigned bmax = __reduce_max_sync(0xffffffffu, mk);
      if (bmax == 0u) {  // fewer rows than columns: every row is chosen
        done = true;
        break;
      }
      const int bw = __ffs(__ballot_sync(0xffffffffu, mk == bmax)) - 1;
      const int bi = sh.idx[par][bw];
      if (t == bi) chosen = j;
      const float* pr = sh.row[par][bw];
      const float pv = pr[jj];
      if (pv == 0.0f && t == 0 && *zero_col < 0) *zero_col = j;
      if (t < nr && chosen < 0) {
        const float l = pv != 0.0f ? vj / pv : 0.0f;
        v[j] = l;
#pragma unroll
        for (int cc = jj + 1; cc < kSub; ++cc) v[jb + cc] = fmaf(-l, pr[cc], v[jb + cc]);
      }
    }
    if (jb + kSub >= W) break;  // no columns right of the last sub-block
    // the sub-block's pivot rows, then U12 = L11^-1 (their entries right of it)
    const bool mine = chosen >= jb && chosen < jb + kSub;
    if (mine) {
#pragma unroll
      for (int c = jb; c < W; ++c) sh.prow[chosen - jb][c] = v[c];
    }
    __syncthreads();
    if (t < W - jb - kSub) {
      const int c = jb + kSub + t;
#pragma unroll
      for (int i = 1; i < kSub; ++i) {
        if (i < nsub) {
          float u = sh.prow[i][c];
#pragma unroll
          for (int k = 0; k < i; ++k) u = fmaf(-sh.prow[i][jb + k], sh.prow[k][c], u);
          sh.prow[i][c] = u;
        }
      }
    }
    __syncthreads();
    if (mine) {
#pragma unroll
      for (int c = jb + kSub; c < W; ++c) v[c] = sh.prow[chosen - jb][c];
    } else if (t < nr && chosen < 0) {
#pragma unroll
      for (int k = 0; k < kSub; ++k) {
        const float l = k < nsub ? v[jb + k] : 0.0f;
#pragma unroll
        for (int c = jb + kSub; c < W; ++c) v[c] = fmaf(-l, sh.prow[k][c], v[c]);
      }
    }
  }
  __syncthreads();
  return chosen;
}

// One level of the tournament. Level 0 (src < 0) reads rows [c0 + 256 g, ...)
// of the panel; later levels read the proposals of children [8 g, 8 g + 8)
// from scratch slot src. Writes this CTA's proposals to slot dst; the single
// CTA of the last level (root) also writes the winners, L11 \ U11, the rows
// at the top before anything moves, ipiv and the list of moved rows.
struct LevelIn {
  const float* a;
  int lda, n, c0, w;
  int* ipiv;
  const int* lab;
  int first_leaf;
  DevStatus* status;
};

// Proposals written by other CTAs are read through L2 (__ldcg): in the
// single-launch form they were written during this launch by other SMs.
template <int W>
__device__ void level_body(const LevelIn& in, int g, int src, int nchild, int dst, bool root, TsluScratch* ws) {
  __shared__ GeppShared box;
  __shared__ int zero_col;
  __shared__ int coff[kFan + 1];
  const float* a = in.a;
  const int lda = in.lda, n = in.n, c0 = in.c0, w = in.w, first_leaf = in.first_leaf;
  int* ipiv = in.ipiv;
  const int* lab = in.lab;
  const int t = threadIdx.x;
  float o[W];  // this row's original values
#pragma unroll
  for (int c = 0; c < W; ++c) o[c] = 0.0f;
  int row = -1, nr = 0;
  if (src < 0) {
    const int r0 = c0 + g * kRows;
    nr = max(0, min(n, r0 + kRows) - r0);
    if (t < nr) {
      row = r0 + t;
#pragma unroll
      for (int c = 0; c < W; ++c) o[c] = c < w ? a[(size_t)row + (size_t)(c0 + c) * lda] : 0.0f;
    }
  } else {
    if (t == 0) {
      int acc = 0;
      for (int k = 0; k < kFan; ++k) {
        coff[k] = acc;
        const int ch = g * kFan + k;
        acc += ch < nchild ? __ldcg(&ws->cand_cnt[src][ch]) : 0;
      }
      coff[kFan] = acc;
    }
    __syncthreads();
    nr = coff[kFan];
    if (t < nr) {
      int k = 0;
      while (k + 1 < kFan && coff[k + 1] <= t) ++k;
      const int ch = g * kFan + k, q = t - coff[k];
      row = __ldcg(&ws->cand_rows[src][ch][q]);
#pragma unroll
      for (int c = 0; c < W; ++c) o[c] = c < w ? __ldcg(&ws->cand_vals[src][ch][c * kW + q]) : 0.0f;
    }
  }
  float v[W];
#pragma unroll
  for (int c = 0; c < W; ++c) v[c] = o[c];

  if (t == 0) zero_col = -1;
  __syncthreads();
  const int step = block_gepp<W>(v, nr, w, box, &zero_col);
  const int cnt = min(w, nr);
  if (!root) {
    if (step >= 0) {
      ws->cand_rows[dst][g][step] = row;
#pragma unroll
      for (int c = 0; c < W; ++c)
        if (c < w) ws->cand_vals[dst][g][c * kW + step] = o[c];
    }
    if (t == 0) ws->cand_cnt[dst][g] = cnt;
    __syncthreads();  // the block's shared state is reused by the next level
    return;
  }
  // ---- root: winners, L11 \ U11, the top rows' original values ------------
  __shared__ int win_s[kW];  // the winners, for the serial steps below (shared, not global, latency)
  if (step >= 0) {
    ws->win[step] = row;
    win_s[step] = row;
#pragma unroll
    for (int c = 0; c < W; ++c)
      if (c < w) ws->top_lu[c * kW + step] = v[c];
  }
  {  // every load first, then the stores (kept in flight together)
    constexpr int kPer = (kW * kW + kRows - 1) / kRows;
    float tv[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = t + u * kRows;
      tv[u] = e < w * w ? a[(size_t)(c0 + e % w) + (size_t)(c0 + e / w) * lda] : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = t + u * kRows;
      if (e < w * w) ws->top_orig[(e / w) * kW + e % w] = tv[u];
    }
  }
  if (t == 0 && zero_col >= 0) atomicMin(&in.status->singular_col, c0 + zero_col);
  __syncthreads();
  // ---- LAPACK sequential interchanges bringing winner j to position c0 + j.
  // Only two kinds of position are ever touched: the top positions c0 + i
  // (i < w) and the original positions of the winners from below the top. A
  // winner from below sits at its original position until its own step, and
  // a row that started in the top moves only by the steps, so one lane keeps
  // the occupant of every touched position and the location of every
  // top-started row in shared memory and runs the w steps in O(1) each.
  if (t < 32) {
    __shared__ int occ_top[kW];  // row at top position c0 + i
    __shared__ int occ_out[kW];  // row at the original position of winner j (a winner from below)
    __shared__ int loc_top[kW];  // where the row that started at c0 + i is: i' < kW top, kW + j outside
    const int lane = t;
    __shared__ int lab_top[kW], lab_win[kW];  // labels of the top rows and of the winners
    if (lane < w) {
      occ_top[lane] = c0 + lane;
      loc_top[lane] = lane;
      occ_out[lane] = win_s[lane];
      // issued before the serial steps, so their latency overlaps them
      if (!first_leaf) {
        lab_top[lane] = lab[c0 + lane];
        lab_win[lane] = lab[win_s[lane]];
      }
    }
    __syncwarp();
    if (lane == 0) {
      for (int j = 0; j < w; ++j) {
        const int gr = win_s[j];
        const bool g_top = gr < c0 + w;  // candidates are rows >= c0
        const int cur = g_top ? loc_top[gr - c0] : kW + j;
        const int pr = cur < kW ? c0 + cur : win_s[cur - kW];
        ipiv[c0 + j] = pr;
        const int h = occ_top[j];  // the row at c0 + j goes where gr was
        occ_top[j] = gr;
        if (g_top) loc_top[gr - c0] = j;
        if (cur < kW) {
          if (cur != j) occ_top[cur] = h;
        } else {
          occ_out[cur - kW] = h;
        }
        if (h < c0 + w && h != gr) loc_top[h - c0] = cur;
      }
    }
    __syncwarp();
    // the moved rows: top positions and the below-top winners' positions
    // whose occupant changed (a set; the apply step's order does not
    // matter), one lane per position, slots by a ballot prefix count
    // the label of a moved row (a top row or a winner)
    auto label_of = [&](int row) {
      if (first_leaf) return row;
      if (row < c0 + w) return lab_top[row - c0];
      int k = 0;
      while (k + 1 < w && win_s[k] != row) ++k;
      return lab_win[k];
    };
    const unsigned below = (1u << lane) - 1u;
    const bool mt = lane < w && occ_top[lane] != c0 + lane;
    const unsigned bt = __ballot_sync(0xffffffffu, mt);
    const int nt = __popc(bt);
    if (mt) {
      const int slot = __popc(bt & below), src = occ_top[lane];
      ws->move_pos[slot] = c0 + lane;
      ws->move_src[slot] = src;
      ws->move_lab[slot] = label_of(src);
    }
    const int gw = lane < w ? win_s[lane] : 0;
    const bool mo = lane < w && gw >= c0 + w && occ_out[lane] != gw;
    const unsigned bo = __ballot_sync(0xffffffffu, mo);
    if (mo) {
      const int slot = nt + __popc(bo & below), src = occ_out[lane];
      ws->move_pos[slot] = gw;
      ws->move_src[slot] = src;
      ws->move_lab[slot] = label_of(src);
    }
    if (lane == 0) ws->nmoves = nt + __popc(bo);
  }
  __syncthreads();
}

// One level of the multi-launch form.
template <int W>
__global__ void __launch_bounds__(kRows, 1) tslu_level_kernel(LevelIn in, int src, int nchild, int dst, int root,
                                                           TsluScratch* ws) {
  level_body<W>(in, blockIdx.x, src, nchild, dst, root != 0, ws);
}

// 3. Blocks [0, side_blocks): the block panel's other columns follow the
//    interchanges (all reads of a column's moved entries before its writes).
//    The rest: rows below the top get l = a U11^-1 (a from the row that ends
//    up there), the top block and the labels.
constexpr int kSideCols = 8;

// CTA `cta` of `ncta`: the first side_blocks CTAs permute the block panel's
// other columns and turn the top rows of its trailing columns into U12; rows
// are spread over the CTAs from row_cta0 on.
template <int W>
__device__ void apply_body(float* a, int lda, int n, int c0, int w, int kb0, int kb1, int* lab, int first_leaf,
                           int cta, int ncta, int side_blocks, int row_cta0, const TsluScratch* ws) {
  __shared__ float U[kW * kW];
  __shared__ int mpos[kMaxMoves], msrc[kMaxMoves], mlab[kMaxMoves];
  __shared__ int nm_s;
  if (threadIdx.x == 0) nm_s = __ldcg(&ws->nmoves);
  for (int t = threadIdx.x; t < kMaxMoves; t += blockDim.x) {
    mpos[t] = __ldcg(&ws->move_pos[t]);
    msrc[t] = __ldcg(&ws->move_src[t]);
    mlab[t] = __ldcg(&ws->move_lab[t]);
  }
  const int side = (kb1 - kb0) - w;
  __syncthreads();
  if (cta < side_blocks) {
    const int nm = nm_s;
    // kSideCols columns x the moves: read all, then write all
    float v[(kSideCols * kMaxMoves + 255) / 256];
#pragma unroll
    for (int u = 0; u < (kSideCols * kMaxMoves + 255) / 256; ++u) {
      const int e = threadIdx.x + u * 256;
      const int cl = e / kMaxMoves, mv = e % kMaxMoves;
      const int cidx = cta * kSideCols + cl;
      v[u] = 0.0f;
      if (cl < kSideCols && cidx < side && mv < nm) {
        int col = kb0 + cidx;
        if (col >= c0) col += w;
        v[u] = a[(size_t)msrc[mv] + (size_t)col * lda];
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < (kSideCols * kMaxMoves + 255) / 256; ++u) {
      const int e = threadIdx.x + u * 256;
      const int cl = e / kMaxMoves, mv = e % kMaxMoves;
      const int cidx = cta * kSideCols + cl;
      if (cl < kSideCols && cidx < side && mv < nm) {
        int col = kb0 + cidx;
        if (col >= c0) col += w;
        a[(size_t)mpos[mv] + (size_t)col * lda] = v[u];
      }
    }
    // U12 = L11^-1 A12 on this CTA's columns right of the leaf (the block
    // panel's trailing columns), from the permuted top rows this CTA just
    // wrote: one warp per column, top row i in lane i, step k's value
    // broadcast by a shuffle; each entry takes its terms in increasing k with
    // one FMA each, the arithmetic of the separate FP32 TRSM kernel
    __syncthreads();
    const int lane = threadIdx.x & 31, cl = threadIdx.x >> 5;
    const int cidx = cta * kSideCols + cl;
    int col = kb0 + cidx;
    if (col >= c0) col += w;
    if (cl < kSideCols && cidx < side && col >= c0 + w) {
      float lrow[kW];  // row `lane` of L11
#pragma unroll
      for (int k = 0; k < kW; ++k) lrow[k] = (k < lane && lane < w) ? __ldcg(&ws->top_lu[k * kW + lane]) : 0.0f;
      float x = lane < w ? a[(size_t)(c0 + lane) + (size_t)col * lda] : 0.0f;
#pragma unroll
      for (int k = 0; k + 1 < kW; ++k) {
        if (k + 1 < w) {
          const float u = __shfl_sync(0xffffffffu, x, k);
          if (lane > k && lane < w) x = __fmaf_rn(-lrow[k], u, x);
        }
      }
      if (lane < w) a[(size_t)(c0 + lane) + (size_t)col * lda] = x;
    }
  }
  if (cta < row_cta0) return;
  __shared__ float rinv[kW];  // 1 / u_jj (0 for a zero pivot, which the factorization reports)
  for (int e = threadIdx.x; e < kW * kW; e += blockDim.x) U[e] = __ldcg(&ws->top_lu[e]);
  if (threadIdx.x < kW) {
    const float d = __ldcg(&ws->top_lu[threadIdx.x * (kW + 1)]);
    rinv[threadIdx.x] = d != 0.0f ? 1.0f / d : 0.0f;
  }
  __syncthreads();
  const int nm = nm_s;
  const int gtid = (cta - row_cta0) * blockDim.x + threadIdx.x;
  const int nth = (ncta - row_cta0) * blockDim.x;
  // rows below the top
  for (int r = c0 + w + gtid; r < n; r += nth) {
    int src = r, hit = -1;
    for (int q = 0; q < nm; ++q)
      if (mpos[q] == r) hit = q;
    if (hit >= 0) src = msrc[hit];
    // a row below the top either stays or is a row displaced from the top
    const bool from_top = src < c0 + w;
    float x[W];
#pragma unroll
    for (int j = 0; j < W; ++j)
      x[j] = j < w ? (from_top ? __ldcg(&ws->top_orig[j * kW + (src - c0)]) : a[(size_t)src + (size_t)(c0 + j) * lda])
                    : 0.0f;
    // l = a U11^-1 by columns, right-looking: step j scales x_j and
    // updates every later entry at once (independent FMAs, row j of U read
    // as a batch), so the dependent chain is one product and one FMA per
    // column instead of a division and a dot product
#pragma unroll
    for (int j = 0; j < W; ++j) {
      if (j < w) {
        x[j] *= rinv[j];
#pragma unroll
        for (int k = j + 1; k < W; ++k) x[k] = fmaf(-x[j], U[j + k * kW], x[k]);
      }
    }
#pragma unroll
    for (int j = 0; j < W; ++j)
      if (j < w) a[(size_t)r + (size_t)(c0 + j) * lda] = x[j];
    if (hit >= 0)
      lab[r] = mlab[hit];
    else if (first_leaf)
      lab[r] = r;
  }
  // the top block (row k = winner k's factored row) and the top labels
  for (int e = gtid; e < w * w; e += nth) {
    const int r = e % w, c = e / w;
    a[(size_t)(c0 + r) + (size_t)(c0 + c) * lda] = U[r + c * kW];
  }
  for (int r = c0 + gtid; r < c0 + w; r += nth) {
    int hit = -1;
    for (int q = 0; q < nm; ++q)
      if (mpos[q] == r) hit = q;
    if (hit >= 0)
      lab[r] = mlab[hit];
    else if (first_leaf)
      lab[r] = r;
  }
}

template <int W>
__global__ void __launch_bounds__(256) tslu_apply_kernel(float* a, int lda, int n, int c0, int w, int kb0, int kb1,
                                                         int* lab, int first_leaf, int side_blocks,
                                                         const TsluScratch* ws) {
  apply_body<W>(a, lda, n, c0, w, kb0, kb1, lab, first_leaf, blockIdx.x, gridDim.x, side_blocks, side_blocks, ws);
}

__device__ __forceinline__ uint64_t tslu_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// The single-launch form (a cooperative launch, so every CTA is resident):
// each CTA factors its 256-row block; the last of each kFan siblings to
// arrive (an atomic count after a fence) merges their proposals and climbs
// on; the CTA that factors the root publishes its results and releases the
// launch's epoch; every CTA waits for it (bounded: 2 s, then the timeout flag)
// and takes its share of the apply step.
template <int W>
__global__ void __launch_bounds__(kRows, 1) tslu_fused_kernel(LevelIn in, int groups0, int kb0, int kb1, int* lab,
                                                           int side_blocks, unsigned epoch, TsluScratch* ws) {
  __shared__ int last_s;
  __shared__ int ok_s;
  int g = blockIdx.x, groups = groups0, src = -1, dst = 0, nchild = 0, level = 0;
  bool ran_root = false;
  // CTAs beyond the level-0 blocks (there only for the side columns) take
  // no part in the tree
  for (; (int)blockIdx.x < groups0;) {
    const bool root = groups == 1;
    level_body<W>(in, g, src, nchild, dst, root, ws);
    if (root) {
      ran_root = true;
      break;
    }
    __threadfence();
    __syncthreads();
    const int parent = g / kFan;
    const int nkids = min(kFan, groups - parent * kFan);
    if (threadIdx.x == 0) {
      const int prev = atomicAdd(&ws->counter[level][parent], 1);
      last_s = prev == nkids - 1 ? 1 : 0;
      if (last_s) ws->counter[level][parent] = 0;  // ready for the next panel
    }
    __syncthreads();
    if (!last_s) break;
    __threadfence();
    nchild = groups;
    groups = (groups + kFan - 1) / kFan;
    src = dst;
    dst = 1 - dst;
    g = parent;
    ++level;
  }
  if (ran_root) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&ws->ready), "r"(epoch) : "memory");
  }
  if (threadIdx.x == 0) {
    const uint64_t t0 = tslu_timer_ns();
    int ok = 0;
    for (;;) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(&ws->ready) : "memory");
      if (v == epoch) {
        ok = 1;
        break;
      }
      if (tslu_timer_ns() - t0 > 2000000000ull) break;
      __nanosleep(64);
    }
    ok_s = ok;
    if (!ok) atomicExch(&in.status->timeout, 1);
  }
  __syncthreads();
  if (!ok_s) return;
  apply_body<W>(const_cast<float*>(in.a), in.lda, in.n, in.c0, in.w, kb0, kb1, lab, in.first_leaf, blockIdx.x,
                gridDim.x, side_blocks, 0, ws);
}

}  // namespace

size_t tslu_scratch_bytes() { return sizeof(TsluScratch); }

// The arrival counts and the release flag start at zero (once per
// factorization; the counts are left at zero by every merge).
int tslu_scratch_reset(alg_ctx* ctx, void* scratch) {
  ALG_CUDA_TRY(cudaMemsetAsync(scratch, 0, offsetof(TsluScratch, cand_rows), ctx->stream));
  return ALG_OK;
}

namespace {

template <int W>
int launch_fused(alg_ctx* ctx, const TsluArgs& p, int groups0, int side_blocks, TsluScratch* ws, bool* done) {
  // co-resident CTAs of the single launch, computed once per process (a
  // thread-safe static initializer; 0 when the query fails)
  static const int max_ctas = [ctx] {
    int per_sm = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tslu_fused_kernel<W>, kRows, 0) == cudaSuccess
               ? per_sm * ctx->sm_count
               : 0;
  }();
  *done = false;
  const int grid = std::max(groups0, side_blocks);
  // the waiting CTAs hold their SMs until the root is done, which the
  // concurrent trailing update of a large matrix needs: tall panels take the
  // multi-launch form (as do grids that cannot be co-resident)
  if (groups0 > kFusedMaxGroups || grid > max_ctas) return ALG_OK;
  static std::atomic<unsigned> epochs{1};
  unsigned epoch = epochs.fetch_add(1);
  if (epoch == 0) epoch = epochs.fetch_add(1);
  LevelIn in{p.a, p.lda, p.n, p.c0, p.w, p.ipiv, p.lab, p.first_leaf, p.status};
  int kb0 = p.kb0, kb1 = p.kb1;
  int* lab = p.lab;
  void* args[] = {(void*)&in, (void*)&groups0, (void*)&kb0, (void*)&kb1, (void*)&lab, (void*)&side_blocks,
                  (void*)&epoch, (void*)&ws};
  ALG_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)tslu_fused_kernel<W>, dim3(grid), dim3(kRows), args, 0,
                                           ctx->stream));
  *done = true;
  return ALG_OK;
}

}  // namespace

// A leaf panel of the FP32 LU by tournament pivoting; the outputs of the
// partial-pivoting cluster kernel (factored panel, ipiv, labels, side
// columns) and U12 of the block panel's trailing columns (the in-block TRSM). Returns ALG_NOT_IMPLEMENTED when the panel does not fit its
// limits (the caller then uses partial pivoting). One cooperative launch when
// the level-0 CTAs fit on the device at once, else one launch per tree level
// and one for the apply step. The scratch is reset once per factorization.
int tslu_panel(alg_ctx* ctx, const TsluArgs& p, void* scratch) {
  const int m = p.n - p.c0, w = p.w;
  if (w > kW || w < 1 || m < w) return ALG_NOT_IMPLEMENTED;
  const int groups0 = (m + kRows - 1) / kRows;
  if (groups0 > kMaxGroups) return ALG_NOT_IMPLEMENTED;
  auto* ws = static_cast<TsluScratch*>(scratch);
  const int side = (p.kb1 - p.kb0) - w;
  const int side_blocks = side > 0 ? (side + kSideCols - 1) / kSideCols : 0;
  double pflops = 0;
  for (int j = 0; j < w; ++j) pflops += double(m - j - 1) * (1.0 + 2.0 * (w - j - 1));
  const int tok = prof_begin(ctx, ALG_K_PANEL);
  if (!std::getenv("ALG_TSLU_SPLIT")) {
    bool done = false;
    if (w <= 16)
      ALG_TRY(launch_fused<16>(ctx, p, groups0, side_blocks, ws, &done));
    else
      ALG_TRY(launch_fused<32>(ctx, p, groups0, side_blocks, ws, &done));
    if (done) {
      count_launches(1);
      prof_end(ctx, tok, pflops, 2.0 * sizeof(float) * m * w);
      ALG_CUDA_TRY(cudaGetLastError());
      return ALG_OK;
    }
  }
  LevelIn in{p.a, p.lda, p.n, p.c0, w, p.ipiv, p.lab, p.first_leaf, p.status};
  // level 0 reads the panel; each later level merges kFan proposals per CTA
  int groups = groups0, src = -1, dst = 0, nchild = 0, launches = 0;
  for (;;) {
    const bool root = groups == 1;
    if (w <= 16)
      tslu_level_kernel<16><<<groups, kRows, 0, ctx->stream>>>(in, src, nchild, dst, root ? 1 : 0, ws);
    else
      tslu_level_kernel<32><<<groups, kRows, 0, ctx->stream>>>(in, src, nchild, dst, root ? 1 : 0, ws);
    ++launches;
    if (root) break;
    nchild = groups;
    groups = (groups + kFan - 1) / kFan;
    src = dst;
    dst = 1 - dst;
  }
  const int row_blocks = std::max(1, std::min(2 * ctx->sm_count, (m + 255) / 256));
  if (w <= 16)
    tslu_apply_kernel<16><<<side_blocks + row_blocks, 256, 0, ctx->stream>>>(p.a, p.lda, p.n, p.c0, w, p.kb0,
                                                                             p.kb1, p.lab, p.first_leaf,
                                                                             side_blocks, ws);
  else
    tslu_apply_kernel<32><<<side_blocks + row_blocks, 256, 0, ctx->stream>>>(p.a, p.lda, p.n, p.c0, w, p.kb0,
                                                                             p.kb1, p.lab, p.first_leaf,
                                                                             side_blocks, ws);
  count_launches(launches + 1);
  prof_end(ctx, tok, pflops, 2.0 * sizeof(float) * m * w);
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

}  // namespace alg
