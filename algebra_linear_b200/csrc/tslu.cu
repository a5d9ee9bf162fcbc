// Tournament pivoting for the leaf panels of the low-precision LU (the
// mixed-precision form only; the FP64 drop-in keeps partial pivoting).
//
// Partial pivoting needs one reduction over all rows per column, and that
// chain is the critical path of the look-ahead LU. Tournament pivoting
// (TSLU: Grigori, Demmel, Xiang, "CALU: a communication optimal LU
// factorization algorithm", SIAM J. Matrix Anal. Appl. 32, 2011) chooses the
// panel's w pivot rows first and factors afterwards:
//   1. select: each CTA runs partial-pivoting LU on its own chunk of rows (in
//      shared memory) and proposes the w rows it pivoted on;
//   2. merge: one CTA runs partial-pivoting LU on the proposed rows'
//      original values; its w pivots are the panel's pivots and its leading
//      w x w block is L11 \ U11;
//   3. apply: the interchanges (LAPACK sequential form, as the partial-
//      pivoting panel records them) move the winners to the top, every other
//      row gets its multipliers l = a U11^-1, the labels of the moved rows
//      and the block panel's other columns follow the interchanges.
// The factorization differs from partial pivoting's (other pivots); the
// mixed form's refinement in FP64 then brings the solution to the FP64
// backward error, which is its contract.
#include <algorithm>
#include <climits>

#include "dense.cuh"

namespace alg {
namespace {

constexpr int kW = 32;             // widest leaf
constexpr int kChunk = 64;         // rows per warp at the tree's leaves
constexpr int kMaxChunks = 1024;   // up to 65 536 panel rows
constexpr int kTreeWarps = 2;      // warps per CTA of the tournament kernel (2 x 16 KB of shared memory)
constexpr int kMaxMoves = 2 * kW;

struct TsluScratch {
  int node_cand[2 * kMaxChunks][kW];  // each tree node's proposed rows (absolute), -1 = none
  float node_vals[2 * kMaxChunks][kW * kW];  // their original values ([col][row], stride kW)
  int counter[2 * kMaxChunks];        // arrivals per node (reset by the merging warp)
  int nmoves;
  int move_pos[kMaxMoves];            // a position whose row changed
  int move_src[kMaxMoves];            // the position that row came from (at the leaf's start)
  int move_lab[kMaxMoves];            // its new label
  float top_lu[kW * kW];              // L11 \ U11 of the winners (column-major w x w)
  float top_orig[kW * kW];            // original values of the rows at the top positions
};

// Partial-pivoting LU, by one warp, of the first w columns of nr <= 64 rows
// held in shared memory ([col][row], stride kChunk), swapping the row ids
// along; returns the first column whose pivot is zero, or -1.
__device__ int warp_gepp(float* s, int* sid, int nr, int w) {
  const int lane = threadIdx.x & 31;
  int zero_col = -1;
  const int kmax = min(w, nr);
  for (int k = 0; k < kmax; ++k) {
    float key = -1.0f;
    int idx = INT_MAX;
    for (int r = k + lane; r < nr; r += 32) {
      const float v = fabsf(s[k * kChunk + r]);
      if (v > key) {
        key = v;
        idx = r;
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const float ok = __shfl_xor_sync(0xffffffffu, key, off);
      const int oi = __shfl_xor_sync(0xffffffffu, idx, off);
      if (ok > key || (ok == key && oi < idx)) {
        key = ok;
        idx = oi;
      }
    }
    const int p = idx;
    if (p != k) {
      if (lane < w) {
        const float t = s[lane * kChunk + k];
        s[lane * kChunk + k] = s[lane * kChunk + p];
        s[lane * kChunk + p] = t;
      }
      if (lane == 0) {
        const int t = sid[k];
        sid[k] = sid[p];
        sid[p] = t;
      }
    }
    __syncwarp();
    const float d = s[k * kChunk + k];
    if (d == 0.0f) {
      if (zero_col < 0) zero_col = k;
    } else {
      const float inv = 1.0f / d;
      for (int r = k + 1 + lane; r < nr; r += 32) s[k * kChunk + r] *= inv;
    }
    __syncwarp();
    for (int r = k + 1 + lane; r < nr; r += 32) {
      const float l = s[k * kChunk + r];
      for (int c = k + 1; c < w; ++c) s[c * kChunk + r] = fmaf(-s[c * kChunk + k], l, s[c * kChunk + r]);
    }
    __syncwarp();
  }
  return zero_col;
}

// 1 + 2. The tournament, one launch: warp g factors rows
// [c0 + 64 g, c0 + 64 (g + 1)) and proposes its w pivot rows, with their
// original values, to its tree node; up a binary tree, the second of two
// sibling warps to finish merges their proposals (partial-pivoting LU of the
// up to 2 w proposed rows' original values, read contiguously from the
// scratch); the warp that merges the root holds the panel's pivots and
// L11 \ U11 and records the interchanges, the moved rows and their labels.
// No warp waits for another: arrivals are counted with atomics after a fence.
__global__ void __launch_bounds__(kTreeWarps * 32) tslu_tree_kernel(const float* a, int lda, int n, int c0, int w,
                                                                    int nchunks, int* ipiv, const int* lab,
                                                                    int first_leaf, DevStatus* status,
                                                                    TsluScratch* ws) {
  __shared__ float work_s[kTreeWarps][kW * kChunk];
  __shared__ float orig_s[kTreeWarps][kW * kChunk];
  __shared__ int sids[kTreeWarps][kChunk];
  __shared__ int rows_s[kTreeWarps][kChunk];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int g = blockIdx.x * kTreeWarps + wl;
  if (g >= nchunks) return;
  float* s = work_s[wl];
  float* o = orig_s[wl];
  int* sid = sids[wl];  // local indices into rows / o
  int* rows = rows_s[wl];
  // leaf: this warp's own chunk
  const int r0 = c0 + g * kChunk;
  int nr = max(0, min(n, r0 + kChunk) - r0);
  for (int e = lane; e < nr * w; e += 32) {
    const int r = e % nr, c = e / nr;
    const float v = a[(size_t)(r0 + r) + (size_t)(c0 + c) * lda];
    o[c * kChunk + r] = v;
    s[c * kChunk + r] = v;
  }
  for (int r = lane; r < nr; r += 32) {
    rows[r] = r0 + r;
    sid[r] = r;
  }
  __syncwarp();
  int zc = warp_gepp(s, sid, nr, w);
  int node = g, base = 0, width = nchunks;  // node index within its level, level's first slot, level width
  auto publish = [&]() {
    const int cnt = min(w, nr);
    for (int k = lane; k < kW; k += 32) ws->node_cand[base + node][k] = k < cnt ? rows[sid[k]] : -1;
    for (int e = lane; e < cnt * w; e += 32) {
      const int k = e % cnt, c = e / cnt;
      ws->node_vals[base + node][c * kW + k] = o[c * kChunk + sid[k]];
    }
  };
  publish();
  // up the tree
  while (width > 1) {
    const int parent = node >> 1, pwidth = (width + 1) >> 1, pbase = base + width;
    const bool has_sibling = (node ^ 1) < width;
    __syncwarp();
    if (has_sibling) {
      __threadfence();
      int arrived = 0;
      if (lane == 0) arrived = atomicAdd(&ws->counter[pbase + parent], 1);
      arrived = __shfl_sync(0xffffffffu, arrived, 0);
      if (arrived == 0) return;  // the sibling merges
      __threadfence();
      if (lane == 0) ws->counter[pbase + parent] = 0;  // ready for the next panel
    }
    // gather the children's proposals and their original values
    nr = 0;
    for (int ch = 2 * parent; ch < min(2 * parent + 2, width); ++ch) {
      const volatile int* cand = ws->node_cand[base + ch];
      const volatile float* vals = ws->node_vals[base + ch];
      int cnt = 0;
      while (cnt < kW && cand[cnt] >= 0) ++cnt;
      for (int k = lane; k < cnt; k += 32) rows[nr + k] = cand[k];
      for (int e = lane; e < cnt * w; e += 32) {
        const int k = e % cnt, c = e / cnt;
        const float v = vals[c * kW + k];
        o[c * kChunk + nr + k] = v;
        s[c * kChunk + nr + k] = v;
      }
      nr += cnt;
    }
    for (int r = lane; r < nr; r += 32) sid[r] = r;
    __syncwarp();
    zc = warp_gepp(s, sid, nr, w);
    node = parent;
    base = pbase;
    width = pwidth;
    publish();
  }
  __syncwarp();
  // the root: pivots, L11 \ U11, the rows at the top before anything moves
  for (int e = lane; e < w * w; e += 32) {
    const int r = e % w, c = e / w;
    ws->top_lu[r + c * kW] = s[c * kChunk + r];
    ws->top_orig[r + c * kW] = a[(size_t)(c0 + r) + (size_t)(c0 + c) * lda];
  }
  if (lane == 0) {
    if (zc >= 0) atomicMin(&status->singular_col, c0 + zc);
    // LAPACK sequential interchanges that bring winner j to position c0 + j;
    // occupant tracking over the touched positions only
    int pos[kMaxMoves], occ[kMaxMoves];
    int nt = 0;
    auto find_pos = [&](int p) {
      for (int t = 0; t < nt; ++t)
        if (pos[t] == p) return t;
      pos[nt] = p;
      occ[nt] = p;  // untouched: the row that started there
      return nt++;
    };
    for (int j = 0; j < w; ++j) {
      const int gr = rows[sid[j]];
      int pr = gr;  // current position of row gr
      for (int t = 0; t < nt; ++t)
        if (occ[t] == gr) {
          pr = pos[t];
          break;
        }
      ipiv[c0 + j] = pr;
      const int tj = find_pos(c0 + j);
      const int tp = find_pos(pr);
      const int h = occ[tj];
      occ[tj] = gr;
      occ[tp] = h;
    }
    int nm = 0;
    for (int t = 0; t < nt; ++t)
      if (occ[t] != pos[t]) {
        ws->move_pos[nm] = pos[t];
        ws->move_src[nm] = occ[t];
        ws->move_lab[nm] = first_leaf ? occ[t] : lab[occ[t]];
        ++nm;
      }
    ws->nmoves = nm;
  }
}

// 3. multipliers of every row below the top, the top block, labels and the
//    block panel's other columns
__global__ void __launch_bounds__(256) tslu_apply_kernel(float* a, int lda, int n, int c0, int w, int kb0, int kb1,
                                                         const int* ipiv, int* lab, int first_leaf,
                                                         const TsluScratch* ws) {
  __shared__ float U[kW * kW];
  __shared__ int mpos[kMaxMoves], msrc[kMaxMoves], mlab[kMaxMoves];
  __shared__ int nm;
  for (int e = threadIdx.x; e < kW * kW; e += blockDim.x) U[e] = ws->top_lu[e];
  if (threadIdx.x == 0) nm = ws->nmoves;
  for (int t = threadIdx.x; t < kMaxMoves; t += blockDim.x) {
    mpos[t] = ws->move_pos[t];
    msrc[t] = ws->move_src[t];
    mlab[t] = ws->move_lab[t];
  }
  __syncthreads();
  const int nmv = nm;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nth = gridDim.x * blockDim.x;
  // rows below the top: l = a U11^-1 (a from the row that ends up there)
  for (int r = c0 + w + gtid; r < n; r += nth) {
    int src = r, t_hit = -1;
    for (int t = 0; t < nmv; ++t)
      if (mpos[t] == r) {
        src = msrc[t];
        t_hit = t;
      }
    float l[kW];
#pragma unroll
    for (int j = 0; j < kW; ++j) {
      if (j < w) {
        // a row displaced from the top reads its saved original values
        float s = src >= c0 + w || src < c0 ? a[(size_t)src + (size_t)(c0 + j) * lda]
                                            : ws->top_orig[(src - c0) + j * kW];
#pragma unroll
        for (int i = 0; i < kW; ++i)
          if (i < j) s = fmaf(-l[i], U[i + j * kW], s);
        l[j] = s / U[j + j * kW];
      }
    }
    // write after every read of this row's source (a source below the top is the row itself)
#pragma unroll
    for (int j = 0; j < kW; ++j)
      if (j < w) a[(size_t)r + (size_t)(c0 + j) * lda] = l[j];
    if (t_hit >= 0)
      lab[r] = mlab[t_hit];
    else if (first_leaf)
      lab[r] = r;
  }
  // the top block and the top positions' labels
  for (int e = gtid; e < w * w; e += nth) {
    const int r = e % w, c = e / w;
    a[(size_t)(c0 + r) + (size_t)(c0 + c) * lda] = U[r + c * kW];
  }
  for (int r = c0 + gtid; r < c0 + w; r += nth) {
    int t_hit = -1;
    for (int t = 0; t < nmv; ++t)
      if (mpos[t] == r) t_hit = t;
    if (t_hit >= 0)
      lab[r] = mlab[t_hit];
    else if (first_leaf)
      lab[r] = r;
  }
  // the block panel's other columns follow the interchanges (in order)
  const int side = (kb1 - kb0) - w;
  for (int cidx = gtid; cidx < side; cidx += nth) {
    int col = kb0 + cidx;
    if (col >= c0) col += w;
    float* cp = a + (size_t)col * lda;
    for (int j = 0; j < w; ++j) {
      const int pr = ipiv[c0 + j];
      if (pr != c0 + j) {
        const float t = cp[c0 + j];
        cp[c0 + j] = cp[pr];
        cp[pr] = t;
      }
    }
  }
}

}  // namespace

size_t tslu_scratch_bytes() { return sizeof(TsluScratch); }

// A leaf panel of the FP32 LU by tournament pivoting; same outputs as the
// partial-pivoting cluster kernel (factored panel, ipiv, labels, side
// columns). Returns ALG_NOT_IMPLEMENTED when the panel does not fit its
// limits (the caller then uses partial pivoting). The scratch's arrival
// counters must be zero on the first call (the caller clears it once).
int tslu_panel(alg_ctx* ctx, const TsluArgs& p, void* scratch) {
  const int m = p.n - p.c0, w = p.w;
  if (w > kW || w < 1 || m < w) return ALG_NOT_IMPLEMENTED;
  const int nchunks = (m + kChunk - 1) / kChunk;
  if (nchunks > kMaxChunks) return ALG_NOT_IMPLEMENTED;
  auto* ws = static_cast<TsluScratch*>(scratch);
  const int tok = prof_begin(ctx, ALG_K_PANEL);
  tslu_tree_kernel<<<(nchunks + kTreeWarps - 1) / kTreeWarps, kTreeWarps * 32, 0, ctx->stream>>>(
      p.a, p.lda, p.n, p.c0, w, nchunks, p.ipiv, p.lab, p.first_leaf, p.status, ws);
  const int grid = std::max(1, std::min(2 * ctx->sm_count, (m + 255) / 256));
  tslu_apply_kernel<<<grid, 256, 0, ctx->stream>>>(p.a, p.lda, p.n, p.c0, w, p.kb0, p.kb1, p.ipiv, p.lab,
                                                   p.first_leaf, ws);
  count_launches(2);
  double pflops = 0;
  for (int j = 0; j < w; ++j) pflops += double(m - j - 1) * (1.0 + 2.0 * (w - j - 1));
  prof_end(ctx, tok, pflops, 2.0 * sizeof(float) * m * w);
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

}  // namespace alg
