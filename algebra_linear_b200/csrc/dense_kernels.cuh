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
// Factors the (m - c0) x w leaf panel whose top-left entry is (c0, c0). Its
// rows are split into C contiguous slabs, one per CTA of the cluster, held in
// shared memory for the whole panel (W = 16 or 32 columns, padded stride).
// Thread (g, c) of a CTA owns column c of the slab rows g, g+G, g+2G, ...
//
// Pivot exchange without cluster barriers: for column j every CTA sends a
// record — its candidate (first index of max |a_ij| with the reference's NaN
// rule, mod.rs:123-134), a copy of that row and its labels — into the
// mailbox of every CTA of the cluster with st.async DSMEM stores that count
// their bytes on the receiver's mbarrier; the owner of row j also sends a
// copy of row j. A CTA waits on its own mbarrier only, and every warp reduces
// the C records redundantly to the same winner. Mailboxes and mbarriers are
// double-buffered by column parity; a sender can only reach column j+2 after
// every CTA has consumed column j (it needs their column j+1 records), so a
// buffer is never overwritten while it is read.
//
// Per column j, after the exchange: swap rows j and p (mod.rs:141-146),
// divide the rows below by the pivot (true division, mod.rs:153-155), apply
// the rank-1 update (mod.rs:156-158) and scan column j+1 for the next
// candidate. Rows carry two labels through the swaps: the original row within
// the enclosing block-panel (for the deferred interchange of the matrix's
// other columns) and within this leaf (for the block-panel's other columns,
// which this kernel swaps itself before it exits).
// ---------------------------------------------------------------------------
template <typename T>
struct PanelArgs {
  T* a;
  int lda;
  int n;           // rows of the matrix
  int c0;          // first row and column of the leaf
  int w;           // leaf width (<= W)
  int kb0, kb1;    // columns of the enclosing block-panel
  int* ipiv;       // global interchanges (0-based global rows)
  int* lab;        // cumulative source labels of rows [kb0, n)
  int first_leaf;  // labels start as the identity
  DevStatus* status;
};

constexpr int kPanelThreads = 512;
constexpr int kPanelWarps = kPanelThreads / 32;
constexpr int kPanelMaxW = 32;
constexpr int kPanelMaxC = 16;
constexpr int kSideCols = 16;  // block-panel columns swapped per pass at exit

// One mailbox record, in 8-byte words: key, (row, cumulative label),
// (leaf label, unused), then the row's W entries.
template <typename T, int W>
struct PanelRec {
  static constexpr int kRowWords = (W * (int)sizeof(T)) / 8;
  static constexpr int kWords = (3 + kRowWords + 1) & ~1;     // padded to 16 bytes
  static constexpr int kBytes = 8 * kWords;
  static constexpr int kDiagWords = (1 + kRowWords + 1) & ~1;  // (cumulative, leaf label), row
  static constexpr int kDiagBytes = 8 * kDiagWords;
};

template <typename T, int W>
struct PanelSmem {
  unsigned long long mbar[2];
  alignas(16) unsigned long long rec[2][kPanelMaxC][PanelRec<T, W>::kWords];
  alignas(16) unsigned long long diag[2][PanelRec<T, W>::kDiagWords];
  alignas(16) unsigned long long outbox[2][PanelRec<T, W>::kWords];
  alignas(16) unsigned long long doutbox[2][PanelRec<T, W>::kDiagWords];
  double cand_key[kPanelWarps];
  int cand_idx[kPanelWarps];
  T side_vals[4 * kPanelMaxW][kSideCols];
  int side_rows[4 * kPanelMaxW];
  int side_cnt;
};

template <typename T, int W>
__host__ __device__ inline size_t panel_smem_bytes(int rows_per_cta) {
  size_t b = sizeof(PanelSmem<T, W>);
  b = (b + 15) & ~size_t(15);
  b += sizeof(T) * (size_t)rows_per_cta * (W + 1);  // slab
  b += sizeof(int) * 2 * (size_t)rows_per_cta;     // labels
  return (b + 127) & ~size_t(127);
}

__device__ __forceinline__ void keyidx_combine(double& k, int& i, double ok, int oi) {
  if (ok > k || (ok == k && oi < i)) {
    k = ok;
    i = oi;
  }
}

__device__ __forceinline__ double pivot_key(double v, bool is_diag) {
  const double a = fabs(v);
  if (isnan(a)) return is_diag ? CUDART_INF : -CUDART_INF;
  return a;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t mapa_u32(uint32_t a, int rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_async_b64(uint32_t remote, unsigned long long v, uint32_t remote_bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];"
               :: "r"(remote), "l"(v), "r"(remote_bar) : "memory");
}
// One bulk copy (async proxy) of `bytes` from this CTA's shared memory into
// the shared memory of a CTA of the cluster, completing on that CTA's mbarrier.
// Addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_to_cta(uint32_t remote_dst, uint32_t local_src, int bytes, uint32_t remote_bar) {
  asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               :: "r"(remote_dst), "r"(local_src), "r"(bytes), "r"(remote_bar) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arm(uint32_t bar, int bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}
// Waits for the phase of the given parity; gives up after kWaitLimitNs and
// returns false.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, int parity) {
  uint32_t done = 0;
  uint64_t t0 = 0;
  for (int it = 0;; ++it) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done) : "r"(bar), "r"(parity) : "memory");
    if (done) return true;
    if ((it & 63) == 0) {
      const uint64_t t = global_timer_ns();
      if (it == 0) t0 = t;
      else if (t - t0 > kWaitLimitNs) return false;
    }
  }
}

template <typename T>
__device__ __forceinline__ unsigned long long pack2(T a, T b);
template <>
__device__ __forceinline__ unsigned long long pack2<float>(float a, float b) {
  return (unsigned long long)__float_as_uint(a) | ((unsigned long long)__float_as_uint(b) << 32);
}
__device__ __forceinline__ unsigned long long pack_ii(int a, int b) {
  return (unsigned long long)(unsigned)a | ((unsigned long long)(unsigned)b << 32);
}

// Word k of a slab row, as the record stores it.
template <typename T, int W>
__device__ __forceinline__ unsigned long long row_word(const T* row, int k) {
  if constexpr (sizeof(T) == 8) {
    return (unsigned long long)__double_as_longlong(static_cast<double>(row[k]));
  } else {
    return pack2<float>(static_cast<float>(row[2 * k]), static_cast<float>(row[2 * k + 1]));
  }
}
template <typename T>
__device__ __forceinline__ T rec_entry(const unsigned long long* words, int c) {
  if constexpr (sizeof(T) == 8) {
    return static_cast<T>(__longlong_as_double((long long)words[c]));
  } else {
    const unsigned long long wv = words[c >> 1];
    return static_cast<T>(__uint_as_float((unsigned)(c & 1 ? (wv >> 32) : wv)));
  }
}

template <typename T>
__device__ __forceinline__ bool div_fast_ok(T x) {
  const double ax = fabs(static_cast<double>(x));
  if constexpr (sizeof(T) == 8) {
    return ax >= 0x1p-500 && ax <= 0x1p500;
  } else {
    return ax >= 0x1p-60f && ax <= 0x1p60f;
  }
}
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

// a / d correctly rounded; y = RN(1/d), fast = d passed div_fast_ok.
template <typename T>
__device__ __forceinline__ T quotient(T a, T d, T y, bool fast) {
  if (fast && div_fast_ok(a)) {
    const T q = mul_rn(a, y);
    const T r = fma_rn(-q, d, a);
    return fma_rn(r, y, q);
  }
  return div_rn(a, d);
}

template <typename T, int W, bool EXACT>
__global__ void __launch_bounds__(kPanelThreads, 1) panel_cluster_kernel(PanelArgs<T> p) {
  using Rec = PanelRec<T, W>;
  constexpr int G = kPanelThreads / W;  // row groups
  constexpr int LD = W + 1;
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks();
  const int q = (int)cl.block_rank();
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int c = tid % W;   // column owned by this thread
  const int g = tid / W;   // row group
  const int m = p.n - p.c0;
  const int R = (m + C - 1) / C;
  const int rb = q * R;
  const int re = min(m, rb + R);
  const int nr = max(0, re - rb);
  const int w = p.w;
  const int step_bytes = C * Rec::kBytes + Rec::kDiagBytes;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  PanelSmem<T, W>& S = *reinterpret_cast<PanelSmem<T, W>*>(smem_raw);
  T* tile = reinterpret_cast<T*>(smem_raw + ((sizeof(PanelSmem<T, W>) + 15) & ~size_t(15)));
  int* lab_s = reinterpret_cast<int*>(tile + (size_t)R * LD);
  int* loc_s = lab_s + R;

  // ---- load the slab, set up the mailboxes ----------------------------------
  for (int cc = 0; cc < W; ++cc) {
    const T* col = p.a + (size_t)(p.c0 + cc) * p.lda + (p.c0 + rb);
    for (int r = tid; r < nr; r += kPanelThreads) tile[r * LD + cc] = cc < w ? col[r] : T(0);
  }
  for (int r = tid; r < nr; r += kPanelThreads) {
    const int gr = p.c0 + rb + r;
    lab_s[r] = p.first_leaf ? gr : p.lab[gr];
    loc_s[r] = gr;
  }
  if (tid == 0) {
    mbar_init(smem_u32(&S.mbar[0]), 1);
    mbar_init(smem_u32(&S.mbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_arm(smem_u32(&S.mbar[0]), step_bytes);
    if (w > 1) mbar_arm(smem_u32(&S.mbar[1]), step_bytes);
  }
  cl.sync();  // mbarriers live in every CTA before anyone sends

  // first candidate (column 0)
  {
    double bk = -CUDART_INF;
    int bi = INT_MAX;
    if (c == 0) {
      for (int r = g; r < nr; r += G) {
        const double key = pivot_key((double)tile[r * LD], rb + r == 0);
        if (key > bk) { bk = key; bi = rb + r; }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ok = __shfl_down_sync(0xffffffffu, bk, off);
      const int oi = __shfl_down_sync(0xffffffffu, bi, off);
      keyidx_combine(bk, bi, ok, oi);
    }
    if (lane == 0) { S.cand_key[warp] = bk; S.cand_idx[warp] = bi; }
  }
  __syncthreads();

  const uint32_t rec_base = smem_u32(&S.rec[0][0][0]);
  const uint32_t diag_base = smem_u32(&S.diag[0][0]);
  const uint32_t bar_base = smem_u32(&S.mbar[0]);
  bool ok_wait = true;

  for (int j = 0; j < w; ++j) {
    const int par = j & 1;
    // ---- send: CTA candidate record (+ row j) to every mailbox -------------
    if (warp == 0) {
      double bk = -CUDART_INF;
      int bi = INT_MAX;
      if (lane < kPanelWarps) { bk = S.cand_key[lane]; bi = S.cand_idx[lane]; }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ok = __shfl_down_sync(0xffffffffu, bk, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        keyidx_combine(bk, bi, ok, oi);
      }
      bk = __shfl_sync(0xffffffffu, bk, 0);
      bi = __shfl_sync(0xffffffffu, bi, 0);
      const bool have = bi != INT_MAX;
      const T* crow = have ? tile + (size_t)(bi - rb) * LD : tile;
      const bool own_j = j >= rb && j < re;
      const T* drow = own_j ? tile + (size_t)(j - rb) * LD : tile;
      unsigned long long* ob = &S.outbox[par][0];
      unsigned long long* dob = &S.doutbox[par][0];
      for (int kw = lane; kw < Rec::kWords; kw += 32) {
        unsigned long long val = 0;
        if (kw == 0) val = (unsigned long long)__double_as_longlong(bk);
        else if (kw == 1) val = pack_ii(bi, have ? lab_s[bi - rb] : 0);
        else if (kw == 2) val = pack_ii(have ? loc_s[bi - rb] : 0, 0);
        else if (kw < 3 + Rec::kRowWords) val = row_word<T, W>(crow, kw - 3);
        ob[kw] = val;
      }
      if (own_j) {
        for (int kw = lane; kw < Rec::kDiagWords; kw += 32) {
          unsigned long long val = 0;
          if (kw == 0) val = pack_ii(lab_s[j - rb], loc_s[j - rb]);
          else if (kw < 1 + Rec::kRowWords) val = row_word<T, W>(drow, kw - 1);
          dob[kw] = val;
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane < C) {
        const uint32_t rbar = mapa_u32(bar_base + 8u * par, lane);
        const uint32_t la = rec_base + 8u * (uint32_t)((par * kPanelMaxC + q) * Rec::kWords);
        bulk_to_cta(mapa_u32(la, lane), smem_u32(ob), Rec::kBytes, rbar);
        if (own_j) {
          const uint32_t ld2 = diag_base + 8u * (uint32_t)(par * Rec::kDiagWords);
          bulk_to_cta(mapa_u32(ld2, lane), smem_u32(dob), Rec::kDiagBytes, rbar);
        }
      }
    }
    // ---- receive: wait for this column's records ---------------------------
    // a wait that ran out stays failed: the rest of the leaf runs through
    // without waiting and the host reports ALG_TIMEOUT
    if (ok_wait && !mbar_wait(bar_base + 8u * par, (j >> 1) & 1)) {
      ok_wait = false;
      atomicExch(&p.status->timeout, 1);
    }
    __syncwarp();
    if (tid == 0 && j + 2 < w) mbar_arm(bar_base + 8u * par, step_bytes);
    // every warp reduces the C records to the same winner
    double wk = -CUDART_INF;
    int wi = INT_MAX, ws = 0;
    if (lane < C) {
      wk = __longlong_as_double((long long)S.rec[par][lane][0]);
      wi = (int)(unsigned)(S.rec[par][lane][1] & 0xffffffffu);
      ws = lane;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ok = __shfl_down_sync(0xffffffffu, wk, off);
      const int oi = __shfl_down_sync(0xffffffffu, wi, off);
      const int os = __shfl_down_sync(0xffffffffu, ws, off);
      if (ok > wk || (ok == wk && oi < wi)) { wk = ok; wi = oi; ws = os; }
    }
    const int pr = __shfl_sync(0xffffffffu, wi, 0);  // winning panel row (>= j)
    const int ps = __shfl_sync(0xffffffffu, ws, 0);  // CTA that sent it
    const unsigned long long* wrow = &S.rec[par][ps][3];
    const T d = rec_entry<T>(wrow, j);
    const T u = rec_entry<T>(wrow, c);
    // swap rows j and pr where this thread owns them (same thread updates them later)
    if (j >= rb && j < re && (j - rb) % G == g) {
      tile[(j - rb) * LD + c] = u;
      if (c == 0) {
        lab_s[j - rb] = (int)(unsigned)(S.rec[par][ps][1] >> 32);
        loc_s[j - rb] = (int)(unsigned)(S.rec[par][ps][2] & 0xffffffffu);
      }
    }
    if (pr != j && pr >= rb && pr < re && (pr - rb) % G == g) {
      tile[(pr - rb) * LD + c] = rec_entry<T>(&S.diag[par][1], c);
      if (c == 0) {
        lab_s[pr - rb] = (int)(unsigned)(S.diag[par][0] & 0xffffffffu);
        loc_s[pr - rb] = (int)(unsigned)(S.diag[par][0] >> 32);
      }
    }
    if (tid == 0 && q == 0) {
      p.ipiv[p.c0 + j] = p.c0 + pr;
      if (fabs((double)d) <= 0.0) atomicMin(&p.status->singular_col, p.c0 + j);
    }
    __syncwarp();
    // multipliers (correctly rounded quotient, as K1r) for the group's rows
    // below j, spread over its lanes
    const int r_first = max(0, j + 1 - rb);
    const int r0 = r_first + ((g - r_first % G) + G) % G;  // first row >= r_first of group g
    {
      const bool fast = div_fast_ok(d);
      const T y = fast ? rcp_rn(d) : T(1);
      int k = 0;
      for (int r = r0 + c * G; r < nr; r += W * G, k += W) {
        const T av = tile[r * LD + j];
        tile[r * LD + j] = quotient<T>(av, d, y, fast);
      }
    }
    __syncwarp();
    // rank-1 update, 8 independent rows per batch; column j+1 yields the next candidate
    double bk = -CUDART_INF;
    int bi = INT_MAX;
    if (c > j && c < w) {
      constexpr int B = 8;
      for (int rs = r0; rs < nr; rs += B * G) {
        T av[B], lv[B];
#pragma unroll
        for (int t = 0; t < B; ++t) {
          const int r = rs + t * G;
          av[t] = r < nr ? tile[r * LD + c] : T(0);
          lv[t] = r < nr ? tile[r * LD + j] : T(0);
        }
#pragma unroll
        for (int t = 0; t < B; ++t) av[t] = msub<EXACT>(av[t], lv[t], u);
#pragma unroll
        for (int t = 0; t < B; ++t) {
          const int r = rs + t * G;
          if (r < nr) {
            tile[r * LD + c] = av[t];
            if (c == j + 1) {
              const double key = pivot_key((double)av[t], rb + r == j + 1);
              if (key > bk) { bk = key; bi = rb + r; }
            }
          }
        }
      }
    }
    if (j + 1 < w) {
      // collect the candidates of the warp's row groups (lanes with c == j+1)
      const int src0 = (lane / W) * W + (j + 1);  // own group's candidate lane
      double k0 = __shfl_sync(0xffffffffu, bk, src0 & 31);
      int i0 = __shfl_sync(0xffffffffu, bi, src0 & 31);
      if constexpr (W == 16) {
        const double k1 = __shfl_sync(0xffffffffu, bk, (j + 1 + 16 - (lane / W) * W) & 31);
        const int i1 = __shfl_sync(0xffffffffu, bi, (j + 1 + 16 - (lane / W) * W) & 31);
        keyidx_combine(k0, i0, k1, i1);
      }
      if (lane == 0) { S.cand_key[warp] = k0; S.cand_idx[warp] = i0; }
    }
    __syncthreads();
  }
  cl.sync();  // every record consumed; no DSMEM access outlives its owner

  // ---- swap the block-panel's other columns by this leaf's interchanges -----
  // Rows whose leaf label moved take the old content of the labelled row; all
  // reads of a pass precede the cluster barrier, all writes follow it.
  if (tid == 0) S.side_cnt = 0;
  __syncthreads();
  for (int r = tid; r < nr; r += kPanelThreads) {
    if (loc_s[r] != p.c0 + rb + r) {
      const int s = atomicAdd(&S.side_cnt, 1);
      if (s < 4 * kPanelMaxW) S.side_rows[s] = r;
    }
  }
  __syncthreads();
  const int n_side = min(S.side_cnt, 4 * kPanelMaxW);
  const int side_w = (p.kb1 - p.kb0) - w;
  for (int cbase = 0; cbase < side_w; cbase += kSideCols) {
    const int ncol = min(kSideCols, side_w - cbase);
    for (int idx = tid; idx < n_side * kSideCols; idx += kPanelThreads) {
      const int s = idx / kSideCols, cc = idx % kSideCols;
      if (cc >= ncol) continue;
      int col = p.kb0 + cbase + cc;
      if (col >= p.c0) col += w;
      S.side_vals[s][cc] = p.a[(size_t)loc_s[S.side_rows[s]] + (size_t)col * p.lda];
    }
    cl.sync();
    for (int idx = tid; idx < n_side * kSideCols; idx += kPanelThreads) {
      const int s = idx / kSideCols, cc = idx % kSideCols;
      if (cc >= ncol) continue;
      int col = p.kb0 + cbase + cc;
      if (col >= p.c0) col += w;
      p.a[(size_t)(p.c0 + rb + S.side_rows[s]) + (size_t)col * p.lda] = S.side_vals[s][cc];
    }
    cl.sync();
  }

  // ---- write the slab back ------------------------------------------------
  for (int cc = 0; cc < w; ++cc) {
    T* col = p.a + (size_t)(p.c0 + cc) * p.lda + (p.c0 + rb);
    for (int r = tid; r < nr; r += kPanelThreads) col[r] = tile[r * LD + cc];
  }
  for (int r = tid; r < nr; r += kPanelThreads) p.lab[p.c0 + rb + r] = lab_s[r];
}

// ---------------------------------------------------------------------------
// K1r: leaf panel LU with register-resident rows (m <= 16 * 256 * RPT).
//
// Same cluster decomposition and st.async pivot exchange as K1, but every
// thread keeps RPT whole rows of the slab (W entries each) in registers for
// the whole panel, so the per-column update is W independent multiply-
// subtracts per row with no shared-memory round trips, and the column loop is
// unrolled (register indices are static). Per column: candidate from
// registers -> warp shuffle -> one CTA barrier -> warp 0 sends the CTA record
// -> every thread waits on its CTA's mbarrier -> swap / divide / update.
//
// Division: the multiplier is the correctly rounded quotient a/d
// (mod.rs:154). With y = RN(1/d) computed once per column, q = RN(a*y) is
// within one ulp of a/d, the remainder a - q*d is exact under an FMA, and
// RN(q + (a - q*d)*y) is the correctly rounded quotient (Markstein's
// theorem), as long as nothing over- or underflows; entries and pivots outside
// [2^-500, 2^500] in magnitude, zeros and non-finite values take the plain
// IEEE division instead.
// ---------------------------------------------------------------------------
constexpr int kPanelRThreads = 256;

template <typename T, int W, int RPT, bool EXACT>
__global__ void __launch_bounds__(kPanelRThreads, 1) panel_reg_kernel(PanelArgs<T> p) {
  using Rec = PanelRec<T, W>;
  constexpr int NT = kPanelRThreads;
  constexpr int NW = NT / 32;
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
  const int step_bytes = C * Rec::kBytes + Rec::kDiagBytes;

  __shared__ unsigned long long mbar[2];
  __shared__ __align__(16) unsigned long long rec[2][kPanelMaxC][Rec::kWords];
  __shared__ __align__(16) unsigned long long diag[2][Rec::kDiagWords];
  __shared__ double cand_key[2][NW];
  __shared__ int cand_idx[2][NW];
  __shared__ int cand_lab[2][NW][2];
  __shared__ T stage[2][NW][W];
  __shared__ T dstage[2][W];
  __shared__ int dlab[2][2];
  __shared__ T side_vals[4 * kPanelMaxW][kSideCols];
  __shared__ int side_rows[4 * kPanelMaxW];
  __shared__ int side_src[4 * kPanelMaxW];
  __shared__ int side_cnt;

  // ---- rows into registers ----------------------------------------------
  T v[RPT][W];
  int lab[RPT], loc[RPT];
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int r = tid + k * NT;  // local row
    const bool in = r < nr;
    const int gr = p.c0 + rb + r;
#pragma unroll
    for (int cc = 0; cc < W; ++cc)
      v[k][cc] = (in && cc < w) ? p.a[(size_t)gr + (size_t)(p.c0 + cc) * p.lda] : T(0);
    lab[k] = in ? (p.first_leaf ? gr : p.lab[gr]) : 0;
    loc[k] = gr;
  }
  if (tid == 0 && C > 1) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_arm(smem_u32(&mbar[0]), step_bytes);
    if (w > 1) mbar_arm(smem_u32(&mbar[1]), step_bytes);
  }
  cl.sync();

  const uint32_t rec_base = smem_u32(&rec[0][0][0]);
  const uint32_t diag_base = smem_u32(&diag[0][0]);
  const uint32_t bar_base = smem_u32(&mbar[0]);
  bool ok_wait = true;

  // The column loop stays rolled: one copy of its code serves every column
  // (an unrolled loop does not fit the instruction cache). Register entries
  // are addressed with static indices under the predicates c == j / c > j.
#pragma unroll 1
  for (int j = 0; j < w; ++j) {
    {
      const int par = j & 1;
      // ---- 1. candidate for column j from the registers ---------------------
      double bk = -CUDART_INF;
      int bi = INT_MAX;
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int r = tid + k * NT;
        T vj = v[k][0];
#pragma unroll
        for (int cc = 1; cc < W; ++cc)
          if (cc == j) vj = v[k][cc];
        if (r < nr && rb + r >= j) {
          const double key = pivot_key((double)vj, rb + r == j);
          if (key > bk) { bk = key; bi = rb + r; }
        }
      }
      // owner of row j stages it (and its labels) for the diagonal record
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        if (tid + k * NT < nr && rb + tid + k * NT == j) {
#pragma unroll
          for (int cc = 0; cc < W; ++cc) dstage[par][cc] = v[k][cc];
          dlab[par][0] = lab[k];
          dlab[par][1] = loc[k];
        }
      }
      double wk = bk;
      int wi = bi;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ok = __shfl_xor_sync(0xffffffffu, wk, off);
        const int oi = __shfl_xor_sync(0xffffffffu, wi, off);
        keyidx_combine(wk, wi, ok, oi);
      }
      // the lane holding the warp's best row stages it
      if (wi != INT_MAX) {
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
          if (tid + k * NT < nr && rb + tid + k * NT == wi) {
            cand_key[par][warp] = wk;
            cand_idx[par][warp] = wi;
            cand_lab[par][warp][0] = lab[k];
            cand_lab[par][warp][1] = loc[k];
#pragma unroll
            for (int cc = 0; cc < W; ++cc) stage[par][warp][cc] = v[k][cc];
          }
        }
      } else if (lane == 0) {
        cand_key[par][warp] = -CUDART_INF;
        cand_idx[par][warp] = INT_MAX;
      }
      __syncthreads();
      // ---- 2. the CTA record (and row j) to every mailbox: each of the first
      // min(NW, C) warps forms the record and sends it to the CTAs t with
      // t % NW == warp (C == 1: warp 0 into the own mailbox) -------------------
      if (warp < (C > 1 ? min(NW, C) : 1)) {
        double ck = -CUDART_INF;
        int ci = INT_MAX, cw = 0;
        if (lane < NW) { ck = cand_key[par][lane]; ci = cand_idx[par][lane]; cw = lane; }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const double ok = __shfl_xor_sync(0xffffffffu, ck, off);
          const int oi = __shfl_xor_sync(0xffffffffu, ci, off);
          const int ow = __shfl_xor_sync(0xffffffffu, cw, off);
          if (ok > ck || (ok == ck && oi < ci)) { ck = ok; ci = oi; cw = ow; }
        }
        const bool have = ci != INT_MAX;
        const T* crow = &stage[par][cw][0];
        const bool own_j = j >= rb && j < re;
        // lane kw builds word kw of the record in a register and stores it
        // into slot q of its CTAs' mailboxes with st.async (each 8-byte store
        // completes on that CTA's mbarrier); C == 1: straight into the own
        // mailbox. No staging in shared memory, no proxy fence, no bulk copy.
        const uint32_t bar_par = bar_base + 8u * par;
        for (int kw = lane; kw < Rec::kWords; kw += 32) {
          unsigned long long val = 0;
          if (kw == 0) val = (unsigned long long)__double_as_longlong(ck);
          else if (kw == 1) val = pack_ii(ci, have ? cand_lab[par][cw][0] : 0);
          else if (kw == 2) val = pack_ii(have ? cand_lab[par][cw][1] : 0, 0);
          else if (kw < 3 + Rec::kRowWords) val = row_word<T, W>(crow, kw - 3);
          if (C > 1) {
            const uint32_t la = rec_base + 8u * (uint32_t)((par * kPanelMaxC + q) * Rec::kWords + kw);
            for (int t = warp; t < C; t += NW) st_async_b64(mapa_u32(la, t), val, mapa_u32(bar_par, t));
          } else {
            rec[par][0][kw] = val;
          }
        }
        if (own_j) {
          for (int kw = lane; kw < Rec::kDiagWords; kw += 32) {
            unsigned long long val = 0;
            if (kw == 0) val = pack_ii(dlab[par][0], dlab[par][1]);
            else if (kw < 1 + Rec::kRowWords) val = row_word<T, W>(&dstage[par][0], kw - 1);
            if (C > 1) {
              const uint32_t ld = diag_base + 8u * (uint32_t)(par * Rec::kDiagWords + kw);
              for (int t = warp; t < C; t += NW) st_async_b64(mapa_u32(ld, t), val, mapa_u32(bar_par, t));
            } else {
              diag[par][kw] = val;
            }
          }
        }
      }
      // ---- 3. wait for this column's records; every warp picks the winner ---
      if (C == 1) {
        __syncthreads();
      } else {
        if (ok_wait && !mbar_wait(bar_base + 8u * par, (j >> 1) & 1)) {
          ok_wait = false;
          atomicExch(&p.status->timeout, 1);
        }
        if (tid == 0 && j + 2 < w) mbar_arm(bar_base + 8u * par, step_bytes);
      }
      double xk = -CUDART_INF;
      int xi = INT_MAX, xs = 0;
      if (lane < C) {
        xk = __longlong_as_double((long long)rec[par][lane][0]);
        xi = (int)(unsigned)(rec[par][lane][1] & 0xffffffffu);
        xs = lane;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ok = __shfl_xor_sync(0xffffffffu, xk, off);
        const int oi = __shfl_xor_sync(0xffffffffu, xi, off);
        const int os = __shfl_xor_sync(0xffffffffu, xs, off);
        if (ok > xk || (ok == xk && oi < xi)) { xk = ok; xi = oi; xs = os; }
      }
      const int pr = xi;  // winning panel row (>= j)
      const int ps = xs;  // CTA that sent it
      T u[W];
#pragma unroll
      for (int cc = 0; cc < W; ++cc) u[cc] = rec_entry<T>(&rec[par][ps][3], cc);
      const T d = rec_entry<T>(&rec[par][ps][3], j);
      // ---- 4. swap rows j and pr (registers of their owners) ----------------
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int r = tid + k * NT;
        if (r < nr) {
          if (rb + r == j) {
#pragma unroll
            for (int cc = 0; cc < W; ++cc) v[k][cc] = u[cc];
            lab[k] = (int)(unsigned)(rec[par][ps][1] >> 32);
            loc[k] = (int)(unsigned)(rec[par][ps][2] & 0xffffffffu);
          } else if (rb + r == pr) {
#pragma unroll
            for (int cc = 0; cc < W; ++cc) v[k][cc] = rec_entry<T>(&diag[par][1], cc);
            lab[k] = (int)(unsigned)(diag[par][0] & 0xffffffffu);
            loc[k] = (int)(unsigned)(diag[par][0] >> 32);
          }
        }
      }
      if (tid == 0 && q == 0) {
        p.ipiv[p.c0 + j] = p.c0 + pr;
        if (fabs((double)d) <= 0.0) atomicMin(&p.status->singular_col, p.c0 + j);
      }
      // ---- 5. divide and update the rows below j -----------------------------
      const bool fast = div_fast_ok(d);
      const T y = fast ? rcp_rn(d) : T(1);
      T l[RPT];
      bool fix = false;
      T av[RPT];
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        av[k] = v[k][0];
#pragma unroll
        for (int cc = 1; cc < W; ++cc)
          if (cc == j) av[k] = v[k][cc];
        const T qv = mul_rn(av[k], y);
        l[k] = fma_rn(fma_rn(-qv, d, av[k]), y, qv);
        fix |= !(fast && div_fast_ok(av[k])) && (tid + k * NT < nr) && (rb + tid + k * NT > j);
      }
      if (fix) {  // zeros, non-finite values, extreme exponents: plain IEEE division
#pragma unroll
        for (int k = 0; k < RPT; ++k)
          if (!(fast && div_fast_ok(av[k]))) l[k] = div_rn(av[k], d);
      }
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int r = tid + k * NT;
        if (r < nr && rb + r > j) {
#pragma unroll
          for (int cc = 0; cc < W; ++cc) {
            if (cc == j) v[k][cc] = l[k];
            else if (cc > j) v[k][cc] = msub<EXACT>(v[k][cc], l[k], u[cc]);
          }
        }
      }
    }
  }
  cl.sync();  // every record consumed; no DSMEM access outlives its owner

  // ---- swap the block-panel's other columns by this leaf's interchanges -----
  if (tid == 0) side_cnt = 0;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int r = tid + k * NT;
    if (r < nr && loc[k] != p.c0 + rb + r) {
      const int s = atomicAdd(&side_cnt, 1);
      if (s < 4 * kPanelMaxW) { side_rows[s] = r; side_src[s] = loc[k]; }
    }
  }
  __syncthreads();
  const int n_side = min(side_cnt, 4 * kPanelMaxW);
  const int side_w = (p.kb1 - p.kb0) - w;
  for (int cbase = 0; cbase < side_w; cbase += kSideCols) {
    const int ncol = min(kSideCols, side_w - cbase);
    for (int idx = tid; idx < n_side * kSideCols; idx += NT) {
      const int s = idx / kSideCols, cc = idx % kSideCols;
      if (cc >= ncol) continue;
      int col = p.kb0 + cbase + cc;
      if (col >= p.c0) col += w;
      side_vals[s][cc] = p.a[(size_t)side_src[s] + (size_t)col * p.lda];
    }
    cl.sync();
    for (int idx = tid; idx < n_side * kSideCols; idx += NT) {
      const int s = idx / kSideCols, cc = idx % kSideCols;
      if (cc >= ncol) continue;
      int col = p.kb0 + cbase + cc;
      if (col >= p.c0) col += w;
      p.a[(size_t)(p.c0 + rb + side_rows[s]) + (size_t)col * p.lda] = side_vals[s][cc];
    }
    cl.sync();
  }

  // ---- registers back to the matrix -------------------------------------
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int r = tid + k * NT;
    if (r < nr) {
      const int gr = p.c0 + rb + r;
#pragma unroll
      for (int cc = 0; cc < W; ++cc)
        if (cc < w) p.a[(size_t)gr + (size_t)(p.c0 + cc) * p.lda] = v[k][cc];
      p.lab[gr] = lab[k];
    }
  }
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
    T* a, int lda, int n, int cb, int ce, int k0, int kb, const int* lab, int* perm, int* perm_tmp) {
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
  // columns of the window [cb, ce) outside the block [k0, k0 + kb)
  const int n_before = max(0, min(ce, k0) - cb);
  const int after0 = max(cb, k0 + kb);
  const int n_out = n_before + max(0, ce - after0);
  constexpr int kPer = kSwapMaxMoves / 32;
  for (int cidx = gwarp; cidx < n_out; cidx += warps_total) {
    const int col = cidx < n_before ? cb + cidx : after0 + (cidx - n_before);
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
// k = r0 .. i-1 in that order (one rounded multiply-subtract each in the
// exact form), the reference's order for those entries. No block barrier
// inside: L11 (kb <= 128) staged in shared memory, each warp owns
// CPW whole columns with lane l holding rows l, l + 32, ... in
// registers; step k broadcasts x_k from its owner lane by a shuffle.
// ---------------------------------------------------------------------------
constexpr int kTrsmThreads = 256;
// CPW columns per warp: 8 for wide right-hand sides, 2 for narrow ones (more
// CTAs and a shorter per-step chain when only a block's columns are solved).
template <typename T, bool EXACT, int RPT, int CPW>
__global__ void __launch_bounds__(kTrsmThreads, 1) trsm_lower_unit_reg_kernel(T* a, int lda, int r0, int kb, int cb,
                                                                           int ce) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* L = reinterpret_cast<T*>(smem_raw);  // kb x kb, column-major
  constexpr int kWarpCols = CPW;
  constexpr int kCtaCols = CPW * (kTrsmThreads / 32);
  const int c_first = cb + blockIdx.x * kCtaCols;
  const int ncol = min(kCtaCols, ce - c_first);
  if (ncol <= 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x[kWarpCols][RPT];
#pragma unroll
  for (int c = 0; c < kWarpCols; ++c) {
    const int cc = warp * kWarpCols + c;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int i = lane + 32 * r;
      x[c][r] = (cc < ncol && i < kb) ? a[(size_t)(r0 + i) + (size_t)(c_first + cc) * lda] : T(0);
    }
  }
  // L's strictly lower part (the rest is never read), kBatch loads in flight
  // per thread before any is stored
  constexpr int kBatch = 16;
  const int total = kb * kb;
  for (int base = threadIdx.x; base < total; base += kTrsmThreads * kBatch) {
    T tmp[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int idx = base + u * kTrsmThreads;
      const int i = idx % kb, k = idx / kb;
      tmp[u] = (idx < total && i > k) ? a[(size_t)(r0 + i) + (size_t)(r0 + k) * lda] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int idx = base + u * kTrsmThreads;
      if (idx < total) L[idx] = tmp[u];
    }
  }
  __syncthreads();
  for (int k = 0; k + 1 < kb; ++k) {
    const int owner = k & 31, rk = k >> 5;
    T u[kWarpCols];
#pragma unroll
    for (int c = 0; c < kWarpCols; ++c) {
      T xv = x[c][0];
#pragma unroll
      for (int r = 1; r < RPT; ++r)
        if (r == rk) xv = x[c][r];
      u[c] = __shfl_sync(0xffffffffu, xv, owner);
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int i = lane + 32 * r;
      if (i > k && i < kb) {
        const T l = L[i + (size_t)k * kb];
#pragma unroll
        for (int c = 0; c < kWarpCols; ++c) x[c][r] = msub<EXACT>(x[c][r], l, u[c]);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < kWarpCols; ++c) {
    const int cc = warp * kWarpCols + c;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int i = lane + 32 * r;
      if (cc < ncol && i < kb) a[(size_t)(r0 + i) + (size_t)(c_first + cc) * lda] = x[c][r];
    }
  }
}

// ---------------------------------------------------------------------------
// K3i: the inverses of the diagonal blocks of packed LU factors, for the
// blocked many-right-hand-side solve (fused arithmetic). Block b = rows and
// columns [b kb, b kb + kb) (the last one may be short; its inverse is
// zero-padded to kb x kb): inv + b kb^2 <- T_bb^{-1}, column-major with
// leading dimension kb, T_bb unit lower (UPPER false) or upper. Grid: column
// groups x blocks. The K3 layout: T_bb (kb <= 128) in shared memory, each
// warp owns CPW columns of the identity with lane l holding rows l, l + 32,
// ... in registers; step k broadcasts row k from its owner lane (upper:
// x_k / u_kk, from the last row up).
// ---------------------------------------------------------------------------
template <typename T, bool UPPER, int RPT, int CPW>
__global__ void __launch_bounds__(kTrsmThreads, 1) tri_block_inverse_kernel(const T* lu, int lda, int n, int kb,
                                                                         T* inv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* M = reinterpret_cast<T*>(smem_raw);  // kb x kb, column-major
  constexpr int kCtaCols = CPW * (kTrsmThreads / 32);
  const int r0 = blockIdx.y * kb;
  const int bk = min(kb, n - r0);
  const int c_first = blockIdx.x * kCtaCols;
  if (c_first >= kb) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T v[CPW][RPT];
#pragma unroll
  for (int c = 0; c < CPW; ++c) {
    const int col = c_first + warp * CPW + c;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int i = lane + 32 * r;
      v[c][r] = (i == col && col < bk) ? T(1) : T(0);
    }
  }
  for (int idx = threadIdx.x; idx < kb * kb; idx += kTrsmThreads) {
    const int i = idx % kb, k = idx / kb;
    const bool keep = (i < bk && k < bk) && (UPPER ? i <= k : i > k);
    M[idx] = keep ? lu[(size_t)(r0 + i) + (size_t)(r0 + k) * lda] : T(0);
  }
  __syncthreads();
  if constexpr (!UPPER) {
    for (int k = 0; k + 1 < bk; ++k) {
      const int owner = k & 31, rk = k >> 5;
      T u[CPW];
#pragma unroll
      for (int c = 0; c < CPW; ++c) {
        T xv = v[c][0];
#pragma unroll
        for (int r = 1; r < RPT; ++r)
          if (r == rk) xv = v[c][r];
        u[c] = __shfl_sync(0xffffffffu, xv, owner);
      }
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        const int i = lane + 32 * r;
        if (i > k && i < bk) {
          const T l = M[i + (size_t)k * kb];
#pragma unroll
          for (int c = 0; c < CPW; ++c) v[c][r] = msub<false>(v[c][r], l, u[c]);
        }
      }
    }
  } else {
    for (int k = bk - 1; k >= 0; --k) {
      const int owner = k & 31, rk = k >> 5;
      const T d = M[k + (size_t)k * kb];
      T u[CPW];
#pragma unroll
      for (int c = 0; c < CPW; ++c) {
        T xv = v[c][0];
#pragma unroll
        for (int r = 1; r < RPT; ++r)
          if (r == rk) xv = v[c][r];
        if (lane == owner) {
          xv = xv / d;
#pragma unroll
          for (int r = 0; r < RPT; ++r)
            if (r == rk) v[c][r] = xv;
        }
        u[c] = __shfl_sync(0xffffffffu, xv, owner);
      }
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        const int i = lane + 32 * r;
        if (i < k) {
          const T m = M[i + (size_t)k * kb];
#pragma unroll
          for (int c = 0; c < CPW; ++c) v[c][r] = msub<false>(v[c][r], m, u[c]);
        }
      }
    }
  }
  T* out = inv + (size_t)blockIdx.y * kb * kb;
#pragma unroll
  for (int c = 0; c < CPW; ++c) {
    const int col = c_first + warp * CPW + c;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int i = lane + 32 * r;
      if (col < kb && i < kb) out[i + (size_t)col * kb] = v[c][r];
    }
  }
}

// ---------------------------------------------------------------------------
// K3b: one step of the blocked many-right-hand-side solve, for the block of
// rows [k0, k0 + kbe): every CTA forms X_new = T_bb^{-1} X[k0:k0+kbe, tile]
// (the block's inverse from K3i; CTA x = 0 stores it in Y), then updates its
// 128 rows of the rows not yet solved, X[rows, tile] -= T[rows, k0:k0+kbe]
// X_new (lower: the rows below the block; upper: the rows above). A tile of
// 128 rows x solve_cols<T>() right-hand sides per CTA, the operands in
// shared memory (kSolveKb x kSolveKb of the factor, the block rows of X).
// Rows of X outside [k0, k0 + kbe) are touched only by the CTA that owns
// them, and X[k0:k0+kbe] is only read in a step, so the CTAs need no sync.
// ---------------------------------------------------------------------------
constexpr int kSolveKb = 128;
// right-hand sides per CTA: 32 in FP32 (two CTAs per SM), 64 in FP64 (one);
// a thread takes 8 rows x kSolveCols / 16 of them
template <typename T>
constexpr int solve_cols() { return sizeof(T) == 4 ? 32 : 64; }

template <typename T, bool UPPER>
__global__ void __launch_bounds__(256) block_solve_step_kernel(const T* __restrict__ lu, int lda, int n, int k0,
                                                               int kbe, const T* __restrict__ inv, T* x,
                                                               T* __restrict__ y, int nrhs) {
  constexpr int kSolveCols = solve_cols<T>(), kSolveTc = kSolveCols / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);  // [k][i], kSolveKb x kSolveKb
  T* Xs = As + kSolveKb * kSolveKb;        // [k][c], kSolveKb x kSolveCols
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int c0 = blockIdx.y * kSolveCols;
  const int nc = min(kSolveCols, nrhs - c0);
  const int ur0 = UPPER ? 0 : k0 + kbe, ur1 = UPPER ? k0 : n;
  const int rt = ur0 + blockIdx.x * kSolveKb;  // this CTA's first update row
  for (int e = tid; e < kSolveKb * kSolveKb; e += 256) {
    const int i = e % kSolveKb, k = e / kSolveKb;
    As[e] = (i < kbe && k < kbe) ? inv[i + (size_t)k * kSolveKb] : T(0);
  }
  for (int e = tid; e < kSolveKb * kSolveCols; e += 256) {
    const int c = e % kSolveCols, k = e / kSolveCols;
    Xs[e] = (k < kbe && c < nc) ? x[(size_t)(k0 + k) + (size_t)(c0 + c) * n] : T(0);
  }
  __syncthreads();
  T acc[8][kSolveTc];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < kSolveTc; ++c) acc[r][c] = T(0);
  for (int k = 0; k < kbe; ++k) {
    T av[8], bv[kSolveTc];
#pragma unroll
    for (int r = 0; r < 8; ++r) av[r] = As[k * kSolveKb + tx + 16 * r];
#pragma unroll
    for (int c = 0; c < kSolveTc; ++c) bv[c] = Xs[k * kSolveCols + ty * kSolveTc + c];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int c = 0; c < kSolveTc; ++c) acc[r][c] = fma_rn(av[r], bv[c], acc[r][c]);
  }
  __syncthreads();  // every thread is done with X_old
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < kSolveTc; ++c) {
      const int i = tx + 16 * r, cc = ty * kSolveTc + c;
      Xs[i * kSolveCols + cc] = acc[r][c];
      if (blockIdx.x == 0 && i < kbe && cc < nc) y[(size_t)(k0 + i) + (size_t)(c0 + cc) * n] = acc[r][c];
    }
  if (rt >= ur1) return;  // no rows left to update (uniform over the CTA)
  for (int e = tid; e < kSolveKb * kSolveKb; e += 256) {
    const int i = e % kSolveKb, k = e / kSolveKb;
    As[e] = (rt + i < ur1 && k < kbe) ? lu[(size_t)(rt + i) + (size_t)(k0 + k) * lda] : T(0);
  }
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < kSolveTc; ++c) {
      const int i = rt + tx + 16 * r, cc = ty * kSolveTc + c;
      acc[r][c] = (i < ur1 && cc < nc) ? x[(size_t)i + (size_t)(c0 + cc) * n] : T(0);
    }
  __syncthreads();
  for (int k = 0; k < kbe; ++k) {
    T av[8], bv[kSolveTc];
#pragma unroll
    for (int r = 0; r < 8; ++r) av[r] = As[k * kSolveKb + tx + 16 * r];
#pragma unroll
    for (int c = 0; c < kSolveTc; ++c) bv[c] = Xs[k * kSolveCols + ty * kSolveTc + c];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int c = 0; c < kSolveTc; ++c) acc[r][c] = msub<false>(acc[r][c], av[r], bv[c]);
  }
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < kSolveTc; ++c) {
      const int i = rt + tx + 16 * r, cc = ty * kSolveTc + c;
      if (i < ur1 && cc < nc) x[(size_t)i + (size_t)(c0 + cc) * n] = acc[r][c];
    }
}

// x[i, c] = b[perm[i], c] (the row interchanges of P, n x ncols)
template <typename T>
__global__ void gather_perm_rows_kernel(const T* __restrict__ b, int ldb, const int* __restrict__ perm, int n,
                                        int ncols, T* __restrict__ x, int ldx) {
  const size_t cnt = (size_t)n * ncols;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    x[(size_t)i + (size_t)c * ldx] = b[(size_t)perm[i] + (size_t)c * ldb];
  }
}

// ---------------------------------------------------------------------------
// K4 (CUDA-core form): C -= A * B with C M x N, A M x K, B K x N, all
// column-major. Each thread owns an 8 x 8 block of C in registers, loads it
// once, applies the K terms in increasing k (EXACT: rounded product then
// rounded difference, the reference's per-entry sequence), and stores it once.
// 128 x BN CTA tile (BN = 128: 256 threads, one CTA per SM; BN = 64: 128
// threads, two CTAs per SM, so one tile's C load and store overlap the
// other's arithmetic), K staged through shared memory 8 at a time with
// register double buffering. Out-of-range A rows / B columns / k are zero,
// which leaves every in-range entry unchanged bit for bit (x - 0*0 = x).
// ---------------------------------------------------------------------------
constexpr int kGemmBM = 128, kGemmBK = 8;

template <typename T, bool EXACT, int BN>
__global__ void __launch_bounds__(2 * BN, BN == 64 ? 2 : 1) gemm_sub_kernel(
    int M, int N, int K, const T* __restrict__ A, int lda, const T* __restrict__ B, int ldb,
    T* __restrict__ Cm, int ldc) {
  constexpr int kThreads = 2 * BN, kHalf = BN / 2, kAPer = kGemmBK * kGemmBM / kThreads,
                kBPer = kGemmBK * BN / kThreads;
  __shared__ __align__(16) T As[2][kGemmBK][kGemmBM];
  __shared__ __align__(16) T Bs[2][kGemmBK][BN + 2];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * BN;

  T acc[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int mi = m0 + (r >> 2) * 64 + tx * 4 + (r & 3);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int nj = n0 + (c >> 2) * kHalf + ty * 4 + (c & 3);
      acc[r][c] = (mi < M && nj < N) ? Cm[(size_t)mi + (size_t)nj * ldc] : T(0);
    }
  }

  // loader mapping: the A chunk is kGemmBK x 128 (k-major in smem), the B
  // chunk kGemmBK x BN
  T ra[kAPer], rb[kBPer];
  auto load_chunk = [&](int k0) {
#pragma unroll
    for (int t = 0; t < kAPer; ++t) {
      const int idx = tid + t * kThreads;
      const int mm = idx & 127, kk = idx >> 7;
      const int gm = m0 + mm, gk = k0 + kk;
      ra[t] = (gm < M && gk < K) ? A[(size_t)gm + (size_t)gk * lda] : T(0);
    }
#pragma unroll
    for (int t = 0; t < kBPer; ++t) {
      const int idx = tid + t * kThreads;
      const int bk = idx & 7, bn = idx >> 3;
      const int gn = n0 + bn, gk2 = k0 + bk;
      rb[t] = (gn < N && gk2 < K) ? B[(size_t)gk2 + (size_t)gn * ldb] : T(0);
    }
  };
  auto store_chunk = [&](int buf) {
#pragma unroll
    for (int t = 0; t < kAPer; ++t) {
      const int idx = tid + t * kThreads;
      As[buf][idx >> 7][idx & 127] = ra[t];
    }
#pragma unroll
    for (int t = 0; t < kBPer; ++t) {
      const int idx = tid + t * kThreads;
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
      for (int c = 0; c < 8; ++c) bf[c] = Bs[buf][kk][(c >> 2) * kHalf + ty * 4 + (c & 3)];
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
      const int nj = n0 + (c >> 2) * kHalf + ty * 4 + (c & 3);
      if (mi < M && nj < N) Cm[(size_t)mi + (size_t)nj * ldc] = acc[r][c];
    }
  }
}

// ---------------------------------------------------------------------------
// K4a: the same update (128 x 64 tile, 128 threads, 8 x 8 per thread, each
// entry's terms in increasing k) with A and B staged by cp.async through a
// three-stage shared-memory ring instead of registers: no prefetch registers,
// and the loads of chunk c + 2 run while chunk c is multiplied. Element-wise
// copies (any leading dimension and offset); out-of-range elements are
// zero-filled, which leaves every in-range entry unchanged bit for bit.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void cp_async_elem_zfill(T* dst, const T* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
  }
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr int kGemmAsyncStages = 3;

template <typename T, bool EXACT>
__global__ void __launch_bounds__(128, 2) gemm_sub_async_kernel(int M, int N, int K, const T* __restrict__ A, int lda,
                                                                const T* __restrict__ B, int ldb, T* __restrict__ Cm,
                                                                int ldc) {
  constexpr int kBN = 64, kHalf = kBN / 2, kThreads = 128, kBS = kBN + 2;
  constexpr int kStage = kGemmBK * kGemmBM + kGemmBK * kBS;
  __shared__ __align__(16) T smem[kGemmAsyncStages * kStage];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * kBN;

  auto load_stage = [&](int stage, int k0) {
    T* As = smem + stage * kStage;  // [k][m]
    T* Bs = As + kGemmBK * kGemmBM;  // [k][n], padded rows
#pragma unroll
    for (int r = 0; r < kGemmBK * kGemmBM / kThreads; ++r) {
      const int e = tid + r * kThreads;
      const int mm = e & (kGemmBM - 1), kk = e / kGemmBM;
      const int gm = m0 + mm, gk = k0 + kk;
      const bool ok = gm < M && gk < K;
      cp_async_elem_zfill(As + kk * kGemmBM + mm, ok ? A + (size_t)gm + (size_t)gk * lda : A, ok);
    }
#pragma unroll
    for (int r = 0; r < kGemmBK * kBN / kThreads; ++r) {
      const int e = tid + r * kThreads;
      const int kk = e % kGemmBK, nn = e / kGemmBK;
      const int gn = n0 + nn, gk = k0 + kk;
      const bool ok = gn < N && gk < K;
      cp_async_elem_zfill(Bs + kk * kBS + nn, ok ? B + (size_t)gk + (size_t)gn * ldb : B, ok);
    }
  };

  const int nch = (K + kGemmBK - 1) / kGemmBK;
#pragma unroll
  for (int st = 0; st < kGemmAsyncStages - 1; ++st) {
    if (st < nch) load_stage(st, st * kGemmBK);
    cp_async_commit_group();
  }
  T acc[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int mi = m0 + (r >> 2) * 64 + tx * 4 + (r & 3);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int nj = n0 + (c >> 2) * kHalf + ty * 4 + (c & 3);
      acc[r][c] = (mi < M && nj < N) ? Cm[(size_t)mi + (size_t)nj * ldc] : T(0);
    }
  }
  for (int ch = 0; ch < nch; ++ch) {
    cp_async_wait_group<kGemmAsyncStages - 2>();  // chunk ch has landed
    __syncthreads();  // ... for every thread, and chunk ch - 1's stage is free
    if (ch + kGemmAsyncStages - 1 < nch)
      load_stage((ch + kGemmAsyncStages - 1) % kGemmAsyncStages, (ch + kGemmAsyncStages - 1) * kGemmBK);
    cp_async_commit_group();
    const T* As = smem + (ch % kGemmAsyncStages) * kStage;
    const T* Bs = As + kGemmBK * kGemmBM;
#pragma unroll
    for (int kk = 0; kk < kGemmBK; ++kk) {
      T af[8], bf[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) af[r] = As[kk * kGemmBM + (r >> 2) * 64 + tx * 4 + (r & 3)];
#pragma unroll
      for (int c = 0; c < 8; ++c) bf[c] = Bs[kk * kBS + (c >> 2) * kHalf + ty * 4 + (c & 3)];
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = msub<EXACT>(acc[r][c], af[r], bf[c]);
    }
  }
  cp_async_wait_group<0>();
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int mi = m0 + (r >> 2) * 64 + tx * 4 + (r & 3);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int nj = n0 + (c >> 2) * kHalf + ty * 4 + (c & 3);
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

// The diagonal blocks are staged in shared memory (Ls, kSolveB x kSolveB)
// before their sequential sweep, so the sweep never waits on global memory.
template <typename T, bool EXACT>
__device__ void solve_diag_block_lower(const T* lu, int lda, T* xc, int j0, int bs, T* xs, T* Ls) {
  // unit lower triangle of rows/cols [j0, j0+bs)
  for (int idx = threadIdx.x; idx < bs * bs; idx += blockDim.x) {
    const int i = idx % bs, k = idx / bs;
    Ls[i + k * kSolveB] = lu[(size_t)(j0 + i) + (size_t)(j0 + k) * lda];
  }
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xs[i] = xc[j0 + i];
  __syncthreads();
  if (threadIdx.x < 32) {
    // one warp: lanes own rows i = lane, lane+32; step k broadcasts x_k
    for (int k = 0; k + 1 < bs; ++k) {
      const T u = xs[k];
      for (int i = k + 1 + threadIdx.x; i < bs; i += 32) xs[i] = msub<EXACT>(xs[i], Ls[i + k * kSolveB], u);
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xc[j0 + i] = xs[i];
}

template <typename T, bool EXACT>
__device__ void solve_diag_block_upper(const T* lu, int lda, T* xc, int j0, int bs, T* xs, T* Ls) {
  for (int idx = threadIdx.x; idx < bs * bs; idx += blockDim.x) {
    const int i = idx % bs, k = idx / bs;
    Ls[i + k * kSolveB] = lu[(size_t)(j0 + i) + (size_t)(j0 + k) * lda];
  }
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xs[i] = xc[j0 + i];
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int k = bs - 1; k >= 0; --k) {
      if (threadIdx.x == 0) xs[k] = div_rn(xs[k], Ls[k + k * kSolveB]);
      __syncwarp();
      const T u = xs[k];
      for (int i = threadIdx.x; i < k; i += 32) xs[i] = msub<EXACT>(xs[i], Ls[i + k * kSolveB], u);
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xc[j0 + i] = xs[i];
}

// Forward: rows [j0+bs, n) take block [j0, j0+bs)'s terms. CTA 0 owns the next
// block's rows and then solves its triangle. j0 = -bs means "only solve block 0".
template <typename T, bool EXACT>
__global__ void __launch_bounds__(kSolveThreads) solve_fwd_kernel(
    const T* __restrict__ lu, int lda, int n, T* __restrict__ x, int ldx, int j0, int bs) {
  __shared__ T xb[kSolveB];
  __shared__ T xs[kSolveB];
  __shared__ T Ls[kSolveB * kSolveB];
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
    solve_diag_block_lower<T, EXACT>(lu, lda, xc, j1, nb1, xs, Ls);
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
  __shared__ T Ls[kSolveB * kSolveB];
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
    solve_diag_block_upper<T, EXACT>(lu, lda, xc, jp, bp, xs, Ls);
  }
}

}  // namespace alg
