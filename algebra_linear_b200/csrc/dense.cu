// Host-side schedule of the blocked right-looking LU (sm_100a) and the
// dense C entry points.
//
// Schedule for an m x nc matrix (m >= nc), block-panel width nb, leaf nbl:
//   for each block-panel [k0, k0+kb):
//     for each leaf [c0, c0+w) inside it:
//       K1 panel_cluster_kernel   : factor rows [c0, m) of the leaf columns,
//                                   swap the block-panel's other columns
//       K3 trsm (w rows)          : U of the leaf's rows, block-panel columns right of it
//       K4 gemm (k = w)           : rows below, block-panel columns right of the leaf
//     K2 laswp_outside            : the block-panel's interchanges, all other columns
//     K3 trsm (kb rows)           : U12 = L11^{-1} A12
//     K4 gemm (k = kb)            : A22 -= L21 U12
// Every entry sees its rank-1 terms in increasing pivot order, so with the
// EXACT arithmetic the result equals the reference's kij loop
// (src/lapack/mod.rs:112-163) bit for bit.
#include <algorithm>
#include <cstdlib>
#include <climits>
#include <cstring>
#include <type_traits>
#include <vector>

#include "dense.cuh"
#include "dense_kernels.cuh"

namespace alg {

LuPlan default_plan(int n, int elem_bytes) {
  LuPlan p;
  p.nb = n >= 8192 ? 128 : 64;  // deeper updates pay off once the update GEMMs dominate
  p.nbl = elem_bytes == 8 ? 16 : 32;
  if (const char* e = std::getenv("ALG_NB")) p.nb = std::max(16, std::atoi(e));
  if (const char* e = std::getenv("ALG_NBL")) p.nbl = std::max(1, std::min(kPanelMaxW, std::atoi(e)));
  (void)n;
  return p;
}

namespace {

// Rows per CTA the cluster size aims for: fewer rows per CTA shorten each
// column step, more CTAs lengthen the cluster barrier. ALG_PANEL_ROWS
// overrides it (tuning). 256 (one register row per thread up to 4 096 rows)
// measured 171.4 ms against 175.4 ms for 512 (fp64_fma, n = 16384) and
// 229 ms against 264 ms per 48^3 sparse round.
int panel_target_rows() {
  static int v = [] {
    const char* e = std::getenv("ALG_PANEL_ROWS");
    return e ? std::max(16, std::atoi(e)) : 256;
  }();
  return v;
}

template <typename T, int W, bool EXACT>
int launch_panel_w(alg_ctx* ctx, const PanelArgs<T>& args) {
  const int m = args.n - args.c0;
  constexpr size_t kMaxSmem = 220 * 1024;
  int C = 1;
  while (C < kPanelMaxC && (m + C - 1) / C > panel_target_rows()) C *= 2;
  size_t smem = panel_smem_bytes<T, W>((m + C - 1) / C);
  while (smem > kMaxSmem && C < kPanelMaxC) {
    C *= 2;
    smem = panel_smem_bytes<T, W>((m + C - 1) / C);
  }
  if (smem > kMaxSmem) return ALG_BAD_SHAPE;  // panel too tall for one cluster
  // kernel attributes set once per process (a thread-safe static initializer)
  static const cudaError_t configured = [] {
    cudaError_t e = cudaFuncSetAttribute(panel_cluster_kernel<T, W, EXACT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(panel_cluster_kernel<T, W, EXACT>, cudaFuncAttributeNonPortableClusterSizeAllowed,
                               1);
    return e;
  }();
  ALG_CUDA_TRY(configured);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(kPanelThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  double pflops = 0;
  for (int j = 0; j < args.w; ++j) pflops += double(m - j - 1) * (1.0 + 2.0 * (args.w - j - 1));
  const int tok = prof_begin(ctx, ALG_K_PANEL);
  ALG_CUDA_TRY(cudaLaunchKernelEx(&cfg, panel_cluster_kernel<T, W, EXACT>, args));
  count_launches();
  prof_end(ctx, tok, pflops, 2.0 * sizeof(T) * m * args.w);
  return ALG_OK;
}

template <typename T, int W, int RPT, bool EXACT>
int launch_panel_reg(alg_ctx* ctx, const PanelArgs<T>& args, int C) {
  static const cudaError_t configured =
      cudaFuncSetAttribute(panel_reg_kernel<T, W, RPT, EXACT>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  ALG_CUDA_TRY(configured);
  const int m = args.n - args.c0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(kPanelRThreads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  double pflops = 0;
  for (int j = 0; j < args.w; ++j) pflops += double(m - j - 1) * (1.0 + 2.0 * (args.w - j - 1));
  const int tok = prof_begin(ctx, ALG_K_PANEL);
  ALG_CUDA_TRY(cudaLaunchKernelEx(&cfg, panel_reg_kernel<T, W, RPT, EXACT>, args));
  count_launches();
  prof_end(ctx, tok, pflops, 2.0 * sizeof(T) * m * args.w);
  return ALG_OK;
}

// Register-resident rows when a 16-CTA cluster can hold the panel's rows at
// up to four rows per thread (two for 32 double columns); the shared-memory
// slab kernel otherwise.
template <typename T, bool EXACT>
int launch_panel(alg_ctx* ctx, const PanelArgs<T>& args) {
  const int m = args.n - args.c0;
  const int max_rpt = (args.w > 16 && sizeof(T) == 8) ? 2 : 4;
  const int target = std::max(1, panel_target_rows());
  if (m <= kPanelMaxC * kPanelRThreads * max_rpt && !std::getenv("ALG_PANEL_SMEM")) {
    int C = 1;
    while (C < kPanelMaxC && (m + C - 1) / C > std::min(target, max_rpt * kPanelRThreads)) C *= 2;
    while (C < kPanelMaxC && (m + C - 1) / C > max_rpt * kPanelRThreads) C *= 2;
    const int R = (m + C - 1) / C;
    const int rpt = R <= kPanelRThreads ? 1 : (R <= 2 * kPanelRThreads ? 2 : 4);
    if (args.w <= 16) {
      if (rpt == 1) return launch_panel_reg<T, 16, 1, EXACT>(ctx, args, C);
      if (rpt == 2) return launch_panel_reg<T, 16, 2, EXACT>(ctx, args, C);
      return launch_panel_reg<T, 16, 4, EXACT>(ctx, args, C);
    }
    if (rpt == 1) return launch_panel_reg<T, 32, 1, EXACT>(ctx, args, C);
    if constexpr (sizeof(T) == 8) {
      return launch_panel_reg<T, 32, 2, EXACT>(ctx, args, C);
    } else {
      if (rpt == 2) return launch_panel_reg<T, 32, 2, EXACT>(ctx, args, C);
      return launch_panel_reg<T, 32, 4, EXACT>(ctx, args, C);
    }
  }
  if (args.w <= 16) return launch_panel_w<T, 16, EXACT>(ctx, args);
  return launch_panel_w<T, 32, EXACT>(ctx, args);
}

template <typename T, bool EXACT>
int launch_trsm_reg(alg_ctx* ctx, T* a, int lda, int r0, int kb, int cb, int ce) {
  const size_t smem = sizeof(T) * (size_t)kb * kb;
  // narrow right-hand sides (a block's columns on the look-ahead chain): two
  // columns per warp for more CTAs; wide ones: eight
  const bool narrow = ce - cb <= 1024;
  auto pick = [&](auto k1, auto k2, auto k4) { return kb <= 32 ? k1 : (kb <= 64 ? k2 : k4); };
  auto kern = narrow ? pick(trsm_lower_unit_reg_kernel<T, EXACT, 1, 2>, trsm_lower_unit_reg_kernel<T, EXACT, 2, 2>,
                            trsm_lower_unit_reg_kernel<T, EXACT, 4, 2>)
                     : pick(trsm_lower_unit_reg_kernel<T, EXACT, 1, 8>, trsm_lower_unit_reg_kernel<T, EXACT, 2, 8>,
                            trsm_lower_unit_reg_kernel<T, EXACT, 4, 8>);
  static const cudaError_t configured = [] {
    for (auto k : {trsm_lower_unit_reg_kernel<T, EXACT, 1, 2>, trsm_lower_unit_reg_kernel<T, EXACT, 2, 2>,
                   trsm_lower_unit_reg_kernel<T, EXACT, 4, 2>, trsm_lower_unit_reg_kernel<T, EXACT, 1, 8>,
                   trsm_lower_unit_reg_kernel<T, EXACT, 2, 8>, trsm_lower_unit_reg_kernel<T, EXACT, 4, 8>}) {
      const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }();
  ALG_CUDA_TRY(configured);
  const int cta_cols = (narrow ? 2 : 8) * (kTrsmThreads / 32);
  const int grid = (ce - cb + cta_cols - 1) / cta_cols;
  const int tok = prof_begin(ctx, ALG_K_TRSM);
  kern<<<grid, kTrsmThreads, smem, ctx->stream>>>(a, lda, r0, kb, cb, ce);
  count_launches();
  prof_end(ctx, tok, double(kb) * (kb - 1) * (ce - cb), sizeof(T) * (double(kb) * kb / 2 + 2.0 * kb * (ce - cb)));
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

// U12 = L11^-1 A12 for the kb x kb unit-lower block at (r0, r0) and columns
// [cb, ce): the register kernel for kb <= 128, else by 128-row diagonal
// blocks with the rows below updated by the trailing GEMM in between (every
// entry still takes its terms in increasing k, so the exact form is kept).
template <typename T, bool EXACT>
int launch_trsm(alg_ctx* ctx, T* a, int lda, int r0, int kb, int cb, int ce) {
  if (ce <= cb || kb <= 1) return ALG_OK;
  if (kb <= 128) return launch_trsm_reg<T, EXACT>(ctx, a, lda, r0, kb, cb, ce);
  for (int k0 = 0; k0 < kb; k0 += 128) {
    const int bk = std::min(128, kb - k0);
    ALG_TRY((launch_trsm_reg<T, EXACT>(ctx, a, lda, r0 + k0, bk, cb, ce)));
    const int below = kb - k0 - bk;
    if (below > 0)
      ALG_TRY((gemm_sub_dev<T, EXACT>(ctx, below, ce - cb, bk, a + (size_t)(r0 + k0 + bk) + (size_t)(r0 + k0) * lda,
                                      lda, a + (size_t)(r0 + k0) + (size_t)cb * lda, lda,
                                      a + (size_t)(r0 + k0 + bk) + (size_t)cb * lda, lda)));
  }
  return ALG_OK;
}

}  // namespace

// ALG_NO_DMMA=1 keeps the fused FP64 updates on the CUDA cores (for comparison).
bool dmma_disabled() {
  static const bool off = [] {
    const char* e = std::getenv("ALG_NO_DMMA");
    return e != nullptr && e[0] == '1';
  }();
  return off;
}

// ALG_GEMM_WIDE=1: the CUDA-core update's former 128 x 128 tiles (one CTA
// per SM) instead of 128 x 64 tiles two to an SM (for comparison).
bool gemm_wide_tiles() {
  static const bool v = [] {
    const char* e = std::getenv("ALG_GEMM_WIDE");
    return e != nullptr && e[0] == '1';
  }();
  return v;
}

template <typename T, bool EXACT>
int gemm_sub_dev(alg_ctx* ctx, int M, int N, int K, const T* A, int lda, const T* B, int ldb,
                 T* C, int ldc) {
  if (M <= 0 || N <= 0 || K <= 0) return ALG_OK;
  if constexpr (std::is_same<T, double>::value && !EXACT) {
    // the fused FP64 form runs on the FP64 tensor cores
    if (!dmma_disabled()) return gemm_dmma_sub_dev(ctx, M, N, K, A, lda, B, ldb, C, ldc);
  }
  const int tok = prof_begin(ctx, ALG_K_GEMM);
  // FP64 (the exact form's update) stages its operands by cp.async:
  // fp64_exact 296.2 ms against 308.7 ms at n = 16384; FP32 keeps the
  // register-prefetch form (mixed_fp32 133.8 ms against 138.3 ms).
  // ALG_GEMM_SYNC=1: the register-prefetch form for FP64 too (measurement switch)
  static const bool sync_env = [] {
    const char* e = std::getenv("ALG_GEMM_SYNC");
    return e != nullptr && e[0] == '1';
  }();
  const bool sync_form = sizeof(T) == 4 || sync_env;
  if (gemm_wide_tiles()) {
    dim3 grid((M + kGemmBM - 1) / kGemmBM, (N + 127) / 128);
    gemm_sub_kernel<T, EXACT, 128><<<grid, 256, 0, ctx->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  } else if (!sync_form) {
    dim3 grid((M + kGemmBM - 1) / kGemmBM, (N + 63) / 64);
    gemm_sub_async_kernel<T, EXACT><<<grid, 128, 0, ctx->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  } else {
    dim3 grid((M + kGemmBM - 1) / kGemmBM, (N + 63) / 64);
    gemm_sub_kernel<T, EXACT, 64><<<grid, 128, 0, ctx->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  }
  count_launches();
  prof_end(ctx, tok, 2.0 * M * N * K, sizeof(T) * (2.0 * M * N + double(M) * K + double(K) * N));
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

template <typename T, bool EXACT>
int lu_factor_dev(alg_ctx* ctx, T* a, int m, int nc, int lda, int* ipiv, int* perm,
                  const LuPlan& plan) {
  return lu_factor_partial_dev<T, EXACT>(ctx, a, m, nc, nc, lda, ipiv, perm, plan);
}

// ALG_LOOKAHEAD=0 factors block after block on one stream (for comparison).
bool lookahead_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("ALG_LOOKAHEAD");
    return !(e != nullptr && e[0] == '0');
  }();
  return on;
}

// SMs the look-ahead's wide tensor-core update leaves to the critical chain:
// its CTAs are persistent, so the chain's kernels (the tournament's
// cooperative launch needs up to 32 SMs at once) run only on SMs it does not
// hold. ALG_TC_RESERVE_SMS overrides the count (tuning).
int tc_reserve_sms() {
  static const int v = [] {
    const char* e = std::getenv("ALG_TC_RESERVE_SMS");
    return e ? std::max(0, std::atoi(e)) : 64;
  }();
  return v;
}

// ALG_INBLOCK_TC=1: the TF32x3 LU's in-block updates on the tensor cores
// instead of the FP32 CUDA cores. Measured slower at n = 16384 (72.4 vs 70.7
// ms per solve: the operand conversion and the persistent launch cost more
// than the narrow K = 32 update saves), so off by default.
bool inblock_tc_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("ALG_INBLOCK_TC");
    return e != nullptr && e[0] == '1';
  }();
  return on;
}

// Cap of the look-ahead chain's persistent tensor-core grids (0: none, every
// SM). Capping them at the SMs the wide update leaves free measured no
// better (72.4 vs 71.9 ms at n = 16384), so off by default; ALG_TC_CHAIN_CTAS
// sets it.
int tc_chain_ctas() {
  static const int v = [] {
    const char* e = std::getenv("ALG_TC_CHAIN_CTAS");
    return e ? std::max(0, std::atoi(e)) : 0;
  }();
  return v;
}

template <typename T, bool EXACT>
int lu_factor_partial_dev(alg_ctx* ctx, T* a, int m, int nc, int ntot, int lda, int* ipiv, int* perm,
                          const LuPlan& plan) {
  if (m < nc || nc < 0 || ntot < nc || lda < std::max(1, m)) return ALG_BAD_SHAPE;
  if (nc == 0) return ALG_OK;
  int* lab = nullptr;  // two label buffers: block k's swaps are applied while block k + 1 is factored
  int* perm_tmp = nullptr;
  ALG_TRY(ws_get(ctx, WS_LAB, 2 * sizeof(int) * (size_t)m, reinterpret_cast<void**>(&lab)));
  ALG_TRY(ws_get(ctx, WS_PERM_TMP, sizeof(int) * kSwapMaxMoves, reinterpret_cast<void**>(&perm_tmp)));
  void* tslu_ws = nullptr;
  if (std::is_same<T, float>::value && plan.tslu) {
    ALG_TRY(ws_get(ctx, WS_TSLU, tslu_scratch_bytes(), &tslu_ws));
    ALG_TRY(tslu_scratch_reset(ctx, tslu_ws));
  }
  if (perm != nullptr) {
    iota_kernel<<<std::min(1024, (m + 255) / 256), 256, 0, ctx->stream>>>(perm, m);
    count_launches();
    ALG_CUDA_TRY(cudaGetLastError());
  }
  // a block's interchanges move at most 2 nb rows, and the deferred-swap
  // kernel holds kSwapMaxMoves of them: wider blocks are cut to that
  const int nb = std::min(std::max(1, plan.nb), kSwapMaxMoves / 2);
  const int nbl = std::max(1, std::min(plan.nbl, kPanelMaxW));
  // persistent tensor-core grids: the wide update's cap (0: every SM) and the
  // look-ahead chain's (its launches must fit on the SMs the wide update
  // leaves free, or their extra CTAs wait for the wide update to retire)
  int wide_ctas = 0, chain_ctas = 0;

  // the leaf panels of block [k0, k0 + kb), with their in-block updates
  auto factor_block = [&](int k0, int kb, int* lb) -> int {
    for (int c0 = k0; c0 < k0 + kb; c0 += nbl) {
      const int w = std::min(nbl, k0 + kb - c0);
      PanelArgs<T> pa;
      pa.a = a;
      pa.lda = lda;
      pa.n = m;
      pa.c0 = c0;
      pa.w = w;
      pa.kb0 = k0;
      pa.kb1 = k0 + kb;
      pa.ipiv = ipiv;
      pa.lab = lb;
      pa.first_leaf = (c0 == k0) ? 1 : 0;
      pa.status = ctx->d_status;
      int prc = ALG_NOT_IMPLEMENTED;
      bool u12_done = false;  // the tournament's apply step also forms U12 of the block's trailing columns
      if constexpr (std::is_same<T, float>::value) {
        if (tslu_ws) {
          prc = tslu_panel(ctx, TsluArgs{a, lda, m, c0, w, k0, k0 + kb, ipiv, lb, pa.first_leaf, ctx->d_status},
                           tslu_ws);
          u12_done = prc == ALG_OK;
        }
      }
      if (prc == ALG_NOT_IMPLEMENTED) prc = launch_panel<T, EXACT>(ctx, pa);
      ALG_TRY(prc);
      const int cr = c0 + w;  // first column right of the leaf
      if (cr < k0 + kb) {
        if (!u12_done) ALG_TRY((launch_trsm<T, EXACT>(ctx, a, lda, c0, w, cr, k0 + kb)));
        bool tc_done = false;
        if constexpr (std::is_same<T, float>::value) {
          // the in-block update on the tensor cores too when their operands
          // keep FP32 accuracy (TF32x3; whole 128-byte K slices only)
          if (plan.tc_prec == ALG_PREC_TF32X3 && inblock_tc_enabled() && w % 32 == 0) {
            ALG_TRY(gemm_tc_sub_dev(ctx, plan.tc_prec, m - cr, k0 + kb - cr, w, a + (size_t)cr + (size_t)c0 * lda,
                                    lda, a + (size_t)c0 + (size_t)cr * lda, lda, a + (size_t)cr + (size_t)cr * lda,
                                    lda, WS_TC_CHAIN, chain_ctas));
            tc_done = true;
          }
        }
        if (!tc_done)
          ALG_TRY((gemm_sub_dev<T, EXACT>(ctx, m - cr, k0 + kb - cr, w, a + (size_t)cr + (size_t)c0 * lda, lda,
                                          a + (size_t)c0 + (size_t)cr * lda, lda,
                                          a + (size_t)cr + (size_t)cr * lda, lda)));
      }
    }
    return ALG_OK;
  };
  // block k's deferred interchanges on the columns of [cb, ce) outside the block
  auto swaps = [&](int k0, int kb, const int* lb, int cb, int ce, int* pm) -> int {
    const int n_out = std::max(0, std::min(ce, k0) - cb) + std::max(0, ce - std::max(cb, k0 + kb));
    if (n_out <= 0 && pm == nullptr) return ALG_OK;
    const int grid = std::max(1, std::min(4 * ctx->sm_count, (std::max(1, n_out) + 7) / 8));
    const int tok = prof_begin(ctx, ALG_K_LASWP);
    laswp_outside_kernel<T><<<grid, kSwapThreads, 0, ctx->stream>>>(a, lda, m, cb, ce, k0, kb, lb, pm, perm_tmp);
    count_launches();
    prof_end(ctx, tok, 0.0, 0.0);
    ALG_CUDA_TRY(cudaGetLastError());
    return ALG_OK;
  };
  // U12 and the trailing update of columns [cb, ce) by block [k0, k0 + kb);
  // wide: the update of the rest of the matrix (off the look-ahead chain);
  // the chain's narrow update converts its tensor-core operands in a
  // workspace of its own, since both can be in flight at once
  auto update = [&](int k0, int kb, int cb, int ce, bool wide) -> int {
    if (ce <= cb) return ALG_OK;
    const int kr = k0 + kb;
    ALG_TRY((launch_trsm<T, EXACT>(ctx, a, lda, k0, kb, cb, ce)));
    if (kr >= m) return ALG_OK;
    if constexpr (std::is_same<T, float>::value) {
      // the tensor-core kernel takes whole 128-byte K slices; a ragged last block stays in FP32
      if (plan.tc_prec >= 0 && kb % (plan.tc_prec == ALG_PREC_BF16 ? 64 : 32) == 0)
        return gemm_tc_sub_dev(ctx, plan.tc_prec, m - kr, ce - cb, kb, a + (size_t)kr + (size_t)k0 * lda, lda,
                               a + (size_t)k0 + (size_t)cb * lda, lda, a + (size_t)kr + (size_t)cb * lda, lda,
                               wide ? WS_KRYLOV : WS_TC_CHAIN, wide ? wide_ctas : chain_ctas);
    }
    return gemm_sub_dev<T, EXACT>(ctx, m - kr, ce - cb, kb, a + (size_t)kr + (size_t)k0 * lda, lda,
                                  a + (size_t)k0 + (size_t)cb * lda, lda, a + (size_t)kr + (size_t)cb * lda, lda);
  };

  const bool la = lookahead_enabled() && nc > nb;
  if (!la) {
    for (int k0 = 0; k0 < nc; k0 += nb) {
      const int kb = std::min(nb, nc - k0);
      ALG_TRY(factor_block(k0, kb, lab));
      ALG_TRY(swaps(k0, kb, lab, 0, ntot, perm));
      ALG_TRY(update(k0, kb, k0 + kb, ntot, true));
    }
    return ALG_OK;
  }

  // Look-ahead by one block: the high-priority stream runs the critical
  // chain (block k's swaps, U12 and update restricted to block k + 1's
  // columns, then block k + 1's panels) while the low-priority stream applies
  // block k to everything else; the two meet once per block.
  ALG_TRY(ctx_lookahead_streams(ctx));
  wide_ctas = std::max(1, ctx->sm_count - tc_reserve_sms());
  chain_ctas = tc_chain_ctas();
  cudaStream_t user = ctx->stream, sa = ctx->la_stream[0], sb = ctx->la_stream[1];
  cudaEvent_t ev_a = ctx->la_event[0], ev_b = ctx->la_event[1], ev_in = ctx->la_event[2];
  ALG_CUDA_TRY(cudaEventRecord(ev_in, user));
  ALG_CUDA_TRY(cudaStreamWaitEvent(sa, ev_in, 0));
  ALG_CUDA_TRY(cudaStreamWaitEvent(sb, ev_in, 0));
  int rc = ALG_OK;
  ctx->stream = sa;
  rc = factor_block(0, std::min(nb, nc), lab);
  for (int blk = 0, k0 = 0; rc == ALG_OK && k0 < nc; k0 += nb, ++blk) {
    const int kb = std::min(nb, nc - k0), kr = k0 + kb;
    const int kb1 = kr < nc ? std::min(nb, nc - kr) : 0;
    int* lk = lab + (size_t)(blk & 1) * m;
    int* ln = lab + (size_t)((blk + 1) & 1) * m;
    // the rest of the update needs block k factored
    if ((rc = cudaEventRecord(ev_a, sa) == cudaSuccess ? ALG_OK : ALG_CUDA_ERROR) != ALG_OK) break;
    if ((rc = cudaStreamWaitEvent(sb, ev_a, 0) == cudaSuccess ? ALG_OK : ALG_CUDA_ERROR) != ALG_OK) break;
    ctx->stream = sa;
    if (kb1 > 0) {
      if ((rc = swaps(k0, kb, lk, kr, kr + kb1, nullptr)) != ALG_OK) break;
      if ((rc = update(k0, kb, kr, kr + kb1, false)) != ALG_OK) break;
      if ((rc = factor_block(kr, kb1, ln)) != ALG_OK) break;
    }
    ctx->stream = sb;
    if ((rc = swaps(k0, kb, lk, 0, k0, perm)) != ALG_OK) break;
    if ((rc = swaps(k0, kb, lk, kr + kb1, ntot, nullptr)) != ALG_OK) break;
    if ((rc = update(k0, kb, kr + kb1, ntot, true)) != ALG_OK) break;
    // block k + 1's swaps touch these columns next
    if ((rc = cudaEventRecord(ev_b, sb) == cudaSuccess ? ALG_OK : ALG_CUDA_ERROR) != ALG_OK) break;
    if ((rc = cudaStreamWaitEvent(sa, ev_b, 0) == cudaSuccess ? ALG_OK : ALG_CUDA_ERROR) != ALG_OK) break;
  }
  ctx->stream = user;
  // join both streams back into the caller's stream, also on an error path
  cudaEventRecord(ev_b, sb);
  cudaStreamWaitEvent(sa, ev_b, 0);
  cudaEventRecord(ev_a, sa);
  cudaStreamWaitEvent(user, ev_a, 0);
  return rc;
}

// Right-hand sides from which the fused forms solve blocked (the dataflow
// sweeps take four right-hand sides per pass).
constexpr int kBlockedSolveRhs = 16;

// b (n x nrhs, ldb) <- (LU)^{-1} P b for many right-hand sides (fused
// arithmetic): the inverses of the 128 x 128 diagonal blocks of L and U
// (K3i, two launches), the rows gathered by perm, then per block one K3b
// launch per sweep: X_block <- T_bb^{-1} X_block by every CTA, the rows not
// yet solved updated by the block's column of the factor. The forward sweep
// reads x1 and writes y into x2; the backward sweep reads x2 and writes x
// into x1.
template <typename T>
int lu_solve_blocked_dev(alg_ctx* ctx, const T* lu, int n, int lda, const int* perm, T* b, int nrhs, int ldb) {
  if (n == 0 || nrhs == 0) return ALG_OK;
  constexpr int kb = kSolveKb;
  const int nblk = (n + kb - 1) / kb;
  T* x1 = nullptr;
  ALG_TRY(ws_get(ctx, WS_X, sizeof(T) * (2 * (size_t)n * nrhs + 2 * (size_t)nblk * kb * kb),
                 reinterpret_cast<void**>(&x1)));
  T* x2 = x1 + (size_t)n * nrhs;
  T* linv = x2 + (size_t)n * nrhs;
  T* uinv = linv + (size_t)nblk * kb * kb;
  constexpr size_t kInvSmem = sizeof(T) * kb * kb;
  constexpr int kSolveCols = solve_cols<T>();
  constexpr size_t kStepSmem = sizeof(T) * (kSolveKb * kSolveKb + kSolveKb * kSolveCols);
  static const cudaError_t configured = [] {
    cudaError_t e = cudaFuncSetAttribute(tri_block_inverse_kernel<T, false, 4, 2>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(tri_block_inverse_kernel<T, true, 4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kInvSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(block_solve_step_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kStepSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(block_solve_step_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kStepSmem);
    return e;
  }();
  ALG_CUDA_TRY(configured);
  const int tok = prof_begin(ctx, ALG_K_SOLVE);
  {
    const dim3 ig(kb / (2 * (kTrsmThreads / 32)), nblk);
    tri_block_inverse_kernel<T, false, 4, 2><<<ig, kTrsmThreads, kInvSmem, ctx->stream>>>(lu, lda, n, kb, linv);
    tri_block_inverse_kernel<T, true, 4, 2><<<ig, kTrsmThreads, kInvSmem, ctx->stream>>>(lu, lda, n, kb, uinv);
    const size_t cnt = (size_t)n * nrhs;
    const int g = (int)std::max<size_t>(1, std::min<size_t>((cnt + 255) / 256, (size_t)ctx->sm_count * 8));
    gather_perm_rows_kernel<T><<<g, 256, 0, ctx->stream>>>(b, ldb, perm, n, nrhs, x1, n);
    count_launches(3);
    ALG_CUDA_TRY(cudaGetLastError());
  }
  const int ctiles = (nrhs + kSolveCols - 1) / kSolveCols;
  for (int k0 = 0; k0 < n; k0 += kb) {  // L y = P b: x1 -> y in x2
    const int kbe = std::min(kb, n - k0);
    const int rows = n - (k0 + kbe);
    const dim3 grid(std::max(1, (rows + kSolveKb - 1) / kSolveKb), ctiles);
    block_solve_step_kernel<T, false><<<grid, 256, kStepSmem, ctx->stream>>>(
        lu, lda, n, k0, kbe, linv + (size_t)(k0 / kb) * kb * kb, x1, x2, nrhs);
    count_launches();
  }
  for (int blk = nblk - 1; blk >= 0; --blk) {  // U x = y: x2 -> x in x1
    const int k0 = blk * kb, kbe = std::min(kb, n - k0);
    const dim3 grid(std::max(1, (k0 + kSolveKb - 1) / kSolveKb), ctiles);
    block_solve_step_kernel<T, true><<<grid, 256, kStepSmem, ctx->stream>>>(
        lu, lda, n, k0, kbe, uinv + (size_t)blk * kb * kb, x2, x1, nrhs);
    count_launches();
  }
  ALG_CUDA_TRY(cudaGetLastError());
  ALG_CUDA_TRY(cudaMemcpy2DAsync(b, sizeof(T) * (size_t)ldb, x1, sizeof(T) * (size_t)n, sizeof(T) * (size_t)n, nrhs,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
  prof_end(ctx, tok, 2.0 * n * n * nrhs, sizeof(T) * (double(n) * n + 4.0 * n * nrhs));
  return ALG_OK;
}

template <typename T, bool EXACT>
int lu_solve_dev(alg_ctx* ctx, const T* lu, int n, int lda, const int* perm, T* b, int nrhs,
                 int ldb) {
  if (nrhs > 65535) return ALG_BAD_SHAPE;
  // the exact form keeps the reference's per-entry order (the dataflow
  // sweeps); the fused forms solve many right-hand sides blocked
  if (!EXACT && nrhs >= kBlockedSolveRhs) return lu_solve_blocked_dev<T>(ctx, lu, n, lda, perm, b, nrhs, ldb);
  return lu_solve_dataflow_dev<T, EXACT>(ctx, lu, n, lda, perm, b, nrhs, ldb);
}

int trsm_lower_unit_f32(alg_ctx* ctx, float* a, int lda, int r0, int kb, int cb, int ce) {
  return launch_trsm<float, false>(ctx, a, lda, r0, kb, cb, ce);
}

// explicit instantiations
#define ALG_INST(T, E)                                                                          \
  template int lu_factor_dev<T, E>(alg_ctx*, T*, int, int, int, int*, int*, const LuPlan&);   \
  template int lu_factor_partial_dev<T, E>(alg_ctx*, T*, int, int, int, int, int*, int*, const LuPlan&); \
  template int lu_solve_dev<T, E>(alg_ctx*, const T*, int, int, const int*, T*, int, int);    \
  template int gemm_sub_dev<T, E>(alg_ctx*, int, int, int, const T*, int, const T*, int, T*, int);
ALG_INST(double, true)
ALG_INST(double, false)
ALG_INST(float, true)
ALG_INST(float, false)
#undef ALG_INST

}  // namespace alg

// ===========================================================================
// C entry points (dense)
// ===========================================================================
namespace {

using alg::LuPlan;

int factor_any(alg_ctx* ctx, int update, double* d_a, int m, int nc, int lda, int* d_ipiv, int* d_perm) {
  const LuPlan plan = alg::default_plan(nc, 8);
  if (update == ALG_UPDATE_EXACT)
    return alg::lu_factor_dev<double, true>(ctx, d_a, m, nc, lda, d_ipiv, d_perm, plan);
  if (update == ALG_UPDATE_FMA)
    return alg::lu_factor_dev<double, false>(ctx, d_a, m, nc, lda, d_ipiv, d_perm, plan);
  return ALG_INVALID_ARGUMENT;
}

int solve_any(alg_ctx* ctx, int update, const double* d_lu, int n, int lda, const int* d_perm,
              double* d_b, int nrhs, int ldb) {
  if (update == ALG_UPDATE_EXACT)
    return alg::lu_solve_dev<double, true>(ctx, d_lu, n, lda, d_perm, d_b, nrhs, ldb);
  return alg::lu_solve_dev<double, false>(ctx, d_lu, n, lda, d_perm, d_b, nrhs, ldb);
}

// Sizes accepted by the int32-indexed kernels.
bool size_ok(size_t n) { return n <= (size_t)INT_MAX / 2; }

struct CtxLock {
  alg_ctx* ctx = nullptr;
  std::unique_lock<std::mutex> lk;
  int rc = ALG_OK;
  CtxLock() {
    rc = alg::default_ctx(&ctx);
    if (rc == ALG_OK) lk = std::unique_lock<std::mutex>(ctx->mu);
  }
};

// Host drop-in core: copy a (and b) in, factor (and solve), copy back.
int host_lu(int update, double* a, size_t m, size_t nc, size_t* ipiv, double* det, double* b,
            size_t nrhs) {
  if (!size_ok(m) || !size_ok(nc) || !size_ok(nrhs)) return ALG_BAD_SHAPE;
  CtxLock L;
  if (L.rc != ALG_OK) return L.rc;
  alg_ctx* ctx = L.ctx;
  const int M = (int)m, N = (int)nc, R = (int)nrhs;
  double* d_a = nullptr;
  double* d_b = nullptr;
  int* d_ipiv = nullptr;
  int* d_perm = nullptr;
  ALG_TRY(alg::ws_get(ctx, alg::WS_A, sizeof(double) * m * nc, reinterpret_cast<void**>(&d_a)));
  ALG_TRY(alg::ws_get(ctx, alg::WS_IPIV, sizeof(int) * nc, reinterpret_cast<void**>(&d_ipiv)));
  ALG_TRY(alg::ws_get(ctx, alg::WS_PERM, sizeof(int) * m, reinterpret_cast<void**>(&d_perm)));
  if (b != nullptr && R > 0)
    ALG_TRY(alg::ws_get(ctx, alg::WS_B, sizeof(double) * m * nrhs, reinterpret_cast<void**>(&d_b)));
  ALG_CUDA_TRY(cudaMemcpyAsync(d_a, a, sizeof(double) * m * nc, cudaMemcpyHostToDevice, ctx->stream));
  if (d_b) ALG_CUDA_TRY(cudaMemcpyAsync(d_b, b, sizeof(double) * m * nrhs, cudaMemcpyHostToDevice, ctx->stream));
  ALG_TRY(alg::status_reset(ctx));
  ALG_TRY(factor_any(ctx, update, d_a, M, N, M, d_ipiv, d_perm));
  ALG_TRY(alg::status_fetch(ctx));
  const bool singular = ctx->h_status->singular_col != INT_MAX;
  if (!singular && d_b) {
    ALG_TRY(solve_any(ctx, update, d_a, M, M, d_perm, d_b, R, M));
    ALG_TRY(alg::status_fetch(ctx));  // a timed-out sweep is an error, not a result
    ALG_CUDA_TRY(cudaMemcpyAsync(b, d_b, sizeof(double) * m * nrhs, cudaMemcpyDeviceToHost, ctx->stream));
  }
  ALG_CUDA_TRY(cudaMemcpyAsync(a, d_a, sizeof(double) * m * nc, cudaMemcpyDeviceToHost, ctx->stream));
  std::vector<int> h_ipiv(nc);
  ALG_CUDA_TRY(cudaMemcpyAsync(h_ipiv.data(), d_ipiv, sizeof(int) * nc, cudaMemcpyDeviceToHost, ctx->stream));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (singular) return ALG_SINGULAR;
  if (ipiv)
    for (size_t k = 0; k < nc; ++k) ipiv[k] = (size_t)h_ipiv[k];
  if (det) {
    // mod.rs:120-150: sign flip per interchange, then times the pivot, in order
    double d = 1.0;
    for (size_t k = 0; k < nc; ++k) {
      if ((size_t)h_ipiv[k] != k) d = -d;
      d *= a[k + k * m];
    }
    *det = d;
  }
  return ALG_OK;
}

// A flag if some u_ii of the factors is zero.
__global__ void zero_diag_kernel(const double* __restrict__ lu, int lda, int n, int* zero_diag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (lu[i + (size_t)i * lda] == 0.0) atomicExch(zero_diag, 1);
}

// Column `col` of the inverse (mod.rs:249-298), one thread per column and the
// reference's loops as they are: b = e_col with dgetrf's interchanges
// applied (row i of P e_col is entry perm[i]), the unit-lower sweep
// sum -= l_ij b_j in increasing j, then the upper sweep sum -= u_ij b_j in
// increasing j and b_i = sum / u_ii, each product and difference rounded on
// its own — so every entry equals the reference's bit for bit. The working
// column lives in w (n x n, w[i * n + col]) so a warp's accesses coalesce.
__global__ void __launch_bounds__(128) inverse_columns_kernel(const double* __restrict__ lu, int lda, int n,
                                                              const int* __restrict__ perm, double* __restrict__ w,
                                                              double* __restrict__ inv) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  double* x = w + col;
  for (int i = 0; i < n; ++i) x[(size_t)i * n] = perm[i] == col ? 1.0 : 0.0;
  for (int i = 0; i < n; ++i) {
    double sum = x[(size_t)i * n];
#pragma unroll 8
    for (int j = 0; j < i; ++j) sum = __dsub_rn(sum, __dmul_rn(lu[i + (size_t)j * lda], x[(size_t)j * n]));
    x[(size_t)i * n] = sum;
  }
  for (int i = n - 1; i >= 0; --i) {
    double sum = x[(size_t)i * n];
#pragma unroll 8
    for (int j = i + 1; j < n; ++j) sum = __dsub_rn(sum, __dmul_rn(lu[i + (size_t)j * lda], x[(size_t)j * n]));
    x[(size_t)i * n] = __ddiv_rn(sum, lu[i + (size_t)i * lda]);
  }
  for (int i = 0; i < n; ++i) inv[i + (size_t)col * n] = x[(size_t)i * n];
}

// The inverse from dgetrf's factors (mod.rs:249-298) into d_inv (ld n);
// ALG_SINGULAR, with nothing written, when some u_ii is zero.
int inverse_dev(alg_ctx* ctx, const double* d_lu, int n, int lda, const int* d_perm, double* d_inv) {
  int* flag = nullptr;
  double* w = nullptr;
  ALG_TRY(alg::ws_get(ctx, alg::WS_MISC, sizeof(int), reinterpret_cast<void**>(&flag)));
  ALG_TRY(alg::ws_get(ctx, alg::WS_X, sizeof(double) * (size_t)n * n, reinterpret_cast<void**>(&w)));
  ALG_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), ctx->stream));
  zero_diag_kernel<<<std::max(1, std::min(ctx->sm_count, (n + 255) / 256)), 256, 0, ctx->stream>>>(d_lu, lda, n,
                                                                                                    flag);
  alg::count_launches();
  ALG_CUDA_TRY(cudaGetLastError());
  int zero = 0;
  ALG_CUDA_TRY(cudaMemcpyAsync(&zero, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  ALG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (zero) return ALG_SINGULAR;
  const int tok = alg::prof_begin(ctx, ALG_K_SOLVE);
  inverse_columns_kernel<<<(n + 127) / 128, 128, 0, ctx->stream>>>(d_lu, lda, n, d_perm, w, d_inv);
  alg::count_launches();
  alg::prof_end(ctx, tok, 2.0 * (double)n * n * n, 8.0 * (double)n * n * 3);
  ALG_CUDA_TRY(cudaGetLastError());
  return ALG_OK;
}

}  // namespace

extern "C" {

int alg_dgetri(double* lu, size_t n, const size_t* ipiv) {
  if (n == 0) return ALG_OK;
  if (lu == nullptr || ipiv == nullptr) return ALG_INVALID_ARGUMENT;
  if (!size_ok(n)) return ALG_BAD_SHAPE;
  for (size_t k = 0; k < n; ++k)
    if (ipiv[k] >= n) return ALG_BAD_SHAPE;
  // the sequential interchanges as one gather: row i of P b is row perm[i] of b
  std::vector<int> perm(n);
  for (size_t i = 0; i < n; ++i) perm[i] = (int)i;
  for (size_t k = 0; k < n; ++k) std::swap(perm[k], perm[ipiv[k]]);
  CtxLock L;
  if (L.rc != ALG_OK) return L.rc;
  alg_ctx* ctx = L.ctx;
  const int N = (int)n;
  double* d_a = nullptr;
  double* d_b = nullptr;
  int* d_perm = nullptr;
  ALG_TRY(alg::ws_get(ctx, alg::WS_A, sizeof(double) * n * n, reinterpret_cast<void**>(&d_a)));
  ALG_TRY(alg::ws_get(ctx, alg::WS_B, sizeof(double) * n * n, reinterpret_cast<void**>(&d_b)));
  ALG_TRY(alg::ws_get(ctx, alg::WS_PERM, sizeof(int) * n, reinterpret_cast<void**>(&d_perm)));
  ALG_CUDA_TRY(cudaMemcpyAsync(d_a, lu, sizeof(double) * n * n, cudaMemcpyHostToDevice, ctx->stream));
  ALG_CUDA_TRY(cudaMemcpyAsync(d_perm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
  ALG_TRY(alg::status_reset(ctx));
  ALG_TRY(inverse_dev(ctx, d_a, N, N, d_perm, d_b));
  ALG_CUDA_TRY(cudaMemcpyAsync(lu, d_b, sizeof(double) * n * n, cudaMemcpyDeviceToHost, ctx->stream));
  return alg::status_fetch(ctx);  // synchronises; reports a timed-out sweep
}

int alg_dgetri_dev(alg_ctx* ctx, double* d_lu, int n, int lda, const int32_t* d_perm) {
  if (ctx == nullptr || (n > 0 && (d_lu == nullptr || d_perm == nullptr))) return ALG_INVALID_ARGUMENT;
  if (n < 0 || lda < std::max(1, n)) return ALG_BAD_SHAPE;
  if (n == 0) return ALG_OK;
  double* d_b = nullptr;
  ALG_TRY(alg::ws_get(ctx, alg::WS_B, sizeof(double) * (size_t)n * n, reinterpret_cast<void**>(&d_b)));
  ALG_TRY(alg::status_reset(ctx));
  ALG_TRY(inverse_dev(ctx, d_lu, n, lda, d_perm, d_b));
  ALG_CUDA_TRY(cudaMemcpy2DAsync(d_lu, sizeof(double) * (size_t)lda, d_b, sizeof(double) * (size_t)n,
                                 sizeof(double) * (size_t)n, n, cudaMemcpyDeviceToDevice, ctx->stream));
  return alg::status_fetch(ctx);
}

int alg_dgetrf(double* a, size_t n, size_t* ipiv, double* det) {
  if (n == 0) {
    if (det) *det = 1.0;
    return ALG_OK;
  }
  if (a == nullptr || ipiv == nullptr) return ALG_INVALID_ARGUMENT;
  return host_lu(ALG_UPDATE_EXACT, a, n, n, ipiv, det, nullptr, 0);
}

int alg_dgetrf_rect(double* a, size_t nrows, size_t ncols, size_t* ipiv) {
  if (nrows < ncols) return ALG_BAD_SHAPE;
  if (ncols == 0) return ALG_OK;
  if (a == nullptr || ipiv == nullptr) return ALG_INVALID_ARGUMENT;
  return host_lu(ALG_UPDATE_EXACT, a, nrows, ncols, ipiv, nullptr, nullptr, 0);
}

int alg_dgesv(double* a, double* b, size_t n) {
  if (n == 0) return ALG_OK;
  if (a == nullptr || b == nullptr) return ALG_INVALID_ARGUMENT;
  return host_lu(ALG_UPDATE_EXACT, a, n, n, nullptr, nullptr, b, 1);
}

int alg_dgesv_nrhs(double* a, double* b, size_t n, size_t nrhs) {
  if (n == 0 || nrhs == 0) return ALG_OK;
  if (a == nullptr || b == nullptr) return ALG_INVALID_ARGUMENT;
  return host_lu(ALG_UPDATE_EXACT, a, n, n, nullptr, nullptr, b, nrhs);
}

int alg_dgesv_ex(int update, double* a, double* b, size_t n, size_t nrhs, size_t* ipiv) {
  if (update != ALG_UPDATE_EXACT && update != ALG_UPDATE_FMA) return ALG_INVALID_ARGUMENT;
  if (n == 0) return ALG_OK;
  if (a == nullptr || (b == nullptr && nrhs > 0)) return ALG_INVALID_ARGUMENT;
  return host_lu(update, a, n, n, ipiv, nullptr, b, nrhs);
}

int alg_dgetrf_dev(alg_ctx* ctx, int update, double* d_a, int n, int lda, int32_t* d_ipiv,
                   int32_t* d_perm) {
  if (ctx == nullptr) return ALG_INVALID_ARGUMENT;
  if (n < 0 || lda < std::max(1, n)) return ALG_BAD_SHAPE;
  if (n == 0) return ALG_OK;
  int* ipiv = d_ipiv;
  if (ipiv == nullptr) ALG_TRY(alg::ws_get(ctx, alg::WS_IPIV, sizeof(int) * n, reinterpret_cast<void**>(&ipiv)));
  ALG_TRY(alg::status_reset(ctx));
  ALG_TRY(factor_any(ctx, update, d_a, n, n, lda, ipiv, d_perm));
  ALG_TRY(alg::status_fetch(ctx));
  return ctx->h_status->singular_col != INT_MAX ? ALG_SINGULAR : ALG_OK;
}

int alg_dgetrf_rect_dev(alg_ctx* ctx, int update, double* d_a, int nrows, int ncols, int lda,
                        int32_t* d_ipiv) {
  if (ctx == nullptr || d_ipiv == nullptr) return ALG_INVALID_ARGUMENT;
  if (nrows < ncols || ncols < 0 || lda < std::max(1, nrows)) return ALG_BAD_SHAPE;
  if (ncols == 0) return ALG_OK;
  ALG_TRY(alg::status_reset(ctx));
  ALG_TRY(factor_any(ctx, update, d_a, nrows, ncols, lda, d_ipiv, nullptr));
  ALG_TRY(alg::status_fetch(ctx));
  return ctx->h_status->singular_col != INT_MAX ? ALG_SINGULAR : ALG_OK;
}

int alg_dgetrs_dev(alg_ctx* ctx, const double* d_lu, int n, int lda, const int32_t* d_perm,
                   double* d_b, int nrhs, int ldb) {
  if (ctx == nullptr || d_perm == nullptr) return ALG_INVALID_ARGUMENT;
  if (n < 0 || nrhs < 0 || lda < std::max(1, n) || ldb < std::max(1, n)) return ALG_BAD_SHAPE;
  ALG_TRY(alg::status_reset(ctx));
  ALG_TRY(solve_any(ctx, ALG_UPDATE_EXACT, d_lu, n, lda, d_perm, d_b, nrhs, ldb));
  return alg::status_fetch(ctx);  // synchronises; reports a timed-out sweep
}

int alg_dgesv_dev(alg_ctx* ctx, int update, double* d_a, int n, int lda, double* d_b, int nrhs,
                  int ldb, int32_t* d_ipiv) {
  if (ctx == nullptr) return ALG_INVALID_ARGUMENT;
  if (update != ALG_UPDATE_EXACT && update != ALG_UPDATE_FMA) return ALG_INVALID_ARGUMENT;
  if (n < 0 || nrhs < 0 || lda < std::max(1, n) || ldb < std::max(1, n)) return ALG_BAD_SHAPE;
  if (n == 0) return ALG_OK;
  int* ipiv = d_ipiv;
  int* perm = nullptr;
  if (ipiv == nullptr) ALG_TRY(alg::ws_get(ctx, alg::WS_IPIV, sizeof(int) * n, reinterpret_cast<void**>(&ipiv)));
  ALG_TRY(alg::ws_get(ctx, alg::WS_PERM, sizeof(int) * n, reinterpret_cast<void**>(&perm)));
  ALG_TRY(alg::status_reset(ctx));
  ALG_TRY(factor_any(ctx, update, d_a, n, n, lda, ipiv, perm));
  ALG_TRY(alg::status_fetch(ctx));
  if (ctx->h_status->singular_col != INT_MAX) return ALG_SINGULAR;
  ALG_TRY(solve_any(ctx, update, d_a, n, lda, perm, d_b, nrhs, ldb));
  return alg::status_fetch(ctx);  // synchronises; reports a timed-out sweep
}

}  // extern "C"
