// Host-side drivers of the blocked dense LU and its solves.
#pragma once

#include "context.cuh"

namespace alg {

struct LuPlan {
  int nb = 64;       // block-panel width (trailing-update depth)
  int nbl = 16;      // leaf-panel width (one cluster kernel)
  int tc_prec = -1;  // FP32 matrices: ALG_PREC_TF32 / ALG_PREC_BF16 puts the
                     // block-level trailing update on the tensor cores
  int tslu = 0;      // FP32 matrices: tournament pivoting for the leaf panels
};

// Tournament-pivoting leaf panel of the FP32 LU (tslu.cu) and its scratch
// size: columns [c0, c0 + w) of rows [c0, n), inside the block panel
// [kb0, kb1); the same outputs as the partial-pivoting leaf kernel.
struct TsluArgs {
  float* a;
  int lda, n, c0, w, kb0, kb1;
  int* ipiv;
  int* lab;
  int first_leaf;
  DevStatus* status;
};
// One multi-CTA triangular sweep over the leading n x n block of LU factors
// (lda): unit-lower or upper; flags: n / 64 + 1 ints, abort_flag zero.
template <typename T>
int tri_solve_dev(alg_ctx* ctx, const T* lu, int lda, int n, T* x, bool upper, int* flags, int* abort_flag);

size_t tslu_scratch_bytes();
int tslu_scratch_reset(alg_ctx* ctx, void* scratch);
int tslu_panel(alg_ctx* ctx, const TsluArgs& p, void* scratch);

// C -= A B on the tensor cores (tcgen05, FP32 accumulation in TMEM) with the
// operands rounded to TF32 or BF16 (or split into TF32 pairs); A, B, C FP32
// column-major. ws_slot: the workspace that holds the converted operands
// (two updates in flight on two streams need two); max_ctas > 0 caps the
// persistent grid below the SM count (SMs left to another stream's kernels).
int gemm_tc_sub_dev(alg_ctx* ctx, int prec, int M, int N, int K, const float* A, int lda, const float* B,
                    int ldb, float* C, int ldc, int ws_slot = WS_KRYLOV, int max_ctas = 0);

// In-place LU of the m x nc (m >= nc) device matrix a (leading dim lda).
// ipiv: nc global interchanges; perm: m net permutation (may be null).
// Status lands in ctx->d_status (singular_col). Stream-ordered, no sync.
template <typename T, bool EXACT>
int lu_factor_dev(alg_ctx* ctx, T* a, int m, int nc, int lda, int* ipiv, int* perm,
                  const LuPlan& plan);

// LU with partial pivoting of the first nc columns of the m x ntot device
// matrix a (m >= nc): the row interchanges span all ntot columns, the block
// row to the right becomes U12 and the trailing (m - nc) x (ntot - nc) block
// becomes the Schur complement. ntot = nc is lu_factor_dev.
template <typename T, bool EXACT>
int lu_factor_partial_dev(alg_ctx* ctx, T* a, int m, int nc, int ntot, int lda, int* ipiv, int* perm,
                          const LuPlan& plan);

// Solves with the packed factors: b (n x nrhs, ldb) becomes x. Stream-ordered.
template <typename T, bool EXACT>
int lu_solve_dev(alg_ctx* ctx, const T* lu, int n, int lda, const int* perm, T* b, int nrhs,
                 int ldb);

// Same contract as lu_solve_dev: gather by perm, then the forward and
// backward sweeps as single dataflow launches (trsv.cu).
template <typename T, bool EXACT>
int lu_solve_dataflow_dev(alg_ctx* ctx, const T* lu, int n, int lda, const int* perm, T* b, int nrhs, int ldb);

// FP64 C -= A B on the FP64 tensor cores (mma.sync m8n8k4), fused arithmetic;
// column-major, any leading dimensions, stream-ordered.
int gemm_dmma_sub_dev(alg_ctx* ctx, int M, int N, int K, const double* A, int lda, const double* B, int ldb,
                      double* C, int ldc);

// C -= A B on the CUDA cores (column-major), stream-ordered.
template <typename T, bool EXACT>
int gemm_sub_dev(alg_ctx* ctx, int M, int N, int K, const T* A, int lda, const T* B, int ldb,
                 T* C, int ldc);

LuPlan default_plan(int n, int elem_bytes);

}  // namespace alg
