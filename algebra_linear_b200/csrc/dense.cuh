// Host-side drivers of the blocked dense LU and its solves.
#pragma once

#include "context.cuh"

namespace alg {

struct LuPlan {
  int nb = 64;       // block-panel width (trailing-update depth)
  int nbl = 16;      // leaf-panel width (one cluster kernel)
  int tc_prec = -1;  // FP32 matrices: ALG_PREC_TF32 / ALG_PREC_BF16 puts the
                     // block-level trailing update on the tensor cores
};

// C -= A B on the tensor cores (tcgen05, FP32 accumulation in TMEM) with the
// operands rounded to TF32 or BF16; A, B, C FP32 column-major.
int gemm_tc_sub_dev(alg_ctx* ctx, int prec, int M, int N, int K, const float* A, int lda, const float* B,
                    int ldb, float* C, int ldc);

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
