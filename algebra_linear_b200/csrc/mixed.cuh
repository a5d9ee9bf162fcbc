// Mixed-precision solve (low-precision LU + FP64 refinement): internal API.
#pragma once

#include "context.cuh"

namespace alg {

// LU of the n x n FP32 matrix a32 (leading dim lda) with trailing updates in
// the chosen precision (ALG_PREC_*). Stream-ordered; status in ctx.
int lu_factor_lowp_dev(alg_ctx* ctx, int precision, float* a32, int n, int lda, int* ipiv, int* perm,
                       bool tournament);

// ||A||_inf of an n x n FP64 matrix (synchronises).
int inf_norm_dev(alg_ctx* ctx, const double* a, int n, int lda, double* out_host);

// r = b - A x (FP64) and, per right-hand side, max|r|, max|x|, max|b| (synchronises).
int residual_dev(alg_ctx* ctx, const double* a, int n, int lda, const double* x, int ldx, const double* b,
                 int ldb, double* r, int ldr, int nrhs, double* rmax, double* xmax, double* bmax);

int dgesv_mixed_dev(alg_ctx* ctx, const alg_mixed_opts& o, double* d_a, int n, int lda, double* d_b, int nrhs,
                    int ldb, alg_mixed_report* rep);

}  // namespace alg
