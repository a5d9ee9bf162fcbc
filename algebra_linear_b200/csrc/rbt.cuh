// Random butterfly transformation + LU without pivoting (mixed form).
#pragma once

#include <cstdint>

#include "context.cuh"

namespace alg {

struct RbtState {
  int n = 0;
  const double* u = nullptr;  // 8 coefficient arrays of length n/4 (left butterfly)
  const double* v = nullptr;  // (right butterfly)
};

// Draws the two depth-2 butterflies of order n (n % 4 == 0) from seed.
int rbt_prepare(alg_ctx* ctx, int n, uint64_t seed, RbtState* st);
// ar (FP32) = U^T a V (a FP64), n x n column-major.
int rbt_transform(alg_ctx* ctx, const RbtState& st, const double* a, int lda, float* ar, int ldr);
// z = U^T x (transpose_u) or z = V x, length-n device vectors.
int rbt_vector(alg_ctx* ctx, const RbtState& st, bool transpose_u, const double* x, double* z);
// LU without pivoting of the n x n FP32 matrix (blocks of nb <= 128); trailing
// updates in prec (ALG_PREC_FP32 on the CUDA cores, TF32/BF16 on tcgen05).
int genp_factor(alg_ctx* ctx, int prec, float* a, int n, int lda, int nb);

// U12 = L11^{-1} A12 for the FP32 matrix (rows [r0, r0+kb), columns [cb, ce)).
int trsm_lower_unit_f32(alg_ctx* ctx, float* a, int lda, int r0, int kb, int cb, int ce);

}  // namespace alg
