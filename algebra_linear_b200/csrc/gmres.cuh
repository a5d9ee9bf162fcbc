// GMRES-IR: FP64 GMRES refinement with a low-precision preconditioner.
#pragma once

#include <functional>

#include "context.cuh"

namespace alg {

// z = M^{-1} v on device vectors of length n (FP64 in and out).
using Precond = std::function<int(alg_ctx*, const double* v, double* z)>;

struct GmresOpts {
  int restart = 30;        // Krylov dimension per outer step
  int max_outer = 10;      // outer refinement steps
  double inner_tol = 1e-6; // relative preconditioned residual that ends an inner solve
  double tol = 0.0;        // backward-error target of the outer loop
};

struct GmresResult {
  int outer = 0;
  int inner = 0;
  double backward_error = 0.0;
  bool converged = false;
};

// y = A x (FP64, n x n column-major); stream-ordered.
int gemv_dev(alg_ctx* ctx, const double* a, int n, int lda, const double* x, double* y);

// Refines x (device, length n) for A x = b; ALG_CONVERGENCE if tol is not met.
int gmres_ir_dev(alg_ctx* ctx, const double* a, int n, int lda, const double* b, double* x, double anorm,
                 const Precond& M, const GmresOpts& go, GmresResult* res);

}  // namespace alg
