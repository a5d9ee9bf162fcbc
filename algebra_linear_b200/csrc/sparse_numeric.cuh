// Device state of one sparse LU handle: the uploaded plan, the numeric
// arenas and two factor sets (a failed factorization keeps the previous
// factors, as the reference's handle does).
//
// Precision. The FP64 form factors and solves in FP64 (the reference's
// arithmetic). The mixed form factors the fronts in FP32 (the large fronts'
// trailing updates in FP32, or on the tensor cores with TF32 / BF16 operands
// and FP32 accumulation) and refines every solve in FP64 against A's values
// (r = b - A x in FP64, x += LU32^-1 r) until the normwise backward error
// meets the target; when it does not, the set is refactored in FP64.
//
// Scalar. A handle's values are real (words = 1) or complex (words = 2:
// SparseLu<Complex64>, interleaved re, im); the arenas are sized in doubles
// times words. Complex factors are FP64 only.
#pragma once

#include <cstdint>
#include <vector>

#include "sparse.cuh"

namespace alg {
namespace sp {

// A work item of the multi-CTA solve kernels: a front, a chunk of its rows
// and a chunk of the columns it sums over.
struct SolveItem {
  int32_t front, chunk, tchunk, pad;
};

struct Stats {
  uint64_t nnz_l = 0, nnz_u = 0, flops_estimate = 0;
};

// Outcome of the last solve of the mixed form.
struct RefineReport {
  int precision = -1;      // -1 FP64, else ALG_PREC_* of the factors used
  int iterations = 0;      // refinement steps (0 on the FP64 form)
  int fell_back = 0;       // 1: the set was refactored in FP64 during this solve
  double backward_error = -1.0;  // ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf); -1 unmeasured
};

struct DeviceLu {
  alg_ctx* ctx = nullptr;
  const FrontPlan* plan = nullptr;
  int words = 1;            // doubles per value: 1 real, 2 complex
  int prec = -1;            // precision of the next factorization (-1: FP64)
  double tol = 0.0;         // backward-error target of the mixed solve (<= 0: 10 n 2^-53)
  int max_ir = 0;           // refinement steps before the FP64 refactorization (<= 0: 10)
  FrontDesc* d_fronts = nullptr;
  int32_t *d_child_idx = nullptr, *d_child_slot = nullptr, *d_struct_cols = nullptr, *d_cb_colmap = nullptr;
  int64_t* d_anew_q = nullptr;
  int32_t *d_anew_slot = nullptr, *d_anew_col = nullptr, *d_new_rows = nullptr;
  int32_t *d_small_levels = nullptr, *d_col_perm = nullptr;
  double* d_values = nullptr;  // A's values (CSC order) of the next factorization
  // arenas sized in doubles (times words); the FP32 form uses their first halves as floats
  double* d_block = nullptr;   // small fronts' blocks
  double* d_stack = nullptr;   // large fronts' contribution blocks
  // per lane (independent subtrees of large fronts run concurrently): a
  // context (stream, workspaces; lane 0 is the handle's own), the front
  // being factored and the pivot scratch
  static constexpr int kMaxLanes = 8;
  int n_lanes = 1;
  alg_ctx* lane_ctx[kMaxLanes] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kMaxLanes] = {};
  double* d_front[kMaxLanes] = {};
  int* d_ipiv[kMaxLanes] = {};
  int* d_perm[kMaxLanes] = {};
  int32_t* d_rowtmp[kMaxLanes] = {};
  double* d_zblock[kMaxLanes] = {};  // complex: a block column of L21 in its real 2x2 form
  int* d_flag = nullptr;       // [0]: a small front met a zero pivot
  double *d_y = nullptr, *d_rhs = nullptr;
  // solve schedule: per level the fronts solved by the one-CTA diagonal
  // kernels, the large fronts solved by the multi-CTA sweep, and the work
  // items of the L21 / U12 kernels; partial sums of the column chunks
  int32_t* d_solve_small = nullptr;
  std::vector<int> solve_small_ptr;
  std::vector<std::vector<int32_t>> solve_big;
  SolveItem *d_fwd_items = nullptr, *d_fin_items = nullptr, *d_bwd_items = nullptr;
  std::vector<int> fwd_item_ptr, fin_item_ptr, bwd_item_ptr;
  int64_t *d_part_off = nullptr, *d_fpart_off = nullptr;
  double *d_partial = nullptr, *d_fpartial = nullptr;
  int* d_tflags = nullptr;     // flags of the multi-CTA sweep, then its abort flag
  int tflag_count = 0;
  // the mixed form's refinement: A in CSR (for r = b - A x), b, x, stats
  int64_t* d_csr_ptr = nullptr;
  int32_t* d_csr_col = nullptr;
  int64_t* d_csr_map = nullptr;  // CSR entry -> CSC index
  double *d_b0 = nullptr, *d_x = nullptr;
  unsigned long long* d_norms = nullptr;
  RefineReport last;
  struct Factors {
    int prec = -1;             // precision of the factors held
    double anorm = 0.0;        // ||A||_inf of the factored values (mixed form)
    double* values = nullptr;  // the factored values (mixed form: the refinement's A)
    double* L = nullptr;
    double* U = nullptr;
    int32_t* rowid = nullptr;
    int32_t* pos_of_row = nullptr;
    int32_t* row_perm = nullptr;
    int32_t* lcount = nullptr;
    unsigned* ucount = nullptr;
  } fac[2];

  int init(alg_ctx* ctx, const FrontPlan* plan, int words = 1);
  void release();
  int factor(int set);                 // d_values -> set, stream-ordered
  int finish(int set, Stats* stats);   // synchronises; SP_OK or SP_SINGULAR
  int solve(int set);                  // d_rhs -> d_rhs (the mixed form synchronises per step)

 private:
  template <typename T>
  int factor_t(int set, const double* values, int tc_prec);
  template <typename T>
  int factor_big(int set, int32_t s, int lane, const double* values, int tc_prec);
  template <typename T>
  int sweep_t(int set);                // d_rhs -> d_rhs with the set's factors, stream-ordered
  int refine(int set);
  int ensure_refine_buffers();
  int refactor_fp64(int set);
};

}  // namespace sp
}  // namespace alg
