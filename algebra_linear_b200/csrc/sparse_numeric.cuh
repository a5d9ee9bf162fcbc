// Device state of one sparse LU handle: the uploaded plan, the numeric
// arenas and two factor sets (a failed factorization keeps the previous
// factors, as the reference's handle does).
#pragma once

#include <cstdint>
#include <vector>

#include "sparse.cuh"

namespace alg {
namespace sp {

// A work item of the multi-CTA solve kernels: a front and a chunk of its
// rows (and of its U12 columns).
struct SolveItem {
  int32_t front, chunk, tchunk, pad;
};

struct Stats {
  uint64_t nnz_l = 0, nnz_u = 0, flops_estimate = 0;
};

struct DeviceLu {
  alg_ctx* ctx = nullptr;
  const FrontPlan* plan = nullptr;
  FrontDesc* d_fronts = nullptr;
  int32_t *d_child_idx = nullptr, *d_child_slot = nullptr, *d_struct_cols = nullptr, *d_cb_colmap = nullptr;
  int64_t* d_anew_q = nullptr;
  int32_t *d_anew_slot = nullptr, *d_anew_col = nullptr, *d_new_rows = nullptr;
  int32_t *d_small_levels = nullptr, *d_solve_levels = nullptr, *d_col_perm = nullptr;
  double* d_values = nullptr;  // A's values (CSC order)
  double* d_block = nullptr;   // small fronts' blocks
  double* d_stack = nullptr;   // large fronts' contribution blocks
  double* d_front = nullptr;   // the large front being factored
  int *d_ipiv = nullptr, *d_perm = nullptr;
  int32_t* d_rowtmp = nullptr;
  int* d_flag = nullptr;       // [0]: a small front met a zero pivot
  double *d_y = nullptr, *d_rhs = nullptr;
  // solve: per-level work items of the multi-CTA kernels, U12 partial sums
  SolveItem* d_fwd_items = nullptr;
  SolveItem* d_bwd_items = nullptr;
  std::vector<int> fwd_item_ptr, bwd_item_ptr;
  int64_t* d_part_off = nullptr;
  double* d_partial = nullptr;
  struct Factors {
    double* L = nullptr;
    double* U = nullptr;
    int32_t* rowid = nullptr;
    int32_t* pos_of_row = nullptr;
    int32_t* row_perm = nullptr;
    int32_t* lcount = nullptr;
    unsigned* ucount = nullptr;
  } fac[2];

  int init(alg_ctx* ctx, const FrontPlan* plan);
  void release();
  int factor(int set);                 // stream-ordered
  int finish(int set, Stats* stats);   // synchronises; SP_OK or SP_SINGULAR
  int solve(int set);                  // d_rhs -> d_rhs, stream-ordered
};

}  // namespace sp
}  // namespace alg
