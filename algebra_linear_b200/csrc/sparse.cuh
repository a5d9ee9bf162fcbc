// Sparse supernodal LU on the device: the static front plan built on the host
// from the reference's symbolic analysis, and the numeric factorization and
// solve that run on the GPU.
//
// The reference (src/sparse/faer/supernodal_lu.rs) factors supernode by
// supernode, left-looking, with row sets that change with the pivots. Here the
// same supernode partition and column order are factored multifrontally over a
// STATIC structure that holds every entry partial pivoting can produce: the
// row structure of chol(A^T A) (George and Ng). Front s holds the rows that
// enter at s (rows of A whose first column, in the new order, is in s) and the
// unpivoted rows of its children; its columns are s's own columns and
// Struct(s), the columns of chol(A^T A) below s. Partial pivoting over all of
// a front's rows is partial pivoting over the whole column, as in the
// reference, so the pivot sequence is the reference's (barring exact ties);
// the order in which the updates of one entry are summed differs, so values
// agree to rounding, not bit for bit.
#pragma once

#include <cstdint>
#include <vector>

#include "context.cuh"
#include "sparse_symbolic.cuh"

namespace alg {
namespace sp {

// Per-front description, uploaded once per pattern.
struct FrontDesc {
  int64_t block_off;    // transient front block (rows x (size + ncb), ld = rows); small fronts only
  int64_t l_off;        // L panel (rows x size, ld = rows)
  int64_t u_off;        // U12 panel (size x ncb, ld = size)
  int64_t rowid_off;    // original row of each slot, after pivoting (rows ints)
  int64_t cb_off;       // where the parent finds this front's contribution block
  int32_t cb_ld;        //   and its leading dimension
  int32_t size, rows, ncb, begin;  // columns, rows, |Struct|, first column (position)
  int32_t child_begin, child_end;  // into child_idx / child_slot
  int32_t anew_begin, anew_end;    // A entries of the rows that enter here
  int32_t new_begin, new_end;      // the rows that enter here
  int32_t struct_begin;            // into struct_cols / cb_colmap
  int32_t small;                   // 1: factored by the batched small-front kernel
};

struct FrontPlan {
  idx n = 0, nnz = 0, ns = 0;
  bool structurally_singular = false;
  std::vector<FrontDesc> fronts;
  std::vector<int32_t> child_idx, child_slot;   // children and their first slot in the parent
  std::vector<int32_t> struct_cols;             // Struct(s), global positions, sorted
  std::vector<int32_t> cb_colmap;               // Struct(c)[t] -> local column in parent(c)
  std::vector<int64_t> anew_q;                  // A entry (CSC index) of each assembled value
  std::vector<int32_t> anew_slot, anew_col;     // its slot and local column in the front
  std::vector<int32_t> new_rows;                // original rows entering each front
  std::vector<int32_t> col_perm;                // position -> original column
  // schedule
  std::vector<int32_t> small_level_ptr, small_level_fronts;  // batched levels (leaves first)
  std::vector<int32_t> big_order;                            // large fronts in postorder
  int n_lanes = 1;                                           // concurrent lanes of large fronts
  std::vector<int32_t> lane_ptr, lane_fronts;                // each lane's large fronts, postorder
  std::vector<int32_t> top_fronts;                           // large fronts after all lanes, postorder
  std::vector<int64_t> lane_front_buf;                       // front buffer (entries) per lane
  std::vector<int32_t> solve_level_ptr, solve_level_fronts;  // all fronts by height (leaves first)
  std::vector<int64_t> csr_ptr, csr_map;                     // A by rows: row starts, CSC index of each entry
  std::vector<int32_t> csr_col;                              //   and its column
  // sizes of the device arenas (doubles / ints)
  int64_t block_total = 0, l_total = 0, u_total = 0, rowid_total = 0;
  int64_t stack_total = 0, front_buf = 0;
  double flops = 0.0;  // multifrontal flops of the plan (structure superset)
};

// Builds the front plan from the validated pattern and the supernodal symbolic
// structure. small_rows: fronts with at most this many rows whose children are
// all small go to the batched kernel. lanes: independent subtrees of large
// fronts are spread over up to this many concurrent lanes.
int build_front_plan(const Pattern& p, const Supernodal& S, int small_rows, int lanes, FrontPlan* out);

// A coarser partition for the GPU plan: chains of only-children merged into
// their parents while the merged front's flops grow by at most tol.
void amalgamate_chains(const FrontPlan& F, const Supernodal& S, double tol, double traffic_scale,
                       std::vector<idx>* ptr_out);
// S with another supernode partition (same order, counts and column etree).
void repartition(const Supernodal& S, const std::vector<idx>& ptr, Supernodal* out);
// S's partition cut wherever a supernode's next column is not the etree
// parent of the one before (the relaxation also merges a supernode into the
// next one in the order when that one is not its parent): every front of the
// GPU plan is then a chain of the column etree, so the unpivoted rows a front
// passes up are those of its own subtree only.
void split_at_etree_breaks(const Supernodal& S, Supernodal* out);

}  // namespace sp
}  // namespace alg
