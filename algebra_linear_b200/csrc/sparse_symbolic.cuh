// Host-side symbolic analysis of the sparse LU: CSC validation, the pattern
// fingerprint, the COLAMD column ordering (postordered through the column
// elimination tree), the column counts of chol(A^T A), the fundamental
// supernode partition and its relaxation. Integer work that runs once per
// pattern on the host, as in the reference (src/sparse/faer/symbolic.rs,
// colamd.rs, etree.rs, supernodal.rs); its results must equal the
// reference's exactly, since they fix the factor structure and the order of
// every floating-point operation of the numeric factorization.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace alg {
namespace sp {

using idx = int64_t;

// Status values (the reference's sparse Error, src/sparse/faer/error.rs:5-24).
enum : int {
  SP_OK = 0,
  SP_BAD_SHAPE = 100,
  SP_INVALID_STRUCTURE = 101,
  SP_UNSORTED_ROWS = 102,
  SP_DUPLICATE_ENTRY = 103,
  SP_SINGULAR = 104,
  SP_INDEX_OVERFLOW = 105,
  SP_STRUCTURE_MISMATCH = 106,
  SP_NOT_FINITE = 107,
  SP_NOT_FACTORIZED = 108,
};

// A borrowed n x n CSC pattern (validated).
struct Pattern {
  idx n = 0;
  const size_t* col_ptr = nullptr;  // n + 1
  const size_t* row_idx = nullptr;  // col_ptr[n]
  idx nnz() const { return (idx)col_ptr[n]; }
};

// CscPattern::new (src/sparse/faer/csc.rs:39-76) for nrows x ncols.
int validate_csc(size_t nrows, size_t ncols, const size_t* col_ptr, size_t col_ptr_len, const size_t* row_idx,
                 size_t row_idx_len);

// FNV-1a over the little-endian bytes of col_ptr then row_idx as 64-bit words
// (src/sparse/faer/symbolic.rs:112-121).
uint64_t fingerprint(const Pattern& p);

// COLAMD ordering with faer's controls (dense_row, dense_col, aggressive);
// perm[new] = old, perm_inv[old] = new (src/sparse/faer/colamd.rs:190-651).
int colamd_order(const Pattern& p, double dense_row, double dense_col, bool aggressive, std::vector<idx>* perm,
                 std::vector<idx>* perm_inv);

// Column elimination tree of A (columns permuted by perm when given) and a
// postorder of a forest (src/sparse/faer/etree.rs:24-105).
void col_etree(const Pattern& p, const idx* perm, std::vector<idx>* etree);
void postorder(const std::vector<idx>& etree, std::vector<idx>* post);

// The supernodal symbolic structure (src/sparse/faer/supernodal.rs).
struct Supernodal {
  idx n = 0;
  std::vector<idx> col_perm, col_perm_inv;  // COLAMD, postordered
  std::vector<idx> col_counts;              // chol(A^T A) column counts, diagonal included
  std::vector<idx> etree;                   // column etree (permuted), -1 = root
  std::vector<idx> supernode_ptr;           // relaxed partition
  std::vector<idx> super_etree;
  idx n_supernodes() const { return (idx)supernode_ptr.size() - 1; }
};

// analyze_with_permutation + with_relaxation(max_child, tol)
// (src/sparse/faer/supernodal.rs:67-208).
int supernodal_analyze(const Pattern& p, const std::vector<idx>& perm, const std::vector<idx>& perm_inv,
                       idx max_child_size, double fill_tolerance, Supernodal* out);

}  // namespace sp
}  // namespace alg
