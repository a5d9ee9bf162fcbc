// ORACLE — test infrastructure only. Not part of the product.
//
// A CPU restatement of the reference crate's complex dense LU and inverse
// (cpmech/algebra_linear 4.0.0, src/lapack/complex.rs), used only by tests/
// as the checker of the GPU complex path. Built by oracle/Makefile with
// -ffp-contract=off -fno-fast-math (rustc's release codegen: every product,
// sum and quotient rounded on its own).
//
// Complex arithmetic. The reference's Complex64 is num_complex::Complex<f64>
// (Cargo.toml: num-complex = "0.4", not vendored). Its published operators,
// restated here:
//   (a + ib)(c + id) = (ac - bd) + i(ad + bc)
//   (a + ib)/(c + id) = ((ac + bd) + i(bc - ad)) / (c c + d d)
//   (a + ib) - (c + id) = (a - c) + i(b - d)
// and the compound assignments `*=`, `/=` assign the binary result, `-=`
// subtracts component-wise. The pivot measure is LAPACK's |Re| + |Im|
// (complex.rs:45-53).
//
// Parity pins (tests/test_oracle_complex.py): the unit tests of
// src/lapack/complex.rs:463-646 (general3 solve, singular 2 x 2, shapes,
// empty input, the tall zgetrf_rect panel) and the complex_sample solve of
// src/parity.rs:76-90 / 518-575 (x_true recovered to 1e-10).

#include <cmath>
#include <cstddef>
#include <vector>

namespace {

struct cplx {
  double re, im;
};

inline cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cplx cdiv(cplx a, cplx b) {
  const double norm_sqr = b.re * b.re + b.im * b.im;
  const double re = a.re * b.re + a.im * b.im;
  const double im = a.im * b.re - a.re * b.im;
  return {re / norm_sqr, im / norm_sqr};
}
inline cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
inline double abs1(cplx z) { return std::fabs(z.re) + std::fabs(z.im); }
inline cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }

}  // namespace

extern "C" {

// Error codes of the dense path; the same numbering as include/algebra_linear_gpu.h.
enum { OZ_OK = 0, OZ_SINGULAR = 1, OZ_BAD_SHAPE = 2 };

// complex.rs:67-124 (zgetrf / zgetf2): per column the first row with the
// largest |Re| + |Im|, singular when that is <= 0 (ZERO_DETERMINANT), the whole
// rows swapped, the column below the pivot divided by it, then the rank-1
// update column by column. On a zero pivot `a` is left as the loop left it.
int oracle_zgetrf(cplx* a, size_t n, size_t* ipiv) {
  for (size_t j = 0; j < n; ++j) {
    double best = abs1(a[j + j * n]);
    size_t jp = j;
    for (size_t i = j + 1; i < n; ++i) {
      const double cand = abs1(a[i + j * n]);
      if (cand > best) {
        best = cand;
        jp = i;
      }
    }
    ipiv[j] = jp;
    if (best <= 0.0) return OZ_SINGULAR;
    if (jp != j) {
      for (size_t k = 0; k < n; ++k) {
        const cplx t = a[k * n + j];
        a[k * n + j] = a[k * n + jp];
        a[k * n + jp] = t;
      }
    }
    const cplx d = a[j + j * n];
    for (size_t i = j + 1; i < n; ++i) a[i + j * n] = cdiv(a[i + j * n], d);
    for (size_t k = j + 1; k < n; ++k) {
      const cplx ajk = a[j + k * n];
      for (size_t i = j + 1; i < n; ++i) a[i + k * n] = csub(a[i + k * n], cmul(a[i + j * n], ajk));
    }
  }
  return OZ_OK;
}

// complex.rs:169-208 (zgetrf_rect): the same on an nrows x ncols panel
// (nrows >= ncols); swaps restricted to the panel's columns; ipiv[k] written
// after the singular test.
int oracle_zgetrf_rect(cplx* a, size_t nrows, size_t ncols, size_t* ipiv) {
  if (nrows < ncols) return OZ_BAD_SHAPE;
  for (size_t k = 0; k < ncols; ++k) {
    size_t pivot = k;
    double best = abs1(a[k + k * nrows]);
    for (size_t i = k + 1; i < nrows; ++i) {
      const double cand = abs1(a[i + k * nrows]);
      if (cand > best) {
        best = cand;
        pivot = i;
      }
    }
    if (best <= 0.0) return OZ_SINGULAR;
    if (pivot != k) {
      for (size_t j = 0; j < ncols; ++j) {
        const cplx t = a[j * nrows + k];
        a[j * nrows + k] = a[j * nrows + pivot];
        a[j * nrows + pivot] = t;
      }
    }
    ipiv[k] = pivot;
    const cplx d = a[k + k * nrows];
    for (size_t i = k + 1; i < nrows; ++i) {
      const cplx factor = cdiv(a[i + k * nrows], d);
      a[i + k * nrows] = factor;
      for (size_t j = k + 1; j < ncols; ++j) a[i + j * nrows] = csub(a[i + j * nrows], cmul(factor, a[k + j * nrows]));
    }
  }
  return OZ_OK;
}

// complex.rs:279-312 (zgesv): zgetrf, the interchanges applied to b in order,
// then the row-oriented sweeps: forward with the unit lower triangle (terms in
// increasing j), backward with the upper one (terms in increasing j, then the
// division by the diagonal). ipiv (n entries) receives the pivots.
int oracle_zgesv(cplx* a, cplx* b, size_t n, size_t* ipiv) {
  if (n == 0) return OZ_OK;
  const int rc = oracle_zgetrf(a, n, ipiv);
  if (rc != OZ_OK) return rc;
  for (size_t k = 0; k < n; ++k) {
    const cplx t = b[k];
    b[k] = b[ipiv[k]];
    b[ipiv[k]] = t;
  }
  for (size_t i = 0; i < n; ++i) {
    cplx sum = b[i];
    for (size_t j = 0; j < i; ++j) sum = csub(sum, cmul(a[i + j * n], b[j]));
    b[i] = sum;
  }
  for (size_t ii = n; ii-- > 0;) {
    cplx sum = b[ii];
    for (size_t j = ii + 1; j < n; ++j) sum = csub(sum, cmul(a[ii + j * n], b[j]));
    b[ii] = cdiv(sum, a[ii + ii * n]);
  }
  return OZ_OK;
}

// complex.rs:130-158 (ztrti2 'Upper', 'Non-unit') and 217-271 (zgetri): U
// inverted in place column by column (the diagonal replaced by its
// reciprocal, the column above it by -inv * (sum over k of a_ik a_kj, k in
// increasing order, from zero)); then, from the last column down, the
// column's L part moved to a work vector and zeroed and the column reduced by
// sum_k a_ik work_k (k increasing, from zero); then the interchanges undone as
// column swaps from the second-to-last pivot down. A zero u_jj returns
// OZ_SINGULAR with the columns before j already inverted.
int oracle_zgetri(cplx* a, size_t n, const size_t* ipiv) {
  for (size_t j = 0; j < n; ++j) {
    if (a[j + j * n].re == 0.0 && a[j + j * n].im == 0.0) return OZ_SINGULAR;
    const cplx inv = cdiv(cplx{1.0, 0.0}, a[j + j * n]);
    a[j + j * n] = inv;
    const cplx ajj{-inv.re, -inv.im};
    std::vector<cplx> x(j);
    for (size_t i = 0; i < j; ++i) {
      cplx sum{0.0, 0.0};
      for (size_t k = i; k < j; ++k) sum = cadd(sum, cmul(a[i + k * n], a[k + j * n]));
      x[i] = sum;
    }
    for (size_t i = 0; i < j; ++i) a[i + j * n] = cmul(ajj, x[i]);
  }
  std::vector<cplx> work(n), y(n);
  for (size_t j = n; j-- > 0;) {
    for (size_t i = j + 1; i < n; ++i) {
      work[i] = a[i + j * n];
      a[i + j * n] = cplx{0.0, 0.0};
    }
    if (j + 1 < n) {
      for (size_t i = 0; i < n; ++i) {
        cplx sum{0.0, 0.0};
        for (size_t k = j + 1; k < n; ++k) sum = cadd(sum, cmul(a[i + k * n], work[k]));
        y[i] = sum;
      }
      for (size_t i = 0; i < n; ++i) a[i + j * n] = csub(a[i + j * n], y[i]);
    }
  }
  for (size_t j = n > 0 ? n - 1 : 0; j-- > 0;) {
    const size_t jp = ipiv[j];
    if (jp != j)
      for (size_t i = 0; i < n; ++i) {
        const cplx t = a[i + j * n];
        a[i + j * n] = a[i + jp * n];
        a[i + jp * n] = t;
      }
  }
  return OZ_OK;
}

}  // extern "C"
