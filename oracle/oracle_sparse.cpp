// TEST INFRASTRUCTURE ONLY. A CPU restatement of the reference's numeric
// supernodal sparse LU, its simplicial LU and their solve, used by the tests
// and the bench's CPU baseline to check the GPU path; nothing in the product
// links or calls it.
//
// Follows src/sparse/faer/supernodal_lu.rs (factorize :145-480, lu_front
// :490-533, solve :118-133) and src/sparse/faer/lu.rs (unit_lower_solve
// :440-449, upper_solve :452-464): a left-looking supernodal LU over a given
// column permutation and supernode partition. For each supernode, the row
// set R_s (rows of A's columns in s and of the stored L columns of the
// supernodes whose U columns reach s, with a current position >= s_begin, plus
// the rows at s's positions) sorted by current position; the L front
// assembled from A and updated by every earlier stored (L, U) pair in the
// order the U entries were stored; partial pivoting on the front (first
// strict maximum of |a| from the diagonal, a zero maximum is singular,
// multipliers by the reciprocal of the pivot); the row permutation updated by
// swaps; the column set C_s after pivoting; the U front assembled, updated
// and solved with the unit lower block; exact zeros dropped on storage; at the
// end L's rows converted to positions and both factors sorted, with L's
// diagonal first and U's last. Compiled without FMA contraction, so every
// product and difference rounds separately, as in the reference.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

namespace {

constexpr size_t kNone = (size_t)-1;

// The scalar operations of the reference's SparseScalar (lu.rs:25-82) for
// f64 and for Complex64 = num_complex::Complex<f64> (num-complex 0.4, not
// vendored): |x| is the modulus hypot(re, im) for a complex entry, recip is
// num-complex's inv() = (re / (re^2 + im^2), -im / (re^2 + im^2)), products
// (ac - bd) + i(ad + bc), sums and differences component-wise.
struct zc {
  double re, im;
};
inline double s_abs(double v) { return std::fabs(v); }
inline double s_abs(zc v) { return std::hypot(v.re, v.im); }
inline double s_recip(double v) { return 1.0 / v; }
inline zc s_recip(zc v) {
  const double ns = v.re * v.re + v.im * v.im;
  return {v.re / ns, -v.im / ns};
}
inline double s_mul(double a, double b) { return a * b; }
inline zc s_mul(zc a, zc b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline void s_add(double& a, double b) { a += b; }
inline void s_add(zc& a, zc b) {
  a.re += b.re;
  a.im += b.im;
}
inline void s_sub(double& a, double b) { a -= b; }
inline void s_sub(zc& a, zc b) {
  a.re -= b.re;
  a.im -= b.im;
}
inline bool s_finite(double v) { return std::isfinite(v); }
inline bool s_finite(zc v) { return std::isfinite(v.re) && std::isfinite(v.im); }
template <typename T>
T s_zero();
template <>
double s_zero<double>() { return 0.0; }
template <>
zc s_zero<zc>() { return {0.0, 0.0}; }
template <typename T>
T s_one();
template <>
double s_one<double>() { return 1.0; }
template <>
zc s_one<zc>() { return {1.0, 0.0}; }

template <typename T>
struct FactorsT {
  size_t n = 0;
  std::vector<size_t> lp, li, up, ui, row_perm, col_perm_inv;
  std::vector<T> lv, uv;
};
using Factors = FactorsT<double>;

size_t owner_of(const std::vector<size_t>& ptr, size_t col) {
  // the supernode whose column range holds col
  return (size_t)(std::upper_bound(ptr.begin(), ptr.end(), col) - ptr.begin()) - 1;
}

// Partial-pivoting LU of the nfac leading columns of an nrows x ncols
// column-major front (supernodal_lu.rs:490-533). Returns false if singular.
template <typename T>
bool factor_front(std::vector<T>& a, size_t nrows, size_t nfac, size_t ncols, std::vector<size_t>& piv) {
  for (size_t k = 0; k < nfac; ++k) {
    size_t p = k;
    double best = s_abs(a[k + k * nrows]);
    for (size_t i = k + 1; i < nrows; ++i) {
      const double v = s_abs(a[i + k * nrows]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (best == 0.0) return false;
    if (p != k)
      for (size_t j = 0; j < ncols; ++j) std::swap(a[j * nrows + k], a[j * nrows + p]);
    piv[k] = p;
    const T inv = s_recip(a[k + k * nrows]);
    for (size_t i = k + 1; i < nrows; ++i) a[i + k * nrows] = s_mul(a[i + k * nrows], inv);
    for (size_t j = k + 1; j < ncols; ++j) {
      const T akj = a[k + j * nrows];
      for (size_t i = k + 1; i < nrows; ++i) s_sub(a[i + j * nrows], s_mul(akj, a[i + k * nrows]));
    }
  }
  return true;
}

template <typename T>
int splu_factorize_t(size_t n, const size_t* cp, const size_t* ri, const T* val, const size_t* col_perm,
                     const size_t* col_perm_inv, const size_t* sn_ptr, size_t n_sn, void** out) {
  *out = nullptr;
  const size_t nnz = cp[n];
  for (size_t q = 0; q < nnz; ++q)
    if (!s_finite(val[q])) return 107;
  std::vector<size_t> ptr(sn_ptr, sn_ptr + n_sn + 1);
  const size_t ns = n_sn;

  // A transposed, each entry's column replaced by its new position
  std::vector<size_t> tp(n + 1, 0), tcol(nnz);
  std::vector<T> tval(nnz);
  for (size_t q = 0; q < nnz; ++q) tp[ri[q] + 1] += 1;
  for (size_t r = 0; r < n; ++r) tp[r + 1] += tp[r];
  {
    std::vector<size_t> fill(tp.begin(), tp.end() - 1);
    for (size_t c = 0; c < n; ++c)
      for (size_t q = cp[c]; q < cp[c + 1]; ++q) {
        const size_t t = fill[ri[q]]++;
        tcol[t] = col_perm_inv[c];
        tval[t] = val[q];
      }
  }

  std::vector<size_t> rperm(n), rpos(n);  // position -> row, row -> position
  for (size_t i = 0; i < n; ++i) rperm[i] = rpos[i] = i;
  std::vector<std::vector<std::pair<size_t, T>>> lcol(n), ucol(n);
  std::vector<std::vector<size_t>> l_rows_to_sn(n);  // row -> supernodes whose L panel holds it
  std::vector<std::vector<size_t>> u_reach(ns);      // supernode -> earlier supernodes whose U reaches it
  std::vector<std::vector<size_t>> panel_cols(ns);   // supernode -> its C_s
  std::vector<size_t> rmark(n, 0), cmark(n, 0), rloc(n, kNone), cloc(n, kNone);
  size_t rtag = 0, ctag = 0;
  std::vector<size_t> R, C;

  auto build_cols = [&](size_t sb, size_t se) {
    ++ctag;
    C.clear();
    for (size_t i = sb; i < se; ++i) {
      const size_t row = rperm[i];
      for (size_t t = tp[row]; t < tp[row + 1]; ++t) {
        const size_t c = tcol[t];
        if (c >= se && cmark[c] != ctag) {
          cmark[c] = ctag;
          C.push_back(c);
        }
      }
      for (size_t d : l_rows_to_sn[row])
        for (size_t c : panel_cols[d])
          if (c >= se && cmark[c] != ctag) {
            cmark[c] = ctag;
            C.push_back(c);
          }
    }
    std::sort(C.begin(), C.end());
  };

  for (size_t s = 0; s < ns; ++s) {
    const size_t sb = ptr[s], se = ptr[s + 1], w = se - sb;
    // R_s
    ++rtag;
    R.clear();
    auto add_row = [&](size_t row) {
      if (rmark[row] != rtag) {
        rmark[row] = rtag;
        R.push_back(row);
      }
    };
    for (size_t j = sb; j < se; ++j) {
      const size_t pj = col_perm[j];
      for (size_t q = cp[pj]; q < cp[pj + 1]; ++q)
        if (rpos[ri[q]] >= sb) add_row(ri[q]);
    }
    for (size_t d : u_reach[s])
      for (size_t j = ptr[d]; j < ptr[d + 1]; ++j)
        for (const auto& e : lcol[j])
          if (rpos[e.first] >= sb) add_row(e.first);
    for (size_t pos = sb; pos < se; ++pos) add_row(rperm[pos]);
    std::stable_sort(R.begin(), R.end(), [&](size_t x, size_t y) { return rpos[x] < rpos[y]; });
    const size_t nr = R.size();
    for (size_t t = 0; t < nr; ++t) rloc[R[t]] = t;

    // L front: A, then every earlier (k, u) stored for each column
    std::vector<T> F(nr * w, s_zero<T>());
    for (size_t jj = 0; jj < w; ++jj) {
      const size_t pj = col_perm[sb + jj];
      for (size_t q = cp[pj]; q < cp[pj + 1]; ++q) {
        const size_t li = rloc[ri[q]];
        if (li != kNone) s_add(F[li + jj * nr], val[q]);
      }
      for (const auto& ku : ucol[sb + jj]) {
        if (ku.first >= sb) continue;
        for (const auto& rl : lcol[ku.first]) {
          const size_t li = rloc[rl.first];
          if (li != kNone) s_sub(F[li + jj * nr], s_mul(rl.second, ku.second));
        }
      }
    }
    std::vector<size_t> piv(w);
    if (!factor_front(F, nr, w, w, piv)) return 104;
    for (size_t k = 0; k < w; ++k) {
      const size_t p = piv[k];
      const size_t prow = R[p];
      const size_t newp = sb + k, oldp = rpos[prow];
      const size_t displaced = rperm[newp];
      if (oldp != newp) {
        std::swap(rperm[newp], rperm[oldp]);
        rpos[prow] = newp;
        rpos[displaced] = oldp;
      }
      if (p != k) {
        std::swap(R[k], R[p]);
        rloc[prow] = k;
        if (displaced != prow) rloc[displaced] = p;
      }
    }
    build_cols(sb, se);
    for (size_t t = 0; t < C.size(); ++t) cloc[C[t]] = t;
    const size_t nc = C.size();
    std::vector<T> U(nr * nc, s_zero<T>());
    for (size_t li = 0; li < nr; ++li) {
      const size_t row = R[li];
      for (size_t t = tp[row]; t < tp[row + 1]; ++t) {
        const size_t c = tcol[t];
        if (c >= se && cloc[c] != kNone) s_add(U[li + cloc[c] * nr], tval[t]);
      }
    }
    for (size_t ci = 0; ci < nc; ++ci)
      for (const auto& ku : ucol[C[ci]]) {
        if (ku.first >= sb) continue;
        for (const auto& rl : lcol[ku.first]) {
          const size_t li = rloc[rl.first];
          if (li != kNone) s_sub(U[li + ci * nr], s_mul(rl.second, ku.second));
        }
      }
    for (size_t jj = 0; jj < w; ++jj)
      for (size_t ii = jj + 1; ii < w; ++ii) {
        const T l = F[ii + jj * nr];
        for (size_t ci = 0; ci < nc; ++ci) s_sub(U[ii + ci * nr], s_mul(l, U[jj + ci * nr]));
      }
    // store, dropping exact zeros
    for (size_t jj = 0; jj < w; ++jj)
      for (size_t li = jj; li < nr; ++li) {
        const T v = li == jj ? s_one<T>() : F[li + jj * nr];
        if (li == jj || s_abs(v) != 0.0) lcol[sb + jj].push_back({R[li], v});
      }
    for (size_t jj = 0; jj < w; ++jj)
      for (size_t ii = 0; ii <= jj; ++ii) {
        const T v = F[ii + jj * nr];
        if (ii == jj || s_abs(v) != 0.0) ucol[sb + jj].push_back({sb + ii, v});
      }
    for (size_t ci = 0; ci < nc; ++ci) {
      const size_t c = C[ci];
      for (size_t ii = 0; ii < w; ++ii) {
        const T v = U[ii + ci * nr];
        if (s_abs(v) != 0.0) ucol[c].push_back({sb + ii, v});
      }
      const size_t node = owner_of(ptr, c);
      if (node > s && (u_reach[node].empty() || u_reach[node].back() != s)) u_reach[node].push_back(s);
    }
    for (size_t row : R)
      if (rpos[row] >= se) l_rows_to_sn[row].push_back(s);
    for (size_t row : R) rloc[row] = kNone;
    for (size_t c : C) cloc[c] = kNone;
    panel_cols[s] = C;
  }

  auto* f = new FactorsT<T>();
  f->n = n;
  f->lp.assign(n + 1, 0);
  f->up.assign(n + 1, 0);
  for (size_t j = 0; j < n; ++j) {
    for (auto& e : lcol[j]) e.first = rpos[e.first];
    std::stable_sort(lcol[j].begin(), lcol[j].end(),
                     [](const std::pair<size_t, T>& x, const std::pair<size_t, T>& y) { return x.first < y.first; });
    if (lcol[j].empty() || lcol[j].front().first != j) {
      delete f;
      return 101;
    }
  }
  for (size_t c = 0; c < n; ++c) {
    std::stable_sort(ucol[c].begin(), ucol[c].end(),
                     [](const std::pair<size_t, T>& x, const std::pair<size_t, T>& y) { return x.first < y.first; });
    if (ucol[c].empty() || ucol[c].back().first != c) {
      delete f;
      return 101;
    }
  }
  for (size_t j = 0; j < n; ++j) {
    f->lp[j + 1] = f->lp[j] + lcol[j].size();
    for (const auto& e : lcol[j]) {
      f->li.push_back(e.first);
      f->lv.push_back(e.second);
    }
    f->up[j + 1] = f->up[j] + ucol[j].size();
    for (const auto& e : ucol[j]) {
      f->ui.push_back(e.first);
      f->uv.push_back(e.second);
    }
  }
  f->row_perm = rperm;
  f->col_perm_inv.assign(col_perm_inv, col_perm_inv + n);
  *out = f;
  return 0;
}

// The simplicial path, lu.rs:209-327 (SymbolicLu::factorize) with
// l_incomplete_solve_sparse, reach and depth_first_search (:349-436), over
// the same column order: for the j-th column, the rows reachable from A's
// column through the L columns stored so far, in the depth-first search's
// finishing order (each search from A's rows in stored order, children in
// stored L order); x = L \ a over that reach; U takes x of the reach's
// pivoted rows at their positions, then the pivot; the pivot is the first
// unpivoted row of the reach with the largest |x| (a NaN, which compares as
// unordered, takes it); L takes 1 for the pivot row, then x_i * (1 / x_piv)
// for every other unpivoted row of the reach, zeros included. L's rows
// become positions at the end; no sorting (L's pivot first, U's diagonal
// last, as the sweeps expect). Same status codes as oracle_splu_factorize.
template <typename T>
int simplicial_factorize_t(size_t n, const size_t* cp, const size_t* ri, const T* val, const size_t* col_perm,
                           const size_t* col_perm_inv, void** out) {
  *out = nullptr;
  for (size_t q = 0; q < cp[n]; ++q)
    if (!s_finite(val[q])) return 107;
  auto* f = new FactorsT<T>;
  f->n = n;
  f->lp.assign(n + 1, 0);
  f->up.assign(n + 1, 0);
  std::vector<T> x(n, s_zero<T>());
  std::vector<size_t> marked(n, 0), reach(n), stack(n), rpi(n, n);
  for (size_t j = 0; j < n; ++j) {
    const size_t pj = col_perm[j], mark = j + 1;
    // depth-first search from b over the L columns 0..j-1; the head of the
    // path lives at reach[0..), finished rows are written down from `tail`
    auto dfs = [&](size_t b0, size_t tail) -> size_t {
      size_t head = 1;
      reach[0] = b0;
      while (head > 0) {
        const size_t b = reach[head - 1];
        const size_t pb = rpi[b];
        const size_t lo = pb < j ? f->lp[pb] : 0, hi = pb < j ? f->lp[pb + 1] : 0;
        if (marked[b] < mark) {
          marked[b] = mark;
          stack[head - 1] = lo;
        }
        bool pushed = false;
        for (size_t ptr = stack[head - 1]; ptr < hi; ++ptr) {
          const size_t i = f->li[ptr];
          if (marked[i] == mark) continue;
          stack[head - 1] = ptr;
          reach[head] = i;
          ++head;
          pushed = true;
          break;
        }
        if (pushed) continue;
        --head;
        reach[--tail] = b;
      }
      return tail;
    };
    size_t tail = n;
    for (size_t q = cp[pj]; q < cp[pj + 1]; ++q)
      if (marked[ri[q]] < mark) tail = dfs(ri[q], tail);
    for (size_t q = cp[pj]; q < cp[pj + 1]; ++q) s_add(x[ri[q]], val[q]);
    for (size_t t = tail; t < n; ++t) {
      const size_t i = reach[t], pi = rpi[i];
      if (pi >= j) continue;
      const T xi = x[i];
      for (size_t k = f->lp[pi] + 1; k < f->lp[pi + 1]; ++k) s_sub(x[f->li[k]], s_mul(f->lv[k], xi));
    }
    size_t piv = n;
    double pval = -1.0;
    for (size_t t = tail; t < n; ++t) {
      const size_t i = reach[t];
      if (rpi[i] == n) {
        const double v = s_abs(x[i]);
        if (std::isnan(v) || std::isnan(pval) || v > pval) {
          piv = i;
          pval = v;
        }
      } else {
        f->ui.push_back(rpi[i]);
        f->uv.push_back(x[i]);
      }
    }
    if (piv == n || pval == 0.0) {
      delete f;
      return 104;
    }
    const T xp = x[piv], xp_inv = s_recip(xp);
    rpi[piv] = j;
    f->ui.push_back(j);
    f->uv.push_back(xp);
    f->up[j + 1] = f->ui.size();
    f->li.push_back(piv);
    f->lv.push_back(s_one<T>());
    for (size_t t = tail; t < n; ++t) {
      const size_t i = reach[t];
      if (rpi[i] == n) {
        f->li.push_back(i);
        f->lv.push_back(s_mul(x[i], xp_inv));
      }
      x[i] = s_zero<T>();
    }
    f->lp[j + 1] = f->li.size();
  }
  for (auto& r : f->li) r = rpi[r];
  f->row_perm.assign(n, 0);
  for (size_t i = 0; i < n; ++i) f->row_perm[rpi[i]] = i;
  f->col_perm_inv.assign(col_perm_inv, col_perm_inv + n);
  *out = f;
  return 0;
}

template <typename T>
void splu_get_t(const void* h, size_t* lp, size_t* li, void* lv, size_t* up, size_t* ui, void* uv,
                size_t* row_perm) {
  const auto* f = static_cast<const FactorsT<T>*>(h);
  std::memcpy(lp, f->lp.data(), sizeof(size_t) * (f->n + 1));
  std::memcpy(up, f->up.data(), sizeof(size_t) * (f->n + 1));
  if (!f->li.empty()) {
    std::memcpy(li, f->li.data(), sizeof(size_t) * f->li.size());
    std::memcpy(lv, f->lv.data(), sizeof(T) * f->lv.size());
  }
  if (!f->ui.empty()) {
    std::memcpy(ui, f->ui.data(), sizeof(size_t) * f->ui.size());
    std::memcpy(uv, f->uv.data(), sizeof(T) * f->uv.size());
  }
  std::memcpy(row_perm, f->row_perm.data(), sizeof(size_t) * f->n);
}

// SupernodalLu::solve (supernodal_lu.rs:118-133), the same as LuFactors::solve
// (lu.rs:177-198), with the sweeps of lu.rs:440-464: permute by rows, unit
// lower sweep by columns, upper sweep from the last column (x_j times the
// reciprocal of the diagonal), permute back.
template <typename T>
void splu_solve_t(const void* h, T* b) {
  const auto* f = static_cast<const FactorsT<T>*>(h);
  const size_t n = f->n;
  std::vector<T> x(n);
  for (size_t i = 0; i < n; ++i) x[i] = b[f->row_perm[i]];
  for (size_t j = 0; j < n; ++j) {
    const T xj = x[j];
    for (size_t k = f->lp[j] + 1; k < f->lp[j + 1]; ++k) s_sub(x[f->li[k]], s_mul(f->lv[k], xj));
  }
  for (size_t j = n; j-- > 0;) {
    const size_t end = f->up[j + 1];
    const T xj = s_mul(x[j], s_recip(f->uv[end - 1]));
    x[j] = xj;
    for (size_t k = f->up[j]; k + 1 < end; ++k) s_sub(x[f->ui[k]], s_mul(f->uv[k], xj));
  }
  for (size_t i = 0; i < n; ++i) b[i] = x[f->col_perm_inv[i]];
}

}  // namespace

extern "C" {

// Status: 0 ok, 104 singular (the reference's Error::Singular), 101 invalid
// structure (a factor lost its diagonal), 107 a non-finite value. The z
// entry points take and return complex values as interleaved (re, im)
// doubles; a handle is used with the entry points of its own scalar type.
int oracle_splu_factorize(size_t n, const size_t* cp, const size_t* ri, const double* val, const size_t* col_perm,
                          const size_t* col_perm_inv, const size_t* sn_ptr, size_t n_sn, void** out) {
  return splu_factorize_t<double>(n, cp, ri, val, col_perm, col_perm_inv, sn_ptr, n_sn, out);
}
int oracle_zsplu_factorize(size_t n, const size_t* cp, const size_t* ri, const double* val, const size_t* col_perm,
                           const size_t* col_perm_inv, const size_t* sn_ptr, size_t n_sn, void** out) {
  return splu_factorize_t<zc>(n, cp, ri, reinterpret_cast<const zc*>(val), col_perm, col_perm_inv, sn_ptr, n_sn,
                              out);
}
int oracle_simplicial_factorize(size_t n, const size_t* cp, const size_t* ri, const double* val,
                                const size_t* col_perm, const size_t* col_perm_inv, void** out) {
  return simplicial_factorize_t<double>(n, cp, ri, val, col_perm, col_perm_inv, out);
}
int oracle_zsimplicial_factorize(size_t n, const size_t* cp, const size_t* ri, const double* val,
                                 const size_t* col_perm, const size_t* col_perm_inv, void** out) {
  return simplicial_factorize_t<zc>(n, cp, ri, reinterpret_cast<const zc*>(val), col_perm, col_perm_inv, out);
}

void oracle_splu_sizes(const void* h, size_t* nnz_l, size_t* nnz_u) {
  const auto* f = static_cast<const Factors*>(h);
  *nnz_l = f->lp[f->n];
  *nnz_u = f->up[f->n];
}
void oracle_zsplu_sizes(const void* h, size_t* nnz_l, size_t* nnz_u) {
  const auto* f = static_cast<const FactorsT<zc>*>(h);
  *nnz_l = f->lp[f->n];
  *nnz_u = f->up[f->n];
}

void oracle_splu_get(const void* h, size_t* lp, size_t* li, double* lv, size_t* up, size_t* ui, double* uv,
                     size_t* row_perm) {
  splu_get_t<double>(h, lp, li, lv, up, ui, uv, row_perm);
}
void oracle_zsplu_get(const void* h, size_t* lp, size_t* li, double* lv, size_t* up, size_t* ui, double* uv,
                      size_t* row_perm) {
  splu_get_t<zc>(h, lp, li, lv, up, ui, uv, row_perm);
}

void oracle_splu_solve(const void* h, double* b) { splu_solve_t<double>(h, b); }
void oracle_zsplu_solve(const void* h, double* b) { splu_solve_t<zc>(h, reinterpret_cast<zc*>(b)); }

void oracle_splu_free(void* h) { delete static_cast<Factors*>(h); }
void oracle_zsplu_free(void* h) { delete static_cast<FactorsT<zc>*>(h); }

}  // extern "C"
