// ORACLE — test infrastructure only. Not part of the product.
//
// A CPU restatement of the reference crate's dense LU path
// (cpmech/algebra_linear 4.0.0, Rust), used only by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg, as the checker.
// The product library (libalgebra_linear_gpu.so) never links or calls it.
//
// Build: oracle/Makefile compiles this with -O3 -ffp-contract=off
// -fno-fast-math -march=x86-64, the codegen rustc uses for the reference in
// release mode (no FMA contraction, SSE2 baseline, IEEE division), so that
// every function below rounds exactly as the Rust does.
//
// Parity pins (tests/test_oracle_kat.py): the larnv known-answer stream from
// src/lapack/families.rs:1183-1261 (captured by the reference from LAPACK's
// libtmglib) and the dense-LU unit tests of src/lapack/mod.rs:461-752.

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// DLARUV / DLARNV stream — src/lapack/families.rs:22-249.
//
// The 48-bit multiplicative generator x <- x * a^i mod 2^48 with
// a = 33952834046453, the state kept as four 12-bit words. The reference holds
// a 128-row table of a^i (i = 1..128) split into 12-bit words
// (families.rs:22-151); here the same table is computed from the multiplier.
// ---------------------------------------------------------------------------
constexpr uint64_t kLaruvMultiplier = 33952834046453ULL;
constexpr uint64_t kMask48 = (1ULL << 48) - 1;
constexpr uint32_t kIpw2 = 4096;  // families.rs:154
constexpr double kR = 1.0 / 4096.0;  // families.rs:157

struct PowerTable {
  uint32_t mm[128][4];
  PowerTable() {
    unsigned __int128 p = 1;
    for (int i = 0; i < 128; ++i) {
      p = (p * kLaruvMultiplier) & kMask48;
      uint64_t v = static_cast<uint64_t>(p);
      mm[i][0] = static_cast<uint32_t>((v >> 36) & 4095);
      mm[i][1] = static_cast<uint32_t>((v >> 24) & 4095);
      mm[i][2] = static_cast<uint32_t>((v >> 12) & 4095);
      mm[i][3] = static_cast<uint32_t>(v & 4095);
    }
  }
};
const PowerTable& power_table() {
  static const PowerTable t;
  return t;
}

// families.rs:166-211 (laruv): n <= 128 uniforms in (0,1); the seed becomes
// the last product computed.
void laruv(uint32_t seed[4], size_t n, double* x) {
  if (n < 1) return;
  const auto& T = power_table();
  uint32_t i1 = seed[0], i2 = seed[1], i3 = seed[2], i4 = seed[3];
  uint32_t it1 = 0, it2 = 0, it3 = 0, it4 = 0;
  for (size_t i = 0; i < n && i < 128; ++i) {
    const uint32_t m1 = T.mm[i][0], m2 = T.mm[i][1], m3 = T.mm[i][2], m4 = T.mm[i][3];
    for (;;) {
      it4 = i4 * m4;
      it3 = it4 / kIpw2;
      it4 -= kIpw2 * it3;
      it3 += i3 * m4 + i4 * m3;
      it2 = it3 / kIpw2;
      it3 -= kIpw2 * it2;
      it2 += i2 * m4 + i3 * m3 + i4 * m2;
      it1 = it2 / kIpw2;
      it2 -= kIpw2 * it1;
      it1 += i1 * m4 + i2 * m3 + i3 * m2 + i4 * m1;
      it1 %= kIpw2;
      const double v = kR * (static_cast<double>(it1) +
                             kR * (static_cast<double>(it2) +
                                   kR * (static_cast<double>(it3) + kR * static_cast<double>(it4))));
      if (v == 1.0) {  // families.rs:191-200: step the seed and draw again
        i1 += 2; i2 += 2; i3 += 2; i4 += 2;
        continue;
      }
      x[i] = v;
      break;
    }
  }
  seed[0] = it1; seed[1] = it2; seed[2] = it3; seed[3] = it4;
}

}  // namespace

extern "C" {

// Error codes of the dense path; the same numbering as include/algebra_linear_gpu.h.
enum { OR_OK = 0, OR_SINGULAR = 1, OR_BAD_SHAPE = 2 };

// families.rs:230-249 (larnv). dist: 1 Uniform(0,1), 2 Symmetric(-1,1), 3 Normal(0,1).
void oracle_larnv(int dist, uint32_t seed[4], size_t n, double* x) {
  double u[128];
  size_t iv = 0;
  while (iv < n) {
    const size_t il = (n - iv) < 64 ? (n - iv) : 64;
    const size_t il2 = dist == 3 ? 2 * il : il;
    laruv(seed, il2, u);
    for (size_t i = 0; i < il; ++i) {
      double v;
      if (dist == 1) {
        v = u[i];
      } else if (dist == 2) {
        v = 2.0 * u[i] - 1.0;
      } else {
        v = std::sqrt(-2.0 * std::log(u[2 * i])) * std::cos(6.283185307179586 * u[2 * i + 1]);
      }
      x[iv + i] = v;
    }
    iv += 64;
  }
}

// mod.rs:112-163 (dgetrf_with_pivots), steps k0 <= k < k1 of the unblocked
// right-looking LU with partial pivoting: pivot search, whole-row swap,
// multipliers by division, rank-1 update. d_acc follows the determinant
// (sign flip per interchange, times the pivot). Returns the first column
// with a zero pivot, or n.
static size_t getrf_steps(double* a, size_t n, size_t k0, size_t k1, size_t* ipiv, double* d_acc) {
  for (size_t k = k0; k < k1; ++k) {
    size_t pivot = k;
    double best = std::fabs(a[k + k * n]);
    for (size_t i = k + 1; i < n; ++i) {
      const double cand = std::fabs(a[i + k * n]);
      if (cand > best) { best = cand; pivot = i; }
    }
    if (best <= 0.0) return k;
    if (pivot != k) {
      for (size_t j = 0; j < n; ++j) {
        const double t = a[j * n + k];
        a[j * n + k] = a[j * n + pivot];
        a[j * n + pivot] = t;
      }
      *d_acc = -*d_acc;
    }
    ipiv[k] = pivot;
    const double d = a[k + k * n];
    *d_acc *= d;
    for (size_t i = k + 1; i < n; ++i) {
      const double factor = a[i + k * n] / d;
      a[i + k * n] = factor;
      for (size_t j = k + 1; j < n; ++j) {
        a[i + j * n] -= factor * a[k + j * n];
      }
    }
  }
  return n;
}

// mod.rs:112-163 (dgetrf_with_pivots). Unblocked right-looking LU with
// partial pivoting; ipiv 0-based sequential interchanges; det = ±prod(u_kk).
// On a zero pivot returns OR_SINGULAR with `a` partially factored, and
// *bad_col (if given) names the column.
int oracle_dgetrf(double* a, size_t n, size_t* ipiv, double* det, size_t* bad_col) {
  if (det) *det = 1.0;
  if (n == 0) return OR_OK;
  double d_acc = 1.0;
  const size_t bad = getrf_steps(a, n, 0, n, ipiv, &d_acc);
  if (bad < n) {
    if (bad_col) *bad_col = bad;
    return OR_SINGULAR;
  }
  if (det) *det = d_acc;
  return OR_OK;
}

// Steps k0 <= k < k1 of the same factorization, continuing where an earlier
// call stopped (a bounded sample of a large LU for timing the reference's
// path); OR_SINGULAR on a zero pivot.
int oracle_dgetrf_range(double* a, size_t n, size_t k0, size_t k1, size_t* ipiv) {
  double d_acc = 1.0;
  if (k1 > n) k1 = n;
  return getrf_steps(a, n, k0, k1, ipiv, &d_acc) < n ? OR_SINGULAR : OR_OK;
}

// mod.rs:202-238 (dgetrf_rect): the same loop on an nrows x ncols panel,
// swaps restricted to the panel's columns, no determinant.
int oracle_dgetrf_rect(double* a, size_t nrows, size_t ncols, size_t* ipiv) {
  if (nrows < ncols) return OR_BAD_SHAPE;
  for (size_t k = 0; k < ncols; ++k) {
    size_t pivot = k;
    double best = std::fabs(a[k + k * nrows]);
    for (size_t i = k + 1; i < nrows; ++i) {
      const double cand = std::fabs(a[i + k * nrows]);
      if (cand > best) { best = cand; pivot = i; }
    }
    if (best <= 0.0) return OR_SINGULAR;
    if (pivot != k) {
      for (size_t j = 0; j < ncols; ++j) {
        const double t = a[j * nrows + k];
        a[j * nrows + k] = a[j * nrows + pivot];
        a[j * nrows + pivot] = t;
      }
    }
    ipiv[k] = pivot;
    const double d = a[k + k * nrows];
    for (size_t i = k + 1; i < nrows; ++i) {
      const double factor = a[i + k * nrows] / d;
      a[i + k * nrows] = factor;
      for (size_t j = k + 1; j < ncols; ++j) {
        a[i + j * nrows] -= factor * a[k + j * nrows];
      }
    }
  }
  return OR_OK;
}

// mod.rs:330-354 (dgetrs), applied column by column to nrhs right-hand sides
// stored column-major (n x nrhs). For nrhs = 1 it is the reference's sweep.
void oracle_dgetrs(const double* lu, const size_t* ipiv, double* b, size_t n, size_t nrhs) {
  for (size_t r = 0; r < nrhs; ++r) {
    double* x = b + r * n;
    for (size_t k = 0; k < n; ++k) {
      const double t = x[k]; x[k] = x[ipiv[k]]; x[ipiv[k]] = t;
    }
    for (size_t i = 0; i < n; ++i) {
      double sum = x[i];
      for (size_t j = 0; j < i; ++j) sum -= lu[i + j * n] * x[j];
      x[i] = sum;
    }
    for (size_t i = n; i-- > 0;) {
      double sum = x[i];
      for (size_t j = i + 1; j < n; ++j) sum -= lu[i + j * n] * x[j];
      x[i] = sum / lu[i + i * n];
    }
  }
}

// mod.rs:249-298 (dgetri): the inverse from dgetrf's factors, column by
// column (the interchanges in dgetrf's order, the unit-lower row-dot sweep,
// the upper sweep dividing by u_ii), written over lu only when every column
// succeeded; OR_SINGULAR on a zero diagonal of U.
int oracle_dgetri(double* lu, size_t n, const size_t* ipiv) {
  if (n == 0) return OR_OK;
  std::vector<double> inverse(n * n, 0.0), b(n);
  for (size_t col = 0; col < n; ++col) {
    std::fill(b.begin(), b.end(), 0.0);
    b[col] = 1.0;
    for (size_t k = 0; k < n; ++k) {
      const double t = b[k]; b[k] = b[ipiv[k]]; b[ipiv[k]] = t;
    }
    for (size_t i = 0; i < n; ++i) {
      double sum = b[i];
      for (size_t j = 0; j < i; ++j) sum -= lu[i + j * n] * b[j];
      b[i] = sum;
    }
    for (size_t i = n; i-- > 0;) {
      double sum = b[i];
      for (size_t j = i + 1; j < n; ++j) sum -= lu[i + j * n] * b[j];
      const double d = lu[i + i * n];
      if (d == 0.0) return OR_SINGULAR;
      b[i] = sum / d;
    }
    for (size_t i = 0; i < n; ++i) inverse[i + col * n] = b[i];
  }
  std::memcpy(lu, inverse.data(), n * n * sizeof(double));
  return OR_OK;
}

// mod.rs:309-323 (dgesv) generalised to nrhs columns: dgetrf then dgetrs.
int oracle_dgesv(double* a, double* b, size_t n, size_t nrhs, size_t* ipiv_out) {
  if (n == 0) return OR_OK;
  std::vector<size_t> ipiv(n);
  const int rc = oracle_dgetrf(a, n, ipiv.data(), nullptr, nullptr);
  if (rc != OR_OK) return rc;
  oracle_dgetrs(a, ipiv.data(), b, n, nrhs);
  if (ipiv_out) std::memcpy(ipiv_out, ipiv.data(), n * sizeof(size_t));
  return OR_OK;
}

// blas.rs:102-130 (dgemv, trans = 'N', alpha = 1, beta = 0): y = A x.
void oracle_dgemv(const double* a, const double* x, double* y, size_t m, size_t n) {
  for (size_t i = 0; i < m; ++i) y[i] = 0.0;
  for (size_t j = 0; j < n; ++j) {
    const double c = x[j];
    if (c == 0.0) continue;
    const double* col = a + j * m;
    for (size_t i = 0; i < m; ++i) y[i] += c * col[i];
  }
}

// blas.rs:77-88 (idamax): first index of max |x_i|; 0 for an empty slice.
size_t oracle_idamax(const double* x, size_t n) {
  size_t best = 0;
  double best_abs = -INFINITY;
  for (size_t i = 0; i < n; ++i) {
    const double v = std::fabs(x[i]);
    if (v > best_abs) { best_abs = v; best = i; }
  }
  return best;
}

// blas.rs:1384-1438 (dtrsm left side, no transpose; alpha = 1):
// B := A^{-1} B for an m x m triangle, B m x n column-major.
void oracle_dtrsm_left(const double* a, double* b, size_t m, size_t n, int lower, int unit) {
  for (size_t c = 0; c < n; ++c) {
    double* x = b + c * m;
    if (lower) {
      for (size_t i = 0; i < m; ++i) {
        double sum = x[i];
        for (size_t k = 0; k < i; ++k) sum -= a[i + k * m] * x[k];
        if (!unit) sum /= a[i + i * m];
        x[i] = sum;
      }
    } else {
      for (size_t i = m; i-- > 0;) {
        double sum = x[i];
        for (size_t k = i + 1; k < m; ++k) sum -= a[i + k * m] * x[k];
        if (!unit) sum /= a[i + i * m];
        x[i] = sum;
      }
    }
  }
}

// accuracy_tests.rs:57-67 (scaled_residual), for column r of an n x nrhs
// system: ||A x - b||_inf / (||A||_inf ||x||_inf + ||b||_inf), the normwise
// backward error. A x is formed row-dot as accuracy_tests.rs:45-53 does.
double oracle_backward_error(const double* a, const double* x, const double* b, size_t n) {
  if (n == 0) return 0.0;
  double rmax = 0.0, anorm = 0.0, xmax = 0.0, bmax = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double s = 0.0, rs = 0.0;
    for (size_t j = 0; j < n; ++j) {
      s += a[i + j * n] * x[j];
      rs += std::fabs(a[i + j * n]);
    }
    rmax = std::fmax(rmax, std::fabs(s - b[i]));
    anorm = std::fmax(anorm, rs);
    xmax = std::fmax(xmax, std::fabs(x[i]));
    bmax = std::fmax(bmax, std::fabs(b[i]));
  }
  const double denom = anorm * xmax + bmax;
  return denom == 0.0 ? rmax : rmax / denom;
}

// checkers.rs:17-63 (get01): ||L U - P A||_1 / (n ||A||_1 eps).
double oracle_get01(const double* a, const double* lu, const size_t* ipiv, size_t m, size_t n) {
  if (m == 0 || n == 0) return 0.0;
  const double eps = 2.220446049250313e-16;
  auto norm1 = [&](const double* x) {
    double best = 0.0;
    for (size_t j = 0; j < n; ++j) {
      double s = 0.0;
      for (size_t i = 0; i < m; ++i) s += std::fabs(x[i + j * m]);
      best = std::fmax(best, s);
    }
    return best;
  };
  const double anorm = norm1(a);
  const size_t k = m < n ? m : n;
  std::vector<double> prod(m * n, 0.0);
  for (size_t j = 0; j < n; ++j) {
    for (size_t i = 0; i < m; ++i) {
      double sum = 0.0;
      for (size_t p = 0; p < k; ++p) {
        if (p > i || p > j) continue;
        const double l = p == i ? 1.0 : lu[i + p * m];
        sum += l * lu[p + j * m];
      }
      prod[i + j * m] = sum;
    }
  }
  for (size_t i = k; i-- > 0;) {
    const size_t p = ipiv[i];
    if (p != i) {
      for (size_t j = 0; j < n; ++j) {
        const double t = prod[i + j * m]; prod[i + j * m] = prod[p + j * m]; prod[p + j * m] = t;
      }
    }
  }
  for (size_t idx = 0; idx < m * n; ++idx) prod[idx] -= a[idx];
  const double resid = norm1(prod.data());
  if (anorm <= 0.0) return resid != 0.0 ? 1.0 / eps : 0.0;
  return (resid / static_cast<double>(n) / anorm) / eps;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// DLATMS for general (nonsymmetric, full) matrices — families.rs:255-370 and
// 903-1078: the spectrum from latm1, scaled to dmax, then A = U D V with U
// and V built one Householder reflection at a time from both sides (dlagge),
// every reflector drawn from the Normal larnv stream and normed by the
// reference BLAS's running-scale dnrm2. The test matrices of the sparse
// accuracy tests (accuracy_tests.rs:15-30) come from here.
// ---------------------------------------------------------------------------
namespace {

// x^i for i >= 0 by binary exponentiation, the algorithm of the __powidf2
// runtime routine that rustc's f64::powi lowers to for a variable exponent
double powi_binary(double a, int b) {
  const bool recip = b < 0;
  unsigned p = recip ? 0u - (unsigned)b : (unsigned)b;
  double r = 1.0;
  for (;;) {
    if (p & 1u) r *= a;
    p >>= 1;
    if (p == 0) break;
    a *= a;
  }
  return recip ? 1.0 / r : r;
}

double laran(uint32_t seed[4]) {
  double x[1];
  laruv(seed, 1, x);
  return x[0];
}

double dnrm2_reference(const double* x, size_t n) {
  double scale = 0.0, ssq = 1.0;
  for (size_t i = 0; i < n; ++i) {
    const double absxi = std::fabs(x[i]);
    if (absxi > 0.0) {
      if (scale < absxi) {
        const double r = scale / absxi;
        ssq = 1.0 + ssq * r * r;
        scale = absxi;
      } else {
        const double r = absxi / scale;
        ssq += r * r;
      }
    }
  }
  return scale * std::sqrt(ssq);
}

}  // namespace

extern "C" {

// families.rs:280-356 (latm1). dist as oracle_larnv. Returns INFO.
int oracle_latm1(int mode, double cond, int irsign, int dist, uint32_t seed[4], size_t n, double* d) {
  const bool ordinary = mode != -6 && mode != 0 && mode != 6;
  if (mode < -6 || mode > 6) return -1;
  if (ordinary && irsign != 0 && irsign != 1) return -2;
  if (ordinary && cond < 1.0) return -3;
  if (n == 0 || mode == 0) return 0;
  switch (mode < 0 ? -mode : mode) {
    case 1:
      for (size_t i = 0; i < n; ++i) d[i] = 1.0 / cond;
      d[0] = 1.0;
      break;
    case 2:
      for (size_t i = 0; i < n; ++i) d[i] = 1.0;
      d[n - 1] = 1.0 / cond;
      break;
    case 3:
      d[0] = 1.0;
      if (n > 1) {
        const double alpha = std::pow(cond, -1.0 / (double)(n - 1));
        for (size_t i = 1; i < n; ++i) d[i] = powi_binary(alpha, (int)i);
      }
      break;
    case 4:
      d[0] = 1.0;
      if (n > 1) {
        const double temp = 1.0 / cond;
        const double alpha = (1.0 - temp) / (double)(n - 1);
        for (size_t i = 1; i < n; ++i) d[i] = (double)(n - i - 1) * alpha + temp;
      }
      break;
    case 5: {
      const double alpha = std::log(1.0 / cond);
      for (size_t i = 0; i < n; ++i) d[i] = std::exp(alpha * laran(seed));
      break;
    }
    default:
      oracle_larnv(dist, seed, n, d);
  }
  if (ordinary && irsign == 1)
    for (size_t i = 0; i < n; ++i)
      if (laran(seed) > 0.5) d[i] = -d[i];
  if (mode < 0)
    for (size_t i = 0, j = n - 1; i < j; ++i, --j) std::swap(d[i], d[j]);
  return 0;
}

// families.rs:903-992 (dlatms) for SYM = nonsymmetric, PACK = full, and
// 994-1078 (dlagge). a is m x n column-major, d min(m, n) entries (read when
// mode == 0). Returns INFO (the reference's codes that apply to this form).
int oracle_dlatms_general(int dist, int mode, double cond, double dmax, size_t m, size_t n, double* a, double* d,
                          uint32_t seed[4]) {
  const size_t mnmin = m < n ? m : n;
  if (m == 0 || n == 0) return 0;
  if (mode < -6 || mode > 6) return -7;
  if (mode != 0 && mode != 6 && mode != -6 && cond < 1.0) return -8;
  for (int k = 0; k < 4; ++k) seed[k] %= 4096;
  if (seed[3] % 2 != 1) seed[3] += 1;
  if (oracle_latm1(mode, cond, 0, dist, seed, mnmin, d) != 0) return 1;
  if (mode != 0 && mode != 6 && mode != -6) {
    double temp = 0.0;
    for (size_t i = 0; i < mnmin; ++i) temp = std::max(temp, std::fabs(d[i]));
    if (!(temp > 0.0)) return 2;
    const double alpha = dmax / temp;
    for (size_t i = 0; i < mnmin; ++i) d[i] *= alpha;
  }
  for (size_t k = 0; k < m * n; ++k) a[k] = 0.0;
  for (size_t i = 0; i < mnmin; ++i) a[i + i * m] = d[i];
  if (m == 1 && n == 1) return 0;
  const size_t lw = m > n ? m : n;
  std::vector<double> w(lw), y(lw);
  auto reflector = [&](size_t len) -> double {  // w <- the reflector, returns tau
    oracle_larnv(3, seed, len, w.data());
    const double wn = dnrm2_reference(w.data(), len);
    const double wa = w[0] < 0.0 ? -wn : wn;
    if (wn == 0.0) return 0.0;
    const double wb = w[0] + wa;
    const double inv = 1.0 / wb;
    for (size_t k = 1; k < len; ++k) w[k] *= inv;
    w[0] = 1.0;
    return wb / wa;
  };
  for (size_t i = mnmin; i-- > 0;) {
    if (i + 1 < m) {  // A(i:m, i:n) -= tau w (w^T A(i:m, i:n))
      const size_t len = m - i;
      const double tau = reflector(len);
      if (tau != 0.0) {
        const size_t ncols = n - i;
        for (size_t j = 0; j < ncols; ++j) {
          double sum = 0.0;
          for (size_t k = 0; k < len; ++k) sum += a[(i + k) + (i + j) * m] * w[k];
          y[j] = sum;
        }
        for (size_t j = 0; j < ncols; ++j)
          for (size_t k = 0; k < len; ++k) a[(i + k) + (i + j) * m] -= tau * w[k] * y[j];
      }
    }
    if (i + 1 < n) {  // A(i:m, i:n) -= tau (A(i:m, i:n) w) w^T
      const size_t len = n - i;
      const double tau = reflector(len);
      if (tau != 0.0) {
        const size_t nrows = m - i;
        for (size_t k = 0; k < nrows; ++k) {
          double sum = 0.0;
          for (size_t j = 0; j < len; ++j) sum += a[(i + k) + (i + j) * m] * w[j];
          y[k] = sum;
        }
        for (size_t j = 0; j < len; ++j)
          for (size_t k = 0; k < nrows; ++k) a[(i + k) + (i + j) * m] -= tau * y[k] * w[j];
      }
    }
  }
  return 0;
}

}  // extern "C"

