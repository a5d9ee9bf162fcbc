"""The complex oracle (a restatement of src/lapack/complex.rs) against the
reference's own complex tests and against LAPACK through scipy (CPU only)."""

import numpy as np
import pytest

from oracle import complex as oz


def _mat_vec(a, x, n):
    return np.array([sum(a[i + j * n] * x[j] for j in range(n)) for i in range(n)])


def _reconstruct(lu, nrows, ncols):
    """L U of a packed rectangular factorization (unit-lower L, upper U)."""
    A = lu.reshape(ncols, nrows).T
    L = np.tril(A, -1)[:, :ncols] + np.eye(nrows, ncols)
    U = np.triu(A[:ncols, :ncols])
    return L @ U


def _permuted(a, nrows, ncols, ipiv):
    pa = a.reshape(ncols, nrows).T.copy()
    for k, p in enumerate(int(v) for v in ipiv):
        pa[[k, p], :] = pa[[p, k], :]
    return pa


def test_zgesv_recovers_a_known_solution():
    # complex.rs:489-500
    a = oz.general3()
    x_true = np.array([1 - 2j, 3 + 0.5j, -1 + 1j])
    b = _mat_vec(a, x_true, 3)
    rc, _, x, _ = oz.zgesv(a, b)
    assert rc == oz.OK
    assert np.all(np.abs(x - x_true) < 1e-12), x


def test_zgetrf_factors_general3():
    # complex.rs:463-486: the last pivot is n - 1; P A = L U
    a = oz.general3()
    rc, lu, ipiv = oz.zgetrf(a, 3)
    assert rc == oz.OK and int(ipiv[-1]) == 2
    np.testing.assert_allclose(_reconstruct(lu, 3, 3), _permuted(a, 3, 3, ipiv), rtol=0, atol=1e-12)


def test_zgetrf_detects_a_singular_matrix():
    # complex.rs:504-516: column 1 = 2 x column 0
    a = np.array([1 + 1j, 3 + 0j, 2 + 2j, 6 + 0j])
    rc, _, _ = oz.zgetrf(a, 2)
    assert rc == oz.SINGULAR


def test_bad_shapes_and_empty_input():
    # complex.rs:518-529, 582-590, 640-645
    assert oz.zgetrf(np.ones(3, dtype=complex), 2)[0] == oz.BAD_SHAPE
    assert oz.zgesv(np.ones(3, dtype=complex), np.ones(2, dtype=complex))[0] == oz.BAD_SHAPE
    assert oz.zgetrf_rect(np.ones(4, dtype=complex), 1, 2)[0] == oz.BAD_SHAPE
    rc, _, ipiv = oz.zgetrf(np.zeros(0, dtype=complex), 0)
    assert rc == oz.OK and ipiv.size == 0
    assert oz.zgesv(np.zeros(0, dtype=complex), np.zeros(0, dtype=complex))[0] == oz.OK


def test_zgetrf_rect_reconstructs_a_tall_panel():
    # complex.rs:601-638
    a0 = np.array([1 + 1j, 3 + 0j, 2 - 1j, 2 + 0j, -1j, 4 + 0j])
    rc, lu, ipiv = oz.zgetrf_rect(a0, 3, 2)
    assert rc == oz.OK
    np.testing.assert_allclose(_reconstruct(lu, 3, 2), _permuted(a0, 3, 2, ipiv), rtol=0, atol=1e-12)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8])
def test_complex_sample_solve(n):
    # parity.rs:518-549: x_true recovered to 1e-10 (relative to max(|x|, 1))
    a = oz.complex_sample(n)
    x_true = np.array([complex(1.0 + 0.5 * i, -0.25 * i) for i in range(n)])
    b = _mat_vec(a, x_true, n)
    rc, _, x, _ = oz.zgesv(a, b)
    assert rc == oz.OK
    assert np.all(np.abs(x - x_true) / np.maximum(np.abs(x_true), 1.0) < 1e-10)


@pytest.mark.parametrize("n", [7, 64])
def test_pivots_and_factors_agree_with_lapack(n):
    # LAPACK's zgetrf picks pivots by the same |Re| + |Im| rule: on random
    # input (no ties) the pivots agree and the factors agree to rounding
    import scipy.linalg as sl

    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    rc, lu, ipiv = oz.zgetrf(A.T.ravel(), n)
    assert rc == oz.OK
    lu_ref, piv_ref = sl.lu_factor(A)
    assert np.array_equal(ipiv.astype(np.int64), piv_ref.astype(np.int64))
    np.testing.assert_allclose(lu.reshape(n, n).T, lu_ref, rtol=0, atol=1e-12 * n)


def test_zgetrf_then_zgetri_inverts():
    # complex.rs:463-486: A * inv(A) = I to 1e-12
    a = oz.general3()
    rc, lu, ipiv = oz.zgetrf(a, 3)
    rc, inv = oz.zgetri(lu, 3, ipiv)
    assert rc == oz.OK
    back = a.reshape(3, 3).T @ inv.reshape(3, 3).T
    assert np.all(np.abs(back - np.eye(3)) < 1e-12)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8])
def test_complex_inverse_agrees_with_lapack(n):
    # parity.rs:463-510 compares with the reference LAPACK at TOL 1e-10 (relative to max(|want|, 1))
    a = oz.complex_sample(n)
    rc, lu, ipiv = oz.zgetrf(a, n)
    rc, inv = oz.zgetri(lu, n, ipiv)
    assert rc == oz.OK
    want = np.linalg.inv(a.reshape(n, n).T)
    got = inv.reshape(n, n).T
    assert np.all(np.abs(got - want) / np.maximum(np.abs(want), 1.0) < 1e-10)


def test_zgetri_zero_diagonal_is_singular():
    # ztrti2's test (complex.rs:134-137): an exactly zero u_jj
    lu = np.array([2 + 0j, 0.5 + 0j, 1 + 1j, 0j])  # u_11 = 0
    rc, inv = oz.zgetri(lu, 2, [0, 1])
    assert rc == oz.SINGULAR
    assert inv[0] == 0.5  # column 0 already inverted: 1 / 2
