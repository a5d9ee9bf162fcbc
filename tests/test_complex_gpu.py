"""GPU parity of the complex twins (src/lapack/complex.rs: zgetrf,
zgetrf_rect, zgesv, zgetri) against the complex oracle: identical pivots and
bit-identical factors and solutions (both run the reference's operations in
the reference's order), on the reference's own test matrices, on sizes whose
rows and columns exceed one CTA's threads and span many 16-column blocks, on
pivot ties, on NaN entries, and on the partial state a zero pivot leaves,
inside a block and at its edges."""

import numpy as np
import pytest

from algebra_linear_b200.lapack import LapackError, zgesv, zgetrf, zgetri, zgetrf_rect

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oz(oracle):
    from oracle import complex as oz

    return oz


def _rand(n_entries, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n_entries) + 1j * rng.standard_normal(n_entries)


def _same(x, y):
    return np.array_equal(x.view(np.float64), y.view(np.float64), equal_nan=True)


@pytest.mark.parametrize("case", ["general3", "sample1", "sample5", "sample8", "sample40", "rand17", "rand1030"])
def test_zgetrf_is_bit_identical(gpu, oz, case):
    if case == "general3":
        a0, n = oz.general3(), 3
    elif case.startswith("sample"):
        n = int(case[6:])
        a0 = oz.complex_sample(n)
    else:
        n = int(case[4:])
        a0 = _rand(n * n, n)
    rc, lu_ref, ipiv_ref = oz.zgetrf(a0, n)
    assert rc == oz.OK
    a = a0.copy()
    ipiv = zgetrf(a, n)
    assert ipiv == [int(v) for v in ipiv_ref]
    assert _same(a, lu_ref)


@pytest.mark.parametrize("shape", [(3, 2), (500, 37), (1100, 1030), (64, 64)])
def test_zgetrf_rect_is_bit_identical(gpu, oz, shape):
    nrows, ncols = shape
    a0 = (np.array([1 + 1j, 3 + 0j, 2 - 1j, 2 + 0j, -1j, 4 + 0j]) if shape == (3, 2)
          else _rand(nrows * ncols, nrows + 7 * ncols))  # complex.rs:601-611 for the first
    rc, lu_ref, ipiv_ref = oz.zgetrf_rect(a0, nrows, ncols)
    assert rc == oz.OK
    a = a0.copy()
    ipiv = [0] * ncols
    zgetrf_rect(a, nrows, ncols, ipiv)
    assert ipiv == [int(v) for v in ipiv_ref]
    assert _same(a, lu_ref)


@pytest.mark.parametrize("n", [1, 3, 8, 300, 1030])
def test_zgesv_is_bit_identical(gpu, oz, n):
    a0 = oz.general3() if n == 3 else (oz.complex_sample(n) if n <= 8 else _rand(n * n, 3 * n))
    x_true = np.array([complex(1.0 + 0.5 * i, -0.25 * i) for i in range(n)])
    A = a0.reshape(n, n).T
    b0 = A @ x_true
    rc, lu_ref, x_ref, _ = oz.zgesv(a0, b0)
    assert rc == oz.OK
    a, b = a0.copy(), b0.copy()
    zgesv(a, b)
    assert _same(a, lu_ref) and _same(b, x_ref)
    if n <= 8:  # parity.rs:518-549 / complex.rs:489-500
        assert np.all(np.abs(b - x_true) / np.maximum(np.abs(x_true), 1.0) < 1e-10)


def _agrees(oz, a0, n):
    """zgetrf on the GPU gives the oracle's outcome: the same pivots and
    factors, or Singular with the same partial state."""
    rc, lu_ref, ipiv_ref = oz.zgetrf(a0, n)
    a = a0.copy()
    if rc == oz.OK:
        assert zgetrf(a, n) == [int(v) for v in ipiv_ref]
    else:
        with pytest.raises(LapackError) as e:
            zgetrf(a, n)
        assert e.value.kind == "Singular"
    assert _same(a, lu_ref)
    return rc


def test_pivot_ties_take_the_first_row(gpu, oz):
    # small integers: many equal |Re| + |Im| in a column, across CTA threads
    n = 1030
    rng = np.random.default_rng(5)
    a0 = (rng.integers(-2, 3, n * n) + 1j * rng.integers(-2, 3, n * n)).astype(np.complex128)
    a0[:: n + 1] += 40.0  # far from singular
    assert _agrees(oz, a0, n) == oz.OK
    # every off-diagonal entry 1 + i, diagonal 1/2: the first column's
    # candidates below the diagonal all tie; the matrix turns singular
    n = 300
    b = np.full(n * n, 1 + 1j)
    b[:: n + 1] = 0.5
    _agrees(oz, b, n)


def test_nan_entries_follow_the_reference_scan(gpu, oz):
    # a NaN below the diagonal is never the pivot; a NaN on the diagonal keeps it
    n = 6
    for pos in [(3, 0), (0, 0), (5, 2)]:
        a0 = _rand(n * n, 11)
        a0[pos[0] + pos[1] * n] = complex(np.nan, 0.0)
        _agrees(oz, a0, n)


def test_zero_pivot_leaves_the_reference_partial_state(gpu, oz):
    # complex.rs:504-516: column 1 = 2 x column 0, singular at the second step
    assert _agrees(oz, np.array([1 + 1j, 3 + 0j, 2 + 2j, 6 + 0j]), 2) == oz.SINGULAR
    # a 5 x 5 with an exactly zero third pivot: rows 2-4 of columns 0-2 are
    # zero and column 2 = column 0 + column 1
    n = 5
    rng = np.random.default_rng(2)
    M = np.zeros((n, n), dtype=np.complex128)
    M[:2, :2] = [[2 + 1j, 0.5j], [1 - 1j, 3 + 0j]]
    M[:, 2] = M[:, 0] + M[:, 1]
    M[2:, 3:] = rng.standard_normal((3, 2)) + 1j * rng.standard_normal((3, 2))
    assert _agrees(oz, M.T.ravel().copy(), n) == oz.SINGULAR


@pytest.mark.parametrize("s", [15, 16, 17, 40, 250])
def test_zero_pivot_at_and_past_block_edges(gpu, oz, s):
    # rows s.. of columns 0..s zero: the pivots of the first s columns come
    # from the rows above, and column s meets an exactly zero pivot. The
    # factorization runs in 16-column blocks, so s = 15, 16, 17 stop at the
    # last column of a block, the first of the next and the second; the
    # columns right of the stopping block must hold exactly the updates of
    # the steps before s, as the reference's early return leaves them.
    n = 300
    rng = np.random.default_rng(s)
    M = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    M[s:, : s + 1] = 0
    assert _agrees(oz, M.T.ravel().copy(), n) == oz.SINGULAR


def _exact_singular(n, s, seed):
    """A = L U in exact dyadic arithmetic: unit-lower L whose entries have
    |Re| + |Im| <= 1 (the diagonal pivot always wins, so no interchange), U
    with a real power-of-two diagonal except u_ss = 0. Elimination then
    reproduces L and U exactly and meets an exactly zero pivot at column s
    after nonzero multipliers, so every column right of s must hold exactly
    the terms of steps 0..s-1."""
    rng = np.random.default_rng(seed)
    entries = np.array([0, 0.5, -0.5, 0.5j, -0.5j, 0.25 + 0.25j, -0.25 + 0.5j, 0.75, -0.25j, 0.5 - 0.25j])
    L = np.tril(rng.choice(entries, (n, n)), -1) + np.eye(n)
    U = np.triu(rng.integers(-3, 4, (n, n)) + 1j * rng.integers(-3, 4, (n, n)), 1).astype(np.complex128)
    U[np.arange(n), np.arange(n)] = rng.choice([1.0, 2.0, 4.0], n)
    U[s, s] = 0
    return (L @ U).T.ravel().copy()


@pytest.mark.parametrize("s", [1, 2, 3, 5, 6, 13, 17, 21, 45, 130])
def test_zero_pivot_after_nonzero_multipliers(gpu, oz, s):
    # the blocked form runs 16-column blocks of 4-column sub-panels: s falls
    # inside a sub-panel, at its edges, and in later blocks
    assert _agrees(oz, _exact_singular(300, s, s), 300) == oz.SINGULAR


@pytest.mark.parametrize("n", [1, 2, 3, 8, 100, 1030])
def test_zgetri_is_bit_identical(gpu, oz, n):
    # complex.rs:463-486 / parity.rs:463-510: zgetrf then zgetri
    a0 = oz.general3() if n == 3 else (oz.complex_sample(n) if n <= 8 else _rand(n * n, 5 * n))
    rc, lu_ref, ipiv_ref = oz.zgetrf(a0, n)
    rc, inv_ref = oz.zgetri(lu_ref, n, ipiv_ref)
    assert rc == oz.OK
    lu = lu_ref.copy()
    zgetri(lu, n, [int(v) for v in ipiv_ref])
    assert _same(lu, inv_ref)
    if n == 3:
        back = a0.reshape(3, 3).T @ lu.reshape(3, 3).T
        assert np.all(np.abs(back - np.eye(3)) < 1e-12)


def test_zgetri_zero_diagonal_leaves_the_partial_inverse(gpu, oz):
    n = 4
    lu0 = _rand(n * n, 9)
    lu0[2 + 2 * n] = 0j  # u_22 = 0: columns 0-1 inverted, then Singular
    rc, inv_ref = oz.zgetri(lu0, n, [0, 1, 2, 3])
    assert rc == oz.SINGULAR
    lu = lu0.copy()
    with pytest.raises(LapackError) as e:
        zgetri(lu, n, [0, 1, 2, 3])
    assert e.value.kind == "Singular"
    assert _same(lu, inv_ref)
