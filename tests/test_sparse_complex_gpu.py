"""GPU parity of SparseLu<Complex64> (the handle generic over SparseScalar,
src/sparse/faer/lu.rs:20-82, sparse_lu.rs:45-156) against the oracle's
complex restatement of the reference's supernodal LU (num-complex
arithmetic, modulus pivots, Complex::inv multipliers), on the same patterns,
symbolic analysis and values.

Bar, as for the real handle: the row permutation (pivot sequence) identical
to the oracle's; nnz(L), nnz(U) and flops_estimate identical; x within 1e-12
relative (max(1, |x|) scale) on the grids, with the reference's own examples
(sparse_lu.rs:279-295, supernodal_lu.rs:763-805, accuracy_tests.rs:120-150)
to their stated tolerances. The GPU sums each entry's updates in another
order (multifrontal, blocked) than the reference, so values agree to
rounding."""

import numpy as np
import pytest

from algebra_linear_b200.sparse import LuMethod, SparseError, SparseLu

pytestmark = pytest.mark.gpu

COL_PTR = [0, 2, 4]
ROW_IDX = [0, 1, 0, 1]


@pytest.fixture(scope="module")
def osp(oracle):
    from oracle import sparse

    return sparse


def _complex_grid(osp, dims, seed=(1988, 1989, 1990, 1991)):
    """Convection-diffusion values with imaginary parts 0.5 U(0,1) - 0.25
    from a second DLARNV stream."""
    cp, ri, kind = osp.grid_pattern(*dims)
    v, s = osp.convection_diffusion_values(kind, list(seed))
    u, _ = osp.dense.larnv("Uniform", [7, 8, 9, 11], kind.size)
    return cp, ri, v + 1j * (0.5 * u - 0.25), s


def _compare(osp, cp, ri, v, tol=1e-12, method=LuMethod.supernodal(), nnz_exact=True):
    n = len(cp) - 1
    lu = SparseLu.analyze(cp, ri, method)
    lu.factorize(cp, ri, v)
    sym = lu.symbolic()
    ref = osp.Factors(n, cp, ri, v, sym["col_perm"], sym["col_perm_inv"], sym["supernode_ptr"])
    assert ref.status == 0 and ref.complex
    assert np.array_equal(lu.row_perm(), ref.row_perm.astype(np.int64)), "pivot sequence"
    s = lu.stats()
    if nnz_exact:
        assert (s["nnz_l"], s["nnz_u"]) == (ref.nnz_l, ref.nnz_u)
        assert s["flops_estimate"] == ref.flops_estimate()
    else:
        assert abs(s["nnz_l"] - ref.nnz_l) <= 1e-3 * ref.nnz_l
        assert abs(s["nnz_u"] - ref.nnz_u) <= 1e-3 * ref.nnz_u
    br, _ = osp.dense.larnv("Symmetric", [3, 5, 7, 9], n)
    bi, _ = osp.dense.larnv("Symmetric", [2, 4, 6, 9], n)
    b = br + 1j * bi
    x = b.copy()
    lu.solve(x)
    xr = ref.solve(b)
    err = np.max(np.abs(x - xr) / np.maximum(np.abs(xr), 1.0))
    assert err <= tol, err
    return lu


def test_every_method_solves_the_reference_example(gpu):
    # sparse_lu.rs:279-295 with complex values: [4 1; 1 3]
    for method in (LuMethod.simplicial(), LuMethod.supernodal(), LuMethod.auto()):
        lu = SparseLu.analyze(COL_PTR, ROW_IDX, method)
        lu.factorize(COL_PTR, ROW_IDX, np.array([4, 1, 1, 3], dtype=np.complex128))
        b = np.array([1.0, 2.0], dtype=np.complex128)
        lu.solve(b)
        assert np.all(np.abs(b - np.array([1 / 11, 7 / 11])) < 1e-14)


def test_tridiagonal_complex_example(gpu):
    # supernodal_lu.rs:763-805: diagonal 6 + i, off-diagonals 0.5 - 0.25 i
    n = 12
    cp, ri = [0], []
    for j in range(n):
        ri.extend(sorted({j, max(j - 1, 0), min(j + 1, n - 1)}))
        cp.append(len(ri))
    v = np.array([6 + 1j if ri[k] == j else 0.5 - 0.25j for j in range(n) for k in range(cp[j], cp[j + 1])])
    x_true = np.arange(n) + 1.0 - 0.5j
    b = np.zeros(n, dtype=np.complex128)
    for j in range(n):
        for k in range(cp[j], cp[j + 1]):
            b[ri[k]] += v[k] * x_true[j]
    for method in (LuMethod.supernodal(), LuMethod.simplicial()):
        lu = SparseLu.analyze(cp, ri, method)
        lu.factorize(cp, ri, v)
        x = b.copy()
        lu.solve(x)
        assert np.all(np.abs(x - x_true) < 1e-12)


def test_dense_dlatms_complex_accuracy(gpu, osp):
    # accuracy_tests.rs:120-150: A = Re + 0.25 i Im from two DLATMS matrices, n = 8
    n = 8
    _, re, _, _ = osp.dense.dlatms_general("Uniform", 3, 1e2, 1.0, n, n, [11, 22, 33, 44])
    _, im, _, _ = osp.dense.dlatms_general("Uniform", 3, 1e2, 1.0, n, n, [55, 66, 77, 88])
    a = re + 0.25j * im
    x_exact = np.array([complex(1.0 + i % 5, -0.5) for i in range(n)])
    b = a.reshape(n, n).T @ x_exact
    cp = list(range(0, n * n + 1, n))
    ri = [i for _ in range(n) for i in range(n)]
    for method in (LuMethod.auto(), LuMethod.supernodal(), LuMethod.simplicial()):
        lu = SparseLu.analyze(cp, ri, method)
        lu.factorize(cp, ri, a)
        x = b.copy()
        lu.solve(x)
        assert np.max(np.abs(x - x_exact)) / np.max(np.abs(x_exact)) < 1e-9


@pytest.mark.parametrize("dims", [(6, 5, 4), (12, 12, 12), (16, 16, 16), (60, 40, 1)],
                         ids=lambda d: "x".join(map(str, d)))
def test_complex_grids_match_the_oracle(gpu, osp, dims):
    # 12^3 and 16^3 have fronts of 570 and 1 299 rows: the blocked large-front path
    cp, ri, v, s = _complex_grid(osp, dims)
    lu = _compare(osp, cp, ri, v)
    # 1 % multiplicative refactorization of both parts
    pr, s = osp.perturb(v.real, s)
    pi, _ = osp.perturb(v.imag, s)
    v2 = pr + 1j * pi
    lu.factorize(cp, ri, v2)
    sym = lu.symbolic()
    ref = osp.Factors(len(cp) - 1, cp, ri, v2, sym["col_perm"], sym["col_perm_inv"], sym["supernode_ptr"])
    assert np.array_equal(lu.row_perm(), ref.row_perm.astype(np.int64))
    b = np.ones(len(cp) - 1, dtype=np.complex128) * (1 - 2j)
    x = b.copy()
    lu.solve(x)
    xr = ref.solve(b)
    assert np.max(np.abs(x - xr) / np.maximum(np.abs(xr), 1.0)) <= 1e-12


def test_heavy_pivoting_matches_the_oracle_pivots(gpu, osp):
    # a weak complex diagonal makes partial pivoting swap rows; distinct moduli
    cp, ri, kind = osp.grid_pattern(9, 8, 7)
    u, _ = osp.dense.larnv("Uniform", [11, 12, 13, 15], kind.size)
    w, _ = osp.dense.larnv("Uniform", [17, 19, 23, 29], kind.size)
    v = np.where(kind == 0, 0.5 + 0.1 * u, -1.0 - 0.3 * u) + 1j * np.where(kind == 0, 0.2 * w, 0.4 * w - 0.2)
    _compare(osp, cp, ri, v, tol=1e-9, nnz_exact=False)


def test_errors_and_scalar_of_the_handle(gpu):
    lu = SparseLu.analyze(COL_PTR, ROW_IDX, LuMethod.supernodal())
    with pytest.raises(SparseError) as e:
        lu.solve(np.ones(2, dtype=np.complex128))
    assert e.value.kind == "NotFactorized"
    with pytest.raises(SparseError) as e:
        lu.factorize(COL_PTR, ROW_IDX, np.array([4, 1, 1j * np.nan, 3]))
    assert e.value.kind == "NotFinite"  # a NaN imaginary part (lu.rs:79-81)
    lu.factorize(COL_PTR, ROW_IDX, np.array([4, 1, 1, 3], dtype=np.complex128))
    with pytest.raises(SparseError) as e:  # rank one: the factors of the first stay
        lu.factorize(COL_PTR, ROW_IDX, np.array([1, 2j, 2j, -4], dtype=np.complex128))
    assert e.value.kind == "Singular"
    b = np.array([1.0, 2.0], dtype=np.complex128)
    lu.solve(b)
    assert np.all(np.abs(b - np.array([1 / 11, 7 / 11])) < 1e-14)
    with pytest.raises(SparseError) as e:
        lu.solve(np.ones(3, dtype=np.complex128))
    assert e.value.kind == "BadShape"
    # the first factorization fixed the scalar: real calls are rejected
    with pytest.raises(SparseError):
        lu.factorize(COL_PTR, ROW_IDX, [4.0, 1.0, 1.0, 3.0])
    with pytest.raises(SparseError):
        lu.solve(np.ones(2))
    real = SparseLu.analyze(COL_PTR, ROW_IDX, LuMethod.supernodal())
    real.factorize(COL_PTR, ROW_IDX, [4.0, 1.0, 1.0, 3.0])
    with pytest.raises(SparseError):
        real.solve(np.ones(2, dtype=np.complex128))
