"""Sparse LU: the host-side analysis through the C ABI and the oracle against
the reference's own tests. CPU only — analyze needs no GPU, and the
factorize/solve checks here are the ones the reference makes before any
numeric work.

Pins: COLAMD permutations (colamd.rs:886-918, tests/golden/colamd_kat.json),
column counts against dense symbolic elimination of (AQ)^T (AQ)
(supernodal.rs:463-531), the supernode partition's invariants
(supernodal.rs:533-560), shape and structure errors (sparse_lu.rs:318-351,
csc.rs), the method choice and flop ratio (sparse_lu.rs:385-503), and the
oracle's solutions of the reference's 2 x 2 examples (sparse_lu.rs:251-309)."""

import json
import pathlib

import numpy as np
import pytest

from algebra_linear_b200.sparse import LuMethod, SparseError, SparseLu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"

COL_PTR = [0, 2, 4]
ROW_IDX = [0, 1, 0, 1]
VALUES = [4.0, 1.0, 1.0, 3.0]


def colamd_cases():
    return json.loads((GOLDEN / "colamd_kat.json").read_text())["cases"]


@pytest.mark.parametrize("case", colamd_cases(), ids=lambda c: c["name"])
def test_colamd_matches_the_reference_fixtures(case):
    lu = SparseLu.analyze(case["col_ptr"], case["row_idx"], LuMethod.supernodal())
    sym = lu.symbolic()
    assert sym["col_perm"].tolist() == case["perm"]
    assert sym["col_perm_inv"].tolist() == case["perm_inv"]


def _dense_pattern(cp, ri, n):
    a = np.zeros((n, n), bool)
    for j in range(n):
        a[ri[cp[j]:cp[j + 1]], j] = True
    return a


def brute_force_counts(cp, ri, perm):
    """Symbolic Cholesky of (A Q)^T (A Q) by dense elimination."""
    n = len(cp) - 1
    a = _dense_pattern(cp, ri, n)[:, perm]
    b = (a.T.astype(int) @ a.astype(int)) > 0
    np.fill_diagonal(b, True)
    counts = np.zeros(n, int)
    for j in range(n):
        col = [i for i in range(j, n) if b[i, j]]
        counts[j] = len(col)
        for i in col:
            if i > j:
                for k in col:
                    if k >= i:
                        b[k, i] = True
    return counts


@pytest.mark.parametrize("case", colamd_cases(), ids=lambda c: c["name"])
def test_column_counts_match_dense_symbolic_elimination(case):
    lu = SparseLu.analyze(case["col_ptr"], case["row_idx"], LuMethod.supernodal())
    sym = lu.symbolic()
    want = brute_force_counts(case["col_ptr"], case["row_idx"], sym["col_perm"])
    assert sym["col_counts"].tolist() == want.tolist()
    ptr = sym["supernode_ptr"]
    n = len(case["col_ptr"]) - 1
    assert ptr[0] == 0 and ptr[-1] == n and np.all(np.diff(ptr) > 0)


def test_diagonal_matrix_has_singleton_supernodes():
    n = 6
    lu = SparseLu.analyze(list(range(n + 1)), list(range(n)), LuMethod.supernodal())
    sym = lu.symbolic()
    assert sym["supernode_ptr"].tolist() == list(range(n + 1))
    assert sym["col_counts"].tolist() == [1] * n


def _raises(code_name, fn, *args):
    with pytest.raises(SparseError) as e:
        fn(*args)
    assert e.value.kind == code_name, e.value.kind
    return e.value


def test_rejects_non_square_and_malformed_input():
    # sparse_lu.rs:340-351 and the CSC validation of csc.rs:39-76
    _raises("BadShape", SparseLu.analyze, [0, 2, 3], [0, 1, 2])
    _raises("BadShape", SparseLu.analyze, [], [])
    _raises("UnsortedRows", SparseLu.analyze, [0, 2, 2], [1, 0])
    _raises("DuplicateEntry", SparseLu.analyze, [0, 2, 2], [1, 1])
    _raises("InvalidStructure", SparseLu.analyze, [1, 2, 2], [1])
    _raises("InvalidStructure", SparseLu.analyze, [0, 2, 1, 2], [0, 1])
    _raises("BadShape", SparseLu.analyze, [0, 2, 3], [0, 1])


def test_factorize_checks_before_numeric_work():
    lu = SparseLu.analyze(COL_PTR, ROW_IDX, LuMethod.auto())
    b = np.array([1.0, 2.0])
    assert _raises("NotFactorized", lu.solve, b)
    # a changed pattern (sparse_lu.rs:301-314)
    _raises("StructureMismatch", lu.factorize, [0, 2, 3], [0, 1, 1], [1.0, 1.0, 1.0])
    for bad in (np.nan, np.inf, -np.inf):  # sparse_lu.rs:327-334
        _raises("NotFinite", lu.factorize, COL_PTR, ROW_IDX, [4.0, 1.0, bad, 3.0])
    _raises("BadShape", lu.factorize, COL_PTR, ROW_IDX, [4.0, 1.0, 1.0])
    assert lu.stats() is None


def test_precision_settings_are_validated_on_the_host():
    # the mixed form's settings (no reference counterpart) need no GPU
    lu = SparseLu.analyze(COL_PTR, ROW_IDX, LuMethod.supernodal())
    for p in ("fp64", "fp32", "tf32", "bf16"):
        lu.set_precision(p, tol=1e-15, max_ir=5)
    with pytest.raises(KeyError):
        lu.set_precision("fp16")
    from algebra_linear_b200 import _lib

    assert lu._lib.alg_splu_set_precision(lu._h, 7, 0.0, 0) == _lib.INVALID_ARGUMENT
    assert lu._lib.alg_splu_set_precision(lu._h, 0, float("nan"), 0) == _lib.INVALID_ARGUMENT
    assert _raises("NotFactorized", lu.last_solve)


def test_large_fronts_split_into_lanes(monkeypatch):
    """Analyze spreads independent subtrees of large fronts over concurrent
    lanes (host-only plan; the 24^3 grid's tree splits into two heavy
    subtrees below a chain of top fronts)."""
    from oracle import sparse as osp

    cp, ri, _ = osp.grid_pattern(24, 24, 24)
    for lanes in ("1", "2"):
        monkeypatch.setenv("ALG_SPLU_LANES", lanes)
        plan = SparseLu.analyze(cp, ri, LuMethod.supernodal()).plan()
        assert plan["n_lanes"] == int(lanes)
        if lanes == "1":
            assert plan["top_fronts"] == 0
            one = plan
        else:
            assert plan["top_fronts"] >= 1
            # same fronts and flops; the lanes only reorder independent work
            assert plan["n_fronts"] == one["n_fronts"] and plan["plan_flops"] == one["plan_flops"]


def test_plan_fronts_follow_the_column_etree(monkeypatch):
    """The GPU plan cuts the reference's relaxed supernodes where the next
    column is not the etree parent of the one before: a front then passes up
    the unpivoted rows of its own subtree only, so the plan's flops stay
    below the cost of the chol(A^T A) columns, sum 2 cc_j^2 (the glued
    partition is several times above it on 3-D grids)."""
    from oracle import sparse as osp

    cp, ri, _ = osp.grid_pattern(24, 24, 24)
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    cc = lu.symbolic()["col_counts"].astype(float)
    bound = 2.0 * (cc ** 2).sum()
    split = lu.plan()
    assert split["plan_flops"] <= bound
    monkeypatch.setenv("ALG_SPLU_KEEP_GLUED", "1")
    glued = SparseLu.analyze(cp, ri, LuMethod.supernodal()).plan()
    assert glued["plan_flops"] > 1.5 * split["plan_flops"]
    assert glued["factor_bytes"] > split["factor_bytes"]


def _tridiag(n, dense=False):
    cp, ri, v = [0], [], []
    for j in range(n):
        rng = range(n) if dense else range(max(j - 1, 0), min(j + 1, n - 1) + 1)
        for i in rng:
            ri.append(i)
            v.append((2.0 * n if dense else 5.0) if i == j else 1.0)
        cp.append(len(ri))
    return cp, ri, v


def test_effective_method_and_flop_ratio():
    # sparse_lu.rs:430-484
    cp, ri, _ = _tridiag(9)
    lu = SparseLu.analyze(cp, ri, LuMethod.simplicial())
    assert lu.effective_method() == "Simplicial" and lu.flop_ratio() is None
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    assert lu.effective_method() == "Supernodal" and lu.flop_ratio() > 0
    lu = SparseLu.analyze(cp, ri, LuMethod.auto())
    r = lu.flop_ratio()
    assert lu.effective_method() == "Simplicial" and 0 < r <= 40
    cp, ri, _ = _tridiag(12, dense=True)
    lu = SparseLu.analyze(cp, ri, LuMethod.auto(1.0))
    assert lu.effective_method() == "Supernodal" and lu.flop_ratio() > 1.0


def test_empty_matrix_has_zero_fill_and_flops():
    # sparse_lu.rs:486-503
    lu = SparseLu.analyze([0], [], LuMethod.auto())
    assert lu.effective_method() == "Simplicial"
    assert lu.flop_ratio() == 0.0
    lu.factorize([0], [], [])
    s = lu.stats()
    assert s["n"] == 0 and s["nnz_a"] == 0 and s["fill_ratio"] == 0.0 and s["flops_estimate"] == 0
    assert s["nnz_l"] + s["nnz_u"] == 0 and s["method"] == "Simplicial" and s["flop_ratio"] == 0.0
    lu.solve(np.zeros(0))


def _oracle_factors(oracle_sparse, cp, ri, v, method=LuMethod.supernodal()):
    lu = SparseLu.analyze(cp, ri, method)
    sym = lu.symbolic()
    return oracle_sparse.Factors(len(cp) - 1, cp, ri, v, sym["col_perm"], sym["col_perm_inv"], sym["supernode_ptr"])


@pytest.fixture(scope="module")
def oracle_sparse(oracle):
    from oracle import sparse

    return sparse


def test_oracle_solves_the_reference_examples(oracle_sparse):
    # sparse_lu.rs:251-309: A = [4 1; 1 3]
    f = _oracle_factors(oracle_sparse, COL_PTR, ROW_IDX, VALUES)
    assert f.status == 0
    np.testing.assert_allclose(f.solve([1.0, 2.0]), [1 / 11, 7 / 11], rtol=0, atol=1e-14 * 2)
    np.testing.assert_allclose(f.solve([1.0, 1.0]), [2 / 11, 3 / 11], rtol=0, atol=1e-14 * 2)
    f = _oracle_factors(oracle_sparse, COL_PTR, ROW_IDX, [5.0, 2.0, 2.0, 2.0])
    np.testing.assert_allclose(f.solve([1.0, 1.0]), [0.0, 0.5], rtol=0, atol=1e-14 * 2)
    assert f.nnz_l >= 3 and f.nnz_u >= 2


def test_oracle_reconstructs_the_permuted_matrix(oracle_sparse):
    # supernodal_lu.rs:707-741: P A Q = L U on the 4 x 5 grid
    case = [c for c in colamd_cases() if c["name"] == "grid4x5"][0]
    cp, ri = case["col_ptr"], case["row_idx"]
    n = len(cp) - 1
    v = np.array([5.0 if ri[k] == j else 1.0 for j in range(n) for k in range(cp[j], cp[j + 1])])
    f = _oracle_factors(oracle_sparse, cp, ri, v)
    assert f.status == 0
    A = np.zeros((n, n))
    for j in range(n):
        A[ri[cp[j]:cp[j + 1]], j] = v[cp[j]:cp[j + 1]]
    L = np.zeros((n, n))
    U = np.zeros((n, n))
    for j in range(n):
        for k in range(int(f.l_col_ptr[j]), int(f.l_col_ptr[j + 1])):
            L[int(f.l_row_idx[k]), j] = f.l_val[k]
        for k in range(int(f.u_col_ptr[j]), int(f.u_col_ptr[j + 1])):
            U[int(f.u_row_idx[k]), j] = f.u_val[k]
    sym = SparseLu.analyze(cp, ri, LuMethod.supernodal()).symbolic()
    PAQ = A[f.row_perm.astype(int)][:, sym["col_perm"]]
    np.testing.assert_allclose(L @ U, PAQ, atol=1e-12)
    assert np.all(np.diag(L) == 1.0)


def test_grid_values_follow_the_stencil(oracle_sparse):
    cp, ri, kind = oracle_sparse.grid_pattern(4, 3, 2)
    v, _ = oracle_sparse.convection_diffusion_values(kind, [1, 2, 3, 5])
    n = len(cp) - 1
    diag = np.array([v[k] for j in range(n) for k in range(int(cp[j]), int(cp[j + 1])) if ri[k] == j])
    assert np.all((diag >= 6.0) & (diag <= 6.1))
    assert np.all(v[kind == 3] == -1.0)
    assert np.all((v[kind == 2] >= -1.0) & (v[kind == 2] <= -0.7))
    assert np.all((v[kind == 1] >= -1.3) & (v[kind == 1] <= -1.0))


def _simplicial(osp, cp, ri, v):
    sym = SparseLu.analyze(cp, ri, LuMethod.simplicial()).symbolic()
    return osp.Factors(len(cp) - 1, cp, ri, v, sym["col_perm"], sym["col_perm_inv"], None), sym


def _csc_dense(cp, ri, v, n):
    A = np.zeros((n, n))
    for j in range(n):
        A[ri[cp[j]:cp[j + 1]], j] = v[cp[j]:cp[j + 1]]
    return A


def _lu_dense(f):
    n = f.n
    L, U = np.zeros((n, n)), np.zeros((n, n))
    for j in range(n):
        for k in range(int(f.l_col_ptr[j]), int(f.l_col_ptr[j + 1])):
            L[int(f.l_row_idx[k]), j] = f.l_val[k]
        for k in range(int(f.u_col_ptr[j]), int(f.u_col_ptr[j + 1])):
            U[int(f.u_row_idx[k]), j] = f.u_val[k]
    return L, U


def test_simplicial_oracle_pins(oracle_sparse):
    # lu.rs:527-533: [4 1; 1 3] x = [1, 2]
    f, _ = _simplicial(oracle_sparse, COL_PTR, ROW_IDX, VALUES)
    assert f.status == 0
    np.testing.assert_allclose(f.solve([1.0, 2.0]), [1 / 11, 7 / 11], rtol=0, atol=1e-14 * 2)
    # lu.rs:536-557: P A Q = L U on the 4 x 4 fill pattern
    cp, ri = [0, 2, 5, 8, 10], [0, 1, 0, 1, 2, 1, 2, 3, 0, 3]
    v = np.array([4.0, 1.0, 1.0, 3.0, 1.0, 1.0, 5.0, 1.0, 1.0, 4.0])
    f, sym = _simplicial(oracle_sparse, cp, ri, v)
    L, U = _lu_dense(f)
    A = _csc_dense(cp, ri, v, 4)
    np.testing.assert_allclose(L @ U, A[f.row_perm.astype(int)][:, sym["col_perm"]], rtol=0, atol=1e-12 * 2)
    # the pivot is stored first in each L column, the diagonal last in each U column
    assert all(f.l_val[int(f.l_col_ptr[j])] == 1.0 for j in range(4))
    assert all(int(f.u_row_idx[int(f.u_col_ptr[j + 1]) - 1]) == j for j in range(4))
    # lu.rs:559-587: banded 8 x 8, x = i + 1/2
    n = 8
    cp, ri, v = [0], [], []
    for j in range(n):
        for i, a in ((j - 1, -1.0), (j, 4.0), (j + 1, -1.0)):
            if 0 <= i < n:
                ri.append(i)
                v.append(a)
        cp.append(len(ri))
    f, _ = _simplicial(oracle_sparse, cp, ri, np.array(v))
    x = np.arange(n) + 0.5
    b = _csc_dense(cp, ri, np.array(v), n) @ x
    np.testing.assert_allclose(f.solve(b), x, rtol=1e-12, atol=1e-12)
    # lu.rs:589-625: diagonal, then an arrow (dense first row and column)
    f, _ = _simplicial(oracle_sparse, list(range(6)), list(range(5)), np.array([2.0, 3.0, 4.0, 5.0, 6.0]))
    np.testing.assert_allclose(f.solve([2.0, 6.0, 12.0, 20.0, 30.0]), [1, 2, 3, 4, 5], rtol=0, atol=1e-15 * 6)
    n = 6
    cp, ri, v = [0], [], []
    for j in range(n):
        col = [(i, 5.0 if i == 0 else 1.0) for i in range(n)] if j == 0 else [(0, 1.0), (j, 4.0)]
        for i, a in col:
            ri.append(i)
            v.append(a)
        cp.append(len(ri))
    f, _ = _simplicial(oracle_sparse, cp, ri, np.array(v))
    x = np.arange(1.0, n + 1)
    np.testing.assert_allclose(f.solve(_csc_dense(cp, ri, np.array(v), n) @ x), x, rtol=1e-12, atol=1e-12)
    # a structurally singular column
    f, _ = _simplicial(oracle_sparse, COL_PTR, ROW_IDX, [1.0, 1.0, 1.0, 1.0])
    assert f.status == 104


@pytest.mark.parametrize("dims", [(8, 8, 8), (30, 30, 1)], ids=lambda d: "x".join(map(str, d)))
def test_simplicial_and_supernodal_oracles_agree(oracle_sparse, dims):
    """The two reference paths share the column order and, without ties, the
    pivots; their solutions agree to rounding, and the simplicial factors keep
    the exact zeros of each column's reach (at least as many entries)."""
    cp, ri, kind = oracle_sparse.grid_pattern(*dims)
    v, _ = oracle_sparse.convection_diffusion_values(kind, [4, 3, 2, 1])
    n = len(cp) - 1
    fs, sym = _simplicial(oracle_sparse, cp, ri, v)
    sup = SparseLu.analyze(cp, ri, LuMethod.supernodal()).symbolic()
    assert np.array_equal(sym["col_perm"], sup["col_perm"])
    f = oracle_sparse.Factors(n, cp, ri, v, sup["col_perm"], sup["col_perm_inv"], sup["supernode_ptr"])
    assert fs.status == 0 and f.status == 0
    assert np.array_equal(fs.row_perm, f.row_perm)
    b = np.linspace(-1.0, 2.0, n)
    xs, x = fs.solve(b), f.solve(b)
    assert np.max(np.abs(xs - x)) / np.max(np.abs(x)) <= 1e-12
    assert fs.nnz_l >= f.nnz_l and fs.nnz_u >= f.nnz_u, (fs.nnz_l, f.nnz_l, fs.nnz_u, f.nnz_u)


@pytest.mark.parametrize("case,n", list(enumerate([4, 8, 16, 32])), ids=lambda v: str(v))
def test_accuracy_on_lapack_random_matrices(oracle_sparse, case, n):
    """accuracy_tests.rs:74-116: DLATMS matrices (mode 3, cond 1e2 and 1e4)
    stored densely as CSC, solved by the simplicial and supernodal
    restatements and by the path Auto(1.0) picks (supernodal from n = 16):
    forward error <= 1e-9 cond, scaled residual <= 1e-13 cond."""
    dense = oracle_sparse.dense
    for ci, cond in enumerate([1e2, 1e4]):
        seed = [1234 + case * 17, 2345 + ci, 3456 + case, 4567]
        info, a, _, _ = dense.dlatms_general("Uniform", 3, cond, 1.0, n, n, seed)
        assert info == 0
        A = a.reshape(n, n).T
        x_exact = 1.0 + (np.arange(n) % 7) * 0.25
        b = A @ x_exact
        cp = list(range(0, n * n + 1, n))
        ri = [i for _ in range(n) for i in range(n)]
        xs = {}
        f, _ = _simplicial(oracle_sparse, cp, ri, a)
        xs["simplicial"] = f.solve(b)
        sup = SparseLu.analyze(cp, ri, LuMethod.supernodal()).symbolic()
        f = oracle_sparse.Factors(n, cp, ri, a, sup["col_perm"], sup["col_perm_inv"], sup["supernode_ptr"])
        xs["supernodal"] = f.solve(b)
        auto = SparseLu.analyze(cp, ri, LuMethod.auto(1.0))
        xs["auto"] = xs["supernodal"] if auto.effective_method() == "Supernodal" else xs["simplicial"]
        if n >= 16:
            assert auto.effective_method() == "Supernodal", n
        anorm = np.max(np.abs(A).sum(axis=1))
        for name, x in xs.items():
            err = np.max(np.abs(x - x_exact)) / max(np.max(np.abs(x_exact)), 1.0)
            res = np.max(np.abs(A @ x - b)) / (anorm * np.max(np.abs(x)) + np.max(np.abs(b)))
            assert err <= 1e-9 * cond, (name, n, cond, err)
            assert res <= 1e-13 * cond, (name, n, cond, res)


def _complex_factors(osp, cp, ri, v, method):
    lu = SparseLu.analyze(cp, ri, method)
    sym = lu.symbolic()
    snp = sym["supernode_ptr"] if lu.effective_method() == "Supernodal" else None
    return osp.Factors(len(cp) - 1, cp, ri, np.asarray(v, dtype=np.complex128), sym["col_perm"],
                       sym["col_perm_inv"], snp)


def test_complex_oracle_pins(oracle_sparse):
    """SparseLu<Complex64> restated (the same loops over num-complex
    arithmetic): sparse_lu.rs:279-295, supernodal_lu.rs:763-805 and
    accuracy_tests.rs:120-150."""
    # sparse_lu.rs:279-295: [4 1; 1 3] as complex values, Auto
    for method in (LuMethod.auto(), LuMethod.supernodal(), LuMethod.simplicial()):
        f = _complex_factors(oracle_sparse, COL_PTR, ROW_IDX, [4, 1, 1, 3], method)
        x = f.solve([1.0, 2.0])
        assert np.all(np.abs(x - np.array([1 / 11, 7 / 11])) < 1e-14)
    # supernodal_lu.rs:763-805: tridiagonal, diagonal 6 + i, off-diagonals 0.5 - 0.25 i
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
        x = _complex_factors(oracle_sparse, cp, ri, v, method).solve(b)
        assert np.all(np.abs(x - x_true) < 1e-12)
    # accuracy_tests.rs:120-150: A = Re + 0.25 i Im from two DLATMS matrices, n = 8
    n = 8
    _, re, _, _ = oracle_sparse.dense.dlatms_general("Uniform", 3, 1e2, 1.0, n, n, [11, 22, 33, 44])
    _, im, _, _ = oracle_sparse.dense.dlatms_general("Uniform", 3, 1e2, 1.0, n, n, [55, 66, 77, 88])
    a = re + 0.25j * im
    x_exact = np.array([complex(1.0 + i % 5, -0.5) for i in range(n)])
    b = a.reshape(n, n).T @ x_exact
    cp = list(range(0, n * n + 1, n))
    ri = [i for _ in range(n) for i in range(n)]
    for method in (LuMethod.auto(), LuMethod.supernodal(), LuMethod.simplicial()):
        x = _complex_factors(oracle_sparse, cp, ri, a, method).solve(b)
        err = np.max(np.abs(x - x_exact)) / np.max(np.abs(x_exact))
        assert err < 1e-9, err


def test_complex_oracle_on_real_values_follows_the_real_oracle(oracle_sparse):
    """With zero imaginary parts the complex restatement takes the real one's
    pivots and structure and keeps every imaginary part zero; its values agree
    to rounding only, since num-complex's reciprocal is re / (re^2 + im^2),
    not 1 / re."""
    cp, ri, kind = oracle_sparse.grid_pattern(7, 6, 5)
    v, _ = oracle_sparse.convection_diffusion_values(kind, [2, 4, 6, 9])
    n = len(cp) - 1
    sym = SparseLu.analyze(cp, ri, LuMethod.supernodal()).symbolic()
    for snp in (sym["supernode_ptr"], None):
        fr = oracle_sparse.Factors(n, cp, ri, v, sym["col_perm"], sym["col_perm_inv"], snp)
        fz = oracle_sparse.Factors(n, cp, ri, v.astype(np.complex128), sym["col_perm"], sym["col_perm_inv"], snp)
        assert np.array_equal(fr.row_perm, fz.row_perm) and fr.nnz_l == fz.nnz_l and fr.nnz_u == fz.nnz_u
        np.testing.assert_allclose(fz.l_val[:fz.nnz_l].real, fr.l_val[:fr.nnz_l], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(fz.u_val[:fz.nnz_u].real, fr.u_val[:fr.nnz_u], rtol=1e-12, atol=1e-15)
        assert not np.any(fz.l_val[:fz.nnz_l].imag) and not np.any(fz.u_val[:fz.nnz_u].imag)


def test_oracle_solves_the_reference_structured_patterns(oracle_sparse):
    """supernodal_lu.rs:686-706 (solve_both, :671-684): the simplicial and
    supernodal restatements agree to 1e-9 on the 2 x 2 example, tridiagonal,
    arrow and grid patterns with 5 on the diagonal and 1 off it."""
    import sparse_patterns as sp

    cases = [(2, ([0, 2, 4], [0, 1, 0, 1]), np.array([4.0, 1.0, 1.0, 3.0]), np.array([1.0, 2.0]))]
    for n, (cp, ri) in sp.STRUCTURED:
        cases.append((n, (cp, ri), sp.diagonal_values(cp, ri, 5.0, 1.0), 1.0 + np.arange(n)))
    for n, (cp, ri), v, b in cases:
        fs, _ = _simplicial(oracle_sparse, cp, ri, v)
        fn = _oracle_factors(oracle_sparse, cp, ri, v)
        assert fs.status == 0 and fn.status == 0
        assert sp.close(fn.solve(b), fs.solve(b), 1e-9), n


def test_oracle_reconstructs_the_reference_patterns(oracle_sparse):
    """supernodal_lu.rs:708-741: P A Q = L U within 1e-10 on tridiag(6),
    arrow(7) and the 3 x 4 grid."""
    import sparse_patterns as sp

    for n, (cp, ri) in [(6, sp.tridiag(6)), (7, sp.arrow(7)), (12, sp.grid(3, 4))]:
        v = sp.diagonal_values(cp, ri, 5.0, 1.0)
        f = _oracle_factors(oracle_sparse, cp, ri, v)
        assert f.status == 0
        L, U = _lu_dense(f)
        col_perm = SparseLu.analyze(cp, ri, LuMethod.supernodal()).symbolic()["col_perm"]
        PAQ = sp.dense(cp, ri, v)[f.row_perm.astype(int)][:, col_perm]
        assert np.max(np.abs(L @ U - PAQ)) < 1e-10, n


def test_oracle_solves_the_reference_random_system(oracle_sparse):
    """supernodal_lu.rs:744-763: the diagonally dominant system of the tests'
    LCG (n = 16, seed 0x1234_5678), x = (i mod 7) - 3: both restatements
    agree to 1e-9 and the supernodal one recovers x to 1e-9; and the 1 x 1
    system [2] x = [6] gives 3 (supernodal_lu.rs:839-852)."""
    import sparse_patterns as sp

    n = 16
    cp, ri, v = sp.diagonally_dominant(n, 0x1234_5678)
    assert cp[-1] == len(ri) == len(v) and all(any(ri[k] == j for k in range(cp[j], cp[j + 1])) for j in range(n))
    x = (np.arange(n) % 7) - 3.0
    b = sp.dense(cp, ri, v) @ x
    fs, _ = _simplicial(oracle_sparse, cp, ri, v)
    fn = _oracle_factors(oracle_sparse, cp, ri, v)
    xn = fn.solve(b)
    assert sp.close(xn, fs.solve(b), 1e-9) and sp.close(xn, x, 1e-9)
    f1 = _oracle_factors(oracle_sparse, [0, 1], [0], np.array([2.0]))
    assert abs(f1.solve([6.0])[0] - 3.0) < 1e-14
