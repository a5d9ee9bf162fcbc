"""Pins the oracle (the C++ restatement of the reference's dense LU path)
against the reference's own known answers before anything is compared with it.
CPU only."""

import json
import pathlib

import numpy as np
import pytest

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
SEEDY = [1988, 1989, 1990, 1991]


def test_larnv_matches_the_reference_stream(oracle):
    # families.rs:1183-1261: values the reference captured from libtmglib
    kat = json.loads((GOLDEN / "larnv_kat.json").read_text())
    assert kat["seed"] == SEEDY
    for case in kat["cases"]:
        x, seed = oracle.larnv(case["dist"], kat["seed"], kat["n"])
        for i, v in enumerate(case["first12"]):
            assert x[i] == float(v), (case["dist"], i)
        for k, v in enumerate(case["last2_at_198"]):
            assert x[198 + k] == float(v), (case["dist"], 198 + k)
        assert seed == case["seed_after"], case["dist"]


@pytest.mark.parametrize("n", [1, 63, 64, 65, 129, 200])
def test_larnv_is_continuous_across_batches(oracle, n):
    # families.rs:1263-1284
    allx, sa = oracle.larnv("Uniform", SEEDY, n)
    s = list(SEEDY)
    one = []
    for _ in range(n):
        v, s = oracle.larnv("Uniform", s, 1)
        one.append(v[0])
    assert list(allx) == one
    assert sa == s


def sample4():
    # mod.rs:467-475, row-major [[4,1,2,1],[1,3,0,1],[2,0,5,2],[1,1,2,6]] as column-major
    return np.array([4.0, 1.0, 2.0, 1.0, 1.0, 3.0, 0.0, 1.0, 2.0, 0.0, 5.0, 2.0, 1.0, 1.0, 2.0, 6.0])


def cofactor_det4():
    # mod.rs:487-491
    return (4.0 * (3.0 * (5.0 * 6.0 - 2.0 * 2.0) - 0.0 * (0.0 * 6.0 - 2.0 * 1.0) + 1.0 * (0.0 * 2.0 - 5.0 * 1.0))
            - 1.0 * (1.0 * (5.0 * 6.0 - 2.0 * 2.0) - 0.0 * (2.0 * 6.0 - 2.0 * 1.0) + 1.0 * (2.0 * 2.0 - 5.0 * 1.0))
            + 2.0 * (1.0 * (0.0 * 6.0 - 2.0 * 1.0) - 3.0 * (2.0 * 6.0 - 2.0 * 1.0) + 1.0 * (2.0 * 1.0 - 0.0 * 1.0))
            - 1.0 * (1.0 * (0.0 * 2.0 - 5.0 * 1.0) - 3.0 * (2.0 * 2.0 - 5.0 * 1.0) + 0.0 * (2.0 * 1.0 - 0.0 * 1.0)))


def test_dgetrf_determinant_and_pivots(oracle):
    a = sample4()
    rc, ipiv, det, _ = oracle.dgetrf(a, 4)
    assert rc == 0 and len(ipiv) == 4
    assert abs(det - cofactor_det4()) < 1e-12


def test_dgetrf_detects_a_singular_matrix(oracle):
    # mod.rs:497-502: second column is twice the first
    a = np.array([1.0, 2.0, 3.0, 2.0, 4.0, 6.0, 1.0, 1.0, 1.0])
    rc, *_ = oracle.dgetrf(a, 3)
    assert rc == 1


def spd(n):
    # checkers.rs:260-279: A = L L^T with integer entries
    l = np.zeros((n, n))
    for j in range(n):
        l[j, j] = j + 2
        for i in range(j + 1, n):
            l[i, j] = (i + j) % 3 - 1.0
    return (l @ l.T).T.reshape(-1).copy()  # column-major storage of the symmetric product


def test_dgetri_inverts_correctly(oracle):
    # mod.rs:510-534: A * A^-1 e_j = e_j for the 4 x 4 sample
    a = sample4()
    lu = a.copy()
    rc, ipiv, _, _ = oracle.dgetrf(lu, 4)
    assert rc == 0
    assert oracle.dgetri(lu, 4, ipiv) == 0
    for j in range(4):
        e = np.zeros(4)
        e[j] = 1.0
        back = oracle.dgemv(lu, oracle.dgemv(a, e, 4, 4), 4, 4)
        assert np.all(np.abs(back - e) < 1e-12)


def test_dgetri_residual_on_spd_matrices(oracle):
    # checkers.rs:307-330 (the DGET03 use): ||I - A A^-1|| small on spd(n)
    for n in (1, 2, 5, 8):
        a = spd(n)
        lu = a.copy()
        rc, ipiv, _, _ = oracle.dgetrf(lu, n)
        assert rc == 0 and oracle.dgetri(lu, n, ipiv) == 0
        am, inv = a.reshape(n, n).T, lu.reshape(n, n).T
        resid = np.abs(np.eye(n) - am @ inv).sum(axis=0).max()
        anorm, inorm = np.abs(am).sum(axis=0).max(), np.abs(inv).sum(axis=0).max()
        assert resid / (n * anorm * inorm * 2.0**-52) <= 20.0


def test_dgetri_reports_a_zero_pivot_and_keeps_the_factors(oracle):
    lu = np.array([2.0, 0.5, 1.0, 0.0])  # U = [[2, 1], [0, 0]]
    before = lu.copy()
    assert oracle.dgetri(lu, 2, [0, 1]) == 1
    assert np.array_equal(lu, before)


def test_dgesv_solves_a_system(oracle):
    # mod.rs:537-551
    a = sample4()
    x_true = np.array([1.0, -2.0, 3.0, 5.0])
    b = oracle.dgemv(a, x_true, 4, 4)
    rc, _ = oracle.dgesv(a.copy(), b, 4)
    assert rc == 0
    assert np.all(np.abs(b - x_true) < 1e-12)


def test_dgesv_reports_a_singular_system(oracle):
    # mod.rs:553-558
    a = np.array([1.0, 2.0, 3.0, 2.0, 4.0, 6.0, 1.0, 1.0, 1.0])
    b = np.ones(3)
    rc, _ = oracle.dgesv(a, b, 3)
    assert rc == 1


def test_empty_matrices_are_handled(oracle):
    # mod.rs:609-616
    a = np.zeros(0)
    rc, ipiv, det, _ = oracle.dgetrf(a, 0)
    assert rc == 0 and ipiv == [] and det == 1.0


def test_pivot_threshold_matches_lapack(oracle):
    # mod.rs:670-683: a 1e-16 pivot is not singular; [[1,2],[2,4]] is
    a = np.array([1e-16, 0.0, 0.0, 1.0])
    rc, ipiv, det, _ = oracle.dgetrf(a, 2)
    assert rc == 0 and len(ipiv) == 2 and abs(det) < 1e-15
    b = np.array([1.0, 2.0, 2.0, 4.0])
    rc, *_ = oracle.dgetrf(b, 2)
    assert rc == 1


def reconstruct_panel(nrows, ncols, a0, a, ipiv):
    # mod.rs:696-721: P A = L U on the panel
    pa = a0.copy()
    for k in range(ncols):
        for j in range(ncols):
            i1, i2 = j * nrows + k, j * nrows + ipiv[k]
            pa[i1], pa[i2] = pa[i2], pa[i1]
    lu = np.zeros(nrows * ncols)
    for j in range(ncols):
        for i in range(nrows):
            s = 0.0
            for l in range(ncols):
                lil = 1.0 if i == l else (a[i + l * nrows] if i > l else 0.0)
                ulj = a[l + j * nrows] if l <= j else 0.0
                s += lil * ulj
            lu[i + j * nrows] = s
    return pa, lu


def test_dgetrf_rect_reconstructs_a_tall_panel(oracle):
    # mod.rs:723-733
    nrows, ncols = 5, 3
    a0 = np.array([1.0, 5.0, 2.0, 3.0, 4.0, 2.0, -1.0, 6.0, 0.0, 1.0, 3.0, 2.0, 1.0, 7.0, -2.0])
    a = a0.copy()
    rc, ipiv = oracle.dgetrf_rect(a, nrows, ncols)
    assert rc == 0
    pa, lu = reconstruct_panel(nrows, ncols, a0, a, ipiv)
    assert np.all(np.abs(pa - lu) < 1e-12)
    assert ipiv[0] == 1


def test_dgetrf_rect_rejects_bad_shapes_and_singular_panels(oracle):
    # mod.rs:735-745
    a = np.array([1.0, 2.0, 3.0, 4.0])
    rc, _ = oracle.dgetrf_rect(a, 1, 2)
    assert rc == 2
    singular = np.array([0.0, 0.0, 2.0, 3.0])
    rc, _ = oracle.dgetrf_rect(singular, 2, 2)
    assert rc == 1


def sample(n):
    # parity.rs:57-70
    a = np.zeros(n * n)
    for i in range(n):
        for j in range(n):
            a[i + j * n] = (n + 1.0 + i * 0.5) if i == j else float((i * 7 + j * 13) % 11) - 5.0
    return a


@pytest.mark.parametrize("n", [1, 2, 3, 5, 9])
def test_dgesv_recovers_the_known_solution(oracle, n):
    # parity.rs:152-195 (the known-solution half; TOL = 1e-10, parity.rs:35)
    a = sample(n)
    x_true = np.array([1.0 + i * 0.25 for i in range(n)])
    b = oracle.dgemv(a, x_true, n, n)
    rc, _ = oracle.dgesv(a.copy(), b, n)
    assert rc == 0
    assert np.all(np.abs(b - x_true) / np.maximum(np.abs(x_true), 1.0) < 1e-10)


def test_idamax_first_maximum_wins(oracle):
    # blas.rs:77-88
    assert oracle.idamax(np.array([1.0, -3.0, 3.0, 2.0])) == 1
    assert oracle.idamax(np.zeros(0)) == 0


def test_random_lu_has_small_get01(oracle):
    # checkers.rs:17-63 ratio bound (checkers.rs:307-352 uses <= 20)
    n = 48
    a0, _ = oracle.larnv("Symmetric", SEEDY, n * n)
    a = a0.copy()
    rc, ipiv, _, _ = oracle.dgetrf(a, n)
    assert rc == 0
    assert oracle.get01(a0, a, ipiv, n, n) < 20.0


def test_oracle_agrees_with_an_independent_lu(oracle):
    """Cross-check against scipy's LAPACK getrf (not the oracle's reference:
    blocked getrf may differ on near-ties, so this compares x, and ipiv here)."""
    scipy_linalg = pytest.importorskip("scipy.linalg")
    n = 200
    a, x_true, b = oracle.c1_system(n)
    lu, piv = scipy_linalg.lu_factor(a.reshape(n, n, order="F"))
    xs = scipy_linalg.lu_solve((lu, piv), b)
    aw = a.copy()
    bw = b.copy()
    rc, ipiv = oracle.dgesv(aw, bw, n)
    assert rc == 0
    assert list(piv) == ipiv
    assert np.max(np.abs(bw - xs)) / np.max(np.abs(xs)) < 1e-12


def _dlatms_general_cases():
    kat = json.loads((GOLDEN / "dlatms_kat.json").read_text())
    return [(kat["seed"], c) for c in kat["cases"] if c["sym"] == "NonSymmetric" and c["pack"] == "Full"]


@pytest.mark.parametrize("seed,case", _dlatms_general_cases(),
                         ids=lambda v: f"mode{v['mode']}_{v['m']}x{v['n']}" if isinstance(v, dict) else "")
def test_dlatms_matches_the_reference_matrices(oracle, seed, case):
    # families.rs:2014-2470: the seed after the call exactly, spectrum and
    # matrix to the reference's own 1e-13 relative (its values come from
    # LAPACK's libtmglib, whose BLAS sums in another order)
    want_d = np.array([float(v) for v in case["d"]])
    want_a = np.array([float(v) for v in case["a"]])
    info, a, d, seed_after = oracle.dlatms_general(case["dist"], case["mode"], float(case["cond"]),
                                                   float(case["dmax"]), case["m"], case["n"], seed, want_d)
    assert info == 0
    assert seed_after == case["seed_after"]
    for got, want in ((d, want_d), (a, want_a)):
        zero = want == 0.0
        assert np.all(got[zero] == 0.0)
        assert np.all(np.abs(got[~zero] - want[~zero]) <= 1e-13 * np.abs(want[~zero]))
