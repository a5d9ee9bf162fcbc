"""GPU tests of the sparse solve's multi-CTA sweeps for large fronts and of the
mixed-precision sparse form (FP32 / TF32 / BF16 fronts with every solve
refined in FP64; no counterpart in the reference, whose sparse LU is FP64).

Bars: the large-front sweeps give the oracle's x within 1e-12 (the bar of
the one-CTA sweeps); the mixed form reaches the FP64 backward error
10 n 2^-53 and agrees with the oracle's x to the accuracy the conditioning
allows (2 cond_inf(A) 10 n 2^-53), and recomputes its factors in FP64 when
refinement cannot get there or the FP32 factorization meets a zero pivot."""

import numpy as np
import pytest

from algebra_linear_b200.sparse import LuMethod, SparseLu

pytestmark = pytest.mark.gpu

SEED = [1988, 1989, 1990, 1991]


@pytest.fixture(scope="module")
def osp(oracle):
    from oracle import sparse

    return sparse


def _ref(osp, lu, cp, ri, v):
    sym = lu.symbolic()
    return osp.Factors(len(cp) - 1, cp, ri, v, sym["col_perm"], sym["col_perm_inv"], sym["supernode_ptr"])


def _dense(cp, ri, v, n):
    a = np.zeros((n, n))
    for j in range(n):
        for q in range(cp[j], cp[j + 1]):
            a[ri[q], j] = v[q]
    return a


def _csr_residual(cp, ri, v, x, b):
    import scipy.sparse as ss

    n = len(cp) - 1
    a = ss.csc_matrix((np.asarray(v), np.asarray(ri), np.asarray(cp)), shape=(n, n))
    r = b - a @ x
    anorm = np.max(np.asarray(abs(a).sum(axis=1)).ravel())
    return np.max(np.abs(r)) / (anorm * np.max(np.abs(x)) + np.max(np.abs(b)))


@pytest.mark.parametrize("dims", [(12, 12, 12), (30, 30, 1)], ids=lambda d: "x".join(map(str, d)))
def test_large_front_sweeps_match_the_oracle(gpu, osp, dims, monkeypatch):
    # every front wider than 32 columns takes the multi-CTA triangular sweeps
    monkeypatch.setenv("ALG_SPLU_SOLVE_BIG", "32")
    cp, ri, kind = osp.grid_pattern(*dims)
    v, _ = osp.convection_diffusion_values(kind, SEED)
    n = len(cp) - 1
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    lu.factorize(cp, ri, v)
    sp = lu.symbolic()["supernode_ptr"]
    assert np.max(np.diff(sp)) > 32 or lu.plan()["max_front_rows"] > 64
    b, _ = osp.dense.larnv("Symmetric", [3, 5, 7, 9], n)
    x = b.copy()
    lu.solve(x)
    xr = _ref(osp, lu, cp, ri, v).solve(b)
    assert np.max(np.abs(x - xr) / np.maximum(np.abs(xr), 1.0)) <= 1e-12


@pytest.mark.parametrize("prec", ["fp32", "tf32", "tf32x3", "bf16"])
def test_mixed_form_reaches_the_fp64_backward_error(gpu, osp, prec):
    cp, ri, kind = osp.grid_pattern(12, 12, 12)
    v, _ = osp.convection_diffusion_values(kind, SEED)
    n = len(cp) - 1
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    lu.set_precision(prec)
    lu.factorize(cp, ri, v)
    b, _ = osp.dense.larnv("Symmetric", [3, 5, 7, 9], n)
    x = b.copy()
    lu.solve(x)
    rep = lu.last_solve()
    target = 10 * n * 2.0**-53
    assert rep["precision"] == prec and rep["factor_precision"] == prec and not rep["fell_back"], rep
    assert 1 <= rep["iterations"] <= 10 and rep["backward_error"] <= target, rep
    a = _dense(cp, ri, v, n)
    eta = np.max(np.abs(b - a @ x)) / (np.max(np.abs(a).sum(axis=1)) * np.max(np.abs(x)) + np.max(np.abs(b)))
    assert eta <= target, eta
    xr = _ref(osp, lu, cp, ri, v).solve(b)
    cond = np.max(np.abs(a).sum(axis=1)) * np.max(np.abs(np.linalg.inv(a)).sum(axis=1))
    fwd = np.max(np.abs(x - xr)) / np.max(np.abs(xr))
    assert fwd <= 2 * cond * target, (fwd, cond)


@pytest.mark.parametrize("prec", ["tf32", "tf32x3", "bf16"])
def test_tensor_core_fronts_on_a_larger_grid(gpu, osp, prec):
    # 20^3: large fronts (factored by the blocked dense LU) exist, so the
    # trailing updates run on the tensor cores
    cp, ri, kind = osp.grid_pattern(20, 20, 20)
    v, s = osp.convection_diffusion_values(kind, SEED)
    n = len(cp) - 1
    ref = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    plan = ref.plan()
    assert plan["n_small_fronts"] < plan["n_fronts"]
    ref.factorize(cp, ri, v)
    b, _ = osp.dense.larnv("Symmetric", [2, 4, 6, 9], n)
    x64 = b.copy()
    ref.solve(x64)
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    lu.set_precision(prec)
    for vals in (v, osp.perturb(v, s)[0]):  # a refactorization with new values too
        lu.factorize(cp, ri, vals)
        x = b.copy()
        lu.solve(x)
        rep = lu.last_solve()
        assert not rep["fell_back"] and rep["backward_error"] <= 10 * n * 2.0**-53, rep
        assert _csr_residual(cp, ri, vals, x, b) <= 10 * n * 2.0**-53
    # back to the first values: the FP64 form's solution, to the conditioning's accuracy
    x_first = b.copy()
    lu.factorize(cp, ri, v)
    lu.solve(x_first)
    assert np.max(np.abs(x_first - x64)) / np.max(np.abs(x64)) <= 1e-8


def test_fp32_zero_pivot_refactors_in_fp64(gpu):
    # [[1, 1], [1, 1 + 1e-10]]: exactly singular once rounded to FP32
    cp, ri, v = [0, 2, 4], [0, 1, 0, 1], [1.0, 1.0, 1.0, 1.0 + 1e-10]
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    lu.set_precision("fp32")
    lu.factorize(cp, ri, v)
    x = np.array([2.0, 2.0 + 1e-10])
    lu.solve(x)
    rep = lu.last_solve()
    assert rep["factor_precision"] == "fp64" and rep["precision"] == "fp64" and rep["iterations"] == 0, rep
    np.testing.assert_allclose(x, [1.0, 1.0], rtol=0, atol=1e-4)  # cond_inf ~ 4e10


def test_refinement_that_cannot_reach_the_target_falls_back(gpu, osp):
    cp, ri, kind = osp.grid_pattern(8, 8, 8)
    v, _ = osp.convection_diffusion_values(kind, SEED)
    n = len(cp) - 1
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    lu.set_precision("fp32", tol=1e-300, max_ir=2)  # an unreachable target
    lu.factorize(cp, ri, v)
    b = np.ones(n)
    x = b.copy()
    lu.solve(x)
    rep = lu.last_solve()
    assert rep["fell_back"] and rep["precision"] == "fp64" and rep["factor_precision"] == "fp64", rep
    assert 1 <= rep["iterations"] <= 2
    xr = _ref(osp, lu, cp, ri, v).solve(b)
    assert np.max(np.abs(x - xr) / np.maximum(np.abs(xr), 1.0)) <= 1e-12
    # the set now holds FP64 factors: the next solve is direct
    x2 = b.copy()
    lu.solve(x2)
    rep = lu.last_solve()
    assert rep["iterations"] == 0 and not rep["fell_back"] and rep["precision"] == "fp64"
    assert np.array_equal(x, x2)


def test_device_resident_mixed_solve_is_deterministic(gpu, osp):
    import torch

    from algebra_linear_b200 import device

    cp, ri, kind = osp.grid_pattern(10, 9, 8)
    v, _ = osp.convection_diffusion_values(kind, [5, 6, 7, 9])
    n = len(cp) - 1
    b = np.linspace(-1.0, 1.0, n)
    host = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    host.set_precision("fp32")
    host.factorize(cp, ri, v)
    xh = b.copy()
    host.solve(xh)
    with device.Context() as ctx:
        lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
        lu.set_precision("fp32")
        lu.bind(ctx)
        lu.factorize_dev(torch.from_numpy(v).cuda())
        db = torch.from_numpy(b.copy()).cuda()
        lu.solve_dev(db)
        torch.cuda.synchronize()
        xd = db.cpu().numpy()
        assert lu.last_solve()["iterations"] >= 1
        lu.close()
    assert np.array_equal(xh, xd)


def test_lanes_do_not_change_the_result(gpu, osp, monkeypatch):
    """Independent subtrees factored on two concurrent lanes give the same
    factors, bit for bit, as one lane (no arithmetic depends on the order)."""
    cp, ri, kind = osp.grid_pattern(20, 20, 20)
    v, _ = osp.convection_diffusion_values(kind, SEED)
    n = len(cp) - 1
    b, _ = osp.dense.larnv("Symmetric", [7, 7, 7, 7], n)
    xs = []
    for lanes in ("1", "2"):
        monkeypatch.setenv("ALG_SPLU_LANES", lanes)
        lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
        assert lu.plan()["n_lanes"] == int(lanes)
        lu.factorize(cp, ri, v)
        x = b.copy()
        lu.solve(x)
        xs.append((x, lu.row_perm(), lu.stats()["nnz_l"]))
    assert np.array_equal(xs[0][0], xs[1][0]) and np.array_equal(xs[0][1], xs[1][1]) and xs[0][2] == xs[1][2]
