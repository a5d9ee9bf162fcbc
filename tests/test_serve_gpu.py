"""The serving loop: every request's result is the same alone and in a mix of
concurrent dense (FP64 and mixed) and sparse requests, and correct against
the oracle (dense: x within 1e-12 relative of the oracle's dgesv on the
shifted systems; sparse: within 1e-12 of the oracle's supernodal LU)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dense_system(oracle, n, k):
    a, s = oracle.larnv("Symmetric", [7, 9, 11, 2 * k + 1], n * n)
    a[:: n + 1] += n
    b, _ = oracle.larnv("Symmetric", s, n)
    return a, b


def _requests(oracle, osp, lu, cp, ri, kind):
    from algebra_linear_b200.serve import Request

    reqs, checks = [], []
    for k, n in enumerate([70, 300, 1000, 64, 2048, 513]):
        a, b = _dense_system(oracle, n, k)
        reqs.append(Request.dense(a, b, mixed=bool(k % 2)))
        checks.append(("dense", a, b, n))
    for k in range(3):
        v, _ = osp.convection_diffusion_values(kind, [3, 4, 5, 2 * k + 1])
        b = np.ones(len(cp) - 1)
        reqs.append(Request.sparse(lu, v, b))
        checks.append(("sparse", v, b, len(cp) - 1))
    return reqs, checks


def test_results_are_the_same_alone_and_in_the_mix(gpu, oracle):
    from algebra_linear_b200.serve import Server
    from algebra_linear_b200.sparse import LuMethod, SparseLu
    from oracle import sparse as osp

    cp, ri, kind = osp.grid_pattern(30, 30, 1)
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    alone, checks = _requests(oracle, osp, lu, cp, ri, kind)
    with Server(workers=1, hbm_budget=8 << 30, max_dense_n=2048) as srv:
        for r in alone:  # one at a time
            srv.submit(r)
            assert srv.wait(r) == 0
    mix, _ = _requests(oracle, osp, lu, cp, ri, kind)
    with Server(workers=4, hbm_budget=8 << 30, max_dense_n=2048) as srv:
        for r in mix[::-1] + []:
            srv.submit(r)
        srv.drain()
    assert len({r.worker for r in mix}) > 1  # the mix really ran concurrently
    for ra, rm in zip(alone, mix):
        assert rm.status == 0
        assert np.array_equal(ra.solution, rm.solution)
    sym = lu.symbolic()
    for r, (kind_, m, b, n) in zip(alone, checks):
        if kind_ == "dense":
            aw, bw = m.copy(), b.copy()
            rc, _ = oracle.dgesv(aw, bw, n)
            assert rc == 0
            err = np.max(np.abs(r.solution - bw) / np.maximum(np.abs(bw), 1.0))
            assert err < 1e-12, (n, err)
        else:
            ref = osp.Factors(n, cp, ri, m, sym["col_perm"], sym["col_perm_inv"], sym["supernode_ptr"])
            xr = ref.solve(b)
            assert np.max(np.abs(r.solution - xr) / np.maximum(np.abs(xr), 1.0)) <= 1e-12


def test_admission_respects_the_budget(gpu, oracle):
    from algebra_linear_b200.serve import Request, Server

    # a budget that holds one n = 1500 system at a time: requests still all
    # complete, one after another
    reqs = []
    for k in range(4):
        a, b = _dense_system(oracle, 1500, 40 + k)
        reqs.append(Request.dense(a, b))
    with Server(workers=4, hbm_budget=8 * 1500 * 1500 + 200000, max_dense_n=1500) as srv:
        for r in reqs:
            srv.submit(r)
        srv.drain()
    spans = sorted((r._r.t_start_ns, r._r.t_done_ns) for r in reqs)
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0  # no two were admitted at once
    assert all(r.status == 0 for r in reqs)


def _eta_extended(a, x, b, n):
    """The normwise backward error of x with the residual in x87 extended
    precision (64-bit significand), so the reference value carries none of
    the FP64 residual's own rounding."""
    import numpy as np

    A = a.reshape(n, n).T.astype(np.longdouble)
    xl, bl = x.astype(np.longdouble), b.astype(np.longdouble)
    r = bl - A @ xl
    return float(np.abs(r).max() / (np.abs(A).sum(axis=1).max() * np.abs(xl).max() + np.abs(bl).max()))


def test_reported_backward_error_matches_the_host(gpu, oracle):
    """A mixed dense request reports the refinement's final normwise
    backward error; it must agree with the error of the returned x computed
    on the host with an extended-precision residual, to a factor of 4 plus
    the FP64 residual's own rounding (about sqrt(n) 2^-53 of the
    normalisation), and be within 10 n 2^-53. Plain FP64 requests report
    -1."""
    import numpy as np

    from algebra_linear_b200.serve import Request, Server

    reqs, systems = [], []
    for k, n in enumerate([64, 257, 1000, 3000]):
        a, b = _dense_system(oracle, n, 60 + k)
        systems.append((a, b, n))
        reqs.append(Request.dense(a, b, mixed=True))
    reqs.append(Request.dense(*_dense_system(oracle, 100, 70), mixed=False))
    with Server(workers=2, hbm_budget=8 << 30, max_dense_n=3000) as srv:
        for r in reqs:
            srv.submit(r)
        srv.drain()
    assert all(r.status == 0 for r in reqs)
    assert reqs[-1].backward_error == -1.0
    for r, (a, b, n) in zip(reqs, systems):
        host = _eta_extended(a, r.solution, b, n)
        rep = r.backward_error
        slack = 4 * np.sqrt(n) * 2.0**-53
        print(f"n={n}: reported eta {rep:.3e}, host eta {host:.3e}")
        assert host <= 10 * n * 2.0**-53, (n, host)
        assert 0 < rep <= 10 * n * 2.0**-53, (n, rep)
        assert host / 4 - slack <= rep <= 4 * host + slack, (n, rep, host)
