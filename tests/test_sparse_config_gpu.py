"""GPU parity of the sparse LU near the benchmark sizes, against the oracle's
results stored by tests/golden/make_sparse_golden.py (the oracle, a C++
restatement of the reference's supernodal LU, supernodal_lu.rs:118-533,
takes minutes to hours per factorization at these sizes on one core).

Cases: 2-D 5-point convection-diffusion patterns (the serving workload's
300 x 300 one, n = 90 000, and 150 x 150) and the 20^3 7-point grid
(n = 8 000), sizes where the GPU plan merges fronts and splits the large ones
over two lanes. Each in two rounds: the generator's values, then a 1 %
multiplicative refactorization on the same handle (the benchmark's round).
Bar per round: the row permutation identical to the oracle's (SHA-256 of the
whole vector); nnz(L), nnz(U) and flops_estimate equal; x within 1e-12
relative (max(1, |x|) scale, parity.rs:134-146) at every stored position;
the normwise backward error of the whole x within 10 n 2^-53."""

import hashlib
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem[len("sparse_"):] for p in GOLDEN.glob("sparse_*.npz"))


def test_fixtures_exist():
    assert "grid20x20x20" in CASES, CASES


@pytest.mark.parametrize("name", CASES)
def test_config_size_grids_match_the_oracle(gpu, name):
    import scipy.sparse as sps

    from algebra_linear_b200.sparse import LuMethod, SparseLu
    from oracle import sparse as osp
    from tests.golden.make_sparse_golden import round_rhs, round_values

    g = dict(np.load(GOLDEN / f"sparse_{name}.npz"))
    cp, ri, kind = osp.grid_pattern(*[int(d) for d in g["dims"]])
    n = len(cp) - 1
    stride = int(g["stride"])
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    for rnd in (0, 1):
        v = round_values(kind, rnd)
        lu.factorize(cp, ri, v)  # round 1 refactorizes the same handle
        rp = lu.row_perm().astype(np.int64)
        assert list(rp[:64]) == list(g[f"r{rnd}_row_perm_head"]), (name, rnd)
        assert hashlib.sha256(rp.tobytes()).digest() == g[f"r{rnd}_row_perm_sha256"].tobytes(), (name, rnd)
        s = lu.stats()
        nnz_l, nnz_u, flops = (int(c) for c in g[f"r{rnd}_counts"])
        assert (s["nnz_l"], s["nnz_u"], s["flops_estimate"]) == (nnz_l, nnz_u, flops), (name, rnd)
        b = round_rhs(n, rnd)
        x = b.copy()
        lu.solve(x)
        xr = g[f"r{rnd}_x"]
        err = float(np.max(np.abs(x[::stride] - xr) / np.maximum(np.abs(xr), 1.0)))
        assert err <= 1e-12, (name, rnd, err)
        A = sps.csc_matrix((v, ri.astype(np.int64), cp.astype(np.int64)), shape=(n, n))
        eta = float(np.abs(b - A @ x).max() / (abs(A).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max()))
        assert eta <= 10 * n * 2.0**-53, (name, rnd, eta)
        print(f"{name} round {rnd}: n {n}, nnz_l {nnz_l}, nnz_u {nnz_u}, x rel err {err:.1e}, eta {eta:.1e}")
    lu.close()
