"""Host-side pieces of bench.py, on the CPU: the workload generators match
the configurations they name (C3 orders, C4 and C5 stencil sizes), the
forward-error comparison between forms, the library-context solve's
reading of the column-major layout, and a failing sub-workload is recorded
instead of ending the benchmark line."""

import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_c3_orders_are_log_uniform_in_8_512():
    n = bench.batched_orders(20000, 1991)
    assert n.size == 20000 and n.min() >= 8 and n.max() <= 512
    # log-uniform: about a sixth of the systems in each factor-2 band
    frac = np.mean((n > 256) & (n <= 512))
    assert 0.13 < frac < 0.20, frac
    assert np.array_equal(n, bench.batched_orders(20000, 1991))  # seeded


@pytest.mark.parametrize("dims,n,nnz", [((48, 48, 48), 110592, 760320), ((300, 300, 1), 90000, 448800)])
def test_stencil_sizes_of_c4_and_c5(dims, n, nnz):
    cp, ri, kind = bench.grid_csc(*dims)
    assert cp.size == n + 1 and int(cp[-1]) == nnz and ri.size == nnz and kind.size == nnz
    # rows sorted within every column, one diagonal entry per column
    cpi = cp.astype(np.int64)
    ends = cpi[1:]
    assert np.all(np.diff(ri.astype(np.int64))[np.setdiff1d(np.arange(nnz - 1), ends[:-1] - 1)] > 0)
    assert int((kind == 0).sum()) == n


def test_forward_error_against_a_reference_form():
    torch = pytest.importorskip("torch")
    x = torch.tensor([1.0, -2.0, 4.0], dtype=torch.float64)
    dx = torch.tensor([0.0, 0.0, 4e-6], dtype=torch.float64)
    res = {"fp64_exact": {"_x": x.clone()}, "mixed": {"_x": x + dx}, "other": {"backward_error": 1.0}}
    bench.forward_vs(res, "fp64_exact")
    assert res["fp64_exact"]["forward_error_vs_fp64_exact"] == 0.0
    assert abs(res["mixed"]["forward_error_vs_fp64_exact"] - 1e-6) < 1e-12
    assert all("_x" not in r for r in res.values())
    res = {"mixed": {"_x": x}}
    bench.forward_vs(res, "fp64_exact")  # no reference form: nothing computed, solutions dropped
    assert res == {"mixed": {}}


def test_a_failing_sub_workload_is_recorded():
    class Args:
        pass

    def boom(args, world, rank, local, pg):
        assert args.steps == 3 and args.warmup == 2 and args.no_cpu and not args.emit
        raise RuntimeError("no device")

    out = bench.sub_arm(boom, Args(), 1, 0, 0, None)
    assert out == {"error": "RuntimeError('no device')"}

    def ok(args, world, rank, local, pg):
        return {"metric": "m", "value": 1.0, "n_gpus": 1, "data": "d", "e2e": {"value": 2.0}}

    assert bench.sub_arm(ok, Args(), 1, 0, 0, None) == {"metric": "m", "value": 1.0, "e2e": {"value": 2.0}}


def test_library_context_solve_reads_the_column_major_layout():
    torch = pytest.importorskip("torch")
    n, nrhs = 37, 3
    g = torch.Generator().manual_seed(3)
    A = torch.rand(n, n, generator=g, dtype=torch.float64) - 0.5  # A[i, j]
    X = torch.rand(n, nrhs, generator=g, dtype=torch.float64)
    B = A @ X
    A0 = A.t().contiguous().view(-1)  # column-major: A0[i + j n] = A[i, j]
    b0 = B.t().contiguous().view(-1)
    x = bench.torch_lu_solve(A0, b0, n, nrhs)
    assert bench.backward_error(A0, x, b0, n, nrhs) < 1e-14
    assert torch.allclose(x.view(nrhs, n).t(), X, atol=1e-10)
    # without a GPU the device-timed context records the failure instead of raising
    if not torch.cuda.is_available():
        assert "error" in bench.cusolver_context(A0, b0, n, nrhs)


def _reference_lattice(m):
    """The loops of bench_sparse_lu (src/sparse/faer/sparse_lu.rs:176-218) as
    they are written there: k outer, i inner, three columns per node, the
    27 surrounding nodes' three rows each, sorted; values -1 off the diagonal
    and 10 + (off-diagonal count) on it."""
    node = lambda i, j, k: (k * m * m + j * m + i) * 3  # noqa: E731
    cp, ri = [0], []
    for k in range(m):
        for j in range(m):
            for i in range(m):
                for _ in range(3):
                    rows = []
                    for dk in range(3):
                        for dj in range(3):
                            for di in range(3):
                                ii, jj, kk = i + di - 1, j + dj - 1, k + dk - 1
                                if min(ii, jj, kk) < 0 or max(ii, jj, kk) >= m:
                                    continue
                                base = node(ii, jj, kk)
                                rows += [base, base + 1, base + 2]
                    rows.sort()
                    ri += rows
                    cp.append(len(ri))
    v = []
    for c in range(len(cp) - 1):
        off = sum(1 for p in range(cp[c], cp[c + 1]) if ri[p] != c)
        v += [10.0 + off if ri[p] == c else -1.0 for p in range(cp[c], cp[c + 1])]
    return cp, ri, v


def test_lattice_is_the_reference_benchmark_matrix():
    cp, ri, v = bench.lattice_csc(4)
    rcp, rri, rv = _reference_lattice(4)
    assert cp.tolist() == rcp and ri.tolist() == rri and v.tolist() == rv
    assert len(cp) - 1 == 192


def test_lattice_fill_is_the_published_one(oracle):
    """README.md:119 and solver.rs:21-25 report fill 2.96 for this matrix:
    the host analysis (COLAMD order, supernodes) and the oracle's simplicial
    and supernodal factorizations over it reproduce it, and Auto picks the
    supernodal method, as the README's second row has it."""
    from algebra_linear_b200.sparse import LuMethod, SparseLu
    from oracle import sparse as osp

    cp, ri, v = bench.lattice_csc(4)
    n = len(cp) - 1
    auto = SparseLu.analyze(cp, ri, LuMethod.auto())
    assert auto.effective_method() == "Supernodal" and auto.flop_ratio() > 40.0
    for method in (LuMethod.simplicial(), LuMethod.supernodal()):
        sym = SparseLu.analyze(cp, ri, method).symbolic()
        snp = sym["supernode_ptr"] if method.kind == LuMethod.supernodal().kind else None
        f = osp.Factors(n, cp, ri, v, sym["col_perm"], sym["col_perm_inv"], snp)
        assert f.status == 0
        assert round((f.nnz_l + f.nnz_u) / len(ri), 2) == 2.96
        x = f.solve(np.ones(n))
        A = np.zeros((n, n))
        A[ri.astype(np.int64), np.repeat(np.arange(n), np.diff(cp).astype(np.int64))] = v
        assert np.max(np.abs(A @ x - 1.0)) < 1e-13


def test_lattice_run_records_a_failure_instead_of_raising():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU run measures it")
    out = bench.lattice_run(reps=2)
    assert set(out) == {"error"} and "device" in out["error"].lower()
