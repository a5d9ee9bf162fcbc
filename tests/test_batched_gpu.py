"""GPU parity of the batched dgesv: every system against the oracle's
dgesv (src/lapack/mod.rs:309-354) on the same inputs.

Tolerances: x within 1e-12 relative (max(1,|x|) scale, as parity.rs:134-146)
for the FP64 form on the shifted systems; the mixed form reaches the FP64
backward error 10 n 2^-53 per system."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORDERS = [1, 2, 7, 8, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 200, 255, 256, 257, 300, 511, 512]


def _systems(oracle, orders, shift=True, seed=11):
    mats, rhs = [], []
    for k, n in enumerate(orders):
        a, s = oracle.larnv("Symmetric", [seed, 3, 5, 2 * k + 1], n * n)
        if shift:
            a[:: n + 1] += n
        x, _ = oracle.larnv("Symmetric", s, n)
        mats.append(a)
        rhs.append(oracle.dgemv(a, x, n, n))
    return mats, rhs


def _pack(plan, mats, rhs):
    import torch

    A = np.zeros(max(plan.a_total, 1))
    B = np.zeros(max(plan.b_total, 1))
    for k, (a, b) in enumerate(zip(mats, rhs)):
        A[plan.a_off[k]:plan.a_off[k] + a.size] = a
        B[plan.b_off[k]:plan.b_off[k] + b.size] = b
    return torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()


@pytest.mark.parametrize("shift", [True, False])
def test_batched_fp64_matches_the_reference(gpu, oracle, shift):
    import torch

    from algebra_linear_b200 import batched, device

    mats, rhs = _systems(oracle, ORDERS, shift=shift)
    with device.Context() as ctx:
        plan = batched.BatchPlan(ctx, ORDERS)
        A, B = _pack(plan, mats, rhs)
        info = torch.zeros(len(ORDERS), dtype=torch.int32, device="cuda")
        plan.solve(A, B, info)
        torch.cuda.synchronize()
        Bh, Ah, ih = B.cpu().numpy(), A.cpu().numpy(), info.cpu().numpy()
        plan.close()
    for k, n in enumerate(ORDERS):
        ra, rb = mats[k].copy(), rhs[k].copy()
        rc, _ = oracle.dgesv(ra, rb, n)
        assert rc == 0 and ih[k] == 0, (n, ih[k])
        x = Bh[plan.b_off[k]:plan.b_off[k] + n]
        err = np.max(np.abs(x - rb) / np.maximum(np.abs(rb), 1.0))
        tol = 1e-12 if shift else 1e-9
        assert err < tol, (n, err)


def test_batched_singular_and_graph_replay(gpu, oracle):
    import torch

    from algebra_linear_b200 import batched, device

    orders = [3, 40, 5]
    mats, rhs = _systems(oracle, orders)
    mats[1][5 * 40:6 * 40] = 0.0  # column 5 of system 1 is zero: singular
    with device.Context() as ctx:
        plan = batched.BatchPlan(ctx, orders)
        A0, B0 = _pack(plan, mats, rhs)
        info = torch.zeros(3, dtype=torch.int32, device="cuda")
        outs = []
        for rep in range(3):  # capture, then replay twice
            A, B = A0.clone(), B0.clone()
            if rep == 0:
                Ag, Bg = A, B
            else:
                Ag.copy_(A0)
                Bg.copy_(B0)
            plan.solve(Ag, Bg, info, graph=True)
            torch.cuda.synchronize()
            outs.append((Bg.cpu().numpy().copy(), info.cpu().numpy().copy()))
        plan.close()
    for B, ih in outs:
        assert ih[0] == 0 and ih[2] == 0 and ih[1] > 0
        assert np.array_equal(B, outs[0][0])


def test_batched_mixed_reaches_fp64_backward_error(gpu, oracle):
    import torch

    from algebra_linear_b200 import batched, device

    orders = [8, 50, 129, 300, 512]
    mats, rhs = _systems(oracle, orders, seed=23)
    with device.Context() as ctx:
        plan = batched.BatchPlan(ctx, orders, mixed=True)
        A, B = _pack(plan, mats, rhs)
        info = torch.zeros(len(orders), dtype=torch.int32, device="cuda")
        plan.solve(A, B, info)
        torch.cuda.synchronize()
        Bh, ih = B.cpu().numpy(), info.cpu().numpy()
        eta = plan.eta()
        plan.close()
    for k, n in enumerate(orders):
        x = Bh[plan.b_off[k]:plan.b_off[k] + n]
        assert ih[k] == 0, (n, ih[k], eta[k])
        assert oracle.backward_error(mats[k], x, rhs[k], n) <= 10 * n * 2.0**-53


def test_batched_fp64_pivots_match_the_reference_without_a_shift(gpu, oracle):
    """Unshifted systems (A iid U(-1,1), cond ~ n), where partial pivoting
    swaps rows at almost every step: the pivot sequence of every system is
    the oracle's (mod.rs:112-163), and x agrees to the conditioning."""
    import torch

    from algebra_linear_b200 import batched, device

    mats, rhs = _systems(oracle, ORDERS, shift=False, seed=29)
    with device.Context() as ctx:
        plan = batched.BatchPlan(ctx, ORDERS)
        A, B = _pack(plan, mats, rhs)
        info = torch.zeros(len(ORDERS), dtype=torch.int32, device="cuda")
        plan.solve(A, B, info)
        torch.cuda.synchronize()
        Bh, ih, piv = B.cpu().numpy(), info.cpu().numpy(), plan.ipiv()
        plan.close()
    swaps = 0
    for k, n in enumerate(ORDERS):
        ra, rb = mats[k].copy(), rhs[k].copy()
        rc, ripiv = oracle.dgesv(ra, rb, n)
        assert rc == 0 and ih[k] == 0, (n, ih[k])
        gp = piv[plan.b_off[k]:plan.b_off[k] + n]
        assert list(gp) == list(ripiv), n
        swaps += int(np.count_nonzero(gp != np.arange(n)))
        x = Bh[plan.b_off[k]:plan.b_off[k] + n]
        assert np.max(np.abs(x - rb) / np.maximum(np.abs(rb), 1.0)) < 1e-9, n
    assert swaps > sum(ORDERS) // 2  # the interchanges were exercised


def test_every_launch_shape_and_the_autotuner(gpu, oracle, tmp_path):
    """Each launch shape the autotuner chooses from (128 / 256 / 512 threads x
    16- / 32-column panels) solves every bucket to the oracle's x and pivots;
    the autotuner's choice is recorded in its JSON cache, and a second plan
    reads the cache instead of timing and gives bit-identical solutions."""
    import torch

    from algebra_linear_b200 import batched, device

    orders = [5, 20, 33, 64, 90, 128, 200, 256, 333, 512]
    mats, rhs = _systems(oracle, orders, shift=False, seed=31)
    refs = []
    for k, n in enumerate(orders):
        ra, rb = mats[k].copy(), rhs[k].copy()
        rc, ripiv = oracle.dgesv(ra, rb, n)
        assert rc == 0
        refs.append((rb, ripiv))
    cache = tmp_path / "tune.json"

    def check(plan, Bh, piv):
        for k, n in enumerate(orders):
            x = Bh[plan.b_off[k]:plan.b_off[k] + n]
            assert np.max(np.abs(x - refs[k][0]) / np.maximum(np.abs(refs[k][0]), 1.0)) < 1e-9, n
            assert list(piv[plan.b_off[k]:plan.b_off[k] + n]) == list(refs[k][1]), n

    with device.Context() as ctx:
        plan = batched.BatchPlan(ctx, orders)
        A0, B0 = _pack(plan, mats, rhs)
        info = torch.zeros(len(orders), dtype=torch.int32, device="cuda")
        nb = len(plan.info()["buckets"])
        for threads in (128, 256, 512):
            for panel in (16, 32):
                for bk in range(nb):
                    assert gpu.alg_batch_set_config(plan.handle, bk, threads, panel) == 0
                A, B = A0.clone(), B0.clone()
                plan.solve(A, B, info)
                torch.cuda.synchronize()
                assert int((info != 0).sum()) == 0
                check(plan, B.cpu().numpy(), plan.ipiv())
        A, B = A0.clone(), B0.clone()
        tuned = plan.autotune(A, B, info, A0, B0, cache=str(cache))
        assert tuned["tuned"] == "timed"
        for bk in tuned["buckets"]:
            assert bk["threads"] in (128, 256, 512) and bk["panel"] in (16, 32), bk
        A, B = A0.clone(), B0.clone()
        plan.solve(A, B, info, graph=True)
        torch.cuda.synchronize()
        x_tuned = B.cpu().numpy()
        check(plan, x_tuned, plan.ipiv())
        plan.close()
        plan2 = batched.BatchPlan(ctx, orders)
        A, B = A0.clone(), B0.clone()
        again = plan2.autotune(A, B, info, A0, B0, cache=str(cache))
        assert again["tuned"] == "cache"
        assert [(b["threads"], b["panel"]) for b in again["buckets"]] == \
            [(b["threads"], b["panel"]) for b in tuned["buckets"]]
        A, B = A0.clone(), B0.clone()
        plan2.solve(A, B, info)
        torch.cuda.synchronize()
        assert np.array_equal(B.cpu().numpy(), x_tuned)
        plan2.close()
