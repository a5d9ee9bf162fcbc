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
