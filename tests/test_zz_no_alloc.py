"""The allocation-free entry point alg_dgesv_mixed_noalloc, called through
the C ABI. It has no counterpart in the reference crate. It exists for
callers that cannot call cudaMalloc (code inside another library's memory
pool, serving loops that must not synchronise the device, callers that must
not meet out-of-memory after start-up): it runs the mixed form of the
batched dgesv kernel on one system with its working memory in a static
device array. On the GPU it must agree bit for bit with a one-system
alg_batch plan (mixed = 1) on the same input (solution, backward error and
pivots), call after call while the static array is reused, and the device's
free memory must not change across the calls after the first. This file is
named to be collected last, so the calls also run after everything the other
test files left on the device."""

import ctypes as C

import numpy as np
import pytest

MAX_N = 512  # ALG_NOALLOC_MAX_N


def _system(oracle, n, seed):
    a, s = oracle.larnv("Symmetric", [seed, 7, 1, 2 * n + 1], n * n)
    x, _ = oracle.larnv("Symmetric", s, n)
    return a, oracle.dgemv(a, x, n, n)


def test_noalloc_rejects_orders_beyond_its_scratch():
    # host-side checks: nothing reaches the device
    from algebra_linear_b200 import _lib

    lib = _lib.load()
    assert lib.alg_dgesv_mixed_noalloc(None, None, None, MAX_N + 1, None, None, None) == _lib.BAD_SHAPE
    assert lib.alg_dgesv_mixed_noalloc(None, None, None, -1, None, None, None) == _lib.BAD_SHAPE
    assert lib.alg_dgesv_mixed_noalloc(None, None, None, 4, None, None, None) == _lib.INVALID_ARGUMENT
    # n = 0 is the set-up call: Ok on a GPU, no-device without one
    assert lib.alg_dgesv_mixed_noalloc(None, None, None, 0, None, None, None) in (_lib.OK, _lib.NO_DEVICE)


def _batched_reference(ctx, a, b, n):
    """The existing entry point: a one-system mixed alg_batch plan."""
    import torch

    from algebra_linear_b200 import batched

    plan = batched.BatchPlan(ctx, [n], mixed=True)
    A = torch.from_numpy(a.copy()).cuda()
    B = torch.from_numpy(b.copy()).cuda()
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    plan.solve(A, B, info)
    torch.cuda.synchronize()
    out = B.cpu().numpy(), int(info.cpu()[0]), float(plan.eta()[0]), plan.ipiv().copy()
    plan.close()
    return out


@pytest.mark.gpu
def test_noalloc_matches_the_batched_entry_point_call_after_call(gpu, oracle):
    import torch

    from algebra_linear_b200 import _lib, device

    lib = gpu
    assert lib.alg_dgesv_mixed_noalloc(None, None, None, 0, None, None, None) == _lib.OK  # set-up call
    orders = [300, 512, 37]  # the second call reuses the array at full size, the third after it
    # every device buffer of the three calls exists before the first, so that
    # nothing but the entry point could change the device's free memory
    calls = []
    for k, n in enumerate(orders):
        a, b = _system(oracle, n, seed=5 + k)
        calls.append((n, a, b, torch.from_numpy(a.copy()).cuda(), torch.from_numpy(b.copy()).cuda(),
                      torch.full((n,), -1, dtype=torch.int32, device="cuda"),
                      torch.full((1,), 99, dtype=torch.int32, device="cuda"),
                      torch.full((1,), -1.0, dtype=torch.float64, device="cuda")))
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free_after = []
    for n, a, b, A, B, ipiv, info, eta in calls:
        rc = lib.alg_dgesv_mixed_noalloc(C.c_void_p(stream), A.data_ptr(), B.data_ptr(), n, ipiv.data_ptr(),
                                         info.data_ptr(), eta.data_ptr())
        assert rc == _lib.OK, _lib.status_string(rc)
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
    # calls 2 and 3 allocated nothing on the device
    assert free_after[1] == free_after[0] and free_after[2] == free_after[0], free_after
    results = [(n, a, b, B.cpu().numpy(), int(info.cpu()[0]), float(eta.cpu()[0]), ipiv.cpu().numpy())
               for n, a, b, A, B, ipiv, info, eta in calls]
    for n, a, b, A, *_ in calls:
        assert np.array_equal(A.cpu().numpy(), a)  # A is only read
    with device.Context() as ctx:
        for n, a, b, x, info, eta, ipiv in results:
            xr, info_r, eta_r, ipiv_r = _batched_reference(ctx, a, b, n)
            assert info == info_r == 0, (n, info, info_r)
            assert np.array_equal(x, xr), n
            assert eta == eta_r, (n, eta, eta_r)
            assert np.array_equal(ipiv, ipiv_r), n
            assert oracle.backward_error(a, x, b, n) <= 10 * n * 2.0**-53


@pytest.mark.gpu
def test_noalloc_reports_a_zero_pivot_like_the_batched_entry_point(gpu, oracle):
    import torch

    from algebra_linear_b200 import _lib, device

    lib = gpu
    n = 40
    a, b = _system(oracle, n, seed=3)
    a[5 * n:6 * n] = 0.0  # column 5 is zero
    A = torch.from_numpy(a.copy()).cuda()
    B = torch.from_numpy(b.copy()).cuda()
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    eta = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    rc = lib.alg_dgesv_mixed_noalloc(None, A.data_ptr(), B.data_ptr(), n, None, info.data_ptr(), eta.data_ptr())
    assert rc == _lib.OK
    torch.cuda.synchronize()
    with device.Context() as ctx:
        _, info_r, _, _ = _batched_reference(ctx, a, b, n)
    assert int(info.cpu()[0]) == info_r > 0
    # on a zero pivot neither b nor the backward error is written
    assert float(eta.cpu()[0]) == -1.0
    assert np.array_equal(B.cpu().numpy(), b)
