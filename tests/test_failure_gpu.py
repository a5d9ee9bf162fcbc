"""The timeout path of the device-side waits, exercised without any fault:
the dataflow triangular solve's first block is made to wait on a flag that
nothing sets (alg_ctx_inject_stuck_wait) under a short host-set limit
(alg_ctx_set_wait_limit). The kernel gives up, every CTA returns, the call
reports ALG_TIMEOUT, and the same context then solves normally — the result
equal to the oracle's (the reference's dgesv, mod.rs:309-354)."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", ["dgetrs_dev", "dgesv_dev"])
def test_a_wait_that_runs_out_reports_timeout_and_the_context_recovers(gpu, oracle, path):
    import torch

    from algebra_linear_b200 import _lib, device
    from algebra_linear_b200.lapack import LapackError

    n = 1024
    a, _, b = oracle.c1_system(n, seed=[5, 6, 7, 9])
    ra, rb = a.copy(), b.copy()
    rc, _ = oracle.dgesv(ra, rb, n)
    assert rc == 0
    with device.Context() as ctx:
        A = torch.from_numpy(a.copy()).cuda()
        perm = ctx.dgetrf(A, n)[1] if path == "dgetrs_dev" else None
        assert gpu.alg_ctx_set_wait_limit(ctx.handle, 1_000_000) == _lib.OK  # 1 ms
        assert gpu.alg_ctx_inject_stuck_wait(ctx.handle, 1) == _lib.OK

        def solve():
            B = torch.from_numpy(b.copy()).cuda()
            if path == "dgetrs_dev":
                ctx.dgetrs(A, perm, B, n)
            else:
                ctx.dgesv(torch.from_numpy(a.copy()).cuda(), B, n)
            return B

        t0 = time.perf_counter()
        with pytest.raises(LapackError) as e:
            solve()
        elapsed = time.perf_counter() - t0
        assert e.value.code == _lib.TIMEOUT, e.value
        assert elapsed < 5.0, elapsed  # the wait gave up; nothing hung
        # the same context, the default limit again: a normal solve
        assert gpu.alg_ctx_set_wait_limit(ctx.handle, 0) == _lib.OK
        x = solve().cpu().numpy()
    err = np.max(np.abs(x - rb) / np.maximum(np.abs(rb), 1.0))
    assert err <= 1e-12, err
