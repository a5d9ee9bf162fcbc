"""GPU tests of the mixed-precision path: the tcgen05 trailing update against
a torch FP32 reference of the same rounded operands, and the refined solve
against the oracle's FP64 solution.

Tolerances: the tensor-core update must match the reference product of the
rounded operands to FP32 accumulation error (1e-4 relative to the largest
|product|); the refined x must reach the FP64 backward-error level
10 n 2^-53 and agree with the oracle's x to cond-scaled FP64 accuracy.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _round_bf16(t):
    import torch

    return t.to(torch.bfloat16).to(torch.float32)


def _round_tf32(t):
    import torch

    u = t.contiguous().view(torch.int32)
    # round-to-nearest (ties away) to 10 mantissa bits, as cvt.rna.tf32.f32
    r = (u + 0x1000) & ~0x1FFF
    return r.view(torch.float32)


@pytest.mark.parametrize("prec", ["bf16", "tf32", "tf32x3"])
@pytest.mark.parametrize("shape", [(128, 256, 64), (300, 500, 128), (1000, 700, 256), (4096, 4096, 128), (17, 9, 128)])
def test_tensor_core_update_matches_reference(gpu, prec, shape):
    import torch

    from algebra_linear_b200 import device, mixed

    M, N, K = shape
    if prec != "bf16" and K % 32 or prec == "bf16" and K % 64:
        pytest.skip("K must be whole slices")
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.rand((K, M), generator=g, device="cuda") * 2 - 1      # storage of a column-major M x K
    B = torch.rand((N, K), generator=g, device="cuda") * 2 - 1      # storage of a column-major K x N
    C0 = torch.rand((N, M), generator=g, device="cuda") * 2 - 1     # storage of a column-major M x N
    C = C0.clone()
    with device.Context() as ctx:
        rc = gpu.alg_gemm_tc_sub_dev(ctx.handle, mixed.PRECISIONS[prec], M, N, K, A.data_ptr(), M, B.data_ptr(),
                                     K, C.data_ptr(), M)
        assert rc == 0, rc
    if prec == "tf32x3":
        # split operands: FP32-level accuracy against the unrounded product
        # (the dropped lo*lo term and FP32 accumulation: (K + 4) 2^-22 relative)
        Am, Bm = A.t().double(), B.t().double()
        bound = (K + 4) * 2.0**-22
    else:
        rnd = _round_bf16 if prec == "bf16" else _round_tf32
        Am = rnd(A).t().double()      # M x K
        Bm = rnd(B).t().double()      # K x N
        bound = 1e-4
    ref = C0.t().double() - Am @ Bm
    err = (C.t().double() - ref).abs().max().item()
    scale = (Am.abs() @ Bm.abs()).max().item()
    assert err <= bound * scale, (err, scale)
    if prec == "tf32x3":
        # and clearly better than plain TF32 (10-bit mantissa, about 5e-4)
        assert err <= 1e-5 * scale, (err, scale)


@pytest.mark.parametrize("pivoting", ["partial", "tournament"])
@pytest.mark.parametrize("prec", ["fp32", "tf32", "tf32x3", "bf16"])
def test_mixed_solve_reaches_fp64_backward_error(gpu, oracle, prec, pivoting):
    import torch

    from algebra_linear_b200 import device, mixed

    n = 1536
    a, x_true, b = oracle.c1_system(n, seed=[7, 7, 7, 9])
    ra, rb = a.copy(), b.copy()
    rc, _ = oracle.dgesv(ra, rb, n)
    assert rc == 0
    with device.Context() as ctx:
        A = torch.from_numpy(a.copy()).cuda()
        B = torch.from_numpy(b.copy()).cuda()
        rep = mixed.dgesv_mixed_dev(ctx, A, B, n, 1, precision=prec, pivoting=pivoting)
        x = B.cpu().numpy()
        assert np.array_equal(A.cpu().numpy(), a), "A must be unchanged on the refinement path"
    assert rep["path"] in ("ir", "gmres"), rep
    assert rep["butterfly"] == (pivoting == "rbt"), rep
    eta = oracle.backward_error(a, x, b, n)
    assert eta <= 10 * n * 2.0**-53, (eta, rep)
    # same solution as the FP64 reference to the accuracy the conditioning
    # allows: forward error <= cond_inf(A) * eta with both solutions at the
    # FP64 backward-error level (cond_inf from numpy's inverse, n = 1536)
    Am = a.reshape(n, n).T
    cond = np.abs(Am).sum(axis=1).max() * np.abs(np.linalg.inv(Am)).sum(axis=1).max()
    fwd = np.max(np.abs(x - rb)) / np.max(np.abs(rb))
    assert fwd <= 2 * cond * 10 * n * 2.0**-53, (fwd, cond)


def test_mixed_host_api_keeps_a(gpu, oracle):
    from algebra_linear_b200 import _lib, mixed

    n = 700
    a, _, b = oracle.c1_system(n, seed=[1, 2, 3, 5])
    ha, hb = a.copy(), b.copy()
    rc = mixed.dgesv_mixed_host(ha.ctypes.data, hb.ctypes.data, n, 1, precision="bf16")
    assert rc == 0, _lib.status_string(rc)
    assert np.array_equal(ha, a)
    assert oracle.backward_error(a, hb, b, n) <= 10 * n * 2.0**-53


def test_mixed_64_rhs(gpu, oracle):
    """64 right-hand sides (the C2 multi-RHS case) through the butterfly form."""
    import torch

    from algebra_linear_b200 import device, mixed

    n, nrhs = 1024, 64
    a, s = oracle.larnv("Symmetric", [4, 4, 4, 5], n * n)
    b, _ = oracle.larnv("Symmetric", s, n * nrhs)
    with device.Context() as ctx:
        A = torch.from_numpy(a.copy()).cuda()
        B = torch.from_numpy(b.copy()).cuda()
        rep = mixed.dgesv_mixed_dev(ctx, A, B, n, nrhs, precision="tf32")
        x = B.cpu().numpy()
    assert rep["path"] in ("ir", "gmres"), rep
    for k in range(nrhs):
        eta = oracle.backward_error(a, x[k * n:(k + 1) * n], b[k * n:(k + 1) * n], n)
        assert eta <= 10 * n * 2.0**-53, (k, eta)


@pytest.mark.parametrize("n,nrhs", [(3001, 17), (1300, 100)])
def test_mixed_many_rhs_odd_orders(gpu, oracle, n, nrhs):
    """From 16 right-hand sides the FP32 solves are blocked (a short last
    128-row block here) and the refinement's residual is one FP64
    tensor-core GEMM: every column reaches the FP64 backward error."""
    import torch

    from algebra_linear_b200 import device, mixed

    a, s = oracle.larnv("Symmetric", [6, 1, 8, 2 * n + 1], n * n)
    b, _ = oracle.larnv("Symmetric", s, n * nrhs)
    with device.Context() as ctx:
        A = torch.from_numpy(a.copy()).cuda()
        B = torch.from_numpy(b.copy()).cuda()
        rep = mixed.dgesv_mixed_dev(ctx, A, B, n, nrhs, precision="tf32x3", no_fallback=True)
        x = B.cpu().numpy()
    assert rep["path"] in ("ir", "gmres"), rep
    for k in range(nrhs):
        eta = oracle.backward_error(a, x[k * n:(k + 1) * n], b[k * n:(k + 1) * n], n)
        assert eta <= 10 * n * 2.0**-53, (k, eta)


def test_butterfly_form_on_a_diagonally_dominant_system(gpu, oracle):
    """The butterfly + no-pivoting form on A + n I (where LU without pivoting
    is stable), refined to the FP64 backward error; A is left unchanged."""
    import torch

    from algebra_linear_b200 import device, mixed

    n = 1024
    a, s = oracle.larnv("Symmetric", [8, 8, 8, 9], n * n)
    a[:: n + 1] += n
    xt, _ = oracle.larnv("Symmetric", s, n)
    b = oracle.dgemv(a, xt, n, n)
    with device.Context() as ctx:
        A = torch.from_numpy(a.copy()).cuda()
        B = torch.from_numpy(b.copy()).cuda()
        rep = mixed.dgesv_mixed_dev(ctx, A, B, n, 1, precision="bf16", pivoting="rbt")
        x = B.cpu().numpy()
        assert np.array_equal(A.cpu().numpy(), a)
    assert rep["butterfly"] and rep["path"] in ("ir", "gmres"), rep
    assert oracle.backward_error(a, x, b, n) <= 10 * n * 2.0**-53


@pytest.mark.parametrize("n", [1536, 5000])
@pytest.mark.parametrize("prec", ["fp32", "tf32x3"])
def test_tournament_pivoting_panels(gpu, oracle, n, prec):
    """Tournament-pivoting leaf panels: the FP32 LU stays a good
    preconditioner (plain refinement, few steps) and x reaches the FP64
    backward error; n = 5000 takes two merge levels."""
    import torch

    from algebra_linear_b200 import device, mixed

    a, _, b = oracle.c1_system(n, seed=[3, 1, 4, 1])
    with device.Context() as ctx:
        A = torch.from_numpy(a.copy()).cuda()
        B = torch.from_numpy(b.copy()).cuda()
        rep = mixed.dgesv_mixed_dev(ctx, A, B, n, 1, precision=prec, pivoting="tournament", no_gmres=True,
                                    no_fallback=True)
        assert rep["tournament"], rep
        x = B.cpu().numpy()
        assert np.array_equal(A.cpu().numpy(), a)
    assert rep["path"] == "ir" and rep["ir_iterations"] <= 8, rep
    assert oracle.backward_error(a, x, b, n) <= 10 * n * 2.0**-53


def test_block_widths_past_the_swap_limit_are_cut(gpu, oracle, monkeypatch):
    """A block's interchanges move up to 2 nb rows and the deferred-swap
    kernel holds 512, so a requested block width over 256 (ALG_NB,
    ALG_NB_TC) is cut to 256: the exact form stays bit-identical to the
    oracle and the mixed form converges by plain refinement."""
    import torch

    from algebra_linear_b200 import device, mixed
    from algebra_linear_b200.lapack import dgetrf

    n = 2048
    a, _, b = oracle.c1_system(n, seed=[4, 4, 2, 7])
    monkeypatch.setenv("ALG_NB", "384")
    g = a.copy()
    ipiv, _ = dgetrf(g, n)
    ref = a.copy()
    rc, ripiv, _, _ = oracle.dgetrf(ref, n)
    assert rc == 0 and ipiv == ripiv and np.array_equal(g.view(np.uint64), ref.view(np.uint64))
    monkeypatch.setenv("ALG_NB_TC", "320")
    with device.Context() as ctx:
        A = torch.from_numpy(a.copy()).cuda()
        B = torch.from_numpy(b.copy()).cuda()
        rep = mixed.dgesv_mixed_dev(ctx, A, B, n, 1, precision="tf32x3", pivoting="tournament", no_gmres=True,
                                    no_fallback=True)
        x = B.cpu().numpy()
    assert rep["path"] == "ir", rep
    assert oracle.backward_error(a, x, b, n) <= 10 * n * 2.0**-53


def test_tournament_single_launch_matches_level_launches(gpu, oracle, monkeypatch):
    """The single cooperative launch per leaf and the one-launch-per-level
    form run the same arithmetic: bit-identical solutions."""
    import torch

    from algebra_linear_b200 import device, mixed

    n = 5000
    a, _, b = oracle.c1_system(n, seed=[2, 7, 1, 9])
    xs = []
    for split in ("0", "1"):
        if split == "1":
            monkeypatch.setenv("ALG_TSLU_SPLIT", "1")
        with device.Context() as ctx:
            A = torch.from_numpy(a.copy()).cuda()
            B = torch.from_numpy(b.copy()).cuda()
            rep = mixed.dgesv_mixed_dev(ctx, A, B, n, 1, precision="tf32x3", pivoting="tournament",
                                        no_gmres=True, no_fallback=True)
            assert rep["tournament"] and rep["path"] == "ir", rep
            xs.append(B.cpu().numpy())
    assert np.array_equal(xs[0], xs[1])


def _c2_system(ctx, n, nrhs, seed):
    """The dense workload at a C2 order, generated on the device by the
    reference's DLARNV stream: A iid U(-1,1) (no shift), x_true continuing
    the stream, b = A x_true."""
    A, s = ctx.larnv(2, seed, n * n)
    xt, _ = ctx.larnv(2, s, n * nrhs)
    b = (A.view(n, n).t() @ xt.view(nrhs, n).t()).t().contiguous().view(-1)
    return A.clone(), b


def _eta(A, x, b, n, nrhs):
    Am = A.view(n, n).t()
    X, B = x.view(nrhs, n).t(), b.view(nrhs, n).t()
    r = (B - Am @ X).abs().amax(dim=0)
    den = Am.abs().sum(dim=1).max() * X.abs().amax(dim=0) + B.abs().amax(dim=0)
    return float((r / den).max())


@pytest.mark.parametrize("nrhs", [1, 64])
def test_c2_order_mixed_forms_reach_fp64_backward_error(gpu, nrhs):
    """C2 at n = 8192: the TF32x3 and FP32 mixed forms (tournament pivoting,
    FP64 refinement) reach eta <= 10 n 2^-53, and their x agrees with the
    FP64 solution of the bit-exact GPU form (which reproduces the oracle's
    LU bit for bit, tests/test_dense_gpu.py) to within cond_inf(A) times
    that backward error. The FP64 refinement path, not the fallback, must
    deliver it."""
    import torch

    from algebra_linear_b200 import _lib, device, mixed

    n = 8192
    tol = 10 * n * 2.0**-53
    with device.Context() as ctx:
        A0, b0 = _c2_system(ctx, n, nrhs, [1988, 1989, 1990, 1991])
        A, x64 = A0.clone(), b0.clone()
        ctx.dgesv(A, x64, n, nrhs, update=_lib.UPDATE_EXACT)
        del A
        eta64 = _eta(A0, x64, b0, n, nrhs)
        assert eta64 <= tol, eta64
        Am = A0.view(n, n).t()
        cond = float(Am.abs().sum(dim=1).max() * torch.linalg.inv(Am).abs().sum(dim=1).max())
        for prec in ("tf32x3", "fp32"):
            x = b0.clone()
            rep = mixed.dgesv_mixed_dev(ctx, A0, x, n, nrhs, precision=prec, no_fallback=True)
            assert rep["path"] in ("ir", "gmres") and rep["tournament"], (prec, rep)
            eta = _eta(A0, x, b0, n, nrhs)
            assert eta <= tol, (prec, eta, rep)
            X, X64 = x.view(nrhs, n), x64.view(nrhs, n)
            fwd = float(((X - X64).abs().amax(dim=1) / X64.abs().amax(dim=1)).max())
            assert fwd <= 2 * cond * tol, (prec, fwd, cond)
            print(f"n={n} nrhs={nrhs} {prec}: eta {eta:.2e} (fp64 exact {eta64:.2e}), forward error vs the "
                  f"FP64 solution {fwd:.2e}, cond_inf {cond:.3g}, {rep}")
