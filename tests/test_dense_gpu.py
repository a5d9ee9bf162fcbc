"""GPU parity of the dense LU path against the oracle, through the C ABI.

Tolerances (the spec's FP64 bar): identical pivot sequence and x within
1e-12 relative. The exact-update form is held to more: the packed LU factors,
pivots and determinant must be bit-identical to the reference's kij loop.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12
SEEDY = [1988, 1989, 1990, 1991]


def rel_err(x, ref):
    return float(np.max(np.abs(x - ref)) / max(np.max(np.abs(ref)), 1e-300))


def same_bits(x, y):
    return np.array_equal(x.view(np.uint64), y.view(np.uint64))


# ---- the reference's own unit tests, through the GPU drop-ins ---------------

def test_reference_unit_cases_on_gpu(gpu, oracle):
    from algebra_linear_b200.lapack import LapackError, dgesv, dgetrf, dgetrf_rect

    from tests.test_oracle_kat import cofactor_det4, reconstruct_panel, sample4

    a = sample4()
    ipiv, det = dgetrf(a, 4)
    assert abs(det - cofactor_det4()) < 1e-12  # mod.rs:483-495
    ref = sample4()
    _, ripiv, rdet, _ = oracle.dgetrf(ref, 4)
    assert ipiv == ripiv and det == rdet and same_bits(a, ref)

    with pytest.raises(LapackError) as e:  # mod.rs:497-502
        dgetrf(np.array([1.0, 2.0, 3.0, 2.0, 4.0, 6.0, 1.0, 1.0, 1.0]), 3)
    assert e.value.kind == "Singular"

    a = sample4()  # mod.rs:537-551
    x_true = np.array([1.0, -2.0, 3.0, 5.0])
    b = oracle.dgemv(a, x_true, 4, 4)
    dgesv(a, b)
    assert np.all(np.abs(b - x_true) < 1e-12)

    with pytest.raises(LapackError) as e:  # mod.rs:553-558
        dgesv(np.array([1.0, 2.0, 3.0, 2.0, 4.0, 6.0, 1.0, 1.0, 1.0]), np.ones(3))
    assert e.value.kind == "Singular"

    a = np.array([1e-16, 0.0, 0.0, 1.0])  # mod.rs:670-683
    ipiv, det = dgetrf(a, 2)
    assert len(ipiv) == 2 and abs(det) < 1e-15
    with pytest.raises(LapackError) as e:
        dgetrf(np.array([1.0, 2.0, 2.0, 4.0]), 2)
    assert e.value.kind == "Singular"

    nrows, ncols = 5, 3  # mod.rs:723-733
    a0 = np.array([1.0, 5.0, 2.0, 3.0, 4.0, 2.0, -1.0, 6.0, 0.0, 1.0, 3.0, 2.0, 1.0, 7.0, -2.0])
    a = a0.copy()
    piv = [0] * ncols
    dgetrf_rect(a, nrows, ncols, piv)
    pa, lu = reconstruct_panel(nrows, ncols, a0, a, piv)
    assert np.all(np.abs(pa - lu) < 1e-12) and piv[0] == 1

    with pytest.raises(LapackError) as e:  # mod.rs:743-744
        dgetrf_rect(np.array([0.0, 0.0, 2.0, 3.0]), 2, 2, [0, 0])
    assert e.value.kind == "Singular"


# ---- bit-exact factors on the larnv workload --------------------------------

SIZES = [1, 2, 3, 5, 15, 16, 17, 31, 33, 63, 64, 65, 100, 127, 129, 200, 257, 513, 1024]


@pytest.mark.parametrize("n", SIZES)
def test_dgetrf_is_bit_identical_to_the_reference(gpu, oracle, n):
    from algebra_linear_b200.lapack import dgetrf

    a0, _ = oracle.larnv("Symmetric", [11, 23, 37, 2 * n + 1], n * n)
    a = a0.copy()
    ipiv, det = dgetrf(a, n)
    ref = a0.copy()
    rc, ripiv, rdet, _ = oracle.dgetrf(ref, n)
    assert rc == 0
    assert ipiv == ripiv
    assert same_bits(a, ref), f"max diff {np.max(np.abs(a - ref))}"
    assert same_bits(np.array([det]), np.array([rdet]))


def test_dgetrf_two_cluster_panel_bit_identical(gpu, oracle):
    """n = 2048 makes the leaf panel span a 2-CTA cluster (rows > one CTA's
    shared memory)."""
    from algebra_linear_b200.lapack import dgetrf

    n = 2048
    a0, _ = oracle.larnv("Symmetric", SEEDY, n * n)
    a = a0.copy()
    ipiv, _ = dgetrf(a, n)
    ref = a0.copy()
    rc, ripiv, _, _ = oracle.dgetrf(ref, n)
    assert rc == 0 and ipiv == ripiv and same_bits(a, ref)


@pytest.mark.parametrize("shape", [(5, 3), (7, 7), (40, 17), (100, 64), (300, 129), (1000, 33), (513, 200)])
def test_dgetrf_rect_is_bit_identical(gpu, oracle, shape):
    from algebra_linear_b200.lapack import dgetrf_rect

    nrows, ncols = shape
    a0, _ = oracle.larnv("Symmetric", [5, 6, 7, 2 * ncols + 1], nrows * ncols)
    a = a0.copy()
    piv = [0] * ncols
    dgetrf_rect(a, nrows, ncols, piv)
    ref = a0.copy()
    rc, rpiv = oracle.dgetrf_rect(ref, nrows, ncols)
    assert rc == 0 and piv == rpiv and same_bits(a, ref)


# ---- the C1 configuration: n = 1024, one RHS ---------------------------------

@pytest.mark.parametrize("update", [0, 1], ids=["exact", "fma"])
def test_c1_dgesv_parity(gpu, oracle, update):
    from algebra_linear_b200.lapack import dgesv_nrhs

    n = 1024
    a, x_true, b = oracle.c1_system(n)
    ra, rb = a.copy(), b.copy()
    rc, ripiv = oracle.dgesv(ra, rb, n)
    assert rc == 0
    ga, gb = a.copy(), b.copy()
    ipiv = dgesv_nrhs(ga, gb, n, 1, update=update)
    assert ipiv == ripiv  # identical pivot sequence
    assert rel_err(gb, rb) <= REL_TOL
    if update == 0:
        assert same_bits(ga, ra)  # bit-identical factors
    assert oracle.backward_error(a, gb, b, n) < 10 * n * 2.0**-53


def test_dgesv_64_rhs_matches_dgetrs_per_column(gpu, oracle):
    from algebra_linear_b200.lapack import dgesv_nrhs

    n, nrhs = 300, 64
    a0, s = oracle.larnv("Symmetric", SEEDY, n * n)
    b0, _ = oracle.larnv("Symmetric", s, n * nrhs)
    ra, rb = a0.copy(), b0.copy()
    rc, ripiv = oracle.dgesv(ra, rb, n, nrhs)
    assert rc == 0
    ga, gb = a0.copy(), b0.copy()
    ipiv = dgesv_nrhs(ga, gb, n, nrhs)
    assert ipiv == ripiv
    assert rel_err(gb, rb) <= REL_TOL


@pytest.mark.parametrize("n,nrhs", [(300, 64), (777, 16), (129, 200), (1000, 33)])
def test_fused_many_rhs_blocked_solve(gpu, oracle, n, nrhs):
    """From 16 right-hand sides the fused form solves blocked (128-row
    triangles in registers, the rest by GEMMs): same pivots as the
    reference, each column's backward error within 10 n 2^-53 and x within
    1e-10 of the oracle's per-column dgetrs (another summation order)."""
    from algebra_linear_b200.lapack import dgesv_nrhs

    a0, s = oracle.larnv("Symmetric", [5, 6, 7, 2 * n + 1], n * n)
    b0, _ = oracle.larnv("Symmetric", s, n * nrhs)
    ra, rb = a0.copy(), b0.copy()
    rc, ripiv = oracle.dgesv(ra, rb, n, nrhs)
    assert rc == 0
    ga, gb = a0.copy(), b0.copy()
    ipiv = dgesv_nrhs(ga, gb, n, nrhs, update=1)
    assert ipiv == ripiv
    assert rel_err(gb, rb) <= 1e-10
    for c in range(0, nrhs, max(1, nrhs // 4)):
        col = slice(c * n, (c + 1) * n)
        assert oracle.backward_error(a0, gb[col].copy(), b0[col].copy(), n) < 10 * n * 2.0**-53


def test_forward_sweep_is_exact_and_solution_close(gpu, oracle):
    """Odd sizes across several solve blocks (64 rows each)."""
    from algebra_linear_b200.lapack import dgesv

    for n in [1, 7, 64, 65, 130, 777]:
        a, _, b = oracle.c1_system(n, seed=[3, 1, 4, 2 * n + 1])
        ra, rb = a.copy(), b.copy()
        oracle.dgesv(ra, rb, n)
        ga, gb = a.copy(), b.copy()
        dgesv(ga, gb)
        assert rel_err(gb, rb) <= REL_TOL, n


# ---- edge cases ---------------------------------------------------------------

def test_nan_and_inf_follow_the_reference_pivot_rule(gpu, oracle):
    """A NaN below the diagonal is never chosen; a NaN on the diagonal keeps
    the pivot in place (strict '>' scan seeded with |a_kk|, mod.rs:123-134)."""
    from algebra_linear_b200.lapack import dgetrf

    n = 40
    for case in range(4):
        a0, _ = oracle.larnv("Symmetric", [9, 9, 9, 2 * case + 1], n * n)
        if case == 0:
            a0[5 + 3 * n] = np.nan          # below the diagonal in column 3
        elif case == 1:
            a0[3 + 3 * n] = np.nan          # on the diagonal
        elif case == 2:
            a0[17 + 0 * n] = np.inf         # an infinite candidate
        else:
            a0[0:n] = 0.0
            a0[n - 1] = np.nan              # column 0 all zero but one NaN
        a = a0.copy()
        try:
            ipiv, _ = dgetrf(a, n)
            grc = 0
        except Exception as e:  # noqa: BLE001
            grc, ipiv = getattr(e, "code", -1), None
        ref = a0.copy()
        rc, ripiv, _, _ = oracle.dgetrf(ref, n)
        assert grc == rc, case
        if rc == 0:
            assert ipiv == ripiv, case
            assert np.array_equal(np.isnan(a), np.isnan(ref)), case
            fin = ~np.isnan(ref)
            assert same_bits(a[fin], ref[fin]), case


def test_exactly_singular_large_matrix(gpu, oracle):
    """A repeated column makes the reference's pivot exactly zero somewhere;
    the GPU reports Singular in the same case (and not otherwise)."""
    from algebra_linear_b200.lapack import LapackError, dgetrf

    n = 96
    a0, _ = oracle.larnv("Symmetric", SEEDY, n * n)
    a0[70 * n:71 * n] = 2.0 * a0[10 * n:11 * n]
    ref = a0.copy()
    rc, *_ = oracle.dgetrf(ref, n)
    a = a0.copy()
    if rc == 1:
        with pytest.raises(LapackError):
            dgetrf(a, n)
    else:
        ipiv, _ = dgetrf(a, n)
        assert same_bits(a, ref)


def test_repeat_runs_are_bitwise_deterministic(gpu, oracle):
    from algebra_linear_b200.lapack import dgesv_nrhs

    n = 700
    a, _, b = oracle.c1_system(n)
    outs = []
    for _ in range(2):
        ga, gb = a.copy(), b.copy()
        dgesv_nrhs(ga, gb, n, 1, update=1)
        outs.append((ga, gb))
    assert same_bits(outs[0][0], outs[1][0]) and same_bits(outs[0][1], outs[1][1])


def test_device_api_matches_host_api(gpu, oracle):
    import torch

    from algebra_linear_b200 import device

    n = 333
    a, _, b = oracle.c1_system(n)
    ra, rb = a.copy(), b.copy()
    oracle.dgesv(ra, rb, n)
    with device.Context() as ctx:
        da = torch.from_numpy(a.copy()).cuda()  # column-major n*n
        db = torch.from_numpy(b.copy()).cuda()
        ipiv = ctx.dgesv(da, db, n)
        assert ipiv.tolist() == oracle.dgesv(a.copy(), b.copy(), n)[1]
        assert rel_err(db.cpu().numpy(), rb) <= REL_TOL


def test_device_larnv_matches_the_reference_stream(gpu, oracle):
    """The device generator reproduces the oracle's larnv bit for bit,
    including the seed it leaves, across batch boundaries."""
    import torch

    from algebra_linear_b200 import device

    with device.Context() as ctx:
        for dist, name in [(1, "Uniform"), (2, "Symmetric")]:
            for n in [1, 63, 64, 65, 200, 4096 + 17]:
                x, s = ctx.larnv(dist, SEEDY, n)
                torch.cuda.synchronize()
                ref, rs = oracle.larnv(name, SEEDY, n)
                assert same_bits(x.cpu().numpy(), ref), (name, n)
                assert s == rs, (name, n)


@pytest.mark.parametrize("shape", [(128, 128, 16), (300, 500, 64), (4032, 4032, 64), (17, 9, 5), (1000, 33, 130)])
def test_fp64_tensor_core_update_matches_torch(gpu, shape):
    """The fused FP64 update on the FP64 tensor cores (mma.sync m8n8k4):
    C - A B against torch's FP64 product, to a few ulps of |A| |B|, with
    leading dimensions larger than the rows (sub-blocks of a front)."""
    import torch

    from algebra_linear_b200 import device

    M, N, K = shape
    lda, ldb, ldc = M + 3, K + 1, M + 5
    g = torch.Generator(device="cuda").manual_seed(M + 7 * N + 11 * K)
    A = torch.rand((K, lda), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    B = torch.rand((N, ldb), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    C0 = torch.rand((N, ldc), generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    C = C0.clone()
    with device.Context() as ctx:
        rc = gpu.alg_gemm_dmma_sub_dev(ctx.handle, M, N, K, A.data_ptr(), lda, B.data_ptr(), ldb, C.data_ptr(), ldc)
        assert rc == 0, rc
    Am, Bm = A[:, :M].t(), B[:, :K].t()
    ref = C0[:, :M].t() - Am @ Bm
    err = (C[:, :M].t() - ref).abs().max().item()
    scale = (Am.abs() @ Bm.abs()).max().item()
    assert err <= 4 * K * 2.0**-53 * scale, (err, scale)
    # padding rows between the leading dimension and M are untouched
    assert torch.equal(C[:, M:], C0[:, M:])


@pytest.mark.parametrize("n", [1, 2, 5, 64, 333, 1024])
def test_dgetri_is_bit_identical_to_the_oracle(gpu, oracle, n):
    """dgetri (mod.rs:249-298) on the GPU from the same factors: the inverse
    equals the oracle's bit for bit (same interchange, row-dot and division
    order per column)."""
    from algebra_linear_b200 import lapack

    a, _ = oracle.larnv("Symmetric", [5, 6, 7, 2 * n + 1], n * n)
    lu = a.copy()
    rc, ipiv, _, _ = oracle.dgetrf(lu, n)
    assert rc == 0
    ref = lu.copy()
    assert oracle.dgetri(ref, n, ipiv) == 0
    got = lu.copy()
    lapack.dgetri(got, n, ipiv)
    assert np.array_equal(got, ref)


def test_dgetri_rejects_zero_pivots_and_bad_shapes(gpu):
    from algebra_linear_b200 import lapack
    from algebra_linear_b200.lapack import LapackError

    lu = np.array([2.0, 0.5, 1.0, 0.0])  # U = [[2, 1], [0, 0]]
    before = lu.copy()
    with pytest.raises(LapackError) as e:
        lapack.dgetri(lu, 2, [0, 1])
    assert e.value.kind == "Singular" and np.array_equal(lu, before)
    with pytest.raises(LapackError):
        lapack.dgetri(np.zeros(4), 2, [0])
    with pytest.raises(LapackError):
        lapack.dgetri(np.eye(2).reshape(-1), 2, [0, 5])


def test_dgetri_device_form_matches_the_host_form(gpu, oracle):
    import ctypes as C

    import torch

    from algebra_linear_b200 import _lib, device

    n = 200
    a, _ = oracle.larnv("Symmetric", [3, 3, 3, 3], n * n)
    with device.Context() as ctx:
        A = torch.from_numpy(a.copy()).cuda()
        perm = torch.zeros(n, dtype=torch.int32, device="cuda")
        lib = _lib.load()
        assert lib.alg_dgetrf_dev(ctx.handle, _lib.UPDATE_EXACT, A.data_ptr(), n, n, None, perm.data_ptr()) == 0
        assert lib.alg_dgetri_dev(ctx.handle, A.data_ptr(), n, n, perm.data_ptr()) == 0
        inv = A.cpu().numpy()
    lu = a.copy()
    rc, ipiv, _, _ = oracle.dgetrf(lu, n)
    assert oracle.dgetri(lu, n, ipiv) == 0
    assert np.array_equal(inv, lu)
