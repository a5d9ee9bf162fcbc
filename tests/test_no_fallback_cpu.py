"""No CPU fallback: on a host without a CUDA device every compute entry point
of the library answers ALG_NO_DEVICE (204) and leaves its inputs as they
were, the Python layer raises, and a missing shared object makes the loader
raise instead of computing anything some other way. Nothing here needs a GPU."""

import ctypes as C

import numpy as np
import pytest

from algebra_linear_b200 import _lib


def _no_device() -> bool:
    import torch

    return not torch.cuda.is_available()


pytestmark = pytest.mark.skipif(not _no_device(), reason="a CUDA device is present: the GPU tests cover this host")


def test_dense_entry_points_report_no_device_and_touch_nothing():
    lib = _lib.load()
    a0 = np.array([4.0, 1.0, 2.0, 1.0, 3.0, 0.0, 2.0, 0.0, 5.0])  # column-major 3 x 3
    b0 = np.array([1.0, 2.0, 3.0])
    a, b = a0.copy(), b0.copy()
    ipiv = np.full(3, 7, dtype=np.uint64)
    det = C.c_double(-9.0)
    assert lib.alg_dgesv(a.ctypes.data, b.ctypes.data, 3) == _lib.NO_DEVICE
    assert lib.alg_dgesv_nrhs(a.ctypes.data, b.ctypes.data, 3, 1) == _lib.NO_DEVICE
    assert lib.alg_dgesv_ex(_lib.UPDATE_FMA, a.ctypes.data, b.ctypes.data, 3, 1, ipiv.ctypes.data) == _lib.NO_DEVICE
    assert lib.alg_dgetrf(a.ctypes.data, 3, ipiv.ctypes.data, C.byref(det)) == _lib.NO_DEVICE
    assert lib.alg_dgetrf_rect(a.ctypes.data, 3, 3, ipiv.ctypes.data) == _lib.NO_DEVICE
    assert (ipiv == 7).all() and det.value == -9.0
    # (dgetri rejects pivots outside 0..n-1 before any device work, where the
    # reference's swap would panic on them, so it is given valid ones)
    perm = np.arange(3, dtype=np.uint64)
    assert lib.alg_dgetri(a.ctypes.data, 3, perm.ctypes.data) == _lib.NO_DEVICE
    assert np.array_equal(a, a0) and np.array_equal(b, b0)


def test_complex_and_mixed_entry_points_report_no_device():
    lib = _lib.load()
    z0 = np.array([4.0, 1.0, 1.0, 0.0, 1.0, -1.0, 3.0, 2.0])  # interleaved 2 x 2
    w0 = np.array([1.0, 0.0, 2.0, 1.0])
    z, w = z0.copy(), w0.copy()
    ipiv = np.zeros(2, dtype=np.uint64)
    assert lib.alg_zgesv(z.ctypes.data, w.ctypes.data, 2) == _lib.NO_DEVICE
    assert lib.alg_zgetrf(z.ctypes.data, 2, ipiv.ctypes.data) == _lib.NO_DEVICE
    assert lib.alg_zgetrf_rect(z.ctypes.data, 2, 2, ipiv.ctypes.data) == _lib.NO_DEVICE
    assert lib.alg_zgetri(z.ctypes.data, 2, ipiv.ctypes.data) == _lib.NO_DEVICE
    assert np.array_equal(z, z0) and np.array_equal(w, w0)
    from algebra_linear_b200 import mixed

    a, b = np.array([4.0, 1.0, 1.0, 3.0]), np.array([1.0, 2.0])
    assert mixed.dgesv_mixed_host(a.ctypes.data, b.ctypes.data, 2, 1, precision="tf32x3") == _lib.NO_DEVICE
    assert np.array_equal(b, [1.0, 2.0])
    # the allocation-free entry point's set-up call, and a context
    assert lib.alg_dgesv_mixed_noalloc(None, None, None, 0, None, None, None) == _lib.NO_DEVICE
    h = C.c_void_p()
    assert lib.alg_ctx_create(None, C.byref(h)) == _lib.NO_DEVICE
    srv = C.c_void_p()
    assert lib.alg_server_create(1, 1 << 20, 64, C.byref(srv)) == _lib.NO_DEVICE


def test_python_layer_raises_instead_of_computing():
    from algebra_linear_b200.lapack import LapackError, dgesv
    from algebra_linear_b200.sparse import LuMethod, SparseError, SparseLu

    a, b = np.array([4.0, 1.0, 1.0, 3.0]), np.array([1.0, 2.0])
    with pytest.raises(LapackError):
        dgesv(a, b)
    assert np.array_equal(b, [1.0, 2.0])
    # the symbolic analysis is host work and runs; the numeric factorization does not
    lu = SparseLu.analyze([0, 2, 4], [0, 1, 0, 1], LuMethod.supernodal())
    with pytest.raises(SparseError):
        lu.factorize([0, 2, 4], [0, 1, 0, 1], [4.0, 1.0, 1.0, 3.0])
    assert lu.stats() is None


def test_a_missing_library_raises(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "libalgebra_linear_gpu.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="missing"):
        _lib.load()
