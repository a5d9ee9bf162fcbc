"""Dense LU drop-ins with the reference's signatures and error behaviour.

Mirrors `algebra_linear::lapack` (src/lapack/mod.rs):

    dgetrf(a, n) -> (ipiv, det)            mod.rs:181-185
    dgetrf_rect(a, nrows, ncols, ipiv)     mod.rs:202-238
    dgesv(a, b)                            mod.rs:309-323
    zgetrf(a, n) -> ipiv                   complex.rs:67-124
    zgetrf_rect(a, nrows, ncols, ipiv)     complex.rs:169-208
    zgesv(a, b)                            complex.rs:279-312
    zgetri(lu, n, ipiv)                    complex.rs:217-271

`a` and `b` are 1-D float64 (complex128 for the z functions) numpy arrays
holding column-major data (`a[i + j*n]`), modified in place exactly as the
Rust slices are. Errors are
raised as LapackError with the reference's variant name. The arithmetic runs
on the GPU through libalgebra_linear_gpu.so; nothing here computes on the CPU.
"""

from __future__ import annotations

import numpy as np

from . import _lib


class LapackError(Exception):
    """lapack::LapackError (mod.rs:76-96): Singular, BadShape, Convergence,
    NotImplemented. GPU-side failures carry the library's own status name."""

    def __init__(self, kind: str, code: int | None = None):
        super().__init__(kind)
        self.kind = kind
        self.code = code

    def __eq__(self, other):
        return isinstance(other, LapackError) and other.kind == self.kind

    __hash__ = Exception.__hash__


_KINDS = {
    _lib.SINGULAR: "Singular",
    _lib.BAD_SHAPE: "BadShape",
    _lib.CONVERGENCE: "Convergence",
    _lib.NOT_IMPLEMENTED: "NotImplemented",
}


def _check(rc: int) -> None:
    if rc != _lib.OK:
        raise LapackError(_KINDS.get(rc, _lib.status_string(rc)), rc)


def _f64(a, name: str) -> np.ndarray:
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or a.ndim != 1 or not a.flags.c_contiguous:
        raise TypeError(f"{name} must be a contiguous 1-D float64 numpy array")
    return a


def dgetrf(a: np.ndarray, n: int):
    """LU with partial pivoting in place; returns (ipiv, det) (mod.rs:181)."""
    _f64(a, "a")
    if a.size != n * n:
        raise LapackError("BadShape", _lib.BAD_SHAPE)
    ipiv = np.zeros(n, dtype=np.uint64)
    det = np.zeros(1, dtype=np.float64)
    if n == 0:
        return [], 1.0
    _check(_lib.load().alg_dgetrf(_lib.ptr(a), n, _lib.ptr(ipiv), _lib.ptr(det)))
    return [int(v) for v in ipiv], float(det[0])


def dgetrf_rect(a: np.ndarray, nrows: int, ncols: int, ipiv) -> None:
    """LU of an nrows x ncols panel (nrows >= ncols), ipiv filled in place (mod.rs:202)."""
    _f64(a, "a")
    if nrows < ncols or a.size != nrows * ncols or len(ipiv) != ncols:
        raise LapackError("BadShape", _lib.BAD_SHAPE)
    if ncols == 0:
        return
    buf = np.zeros(ncols, dtype=np.uint64)
    _check(_lib.load().alg_dgetrf_rect(_lib.ptr(a), nrows, ncols, _lib.ptr(buf)))
    for k in range(ncols):
        ipiv[k] = int(buf[k])


def dgetri(lu: np.ndarray, n: int, ipiv) -> None:
    """Inverse from dgetrf's factors, in place (mod.rs:249-298)."""
    _f64(lu, "lu")
    if lu.size != n * n or len(ipiv) != n:
        raise LapackError("BadShape", _lib.BAD_SHAPE)
    if n == 0:
        return
    iv = np.ascontiguousarray(ipiv, dtype=np.uint64)
    _check(_lib.load().alg_dgetri(_lib.ptr(lu), n, _lib.ptr(iv)))


def dgesv(a: np.ndarray, b: np.ndarray) -> None:
    """Solves A x = b for one right-hand side; n = len(b) (mod.rs:309)."""
    _f64(a, "a")
    _f64(b, "b")
    n = b.size
    if a.size != n * n:
        raise LapackError("BadShape", _lib.BAD_SHAPE)
    if n == 0:
        return
    _check(_lib.load().alg_dgesv(_lib.ptr(a), _lib.ptr(b), n))


def _c128(a, name: str) -> np.ndarray:
    if not isinstance(a, np.ndarray) or a.dtype != np.complex128 or a.ndim != 1 or not a.flags.c_contiguous:
        raise TypeError(f"{name} must be a contiguous 1-D complex128 numpy array")
    return a


def zgetrf(a: np.ndarray, n: int):
    """Complex LU with partial pivoting in place; returns ipiv (complex.rs:67)."""
    _c128(a, "a")
    if a.size != n * n:
        raise LapackError("BadShape", _lib.BAD_SHAPE)
    if n == 0:
        return []
    ipiv = np.zeros(n, dtype=np.uint64)
    _check(_lib.load().alg_zgetrf(_lib.ptr(a), n, _lib.ptr(ipiv)))
    return [int(v) for v in ipiv]


def zgetrf_rect(a: np.ndarray, nrows: int, ncols: int, ipiv) -> None:
    """Complex LU of an nrows x ncols panel, ipiv filled in place (complex.rs:169)."""
    _c128(a, "a")
    if nrows < ncols or a.size != nrows * ncols or len(ipiv) != ncols:
        raise LapackError("BadShape", _lib.BAD_SHAPE)
    if ncols == 0:
        return
    buf = np.zeros(ncols, dtype=np.uint64)
    _check(_lib.load().alg_zgetrf_rect(_lib.ptr(a), nrows, ncols, _lib.ptr(buf)))
    for k in range(ncols):
        ipiv[k] = int(buf[k])


def zgesv(a: np.ndarray, b: np.ndarray) -> None:
    """Solves A x = b for one complex right-hand side; n = len(b) (complex.rs:279)."""
    _c128(a, "a")
    _c128(b, "b")
    n = b.size
    if a.size != n * n:
        raise LapackError("BadShape", _lib.BAD_SHAPE)
    if n == 0:
        return
    _check(_lib.load().alg_zgesv(_lib.ptr(a), _lib.ptr(b), n))


def zgetri(lu: np.ndarray, n: int, ipiv) -> None:
    """Complex inverse from zgetrf's factors, in place (complex.rs:217)."""
    _c128(lu, "lu")
    if lu.size != n * n or len(ipiv) != n:
        raise LapackError("BadShape", _lib.BAD_SHAPE)
    if n == 0:
        return
    iv = np.ascontiguousarray(ipiv, dtype=np.uint64)
    _check(_lib.load().alg_zgetri(_lib.ptr(lu), n, _lib.ptr(iv)))


def dgesv_nrhs(a: np.ndarray, b: np.ndarray, n: int, nrhs: int, update: int = _lib.UPDATE_EXACT):
    """dgesv with nrhs columns in b (n x nrhs column-major). Returns ipiv."""
    _f64(a, "a")
    _f64(b, "b")
    if a.size != n * n or b.size != n * nrhs:
        raise LapackError("BadShape", _lib.BAD_SHAPE)
    ipiv = np.zeros(max(n, 1), dtype=np.uint64)
    if n == 0:
        return []
    _check(_lib.load().alg_dgesv_ex(update, _lib.ptr(a), _lib.ptr(b), n, nrhs, _lib.ptr(ipiv)))
    return [int(v) for v in ipiv[:n]]
