"""ORACLE — test infrastructure only: ctypes wrapper of oracle_complex.cpp,
the C++ restatement of src/lapack/complex.rs (zgetrf, zgetrf_rect, zgesv, zgetri) with
num-complex 0.4's operator formulas. Matrices are numpy complex128,
column-major (`a[i + j * n]`), as the reference stores them.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from oracle import dense as _dense

OK, SINGULAR, BAD_SHAPE = 0, 1, 2

_bound = False


def _lib() -> C.CDLL:
    global _bound
    lib = _dense.load()
    if not _bound:
        P, SZ = C.c_void_p, C.c_size_t
        lib.oracle_zgetrf.argtypes = [P, SZ, P]
        lib.oracle_zgetrf_rect.argtypes = [P, SZ, SZ, P]
        lib.oracle_zgesv.argtypes = [P, P, SZ, P]
        lib.oracle_zgetri.argtypes = [P, SZ, P]
        _bound = True
    return lib


def _cm(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a.copy()


def zgetrf(a, n: int):
    """complex.rs:67-124. Returns (status, lu, ipiv) on a copy of `a`
    (flat column-major, n*n entries); on Singular, `lu` is the partial state."""
    lu = _cm(a)
    if lu.size != n * n:
        return BAD_SHAPE, lu, np.zeros(0, dtype=np.uintp)
    ipiv = np.zeros(max(n, 1), dtype=np.uintp)
    rc = _lib().oracle_zgetrf(lu.ctypes.data, n, ipiv.ctypes.data)
    return rc, lu, ipiv[:n]


def zgetrf_rect(a, nrows: int, ncols: int):
    """complex.rs:169-208. Returns (status, lu, ipiv)."""
    lu = _cm(a)
    if nrows < ncols or lu.size != nrows * ncols:
        return BAD_SHAPE, lu, np.zeros(0, dtype=np.uintp)
    ipiv = np.zeros(max(ncols, 1), dtype=np.uintp)
    rc = _lib().oracle_zgetrf_rect(lu.ctypes.data, nrows, ncols, ipiv.ctypes.data)
    return rc, lu, ipiv[:ncols]


def zgesv(a, b):
    """complex.rs:279-312. Returns (status, lu, x, ipiv); n = len(b)."""
    x = _cm(b)
    n = x.size
    lu = _cm(a)
    if lu.size != n * n:
        return BAD_SHAPE, lu, x, np.zeros(0, dtype=np.uintp)
    ipiv = np.zeros(max(n, 1), dtype=np.uintp)
    rc = _lib().oracle_zgesv(lu.ctypes.data, x.ctypes.data, n, ipiv.ctypes.data)
    return rc, lu, x, ipiv[:n]


def zgetri(lu, n: int, ipiv):
    """complex.rs:217-271 on a copy of the factors; returns (status, inverse)."""
    inv = _cm(lu)
    iv = np.ascontiguousarray(ipiv, dtype=np.uintp)
    if inv.size != n * n or iv.size != n:
        return BAD_SHAPE, inv
    rc = _lib().oracle_zgetri(inv.ctypes.data, n, iv.ctypes.data if n else None)
    return rc, inv


def complex_sample(n: int) -> np.ndarray:
    """src/parity.rs:76-90: the deterministic complex test matrix (flat column-major)."""
    a = np.zeros(n * n, dtype=np.complex128)
    for i in range(n):
        for j in range(n):
            re = (n + 2.0 + i * 0.5) if i == j else float((i * 5 + j * 7) % 9) - 4.0
            im = float((i * 3 + j * 11) % 7) - 3.0 + (1.0 if i == j else 0.0)
            a[i + j * n] = complex(re, im)
    return a


def general3() -> np.ndarray:
    """src/lapack/complex.rs:438-452 (flat column-major)."""
    return np.array([4 + 1j, 1 + 3j, 2 - 1j, 1 - 2j, 3 + 0j, 1 + 1j, 2 + 0j, -1j, 5 + 2j], dtype=np.complex128)
