"""ORACLE — test infrastructure only: ctypes wrapper of oracle_dense.cpp,
the C++ restatement of src/lapack/mod.rs (dgetrf, dgetrf_rect, dgetrs,
dgesv), src/lapack/families.rs (larnv) and the reference's checkers.
"""

from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None

DIST = {"Uniform": 1, "Symmetric": 2, "Normal": 3}


def build() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        srcs = list(HERE.glob("oracle_*.cpp"))
        if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
            build()
        lib = C.CDLL(str(LIB))
        P, SZ = C.c_void_p, C.c_size_t
        lib.oracle_larnv.argtypes = [C.c_int, P, SZ, P]
        lib.oracle_dgetrf.argtypes = [P, SZ, P, P, P]
        lib.oracle_dgetrf_range.argtypes = [P, SZ, SZ, SZ, P]
        lib.oracle_dgetrf_rect.argtypes = [P, SZ, SZ, P]
        lib.oracle_dgetrs.argtypes = [P, P, P, SZ, SZ]
        lib.oracle_dgesv.argtypes = [P, P, SZ, SZ, P]
        lib.oracle_dgetri.argtypes = [P, SZ, P]
        lib.oracle_dgemv.argtypes = [P, P, P, SZ, SZ]
        lib.oracle_idamax.argtypes = [P, SZ]
        lib.oracle_idamax.restype = SZ
        lib.oracle_dtrsm_left.argtypes = [P, P, SZ, SZ, C.c_int, C.c_int]
        lib.oracle_backward_error.argtypes = [P, P, P, SZ]
        lib.oracle_backward_error.restype = C.c_double
        lib.oracle_get01.argtypes = [P, P, P, SZ, SZ]
        lib.oracle_get01.restype = C.c_double
        lib.oracle_latm1.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, P, SZ, P]
        lib.oracle_dlatms_general.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, SZ, SZ, P, P, P]
        _lib = lib
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def larnv(dist: str, seed, n: int):
    """Returns (x, seed_after) for the DLARNV stream (families.rs:230-249)."""
    s = (C.c_uint32 * 4)(*seed)
    x = np.zeros(n, dtype=np.float64)
    load().oracle_larnv(DIST[dist], s, n, _p(x))
    return x, [int(v) for v in s]


def dgetrf(a: np.ndarray, n: int):
    """In place; returns (rc, ipiv, det, bad_col)."""
    ipiv = np.zeros(max(n, 1), dtype=np.uint64)
    det = np.zeros(1)
    bad = np.zeros(1, dtype=np.uint64)
    rc = load().oracle_dgetrf(_p(a), n, _p(ipiv), _p(det), _p(bad))
    return rc, [int(v) for v in ipiv[:n]], float(det[0]), int(bad[0])


def dgetrf_range(a: np.ndarray, n: int, k0: int, k1: int, ipiv: np.ndarray) -> int:
    """Steps k0 <= k < k1 of dgetrf (mod.rs:112-163) on a (n x n, in place),
    continuing an earlier call; ipiv: a uint64 array of n entries."""
    return load().oracle_dgetrf_range(_p(a), n, k0, k1, _p(ipiv))


def dgetrf_rect(a: np.ndarray, nrows: int, ncols: int):
    ipiv = np.zeros(max(ncols, 1), dtype=np.uint64)
    rc = load().oracle_dgetrf_rect(_p(a), nrows, ncols, _p(ipiv))
    return rc, [int(v) for v in ipiv[:ncols]]


def dgetrs(lu: np.ndarray, ipiv, b: np.ndarray, n: int, nrhs: int = 1) -> None:
    iv = np.asarray(ipiv, dtype=np.uint64)
    load().oracle_dgetrs(_p(lu), _p(iv), _p(b), n, nrhs)


def dgetri(lu: np.ndarray, n: int, ipiv) -> int:
    """mod.rs:249-298: lu (n*n, column-major) becomes the inverse; returns
    the status (0, or OR_SINGULAR leaving lu unchanged)."""
    iv = np.ascontiguousarray(ipiv, dtype=np.uint64)
    return int(load().oracle_dgetri(_p(lu), n, _p(iv)))


def dgesv(a: np.ndarray, b: np.ndarray, n: int, nrhs: int = 1):
    ipiv = np.zeros(max(n, 1), dtype=np.uint64)
    rc = load().oracle_dgesv(_p(a), _p(b), n, nrhs, _p(ipiv))
    return rc, [int(v) for v in ipiv[:n]]


def dgemv(a: np.ndarray, x: np.ndarray, m: int, n: int) -> np.ndarray:
    y = np.zeros(m)
    load().oracle_dgemv(_p(a), _p(x), _p(y), m, n)
    return y


def idamax(x: np.ndarray) -> int:
    return int(load().oracle_idamax(_p(x), x.size))


def dtrsm_left(a: np.ndarray, b: np.ndarray, m: int, n: int, lower: bool, unit: bool) -> None:
    load().oracle_dtrsm_left(_p(a), _p(b), m, n, int(lower), int(unit))


def backward_error(a: np.ndarray, x: np.ndarray, b: np.ndarray, n: int) -> float:
    return float(load().oracle_backward_error(_p(a), _p(x), _p(b), n))


def get01(a: np.ndarray, lu: np.ndarray, ipiv, m: int, n: int) -> float:
    iv = np.asarray(ipiv, dtype=np.uint64)
    return float(load().oracle_get01(_p(a), _p(lu), _p(iv), m, n))


def c1_system(n: int, seed=(1988, 1989, 1990, 1991)):
    """The dense workload of the spec: A iid U(-1,1) from the larnv stream in
    storage order, x_true continuing the same stream, b = A x_true (dgemv)."""
    a, s = larnv("Symmetric", list(seed), n * n)
    x, _ = larnv("Symmetric", s, n)
    b = dgemv(a, x, n, n)
    return a, x, b


def dlatms_general(dist: str, mode: int, cond: float, dmax: float, m: int, n: int, seed, d=None):
    """families.rs:903-1078 (DLATMS, nonsymmetric, full storage): returns
    (info, a column-major m*n, d, seed_after)."""
    s = (C.c_uint32 * 4)(*seed)
    a = np.zeros(max(m * n, 1), dtype=np.float64)
    dv = np.zeros(max(min(m, n), 1), dtype=np.float64)
    if d is not None:
        dv[: len(d)] = d
    info = load().oracle_dlatms_general(DIST[dist], mode, cond, dmax, m, n, _p(a), _p(dv), s)
    return info, a[: m * n], dv[: min(m, n)], list(s)
