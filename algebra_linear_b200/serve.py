"""The serving loop (alg_server_*): a device-resident queue of dense dgesv
and sparse refactorize+solve requests, admitted by worker streams under an
HBM budget. No counterpart in the reference crate.

    with Server(workers=4, hbm_budget=32 << 30, max_dense_n=4096) as srv:
        r = Request.dense(a, b, mixed=False)      # a: n*n column-major float64
        srv.submit(r); srv.wait(r); r.x           # the solution
        r = Request.sparse(lu, values, b)         # lu: an analyzed SparseLu

Host arrays must stay alive until the request is done; Request keeps them.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

DENSE, SPARSE = 0, 1
FP64, MIXED = 0, 1


class _Req(C.Structure):
    _fields_ = [("kind", C.c_int), ("precision", C.c_int), ("n", C.c_size_t), ("a", C.c_void_p),
                ("values", C.c_void_p), ("pattern", C.c_void_p), ("b", C.c_void_p), ("x", C.c_void_p),
                ("status", C.c_int), ("worker", C.c_int), ("backward_error", C.c_double),
                ("t_submit_ns", C.c_int64), ("t_start_ns", C.c_int64), ("t_done_ns", C.c_int64),
                ("done", C.c_int)]


def _f64(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a


class Request:
    def __init__(self, kind, n, b, a=None, values=None, pattern=None, mixed=False):
        self.kind = kind
        self.n = int(n)
        self.b = _f64(b)
        self.a = None if a is None else _f64(a)
        self.values = None if values is None else _f64(values)
        self.pattern = pattern
        self.x = np.zeros(max(self.n, 1))
        r = _Req()
        r.kind = kind
        r.precision = MIXED if mixed else FP64
        r.n = self.n
        r.a = self.a.ctypes.data if self.a is not None else None
        r.values = self.values.ctypes.data if self.values is not None else None
        r.pattern = pattern._h if pattern is not None else None
        r.b = self.b.ctypes.data
        r.x = self.x.ctypes.data
        self._r = r

    @classmethod
    def dense(cls, a, b, mixed=False) -> "Request":
        """A x = b, a column-major n x n with n = len(b). The loop reads n^2
        entries of a and n of b from these host arrays, so their lengths are
        checked here (the C ABI cannot see them)."""
        b = _f64(b)
        if np.size(a) != b.size * b.size:
            raise ValueError(f"a holds {np.size(a)} entries, an n x n matrix with n = len(b) = {b.size} needs "
                             f"{b.size * b.size}")
        return cls(DENSE, b.size, b, a=a, mixed=mixed)

    @classmethod
    def sparse(cls, pattern, values, b) -> "Request":
        """Refactorize the analyzed `pattern` (a SparseLu) with `values` (one
        per entry of its pattern) and solve for b (length n); both lengths
        are checked here, as the loop reads that many entries."""
        b = _f64(b)
        if b.size != pattern.n or np.size(values) != pattern.nnz:
            raise ValueError(f"the pattern has n = {pattern.n} and {pattern.nnz} entries; got len(b) = {b.size} "
                             f"and {np.size(values)} values")
        return cls(SPARSE, b.size, b, values=values, pattern=pattern)

    @property
    def solution(self) -> np.ndarray:
        return self.x[: self.n]

    @property
    def status(self) -> int:
        return self._r.status

    @property
    def latency_ms(self) -> float:
        return (self._r.t_done_ns - self._r.t_submit_ns) / 1e6

    @property
    def service_ms(self) -> float:
        return (self._r.t_done_ns - self._r.t_start_ns) / 1e6

    @property
    def worker(self) -> int:
        return self._r.worker

    @property
    def backward_error(self) -> float:
        return self._r.backward_error


class Server:
    def __init__(self, workers: int = 4, hbm_budget: int = 32 << 30, max_dense_n: int = 4096):
        self._lib = _lib.load()
        h = C.c_void_p()
        rc = self._lib.alg_server_create(workers, hbm_budget, max_dense_n, C.byref(h))
        if rc != _lib.OK:
            raise RuntimeError(f"alg_server_create: {_lib.status_string(rc)}")
        self._h = h

    def submit(self, req: Request) -> None:
        rc = self._lib.alg_server_submit(self._h, C.byref(req._r))
        if rc != _lib.OK:
            raise RuntimeError(f"alg_server_submit: {_lib.status_string(rc)}")

    def wait(self, req: Request) -> int:
        return self._lib.alg_server_wait(self._h, C.byref(req._r))

    def drain(self) -> None:
        self._lib.alg_server_drain(self._h)

    def now_ns(self) -> int:
        return self._lib.alg_server_now_ns()

    def close(self) -> None:
        if self._h:
            self._lib.alg_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
