"""Mixed-precision dgesv (low-precision LU + FP64 iterative refinement).

The dsgesv contract over the C ABI (alg_dgesv_mixed / alg_dgesv_mixed_dev):
A is factorized in FP32 (trailing updates FP32, TF32 or BF16 with FP32
accumulation) and x is refined in FP64 until the normwise backward error is
within 10 n 2^-53; A stays unchanged unless the FP64 fallback ran.
"""

from __future__ import annotations

import ctypes as C

from . import _lib
from .lapack import LapackError, _KINDS

PRECISIONS = {"fp32": 0, "tf32": 1, "bf16": 2, "tf32x3": 3}
PATHS = {1: "ir", 2: "gmres", 3: "fp64"}


class Opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("tol", C.c_double), ("max_ir", C.c_int), ("no_fallback", C.c_int),
                ("no_gmres", C.c_int), ("gmres_restart", C.c_int), ("pivoting", C.c_int), ("reserved", C.c_int)]


class Report(C.Structure):
    _fields_ = [("path", C.c_int), ("precision", C.c_int), ("ir_iterations", C.c_int),
                ("gmres_iterations", C.c_int), ("backward_error", C.c_double), ("reserved", C.c_double * 4)]

    def as_dict(self) -> dict:
        return {"path": PATHS.get(self.path, "none"), "ir_iterations": self.ir_iterations,
                "gmres_iterations": self.gmres_iterations, "backward_error": self.backward_error,
                "butterfly": bool(self.reserved[0]), "tournament": bool(self.reserved[1])}


PIVOTING = {"auto": 0, "partial": 1, "rbt": 2, "tournament": 3}


def opts(precision: str = "fp32", tol: float = 0.0, max_ir: int = 30, no_fallback: bool = False,
         pivoting: str = "auto", no_gmres: bool = False) -> Opts:
    o = Opts()
    _lib.load().alg_mixed_opts_default(C.byref(o))
    o.precision = PRECISIONS[precision]
    o.pivoting = PIVOTING[pivoting]
    o.no_gmres = 1 if no_gmres else 0
    o.tol = tol
    o.max_ir = max_ir
    o.no_fallback = 1 if no_fallback else 0
    return o


last_report: dict = {}


def _check(rc: int) -> None:
    if rc != _lib.OK:
        raise LapackError(_KINDS.get(rc, _lib.status_string(rc)), rc)


def dgesv_mixed_dev(ctx, A, b, n: int, nrhs: int = 1, precision: str = "fp32", **kw) -> dict:
    """A (n*n float64 CUDA tensor, column-major) is read; b (n*nrhs) becomes x."""
    from .device import _dev_f64

    _dev_f64(A, n * n, "A")
    _dev_f64(b, n * nrhs, "b")
    o = opts(precision, **kw)
    rep = Report()
    _check(_lib.load().alg_dgesv_mixed_dev(ctx.handle, C.byref(o), A.data_ptr(), n, n, b.data_ptr(), nrhs, n,
                                           C.byref(rep)))
    last_report.clear()
    last_report.update(rep.as_dict())
    return rep.as_dict()


def dgesv_mixed_host(a_ptr: int, b_ptr: int, n: int, nrhs: int = 1, precision: str = "fp32", **kw) -> int:
    """Host-pointer drop-in; returns the status code."""
    o = opts(precision, **kw)
    rep = Report()
    rc = _lib.load().alg_dgesv_mixed(C.byref(o), a_ptr, b_ptr, n, nrhs, C.byref(rep))
    last_report.clear()
    last_report.update(rep.as_dict())
    return rc
