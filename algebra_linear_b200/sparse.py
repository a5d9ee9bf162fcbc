"""Sparse LU with the reference's handle API (src/sparse/faer/sparse_lu.rs).

    lu = SparseLu.analyze(col_ptr, row_idx, LuMethod.auto())   sparse_lu.rs:64
    lu.factorize(col_ptr, row_idx, values)                     sparse_lu.rs:91
    lu.solve(b)             # b (float64) becomes x            sparse_lu.rs:125
    lu.effective_method(), lu.flop_ratio(), lu.stats()         sparse_lu.rs:137-155

CSC arrays: col_ptr (n + 1) and row_idx (nnz) as integer numpy arrays,
values (nnz) float64, or complex128 for SparseLu<Complex64> (lu.rs:61-82;
then b is complex128 too; the first factorization fixes the handle's
scalar). Errors are raised as SparseError whose `kind` is the
reference's Error variant and whose message is its Display string. analyze
runs on the host (COLAMD and the supernodal symbolic analysis); factorize and
solve run on the GPU through libalgebra_linear_gpu.so.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib

_ERR_KINDS = {
    _lib.SP_BAD_SHAPE: "BadShape",
    _lib.SP_INVALID_STRUCTURE: "InvalidStructure",
    _lib.SP_UNSORTED_ROWS: "UnsortedRows",
    _lib.SP_DUPLICATE_ENTRY: "DuplicateEntry",
    _lib.SP_SINGULAR: "Singular",
    _lib.SP_INDEX_OVERFLOW: "IndexOverflow",
    _lib.SP_STRUCTURE_MISMATCH: "StructureMismatch",
    _lib.SP_NOT_FINITE: "NotFinite",
    _lib.SP_NOT_FACTORIZED: "NotFactorized",
}

SIMPLICIAL, SUPERNODAL, AUTO = 0, 1, 2


class SparseError(Exception):
    """sparse::faer::Error (error.rs:5-24); str() is the reference's message."""

    def __init__(self, code: int):
        super().__init__(_lib.status_string(code))
        self.code = code
        self.kind = _ERR_KINDS.get(code, "Gpu")

    def __eq__(self, other):
        return isinstance(other, SparseError) and other.code == self.code

    __hash__ = Exception.__hash__


def _check(rc: int) -> None:
    if rc != _lib.OK:
        raise SparseError(rc)


@dataclass(frozen=True)
class LuMethod:
    """LuMethod (solver.rs:71-96): Simplicial, Supernodal or Auto(threshold)."""

    kind: int = SIMPLICIAL
    flop_ratio_threshold: float = 40.0

    @staticmethod
    def simplicial() -> "LuMethod":
        return LuMethod(SIMPLICIAL)

    @staticmethod
    def supernodal() -> "LuMethod":
        return LuMethod(SUPERNODAL)

    @staticmethod
    def auto(flop_ratio_threshold: float = 40.0) -> "LuMethod":
        return LuMethod(AUTO, float(flop_ratio_threshold))


class _Stats(C.Structure):
    _fields_ = [("n", C.c_size_t), ("nnz_a", C.c_size_t), ("nnz_l", C.c_size_t), ("nnz_u", C.c_size_t),
                ("fill_ratio", C.c_double), ("flops_estimate", C.c_size_t), ("method", C.c_int),
                ("has_flop_ratio", C.c_int), ("flop_ratio", C.c_double), ("ordering_time", C.c_double),
                ("factorization_time", C.c_double)]


class _Plan(C.Structure):
    _fields_ = [("n_fronts", C.c_size_t), ("n_small_fronts", C.c_size_t), ("small_levels", C.c_size_t),
                ("solve_levels", C.c_size_t), ("max_front_rows", C.c_size_t), ("max_front_cols", C.c_size_t),
                ("factor_bytes", C.c_size_t), ("work_bytes", C.c_size_t), ("plan_flops", C.c_double),
                ("structurally_singular", C.c_int), ("n_lanes", C.c_int), ("top_fronts", C.c_size_t)]


class _Refine(C.Structure):
    _fields_ = [("precision", C.c_int), ("iterations", C.c_int), ("fell_back", C.c_int),
                ("factor_precision", C.c_int), ("backward_error", C.c_double)]


# precisions of the factors (no counterpart in the reference, which is FP64 only)
PRECISIONS = {"fp64": -1, "fp32": 0, "tf32": 1, "bf16": 2, "tf32x3": 3}
_PREC_NAMES = {v: k for k, v in PRECISIONS.items()}


def _idx(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


def _dev_f64(t, numel: int, name: str) -> None:
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
            and t.numel() >= numel):
        raise TypeError(f"{name} must be a contiguous float64 CUDA tensor with >= {numel} entries")


class SparseLu:
    """Opaque sparse LU handle (sparse_lu.rs:45-156)."""

    def __init__(self, handle, n: int, nnz: int):
        self._lib = _lib.load()
        self._h = handle
        self.n = n
        self.nnz = nnz  # the analyzed pattern's entries: every values array has this length

    @classmethod
    def analyze(cls, col_ptr, row_idx, method: LuMethod = LuMethod()) -> "SparseLu":
        lib = _lib.load()
        cp, ri = _idx(col_ptr), _idx(row_idx)
        h = C.c_void_p()
        _check(lib.alg_splu_analyze(cp.ctypes.data if cp.size else None, cp.size,
                                    ri.ctypes.data if ri.size else None, ri.size, method.kind,
                                    method.flop_ratio_threshold, C.byref(h)))
        return cls(h, cp.size - 1, ri.size)

    def factorize(self, col_ptr, row_idx, values) -> None:
        cp, ri = _idx(col_ptr), _idx(row_idx)
        cplx = np.iscomplexobj(values)
        v = np.ascontiguousarray(values, dtype=np.complex128 if cplx else np.float64)
        fn = self._lib.alg_zsplu_factorize if cplx else self._lib.alg_splu_factorize
        _check(fn(self._h, cp.ctypes.data if cp.size else None, cp.size, ri.ctypes.data if ri.size else None,
                  ri.size, v.ctypes.data if v.size else None, v.size))

    def solve(self, b: np.ndarray) -> None:
        if (not isinstance(b, np.ndarray) or b.dtype not in (np.float64, np.complex128) or b.ndim != 1
                or not b.flags.c_contiguous):
            raise TypeError("b must be a contiguous 1-D float64 or complex128 numpy array")
        fn = self._lib.alg_zsplu_solve if b.dtype == np.complex128 else self._lib.alg_splu_solve
        _check(fn(self._h, b.ctypes.data if b.size else None, b.size))

    def effective_method(self) -> str:
        return "Supernodal" if self._lib.alg_splu_effective_method(self._h) == SUPERNODAL else "Simplicial"

    def flop_ratio(self):
        r = C.c_double()
        return r.value if self._lib.alg_splu_flop_ratio(self._h, C.byref(r)) == 1 else None

    def stats(self):
        s = _Stats()
        rc = self._lib.alg_splu_get_stats(self._h, C.byref(s))
        if rc == _lib.SP_NOT_FACTORIZED:
            return None
        _check(rc)
        return {"n": s.n, "nnz_a": s.nnz_a, "nnz_l": s.nnz_l, "nnz_u": s.nnz_u, "fill_ratio": s.fill_ratio,
                "flops_estimate": s.flops_estimate,
                "method": "Supernodal" if s.method == SUPERNODAL else "Simplicial",
                "flop_ratio": s.flop_ratio if s.has_flop_ratio else None, "ordering_time": s.ordering_time,
                "factorization_time": s.factorization_time}

    # ---- inspection (no reference counterpart) ------------------------------
    def symbolic(self) -> dict:
        n = self.n
        perm, inv, counts = (np.zeros(max(n, 1), np.uint64) for _ in range(3))
        ptr = np.zeros(n + 2, np.uint64)
        ns = C.c_size_t()
        _check(self._lib.alg_splu_symbolic(self._h, perm.ctypes.data, inv.ctypes.data, counts.ctypes.data,
                                           ptr.ctypes.data, C.byref(ns)))
        k = ns.value
        return {"col_perm": perm[:n].astype(np.int64), "col_perm_inv": inv[:n].astype(np.int64),
                "col_counts": counts[:n].astype(np.int64), "supernode_ptr": ptr[:k + 1].astype(np.int64)}

    def row_perm(self) -> np.ndarray:
        out = np.zeros(max(self.n, 1), np.uint64)
        _check(self._lib.alg_splu_row_perm(self._h, out.ctypes.data))
        return out[: self.n].astype(np.int64)

    def plan(self) -> dict:
        p = _Plan()
        _check(self._lib.alg_splu_plan_info(self._h, C.byref(p)))
        return {f: getattr(p, f) for f, _ in _Plan._fields_}

    # ---- mixed precision (no reference counterpart) ----------------------------
    def set_precision(self, precision: str = "fp64", tol: float = 0.0, max_ir: int = 0) -> None:
        """Precision of the next factorizations: "fp64" (the reference's
        arithmetic), or "fp32" / "tf32" / "tf32x3" / "bf16" fronts with every solve
        refined in FP64 to the backward error tol (<= 0: 10 n 2^-53), else
        the factors are recomputed in FP64."""
        _check(self._lib.alg_splu_set_precision(self._h, PRECISIONS[precision], float(tol), int(max_ir)))

    def last_solve(self) -> dict:
        r = _Refine()
        _check(self._lib.alg_splu_last_solve(self._h, C.byref(r)))
        return {"precision": _PREC_NAMES[r.precision], "iterations": r.iterations, "fell_back": bool(r.fell_back),
                "factor_precision": _PREC_NAMES[r.factor_precision],
                "backward_error": r.backward_error if r.backward_error >= 0 else None}

    # ---- device-resident ------------------------------------------------------
    def bind(self, ctx) -> None:
        """Factor and solve on ctx's stream; ctx closes this handle first."""
        _check(self._lib.alg_splu_set_ctx(self._h, ctx.handle))
        ctx.adopt(self)

    def factorize_dev(self, values) -> None:
        """values: the pattern's nnz entries, a float64 CUDA tensor (read
        through a raw device pointer, so its reach is checked here)."""
        _dev_f64(values, self.nnz, "values")
        _check(self._lib.alg_splu_factorize_dev(self._h, _lib.ptr(values)))

    def solve_dev(self, b) -> None:
        """b (n entries, a float64 CUDA tensor) becomes x."""
        _dev_f64(b, self.n, "b")
        _check(self._lib.alg_splu_solve_dev(self._h, _lib.ptr(b)))

    def close(self) -> None:
        if self._h:
            self._lib.alg_splu_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass
