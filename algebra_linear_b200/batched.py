"""Batched dgesv over many independent systems of uneven order (device).

Each system is the reference's dgesv (src/lapack/mod.rs:309-354). Matrices
(column-major, leading dimension n_i) and right-hand sides are packed in two
float64 CUDA tensors at the offsets the plan reports.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .lapack import LapackError, _KINDS


def _check(rc: int) -> None:
    if rc != _lib.OK:
        raise LapackError(_KINDS.get(rc, _lib.status_string(rc)), rc)


class BatchPlan:
    def __init__(self, ctx, orders, mixed: bool = False):
        self._lib = _lib.load()
        self.ctx = ctx
        self.orders = np.asarray(orders, dtype=np.int32)
        self.count = int(self.orders.size)
        h = C.c_void_p()
        _check(self._lib.alg_batch_create(ctx.handle, self.count, self.orders.ctypes.data, 1 if mixed else 0,
                                          C.byref(h)))
        self.handle = h
        self.a_off = np.zeros(max(self.count, 1), dtype=np.int64)
        self.b_off = np.zeros(max(self.count, 1), dtype=np.int64)
        _check(self._lib.alg_batch_offsets(h, self.a_off.ctypes.data, self.b_off.ctypes.data))
        ctx.adopt(self)
        self.a_total = int((self.orders.astype(np.int64) ** 2).sum())
        self.b_total = int(self.orders.sum())

    def close(self):
        if self.handle:
            self._lib.alg_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def solve(self, a: torch.Tensor, b: torch.Tensor, info: torch.Tensor, graph: bool = False):
        fn = self._lib.alg_batch_solve_graph if graph else self._lib.alg_batch_solve
        _check(fn(self.handle, a.data_ptr(), b.data_ptr(), info.data_ptr()))

    def autotune(self, a, b, info, a_src, b_src):
        out = np.zeros(8, dtype=np.int32)
        _check(self._lib.alg_batch_autotune(self.handle, a.data_ptr(), b.data_ptr(), info.data_ptr(),
                                            a_src.data_ptr(), b_src.data_ptr(), out.ctypes.data))
        return self.info()

    def info(self) -> dict:
        nb = C.c_int()
        caps = np.zeros(8, dtype=np.int32)
        thr = np.zeros(8, dtype=np.int32)
        cnt = np.zeros(8, dtype=np.int32)
        fl = C.c_double()
        _check(self._lib.alg_batch_info(self.handle, C.byref(nb), caps.ctypes.data, thr.ctypes.data,
                                        cnt.ctypes.data, C.byref(fl)))
        k = nb.value
        return {"buckets": [{"cap": int(caps[i]), "threads": int(thr[i]), "count": int(cnt[i])} for i in range(k)],
                "flops": fl.value}

    def eta(self) -> np.ndarray:
        out = np.zeros(max(self.count, 1))
        _check(self._lib.alg_batch_eta(self.handle, out.ctypes.data))
        return out[: self.count]
