"""Batched dgesv over many independent systems of uneven order (device).

Each system is the reference's dgesv (src/lapack/mod.rs:309-354). Matrices
(column-major, leading dimension n_i) and right-hand sides are packed in two
float64 CUDA tensors at the offsets the plan reports.
"""

from __future__ import annotations

import ctypes as C
import json
import pathlib

import numpy as np
import torch

from . import _lib
from .lapack import LapackError, _KINDS


def _check(rc: int) -> None:
    if rc != _lib.OK:
        raise LapackError(_KINDS.get(rc, _lib.status_string(rc)), rc)


def _dev_tensor(t, dtype, numel: int, name: str) -> None:
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()
            and t.numel() >= numel):
        raise TypeError(f"{name} must be a contiguous {dtype} CUDA tensor with >= {numel} entries")


class BatchPlan:
    def __init__(self, ctx, orders, mixed: bool = False):
        self._lib = _lib.load()
        self.ctx = ctx
        self.orders = np.asarray(orders, dtype=np.int32)
        self.count = int(self.orders.size)
        self.mixed = bool(mixed)
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
        # the packed arrays must reach the end of the last system at its offset
        n64 = self.orders.astype(np.int64)
        self._a_need = int((self.a_off[: self.count] + n64 * n64).max()) if self.count else 0
        self._b_need = int((self.b_off[: self.count] + n64).max()) if self.count else 0

    def _check_operands(self, a, b, info):
        """The kernels read and write the packed systems through raw device
        pointers: the tensors must be contiguous CUDA tensors of the right
        type that reach every system, or the launch would touch memory past
        them."""
        _dev_tensor(a, torch.float64, self._a_need, "a")
        _dev_tensor(b, torch.float64, self._b_need, "b")
        _dev_tensor(info, torch.int32, self.count, "info")

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
        self._check_operands(a, b, info)
        fn = self._lib.alg_batch_solve_graph if graph else self._lib.alg_batch_solve
        _check(fn(self.handle, a.data_ptr(), b.data_ptr(), info.data_ptr()))

    def autotune(self, a, b, info, a_src, b_src, cache: str | None = None) -> dict:
        """Picks each size bucket's launch shape (CTA size x panel width) by
        timing them on this batch (a, b are scratch: restored from a_src,
        b_src before every trial). With `cache` (a JSON file), shapes already
        chosen for the same bucket (its cap, the form and the device name) are
        reused without timing, and new choices are added to the file."""
        key = None
        entries = {}
        if cache:
            path = pathlib.Path(cache)
            if path.exists():
                entries = json.loads(path.read_text())
            dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "none"
            key = lambda cap: f"{dev}|{'mixed' if self.mixed else 'fp64'}|cap{cap}"  # noqa: E731
            buckets = self.info()["buckets"]
            if all(key(bk["cap"]) in entries for bk in buckets):
                for i, bk in enumerate(buckets):
                    e = entries[key(bk["cap"])]
                    _check(self._lib.alg_batch_set_config(self.handle, i, int(e["threads"]), int(e["panel"])))
                out = self.info()
                out["tuned"] = "cache"
                return out
        self._check_operands(a, b, info)
        self._check_operands(a_src, b_src, info)
        th = np.zeros(8, dtype=np.int32)
        _check(self._lib.alg_batch_autotune(self.handle, a.data_ptr(), b.data_ptr(), info.data_ptr(),
                                            a_src.data_ptr(), b_src.data_ptr(), th.ctypes.data))
        out = self.info()
        out["tuned"] = "timed"
        if key is not None:
            for bk in out["buckets"]:
                entries[key(bk["cap"])] = {"threads": bk["threads"], "panel": bk["panel"]}
            pathlib.Path(cache).write_text(json.dumps(entries, indent=1, sort_keys=True) + "\n")
        return out

    def info(self) -> dict:
        nb = C.c_int()
        caps = np.zeros(8, dtype=np.int32)
        thr = np.zeros(8, dtype=np.int32)
        cnt = np.zeros(8, dtype=np.int32)
        fl = C.c_double()
        _check(self._lib.alg_batch_info(self.handle, C.byref(nb), caps.ctypes.data, thr.ctypes.data,
                                        cnt.ctypes.data, C.byref(fl)))
        k = nb.value
        pan = np.zeros(8, dtype=np.int32)
        _check(self._lib.alg_batch_panels(self.handle, pan.ctypes.data))
        return {"buckets": [{"cap": int(caps[i]), "threads": int(thr[i]), "panel": int(pan[i]), "count": int(cnt[i])}
                            for i in range(k)], "flops": fl.value}

    def eta(self) -> np.ndarray:
        out = np.zeros(max(self.count, 1))
        _check(self._lib.alg_batch_eta(self.handle, out.ctypes.data))
        return out[: self.count]

    def ipiv(self) -> np.ndarray:
        """Pivots of the last solve (0-based pivot rows), packed at the b offsets."""
        out = np.zeros(max(self.b_total, 1), dtype=np.int32)
        _check(self._lib.alg_batch_ipiv(self.handle, out.ctypes.data))
        return out[: self.b_total]
