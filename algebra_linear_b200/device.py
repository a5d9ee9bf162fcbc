"""Device-resident entry points over torch tensors (the alg_*_dev C ABI).

Matrices are 1-D (or any contiguous) float64 CUDA tensors holding
column-major data, leading dimension n, as the host drop-ins take them. The
context runs on torch's current CUDA stream.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from .lapack import LapackError, _KINDS


def _check(rc: int) -> None:
    if rc != _lib.OK:
        raise LapackError(_KINDS.get(rc, _lib.status_string(rc)), rc)


def _dev_f64(t: torch.Tensor, numel: int, name: str) -> torch.Tensor:
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.numel() >= numel):
        raise TypeError(f"{name} must be a contiguous float64 CUDA tensor with >= {numel} entries")
    return t


# cudaStreamLegacy: torch's default stream is the legacy NULL stream, and a
# NULL handle would make the library create its own unordered stream.
_CUDA_STREAM_LEGACY = 0x1


def _current_stream() -> int:
    h = torch.cuda.current_stream().cuda_stream
    return h if h else _CUDA_STREAM_LEGACY


class Context:
    """Owns an alg_ctx bound to torch's current stream."""

    def __init__(self):
        self._lib = _lib.load()
        h = C.c_void_p()
        _check(self._lib.alg_ctx_create(C.c_void_p(_current_stream()), C.byref(h)))
        self.handle = h

    def adopt(self, child):
        """Children (plans, sparse handles) are closed before the context."""
        import weakref

        self.__dict__.setdefault("_children", []).append(weakref.ref(child))
        return child

    def close(self):
        for ref in self.__dict__.get("_children", []):
            child = ref()
            if child is not None:
                child.close()
        if self.handle:
            self._lib.alg_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def sync_stream(self):
        _check(self._lib.alg_ctx_set_stream(self.handle, C.c_void_p(_current_stream())))

    def larnv(self, dist: int, seed, n: int, out: torch.Tensor | None = None):
        """The reference's DLARNV stream on the device; returns (x, seed_after)."""
        if out is not None:
            _dev_f64(out, n, "out")
        x = out if out is not None else torch.empty(max(n, 1), dtype=torch.float64, device="cuda")
        s_in = (C.c_uint32 * 4)(*seed)
        s_out = (C.c_uint32 * 4)()
        _check(self._lib.alg_larnv_dev(self.handle, dist, s_in, n, x.data_ptr(), s_out))
        return x[:n], [int(v) for v in s_out]

    def dgetrf(self, a: torch.Tensor, n: int, update: int = _lib.UPDATE_EXACT):
        """In-place LU; returns (ipiv, perm) int32 CUDA tensors."""
        _dev_f64(a, n * n, "a")
        ipiv = torch.empty(max(n, 1), dtype=torch.int32, device=a.device)
        perm = torch.empty(max(n, 1), dtype=torch.int32, device=a.device)
        _check(self._lib.alg_dgetrf_dev(self.handle, update, a.data_ptr(), n, n, ipiv.data_ptr(), perm.data_ptr()))
        return ipiv[:n], perm[:n]

    def dgetrs(self, lu: torch.Tensor, perm: torch.Tensor, b: torch.Tensor, n: int, nrhs: int = 1):
        _dev_f64(lu, n * n, "lu")
        _dev_f64(b, n * nrhs, "b")
        if not (perm.is_cuda and perm.dtype == torch.int32 and perm.is_contiguous() and perm.numel() >= n):
            raise TypeError(f"perm must be a contiguous int32 CUDA tensor with >= {n} entries")
        _check(self._lib.alg_dgetrs_dev(self.handle, lu.data_ptr(), n, n, perm.data_ptr(), b.data_ptr(), nrhs, n))

    def dgesv(self, a: torch.Tensor, b: torch.Tensor, n: int, nrhs: int = 1, update: int = _lib.UPDATE_EXACT):
        """Solves in place (a -> LU, b -> x); returns ipiv (int32 CUDA tensor)."""
        _dev_f64(a, n * n, "a")
        _dev_f64(b, n * nrhs, "b")
        ipiv = torch.empty(max(n, 1), dtype=torch.int32, device=a.device)
        _check(self._lib.alg_dgesv_dev(self.handle, update, a.data_ptr(), n, n, b.data_ptr(), nrhs, n,
                                       ipiv.data_ptr()))
        return ipiv[:n]


def _profile_methods():
    def set_profiling(self, on: bool = True):
        _check(self._lib.alg_ctx_set_profiling(self.handle, 1 if on else 0))

    def profile_reset(self):
        _check(self._lib.alg_ctx_profile_reset(self.handle))

    def profile(self) -> dict:
        """{class: {"launches", "ms", "flops", "bytes"}} for classes that ran."""
        out = {}
        for i, name in enumerate(_lib.KERNEL_CLASSES):
            n = C.c_ulonglong()
            ms, fl, by = C.c_double(), C.c_double(), C.c_double()
            _check(self._lib.alg_ctx_profile_get(self.handle, i, C.byref(n), C.byref(ms), C.byref(fl), C.byref(by)))
            if n.value:
                out[name] = {"launches": n.value, "ms": ms.value, "flops": fl.value, "bytes": by.value}
        return out

    Context.set_profiling = set_profiling
    Context.profile_reset = profile_reset
    Context.profile = profile


_profile_methods()
