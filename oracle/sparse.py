"""ORACLE — test infrastructure only: ctypes wrapper of oracle_sparse.cpp, the
C++ restatement of the reference's numeric supernodal LU and its solve
(src/sparse/faer/supernodal_lu.rs, lu.rs), plus the grid patterns and value
streams the sparse tests and the bench's CPU baseline use.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import dense

SINGULAR = 104


def _lib():
    lib = dense.load()
    if not getattr(lib, "_sparse_bound", False):
        P, SZ = C.c_void_p, C.c_size_t
        lib.oracle_splu_factorize.argtypes = [SZ, P, P, P, P, P, P, SZ, C.POINTER(C.c_void_p)]
        lib.oracle_splu_sizes.argtypes = [P, C.POINTER(SZ), C.POINTER(SZ)]
        lib.oracle_splu_get.argtypes = [P, P, P, P, P, P, P, P]
        lib.oracle_splu_solve.argtypes = [P, P]
        lib.oracle_splu_free.argtypes = [P]
        lib.oracle_simplicial_factorize.argtypes = [SZ, P, P, P, P, P, C.POINTER(C.c_void_p)]
        lib.oracle_zsplu_factorize.argtypes = [SZ, P, P, P, P, P, P, SZ, C.POINTER(C.c_void_p)]
        lib.oracle_zsimplicial_factorize.argtypes = [SZ, P, P, P, P, P, C.POINTER(C.c_void_p)]
        lib.oracle_zsplu_sizes.argtypes = [P, C.POINTER(SZ), C.POINTER(SZ)]
        lib.oracle_zsplu_get.argtypes = [P, P, P, P, P, P, P, P]
        lib.oracle_zsplu_solve.argtypes = [P, P]
        lib.oracle_zsplu_free.argtypes = [P]
        lib._sparse_bound = True
    return lib


def _u(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


class Factors:
    """The reference's supernodal factors of one matrix (positions, CSC);
    with supernode_ptr None, its simplicial factors (lu.rs:209-327). Complex
    values (numpy complex128) give the SparseLu<Complex64> factors."""

    def __init__(self, n, col_ptr, row_idx, values, col_perm, col_perm_inv, supernode_ptr):
        lib = _lib()
        self.n = int(n)
        self.complex = np.iscomplexobj(values)
        dt = np.complex128 if self.complex else np.float64
        z = "z" if self.complex else ""
        self._fn = {k: getattr(lib, f"oracle_{z}splu_{k}") for k in ("sizes", "get", "solve", "free")}
        cp, ri = _u(col_ptr), _u(row_idx)
        v = np.ascontiguousarray(values, dtype=dt)
        cpm, cpi = _u(col_perm), _u(col_perm_inv)
        snp = _u(supernode_ptr) if supernode_ptr is not None else None
        h = C.c_void_p()
        if supernode_ptr is None:  # the simplicial path
            self.status = getattr(lib, f"oracle_{z}simplicial_factorize")(
                self.n, cp.ctypes.data, ri.ctypes.data, v.ctypes.data, cpm.ctypes.data, cpi.ctypes.data, C.byref(h))
        else:
            self.status = getattr(lib, f"oracle_{z}splu_factorize")(
                self.n, cp.ctypes.data, ri.ctypes.data, v.ctypes.data, cpm.ctypes.data, cpi.ctypes.data,
                snp.ctypes.data, len(snp) - 1, C.byref(h))
        self.h = h if self.status == 0 else None
        if self.h is None:
            return
        nl, nu = C.c_size_t(), C.c_size_t()
        self._fn["sizes"](h, C.byref(nl), C.byref(nu))
        self.l_col_ptr = np.zeros(self.n + 1, np.uint64)
        self.u_col_ptr = np.zeros(self.n + 1, np.uint64)
        self.l_row_idx = np.zeros(max(nl.value, 1), np.uint64)
        self.u_row_idx = np.zeros(max(nu.value, 1), np.uint64)
        self.l_val = np.zeros(max(nl.value, 1), dtype=dt)
        self.u_val = np.zeros(max(nu.value, 1), dtype=dt)
        self.row_perm = np.zeros(max(self.n, 1), np.uint64)
        self._fn["get"](h, self.l_col_ptr.ctypes.data, self.l_row_idx.ctypes.data, self.l_val.ctypes.data,
                        self.u_col_ptr.ctypes.data, self.u_row_idx.ctypes.data, self.u_val.ctypes.data,
                        self.row_perm.ctypes.data)
        self.nnz_l, self.nnz_u = nl.value, nu.value

    def solve(self, b) -> np.ndarray:
        x = np.array(b, dtype=np.complex128 if self.complex else np.float64, copy=True)
        self._fn["solve"](self.h, x.ctypes.data)
        return x

    def flops_estimate(self) -> int:
        """stats.rs:47-57: sum over columns of nnz(L col) * nnz(U col)."""
        nl = np.diff(self.l_col_ptr.astype(np.int64))
        nu = np.diff(self.u_col_ptr.astype(np.int64))
        return int((nl * nu).sum())

    def __del__(self):
        if getattr(self, "h", None):
            self._fn["free"](self.h)
            self.h = None


def grid_pattern(nx: int, ny: int, nz: int = 1):
    """CSC pattern of the 7-point (nz > 1) or 5-point (nz == 1) stencil on an
    nx x ny x nz grid, node index x + nx (y + ny z), rows sorted per column."""
    n = nx * ny * nz
    idx = np.arange(n, dtype=np.int64)
    x, y, z = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    cols = [idx]
    offs = [(-1, x > 0), (1, x < nx - 1), (-nx, y > 0), (nx, y < ny - 1)]
    if nz > 1:
        offs += [(-nx * ny, z > 0), (nx * ny, z < nz - 1)]
    rows, cidx, kind = [idx], [idx], [np.zeros(n, np.int8)]
    # row = column + off: off = -1 makes the column the row's east neighbour
    kinds = {-1: 2, 1: 1, -nx: 3, nx: 3, -nx * ny: 3, nx * ny: 3}
    for off, ok in offs:
        c = idx[ok]
        rows.append(c + off)
        cidx.append(c)
        kind.append(np.full(c.size, kinds[off], np.int8))
    r = np.concatenate(rows)
    c = np.concatenate(cidx)
    k = np.concatenate(kind)
    order = np.lexsort((r, c))
    r, c, k = r[order], c[order], k[order]
    col_ptr = np.zeros(n + 1, np.uint64)
    np.add.at(col_ptr, c + 1, 1)
    col_ptr = np.cumsum(col_ptr).astype(np.uint64)
    del cols
    return col_ptr, r.astype(np.uint64), k


def convection_diffusion_values(kind: np.ndarray, seed, scale_seed=None):
    """Values of the convection-diffusion stencil: diagonal 6 + 0.1 U(0,1);
    neighbours -1, with the x-neighbours -1 + 0.3 U(0,1) (the row's east
    neighbour, kind 2) and -1 - 0.3 U(0,1) (west, kind 1). U(0,1) comes from
    the reference's DLARNV stream (families.rs:230-249) in storage order."""
    u, s = dense.larnv("Uniform", seed, kind.size)
    v = np.where(kind == 0, 6.0 + 0.1 * u,
                 np.where(kind == 2, -1.0 + 0.3 * u, np.where(kind == 1, -1.0 - 0.3 * u, -1.0)))
    return v, s


def perturb(values: np.ndarray, seed):
    """values * (1 + 0.01 U(-1,1)), U(-1,1) from the DLARNV Symmetric stream."""
    u, s = dense.larnv("Symmetric", seed, values.size)
    return values * (1.0 + 0.01 * u), s
