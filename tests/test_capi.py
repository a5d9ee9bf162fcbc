"""The C ABI library loads, exports every entry point include/*.h declares,
and the Python mirror enforces the reference's shape errors before any GPU
call. CPU only: no compute entry point is called here."""

import pathlib
import re

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(alg_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_entry_points():
    names = declared_symbols()
    for want in ["alg_dgetrf", "alg_dgetrf_rect", "alg_dgesv", "alg_dgesv_nrhs", "alg_dgetrf_dev",
                 "alg_dgetrs_dev", "alg_dgesv_dev", "alg_ctx_create", "alg_ctx_destroy"]:
        assert want in names


def test_library_exports_every_declared_symbol():
    import ctypes

    from algebra_linear_b200 import _lib

    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
        assert ctypes.cast(getattr(lib, name), ctypes.c_void_p).value


def test_python_signatures_cover_the_header():
    from algebra_linear_b200 import _lib

    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_python_argument_counts_match_the_header():
    # every prototype's parameter count equals the ctypes binding's, so a
    # changed C signature cannot be called with a stale argument list
    from algebra_linear_b200 import _lib

    protos = {}
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(alg_[a-z0-9_]+)\s*\(([^;{}]*?)\)\s*;", text, flags=re.S):
            params = m.group(2).strip()
            protos[m.group(1)] = 0 if params in ("", "void") else len(params.split(","))
    bound = {name: len(args) for name, _, args in _lib.SIGNATURES}
    assert protos and {k: v for k, v in protos.items() if bound.get(k) != v} == {}


def test_status_strings_are_the_reference_messages():
    # src/sparse/faer/error.rs:52-64 (display_messages_are_exact)
    from algebra_linear_b200 import _lib

    want = {
        _lib.SP_BAD_SHAPE: "inconsistent shape or length",
        _lib.SP_INVALID_STRUCTURE: "invalid CSC structure",
        _lib.SP_UNSORTED_ROWS: "row indices must be strictly increasing within a column",
        _lib.SP_DUPLICATE_ENTRY: "duplicate entry in a column",
        _lib.SP_SINGULAR: "the matrix is singular",
        _lib.SP_INDEX_OVERFLOW: "index or workspace size overflow",
        _lib.SP_STRUCTURE_MISMATCH: "the matrix pattern differs from the symbolic analysis",
        _lib.SP_NOT_FINITE: "the matrix has a NaN or infinite entry",
        _lib.SP_NOT_FACTORIZED: "the matrix has not been factorized",
    }
    for code, msg in want.items():
        assert _lib.status_string(code) == msg


def test_dense_shape_errors_match_the_reference():
    from algebra_linear_b200.lapack import LapackError, dgesv, dgetrf, dgetrf_rect

    # mod.rs:504-508
    with pytest.raises(LapackError) as e:
        dgetrf(np.array([1.0, 2.0, 3.0]), 2)
    assert e.value.kind == "BadShape"
    # mod.rs:609-616 (n = 0 succeeds without touching the device)
    assert dgetrf(np.zeros(0), 0) == ([], 1.0)
    dgesv(np.zeros(0), np.zeros(0))
    # mod.rs:735-741
    a = np.array([1.0, 2.0, 3.0, 4.0])
    with pytest.raises(LapackError) as e:
        dgetrf_rect(a, 1, 2, [0, 0])
    assert e.value.kind == "BadShape"
    with pytest.raises(LapackError) as e:
        dgetrf_rect(a, 2, 2, [0])
    assert e.value.kind == "BadShape"
    # mod.rs:747-751
    dgetrf_rect(np.zeros(0), 3, 0, [])
    with pytest.raises(LapackError) as e:
        dgesv(np.zeros(5), np.zeros(2))
    assert e.value.kind == "BadShape"
    # mod.rs:250-255 (dgetri: lengths checked first, n = 0 succeeds)
    from algebra_linear_b200.lapack import dgetri

    with pytest.raises(LapackError) as e:
        dgetri(np.zeros(4), 2, [0])
    assert e.value.kind == "BadShape"
    with pytest.raises(LapackError) as e:
        dgetri(np.zeros(3), 2, [0, 1])
    assert e.value.kind == "BadShape"
    dgetri(np.zeros(0), 0, [])


def test_complex_shape_errors_match_the_reference():
    # complex.rs:518-529, 582-590, 640-645: lengths checked before any work,
    # n = 0 succeeds; the C ABI rejects nrows < ncols without touching a GPU
    from algebra_linear_b200 import _lib
    from algebra_linear_b200.lapack import LapackError, zgesv, zgetrf, zgetrf_rect

    with pytest.raises(LapackError) as e:
        zgetrf(np.ones(3, dtype=np.complex128), 2)
    assert e.value.kind == "BadShape"
    with pytest.raises(LapackError) as e:
        zgesv(np.ones(3, dtype=np.complex128), np.ones(2, dtype=np.complex128))
    assert e.value.kind == "BadShape"
    with pytest.raises(LapackError) as e:
        zgetrf_rect(np.ones(4, dtype=np.complex128), 1, 2, [0, 0])
    assert e.value.kind == "BadShape"
    with pytest.raises(TypeError):
        zgetrf(np.ones(4), 2)  # float64 is not a complex matrix
    assert zgetrf(np.zeros(0, dtype=np.complex128), 0) == []
    zgesv(np.zeros(0, dtype=np.complex128), np.zeros(0, dtype=np.complex128))
    lib = _lib.load()
    assert lib.alg_zgetrf_rect(None, 1, 2, None) == _lib.BAD_SHAPE
    assert lib.alg_zgetrf(None, 0, None) == _lib.OK
    assert lib.alg_zgesv(None, None, 0) == _lib.OK
    from algebra_linear_b200.lapack import zgetri

    with pytest.raises(LapackError) as e:
        zgetri(np.zeros(4, dtype=np.complex128), 2, [0])
    assert e.value.kind == "BadShape"
    zgetri(np.zeros(0, dtype=np.complex128), 0, [])
    assert lib.alg_zgetri(None, 0, None) == _lib.OK
