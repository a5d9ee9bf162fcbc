"""The Rust binding crate (rust/algebra_linear_gpu) against the C header and
the built library, on the CPU (no Rust toolchain is needed): src/ffi.rs is
exactly what gen_ffi.py writes from include/algebra_linear_gpu.h; its
extern block names every prototype with the header's parameter count; the
safe wrappers name only declared functions and constants; the library
exports every function the crate links; the sparse error variants are in
the order of the status codes (the reference's declaration order)."""

import pathlib
import re
import subprocess
import sys

ROOT = pathlib.Path(__file__).resolve().parent.parent
CRATE = ROOT / "rust" / "algebra_linear_gpu"


def _header_protos():
    text = (ROOT / "include" / "algebra_linear_gpu.h").read_text()
    text = re.sub(r"//[^\n]*", "", re.sub(r"/\*.*?\*/", "", text, flags=re.S))
    out = {}
    for m in re.finditer(r"\b(alg_[a-z0-9_]+)\s*\(([^;{}]*?)\)\s*;", text, flags=re.S):
        params = " ".join(m.group(2).split())
        out[m.group(1)] = 0 if params in ("", "void") else len(params.split(","))
    return out


def _rust_externs():
    text = (CRATE / "src" / "ffi.rs").read_text()
    block = text[text.index('extern "C" {'):]
    out = {}
    for m in re.finditer(r"pub fn (alg_\w+)\(([^)]*)\)", block):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if not params else len(params.split(","))
    return out


def test_ffi_rs_is_generated_from_the_header():
    r = subprocess.run([sys.executable, str(CRATE / "gen_ffi.py"), "--check"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_every_prototype_is_declared_with_its_parameter_count():
    assert _rust_externs() == _header_protos()


def test_wrappers_name_only_declared_items():
    ffi = (CRATE / "src" / "ffi.rs").read_text()
    declared = set(re.findall(r"pub fn (alg_\w+)", ffi)) | set(re.findall(r"pub const (ALG_\w+)", ffi))
    declared |= set(re.findall(r"pub struct (alg_\w+)", ffi))
    used = set()
    for f in ("lib.rs", "lapack.rs", "complex.rs", "sparse.rs"):
        used |= set(re.findall(r"ffi::((?:alg|ALG)_\w+)", (CRATE / "src" / f).read_text()))
    assert used and used <= declared, used - declared
    # every reference entry point of the path has its safe wrapper
    lapack = (CRATE / "src" / "lapack.rs").read_text()
    for fn in ("dgetrf", "dgetrf_rect", "dgesv", "dgetri"):
        assert re.search(rf"pub fn {fn}\(", lapack), fn
    cplx = (CRATE / "src" / "complex.rs").read_text()
    for fn in ("zgetrf", "zgetrf_rect", "zgesv", "zgetri"):
        assert re.search(rf"pub fn {fn}\(", cplx), fn
    sp = (CRATE / "src" / "sparse.rs").read_text()
    for fn in ("analyze", "factorize", "solve", "effective_method", "flop_ratio", "stats"):
        assert re.search(rf"pub fn {fn}\(", sp), fn


def test_library_exports_what_the_crate_links():
    import ctypes

    from algebra_linear_b200 import _lib

    lib = _lib.load()
    for name in _rust_externs():
        assert ctypes.cast(getattr(lib, name), ctypes.c_void_p).value, name


def test_sparse_error_variants_follow_the_status_codes():
    sp = (CRATE / "src" / "sparse.rs").read_text()
    enum = sp[sp.index("pub enum Error {"):]
    enum = enum[:enum.index("}")]
    variants = re.findall(r"^\s*(\w+)(?:\(i32\))?,", enum, flags=re.M)
    ffi = (CRATE / "src" / "ffi.rs").read_text()
    codes = dict((k, int(v)) for k, v in re.findall(r"pub const (ALG_SP_\w+): c_int = (-?\d+);", ffi))
    names = ["BadShape", "InvalidStructure", "UnsortedRows", "DuplicateEntry", "Singular", "IndexOverflow",
             "StructureMismatch", "NotFinite", "NotFactorized"]
    assert variants[:9] == names and variants[9:] == ["Device"]
    snake = re.compile(r"(?<!^)(?=[A-Z])")
    for k, v in enumerate(names):
        assert codes["ALG_SP_" + snake.sub("_", v).upper()] == 100 + k, v
