"""Writes src/ffi.rs, the raw Rust declarations of the C ABI, from
include/algebra_linear_gpu.h (status and option constants, the #[repr(C)]
structs, the opaque handles and every extern "C" function):

    python rust/algebra_linear_gpu/gen_ffi.py [--check]

--check compares the file on disk with what the header gives and exits 1 when
they differ (the repository's CPU tests run the same comparison), so the Rust
binding cannot drift from the header the library is built with.
"""

from __future__ import annotations

import pathlib
import re
import sys

HERE = pathlib.Path(__file__).resolve().parent
HEADER = HERE.parent.parent / "include" / "algebra_linear_gpu.h"
OUT = HERE / "src" / "ffi.rs"

SCALARS = {
    "double": "f64", "float": "f32", "int": "c_int", "size_t": "usize", "int32_t": "i32", "uint32_t": "u32",
    "int64_t": "i64", "unsigned long long": "c_ulonglong", "char": "c_char", "void": "c_void",
}


def strip_comments(text: str) -> str:
    return re.sub(r"//[^\n]*", "", re.sub(r"/\*.*?\*/", "", text, flags=re.S))


def rust_type(ctype: str, array: bool = False) -> str:
    """C type of a parameter or field (without its name) -> Rust type."""
    c = ctype.replace("volatile", "").strip()
    const = c.startswith("const ")
    if const:
        c = c[len("const "):].strip()
    stars = c.count("*")
    base = c.replace("*", "").strip()
    rt = SCALARS.get(base, base)
    if array:  # a parameter declared as an array decays to a pointer
        stars += 1
    if stars == 0:
        return rt
    # the innermost pointer carries the const of the pointee (const T* / const T**)
    for k in range(stars):
        rt = f"*{'const' if const and k == 0 else 'mut'} {rt}"
    return rt


def split_decl(decl: str):
    """'const uint32_t seed[4]' -> ('const uint32_t', 'seed', '4')."""
    m = re.match(r"^(.*?)(\w+)\s*(?:\[(\d*)\])?$", decl.strip(), flags=re.S)
    return m.group(1).strip(), m.group(2), m.group(3)


def parse(text: str):
    t = strip_comments(text)
    consts = []
    for m in re.finditer(r"^#define\s+(ALG_\w+)\s+(\(?-?\d+\)?)\s*$", t, flags=re.M):
        consts.append((m.group(1), int(m.group(2).strip("()"))))
    structs = []
    for m in re.finditer(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", t, flags=re.S):
        fields = []
        for line in m.group(1).split(";"):
            line = " ".join(line.split())
            if not line:
                continue
            first, *rest = [p.strip() for p in line.split(",")]
            ctype, name, dim = split_decl(first)
            fields.append((name, rust_type(ctype) if not dim else f"[{rust_type(ctype)}; {dim}]"))
            for extra in rest:  # 'size_t a, b, c'
                fields.append((extra, rust_type(ctype)))
        structs.append((m.group(2), fields))
    opaque = [m.group(2) for m in re.finditer(r"typedef struct (\w+) (\w+);", t)]
    funcs = []
    for m in re.finditer(r"^([A-Za-z_][\w\s\*]*?)\b(alg_\w+)\s*\(([^;{}]*?)\)\s*;", t, flags=re.S | re.M):
        ret = " ".join(m.group(1).split())
        params = " ".join(m.group(3).split())
        args = []
        if params not in ("", "void"):
            for p in params.split(","):
                ctype, name, dim = split_decl(p)
                args.append((name, rust_type(ctype, array=dim is not None)))
        funcs.append((m.group(2), rust_type(ret) if ret != "void" else None, args))
    return consts, structs, opaque, funcs


def render(text: str) -> str:
    consts, structs, opaque, funcs = parse(text)
    out = [
        "// Raw declarations of the C ABI of libalgebra_linear_gpu, written by",
        "// gen_ffi.py from include/algebra_linear_gpu.h; do not edit by hand.",
        "// The meaning of every constant, field and function is documented in the header.",
        "#![allow(non_camel_case_types, non_snake_case, dead_code)]",
        "",
        "use core::ffi::{c_char, c_int, c_ulonglong, c_void};",
        "",
    ]
    for name, value in consts:
        out.append(f"pub const {name}: c_int = {value};")
    out.append("")
    for name in opaque:
        out += ["#[repr(C)]", f"pub struct {name} {{", "    _private: [u8; 0],", "}", ""]
    for name, fields in structs:
        out += ["#[repr(C)]", "#[derive(Clone, Copy, Debug)]", f"pub struct {name} {{"]
        out += [f"    pub {f}: {ty}," for f, ty in fields]
        out += ["}", ""]
    out.append('#[link(name = "algebra_linear_gpu")]')
    out.append('unsafe extern "C" {')
    for name, ret, args in funcs:
        sig = ", ".join(f"{a}: {ty}" for a, ty in args)
        out.append(f"    pub fn {name}({sig})" + (f" -> {ret};" if ret else ";"))
    out.append("}")
    return "\n".join(out) + "\n"


def main() -> None:
    want = render(HEADER.read_text())
    if "--check" in sys.argv:
        if not OUT.exists() or OUT.read_text() != want:
            sys.exit(f"{OUT} is out of date: run {pathlib.Path(__file__).name}")
        return
    OUT.parent.mkdir(parents=True, exist_ok=True)
    OUT.write_text(want)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
