"""Extracts the reference crate's own known-answer vectors into JSON fixtures.

Run in a container where the reference sources are mounted (they are read as
text; nothing of the reference is executed):

    python tests/golden/make_golden.py /path/to/algebra_linear

Writes tests/golden/larnv_kat.json from the test
`larnv_matches_the_reference_stream` in src/lapack/families.rs:1176-1261,
whose values the reference captured from LAPACK 3.12.1's libtmglib (`dlarnv_`)
for seed [1988, 1989, 1990, 1991], n = 200: x[0..12], x[198..200] and the seed
after the call, for the Uniform, Symmetric and Normal distributions.

Writes tests/golden/dlatms_kat.json from the test
`dlatms_matches_the_reference_matrices` in src/lapack/families.rs:2014-2470
(twelve DLATMS calls whose spectra, matrices and final seeds the reference
captured from LAPACK 3.12.1's libtmglib).

Writes tests/golden/colamd_kat.json from the test `matches_faer_on_fixtures`
in src/sparse/faer/colamd.rs:886-918 (permutations the reference captured from
faer's colamd::order): each fixture's CSC pattern, built here from the
fixture's definition in the same test module (colamd.rs:800-880), and the
expected perm and perm_inv read from the test's text.
"""

import json
import pathlib
import re
import sys

HERE = pathlib.Path(__file__).resolve().parent


def extract_larnv(src: str) -> dict:
    start = src.index("fn larnv_matches_the_reference_stream")
    body = src[start:src.index("fn larnv_is_continuous_across_batches", start)]
    seedy = re.search(r"const SEEDY: \[u32; 4\] = \[([^\]]+)\]", src)
    cases = []
    for m in re.finditer(r"Dist::(\w+),\s*\[([^\]]+)\],\s*\[([^\]]+)\]", body):
        dist = m.group(1)
        values = [v.strip() for v in m.group(2).split(",") if v.strip()]
        seed = [int(v) for v in m.group(3).split(",") if v.strip()]
        assert len(values) == 14 and len(seed) == 4, dist
        cases.append({
            "dist": dist,
            # kept as text so the exact decimal strings round-trip to the same bits
            "first12": values[:12],
            "last2_at_198": values[12:],
            "seed_after": seed,
        })
    assert [c["dist"] for c in cases] == ["Uniform", "Symmetric", "Normal"], cases
    return {
        "source": "src/lapack/families.rs:1176-1261 (larnv_matches_the_reference_stream)",
        "seed": [int(v) for v in seedy.group(1).split(",")],
        "n": 200,
        "cases": cases,
    }


def _from_cols(cols):
    col_ptr, row_idx = [0], []
    for c in cols:
        c = sorted(set(c))
        row_idx.extend(c)
        col_ptr.append(len(row_idx))
    return col_ptr, row_idx


def colamd_fixtures():
    """The fixture patterns of colamd.rs's tests (tridiag5, arrow8, grid4x5,
    ring12, lcg30), in the test's order."""
    out = {}
    out["tridiag5"] = _from_cols([[0, 1], [0, 1, 2], [1, 2, 3], [2, 3, 4], [3, 4]])
    out["arrow8"] = _from_cols([list(range(8)) if j == 0 else [0, j] for j in range(8)])
    rows, cn = 4, 5
    cols = []
    for i in range(rows * cn):
        r, c = divmod(i, cn)
        v = [i]
        if r > 0:
            v.append((r - 1) * cn + c)
        if r + 1 < rows:
            v.append((r + 1) * cn + c)
        if c > 0:
            v.append(r * cn + c - 1)
        if c + 1 < cn:
            v.append(r * cn + c + 1)
        cols.append(v)
    out["grid4x5"] = _from_cols(cols)
    out["ring12"] = _from_cols([[j, (j + 1) % 12, (j + 3) % 12, (j + 7) % 12] for j in range(12)])
    state, m64, cols = 0x2545F4914F6CDD1D, (1 << 64) - 1, []
    for j in range(30):
        v = [j]
        for _ in range(4):
            state = (state * 6364136223846793005 + 1442695040888963407) & m64
            v.append((state >> 33) % 30)
        cols.append(v)
    out["lcg30"] = _from_cols(cols)
    return out


def extract_colamd(src: str) -> dict:
    start = src.index("fn matches_faer_on_fixtures")
    body = src[start:src.index("fn returns_valid_permutations", start)]
    vecs = [[int(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()]
            for m in re.finditer(r"vec!\[([0-9,\s]+)\]", body)]
    fx = colamd_fixtures()
    names = list(fx)
    assert len(vecs) == 2 * len(names), len(vecs)
    cases = []
    for i, name in enumerate(names):
        cp, ri = fx[name]
        perm, inv = vecs[2 * i], vecs[2 * i + 1]
        assert len(perm) == len(cp) - 1 == len(inv), name
        cases.append({"name": name, "col_ptr": cp, "row_idx": ri, "perm": perm, "perm_inv": inv})
    return {"source": "src/sparse/faer/colamd.rs:886-918 (matches_faer_on_fixtures)", "cases": cases}


def extract_dlatms(src: str) -> dict:
    """families.rs:2014-2470 (dlatms_matches_the_reference_matrices): twelve
    DLATMS calls from seed SEEDY with the spectrum, the matrix and the seed
    after the call that the reference captured from LAPACK's libtmglib."""
    start = src.index("fn dlatms_matches_the_reference_matrices")
    body = src[start:src.index("fn dlatms_reports_what_the_reference_reports", start)]
    arrays = {}
    for m in re.finditer(r"let ([ad]\d+): \[f64; \d+\] = \[(.*?)\];", body, flags=re.S):
        text = re.sub(r"//[^\n]*", "", m.group(2))
        arrays[m.group(1)] = [v.strip() for v in text.split(",") if v.strip()]
    cases = []
    pat = (r"Dlatms \{\s*dist: Dist::(\w+),\s*sym: DlatmsSym::(\w+),\s*mode: (-?\d+),\s*cond: ([^,]+),"
           r"\s*dmax: ([^,]+),\s*pack: DlatmsPack::(\w+),\s*\},\s*(\d+),\s*(\d+),\s*\[([^\]]+)\],"
           r"\s*&(d\d+),\s*&(a\d+),")
    for m in re.finditer(pat, body):
        dist, sym, mode, cond, dmax, pack, mm, nn, seed, dn, an = m.groups()
        cases.append({"dist": dist, "sym": sym, "mode": int(mode), "cond": cond.strip(), "dmax": dmax.strip(),
                      "pack": pack, "m": int(mm), "n": int(nn), "seed_after": [int(v) for v in seed.split(",")],
                      "d": arrays[dn], "a": arrays[an]})
    assert len(cases) == 12, len(cases)
    seedy = re.search(r"const SEEDY: \[u32; 4\] = \[([^\]]+)\]", src)
    return {"source": "src/lapack/families.rs:2014-2470 (dlatms_matches_the_reference_matrices)",
            "seed": [int(v) for v in seedy.group(1).split(",")], "cases": cases}


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/algebra_linear")
    root = pathlib.Path(sys.argv[1])
    fam = (root / "src/lapack/families.rs").read_text()
    out = HERE / "larnv_kat.json"
    out.write_text(json.dumps(extract_larnv(fam), indent=1) + "\n")
    print("wrote", out)
    out = HERE / "dlatms_kat.json"
    out.write_text(json.dumps(extract_dlatms(fam), indent=1) + "\n")
    print("wrote", out)
    col = (root / "src/sparse/faer/colamd.rs").read_text()
    out = HERE / "colamd_kat.json"
    out.write_text(json.dumps(extract_colamd(col)) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
