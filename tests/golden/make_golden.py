"""Extracts the reference crate's own known-answer vectors into JSON fixtures.

Run in a container where the reference sources are mounted (they are read as
text; nothing of the reference is executed):

    python tests/golden/make_golden.py /path/to/algebra_linear

Writes tests/golden/larnv_kat.json from the test
`larnv_matches_the_reference_stream` in src/lapack/families.rs:1176-1261,
whose values the reference captured from LAPACK 3.12.1's libtmglib (`dlarnv_`)
for seed [1988, 1989, 1990, 1991], n = 200: x[0..12], x[198..200] and the seed
after the call, for the Uniform, Symmetric and Normal distributions.
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


def main() -> None:
    root = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    fam = (root / "src/lapack/families.rs").read_text()
    out = HERE / "larnv_kat.json"
    out.write_text(json.dumps(extract_larnv(fam), indent=1) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
