"""Runs the oracle (the C++ restatement of the reference's supernodal LU,
supernodal_lu.rs:118-533) on sparse workloads near the benchmark sizes and
stores what the GPU parity tests compare against, so the tests need not
re-run the oracle (minutes to hours of one host core at these sizes):

    python tests/golden/make_sparse_golden.py [case ...]

Cases: 2-D 5-point convection-diffusion patterns (the serving workload's
300 x 300 one, n = 90 000, and 150 x 150) and the 20^3 7-point grid
(n = 8 000); each in two rounds: the values of the benchmark's generator
(diagonal 6 + 0.1 U(0,1), neighbours -1, x-neighbours -1 -/+ 0.3 U(0,1),
DLARNV seed [1988, 1989, 1990, 1991]) and a 1 % multiplicative
refactorization of them. The column order and supernode partition are the
library's host analysis (itself pinned on the reference's COLAMD outputs and
column counts).

Per case and round, tests/golden/sparse_<case>.npz holds: the SHA-256 of the
oracle's row permutation (int64) and its first 64 entries; nnz(L), nnz(U)
and flops_estimate; the oracle's solution x at every `stride`-th position for
the round's right-hand side (round 0: the DLARNV Symmetric stream from seed
[3, 5, 7, 9]; round 1: all ones).
"""

from __future__ import annotations

import hashlib
import multiprocessing as mp
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
CASES = {"grid300x300": (300, 300, 1), "grid150x150": (150, 150, 1), "grid20x20x20": (20, 20, 20)}
SEED = [1988, 1989, 1990, 1991]
RHS_SEED = [3, 5, 7, 9]
SAMPLES = 4000


def stride_of(n: int) -> int:
    return max(1, n // SAMPLES)


def round_values(kind, rnd: int):
    from oracle import sparse as osp

    v, s = osp.convection_diffusion_values(kind, SEED)
    if rnd == 1:
        v, _ = osp.perturb(v, s)
    return v


def round_rhs(n: int, rnd: int):
    from oracle import dense

    if rnd == 0:
        b, _ = dense.larnv("Symmetric", list(RHS_SEED), n)
        return b
    return np.ones(n)


def _job(args):
    name, rnd = args
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    from algebra_linear_b200.sparse import LuMethod, SparseLu
    from oracle import sparse as osp

    cp, ri, kind = osp.grid_pattern(*CASES[name])
    n = len(cp) - 1
    v = round_values(kind, rnd)
    sym = SparseLu.analyze(cp, ri, LuMethod.supernodal()).symbolic()
    t0 = time.perf_counter()
    f = osp.Factors(n, cp, ri, v, sym["col_perm"], sym["col_perm_inv"], sym["supernode_ptr"])
    assert f.status == 0, f.status
    x = f.solve(round_rhs(n, rnd))
    rp = f.row_perm.astype(np.int64)
    out = {
        f"r{rnd}_row_perm_sha256": np.frombuffer(hashlib.sha256(rp.tobytes()).digest(), np.uint8),
        f"r{rnd}_row_perm_head": rp[:64],
        f"r{rnd}_counts": np.array([f.nnz_l, f.nnz_u, f.flops_estimate()], np.int64),
        f"r{rnd}_x": x[::stride_of(n)].copy(),
        f"r{rnd}_oracle_s": np.array(time.perf_counter() - t0),
    }
    print(f"{name} round {rnd}: oracle {time.perf_counter() - t0:.1f} s, nnz_l {f.nnz_l}, nnz_u {f.nnz_u}",
          flush=True)
    return name, out


def main() -> None:
    names = sys.argv[1:] or list(CASES)
    jobs = [(nm, r) for nm in names for r in (0, 1)]
    done = {}
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        # each case is written as soon as both of its rounds are done
        for name, out in pool.imap_unordered(_job, jobs):
            done.setdefault(name, {}).update(out)
            if len(done[name]) == 2 * len(out):
                _write(name, done[name])


def _write(nm, rounds):
    arrays = {"dims": np.array(CASES[nm], np.int64), "stride": np.array(stride_of(int(np.prod(CASES[nm]))))}
    arrays.update(rounds)
    path = HERE / f"sparse_{nm}.npz"
    np.savez_compressed(path, **arrays)
    print("wrote", path, flush=True)


if __name__ == "__main__":
    main()
