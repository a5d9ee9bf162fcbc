"""The small sparse systems of the reference's supernodal tests
(src/sparse/faer/supernodal_lu.rs:541-662), restated for the tests here:
tridiagonal, arrow and 5-point grid patterns in CSC with sorted rows, the
diagonal/off-diagonal value fill, and the diagonally dominant system drawn
from the tests' 64-bit LCG (seed 0x1234_5678)."""

import numpy as np

MASK = (1 << 64) - 1


def from_cols(cols):
    """supernodal_lu.rs:541-552: each column's rows sorted and deduplicated."""
    cp, ri = [0], []
    for c in cols:
        ri.extend(sorted(set(c)))
        cp.append(len(ri))
    return cp, ri


def tridiag(n):
    """supernodal_lu.rs:554-569."""
    return from_cols([[j] + ([j - 1] if j > 0 else []) + ([j + 1] if j + 1 < n else []) for j in range(n)])


def arrow(n):
    """supernodal_lu.rs:571-582: a full first column, then [0, j]."""
    return from_cols([list(range(n)) if j == 0 else [0, j] for j in range(n)])


def grid(rows, cols_n):
    """supernodal_lu.rs:584-607: node i = r * cols_n + c and its four
    neighbours (this numbering is not the one of the oracle's grid_pattern)."""
    cols = []
    for i in range(rows * cols_n):
        r, c = divmod(i, cols_n)
        v = [i]
        if r > 0:
            v.append((r - 1) * cols_n + c)
        if r + 1 < rows:
            v.append((r + 1) * cols_n + c)
        if c > 0:
            v.append(r * cols_n + c - 1)
        if c + 1 < cols_n:
            v.append(r * cols_n + c + 1)
        cols.append(v)
    return from_cols(cols)


def diagonal_values(cp, ri, diag, off):
    """supernodal_lu.rs:644-652."""
    n = len(cp) - 1
    return np.array([diag if ri[k] == j else off for j in range(n) for k in range(cp[j], cp[j + 1])])


def diagonally_dominant(n, seed):
    """supernodal_lu.rs:609-642: per column the diagonal and two rows drawn
    from the LCG state * 6364136223846793005 + 1442695040888963407 (mod 2^64),
    next() = (state >> 33) / 2^31; diagonal values 8 + next(), the others
    0.5 - next(), drawn column by column after the pattern."""
    state = seed

    def nxt():
        nonlocal state
        state = (state * 6364136223846793005 + 1442695040888963407) & MASK
        return (state >> 33) / 2147483648.0

    cols = []
    for j in range(n):
        c = [j]
        for _ in range(2):
            i = int(nxt() * 1e6) % n
            if i != j:
                c.append(i)
        cols.append(c)
    cp, ri, v = [0], [], []
    for j in range(n):
        for i in sorted(set(cols[j])):
            ri.append(i)
            v.append(8.0 + nxt() if i == j else 0.5 - nxt())
        cp.append(len(ri))
    return cp, ri, np.array(v)


def dense(cp, ri, v):
    n = len(cp) - 1
    a = np.zeros((n, n))
    for j in range(n):
        for k in range(cp[j], cp[j + 1]):
            a[ri[k], j] = v[k]
    return a


# supernodal_lu.rs:691-706
STRUCTURED = [(1, tridiag(1)), (4, grid(2, 2)), (6, grid(2, 3)), (9, grid(3, 3)), (5, tridiag(5)), (8, arrow(8)),
              (12, grid(3, 4))]


def close(got, want, tol):
    """supernodal_lu.rs:664-669: |g - w| <= tol (1 + |w|) entry by entry."""
    got, want = np.asarray(got), np.asarray(want)
    return got.shape == want.shape and bool(np.all(np.abs(got - want) <= tol * (1.0 + np.abs(want))))
