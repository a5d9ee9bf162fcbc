"""Host-side checks of the serving loop's requests, on the CPU: the loop
reads n^2 entries of a dense request's matrix and one value per pattern
entry of a sparse one straight from the caller's host arrays, so a request
whose arrays are too short is refused when it is built, before anything is
queued. Nothing here needs a GPU."""

import numpy as np
import pytest

from algebra_linear_b200.serve import DENSE, SPARSE, Request
from algebra_linear_b200.sparse import LuMethod, SparseLu


def test_dense_request_needs_an_n_by_n_matrix():
    r = Request.dense(np.eye(3).ravel(), np.ones(3))
    assert r.kind == DENSE and r.n == 3 and r.solution.shape == (3,)
    with pytest.raises(ValueError):
        Request.dense(np.ones(8), np.ones(3))
    with pytest.raises(ValueError):
        Request.dense(np.ones(16), np.ones(3))


def test_sparse_request_needs_the_pattern_sizes():
    cp, ri = [0, 2, 4], [0, 1, 0, 1]
    lu = SparseLu.analyze(cp, ri, LuMethod.supernodal())
    assert (lu.n, lu.nnz) == (2, 4)
    r = Request.sparse(lu, [4.0, 1.0, 1.0, 3.0], [1.0, 2.0])
    assert r.kind == SPARSE and r.n == 2
    with pytest.raises(ValueError):
        Request.sparse(lu, [4.0, 1.0, 1.0], [1.0, 2.0])
    with pytest.raises(ValueError):
        Request.sparse(lu, [4.0, 1.0, 1.0, 3.0], [1.0, 2.0, 3.0])
