"""algebra_linear_b200: a B200 (sm_100a) LU solver behind the API of the
cpmech/algebra_linear crate's dense and sparse LU path.

The compute lives in libalgebra_linear_gpu.so (CUDA, built in-tree by
`python -m algebra_linear_b200.build`); the Python modules mirror the
reference's functions over its C ABI (include/algebra_linear_gpu.h).
"""

__all__ = ["lapack"]
