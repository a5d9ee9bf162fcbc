"""The device-tensor wrappers check their operands before any launch: the
kernels address the packed systems (batched) and the matrix and right-hand
sides (mixed) through raw pointers, so a tensor on the wrong device, of the
wrong type, not contiguous or too short is refused with a TypeError instead
of letting a launch touch memory past it. The checks run before the library
is called, so they are tested here without a GPU."""

import types

import pytest
import torch

from algebra_linear_b200 import batched, mixed


def test_batched_operand_check():
    ok = torch.zeros(10, dtype=torch.float64)
    with pytest.raises(TypeError, match="CUDA"):
        batched._dev_tensor(ok, torch.float64, 10, "a")  # a host tensor
    with pytest.raises(TypeError):
        batched._dev_tensor(ok.numpy(), torch.float64, 10, "a")


def test_batched_plan_checks_reach_and_type_before_launching():
    # a plan's operand check without a device: the sizes it demands come from
    # the offsets (the last system's end), the types from the kernels
    plan = object.__new__(batched.BatchPlan)
    plan.count, plan._a_need, plan._b_need = 2, 13, 5
    a, b = torch.zeros(13, dtype=torch.float64), torch.zeros(5, dtype=torch.float64)
    info = torch.zeros(2, dtype=torch.int32)
    with pytest.raises(TypeError, match="a must be"):
        plan.solve(a, b, info)
    with pytest.raises(TypeError, match="a must be"):
        plan.solve(a[:12], b, info)


def test_mixed_device_solve_checks_before_launching():
    ctx = types.SimpleNamespace(handle=None)
    n = 4
    with pytest.raises(TypeError, match="A must be"):
        mixed.dgesv_mixed_dev(ctx, torch.zeros(n * n, dtype=torch.float64), torch.zeros(n, dtype=torch.float64), n)
    with pytest.raises(TypeError, match="A must be"):
        mixed.dgesv_mixed_dev(ctx, torch.zeros(n * n, dtype=torch.float32), torch.zeros(n, dtype=torch.float64), n)


def test_sparse_device_calls_check_before_launching():
    from algebra_linear_b200.sparse import LuMethod, SparseLu

    lu = SparseLu.analyze([0, 2, 4], [0, 1, 0, 1], LuMethod.supernodal())
    with pytest.raises(TypeError, match="values must be"):
        lu.factorize_dev(torch.tensor([4.0, 1.0, 1.0, 3.0], dtype=torch.float64))  # a host tensor
    with pytest.raises(TypeError, match="b must be"):
        lu.solve_dev(torch.ones(2, dtype=torch.float64))
