"""Ordered sliced Gauss-Seidel: CUDA (dependency-scheduled) vs the oracle's sequential order.

Bitwise equality, as warp-psr requires of its wavefront graphs
(tests/test_relaxation.py:110-147).
"""
import numpy as np
import pytest
import torch

import oracle
from relax_cases import local_system

pytestmark = pytest.mark.gpu


def gpu_relax(keys, offsets, columns, values, b, x, depth, iters):
    from warp_psr_b200 import ops
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    xx = t(x)
    ops.relax_sliced(t(keys), depth, t(offsets), t(columns), t(values), t(b), xx, iters)
    return xx.cpu().numpy()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("iters", [0, 1, 3, 8])
@pytest.mark.parametrize("pattern", ["full", "sparse", "empty_slices"])
def test_matches_serialized_updates_for_arbitrary_local_matrices(dtype, iters, pattern):
    keys, offsets, columns, values, b, x = local_system(pattern, dtype=dtype)
    expected = oracle.relax_sliced(keys, 3, offsets, columns, values, b, x, iters)
    actual = gpu_relax(keys, offsets, columns, values, b, x, 3, iters)
    np.testing.assert_array_equal(actual, expected)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("seed", [0, 1])
def test_many_concurrent_slices(dtype, seed):
    # 33^3 nodes at depth 5: 33 slices x 8 visits keep the whole persistent grid busy.
    keys, offsets, columns, values, b, x = local_system("random", size=33, depth=5, dtype=dtype, seed=seed)
    expected = oracle.relax_sliced(keys, 5, offsets, columns, values, b, x, 8)
    actual = gpu_relax(keys, offsets, columns, values, b, x, 5, 8)
    np.testing.assert_array_equal(actual, expected)


def test_repeated_calls_are_deterministic():
    keys, offsets, columns, values, b, x = local_system("full", size=17, depth=4, dtype=np.float32)
    first = gpu_relax(keys, offsets, columns, values, b, x, 4, 8)
    for _ in range(3):
        np.testing.assert_array_equal(gpu_relax(keys, offsets, columns, values, b, x, 4, 8), first)


def test_rejects_rows_wider_than_the_stencil():
    from warp_psr_b200 import ops
    keys, offsets, columns, values, b, x = local_system("full", dtype=np.float32)
    bad = columns.copy()
    bad[0] = len(keys) + 5
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    with pytest.raises(ValueError, match="out of range"):
        ops.relax_sliced(t(keys), 3, t(offsets), t(bad), t(values), t(b), t(x), 2)
