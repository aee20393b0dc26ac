"""Weighted-mean isovalue reduction (warp-psr tests/test_isovalue_reduction.py:10-33)."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def blocked(values, weights):
    """The fixed order of the CUDA kernel: 1024-blocks, 256 lanes x 4, pairwise lanes."""
    total = mass = 0.0
    n = len(values)
    prods = (values * weights).astype(np.float64)
    w = weights.astype(np.float64)
    for b in range(0, n, 1024):
        tv = np.zeros(256)
        tw = np.zeros(256)
        for j in range(4):
            idx = b + np.arange(256) + 256 * j
            m = idx < n
            tv[m] += prods[idx[m]]
            tw[m] += w[idx[m]]
        stride = 128
        while stride >= 1:
            tv[:stride] = tv[:stride] + tv[stride:2 * stride]
            tw[:stride] = tw[:stride] + tw[stride:2 * stride]
            stride //= 2
        total += tv[0]
        mass += tw[0]
    return total / mass


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("count", [1, 1023, 1024, 1025, 65537, 1048577])
def test_weighted_mean_matches_accurate_sum(dtype, count):
    from warp_psr_b200 import ops
    rng = np.random.default_rng(235)
    values = rng.normal(size=count).astype(dtype)
    weights = np.exp2(rng.uniform(-20, 20, size=count)).astype(dtype)
    weights[::13] = 0
    weights[0] = 1
    products = values * weights
    expected = dtype(math.fsum(products) / math.fsum(weights))
    v, w = torch.from_numpy(values).cuda(), torch.from_numpy(weights).cuda()
    first = ops.isovalue(v, w).cpu().numpy()[0]
    second = ops.isovalue(v, w).cpu().numpy()[0]
    np.testing.assert_array_equal(first, second)
    if dtype == np.float64:
        np.testing.assert_allclose(first, expected, atol=3e-15, rtol=3e-14)
    else:
        np.testing.assert_allclose(first, expected, atol=3e-8, rtol=1e-7)
    assert first == dtype(blocked(values, weights))
