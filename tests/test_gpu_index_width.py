"""The 32-bit neighbour-index rows of the ordered relaxation (taken when a (slice, colour)
group reaches 2^15 rows, i.e. on very large levels) forced on small cases with
PSR_INDEX_WIDTH=32: the relaxation stays bitwise the oracle's, and reconstructions and
their reverse passes agree with the 16-bit path."""
import numpy as np
import pytest
import torch

import oracle
from relax_cases import local_system
from test_gpu_adjoint import CASES, QUERIES, SEED, cloud
from test_gpu_relaxation import gpu_relax

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("pattern,size,depth,iters", [("full", 9, 3, 3), ("sparse", 9, 3, 8), ("random", 33, 5, 8)])
def test_relaxation_with_32_bit_rows_matches_oracle(monkeypatch, dtype, pattern, size, depth, iters):
    monkeypatch.setenv("PSR_INDEX_WIDTH", "32")
    keys, offsets, columns, values, b, x = local_system(pattern, size=size, depth=depth, dtype=dtype)
    expected = oracle.relax_sliced(keys, depth, offsets, columns, values, b, x, iters)
    np.testing.assert_array_equal(gpu_relax(keys, offsets, columns, values, b, x, depth, iters), expected)


@pytest.mark.parametrize("precision", ["input", "mixed"])
def test_reconstruction_with_32_bit_rows_is_identical(monkeypatch, precision):
    from warp_psr_b200 import reconstruct
    p0, m0 = cloud()
    opts = dict(depth=6, full_depth=3, point_weight=2.0, precision=precision)
    runs = []
    for width in (None, "32"):
        if width:
            monkeypatch.setenv("PSR_INDEX_WIDTH", width)
        r = reconstruct(torch.tensor(p0, device="cuda"), torch.tensor(m0, device="cuda"), **opts)
        runs.append((r.field.coefficients.cpu().numpy(), r.iso_value))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]


def test_reverse_pass_with_32_bit_rows_agrees(monkeypatch):
    from warp_psr_b200 import reconstruct_differentiable
    p0, m0 = cloud()
    q = torch.tensor(QUERIES, device="cuda", dtype=torch.float64)
    seed = torch.tensor(SEED, device="cuda", dtype=torch.float64)
    grads = []
    for width in (None, "32"):
        if width:
            monkeypatch.setenv("PSR_INDEX_WIDTH", width)
        P = torch.tensor(p0, device="cuda", requires_grad=True)
        N = torch.tensor(m0, device="cuda", requires_grad=True)
        res = reconstruct_differentiable(P, N, **CASES["sliced_levels_8_sweeps"])
        v, _, _ = res.evaluate(q, centered=True)
        (v * seed).sum().backward()
        grads.append(torch.cat([P.grad.flatten(), N.grad.flatten()]))
    # equal up to the summation order of atomic accumulations
    torch.testing.assert_close(grads[1], grads[0], rtol=1e-10, atol=1e-13)
