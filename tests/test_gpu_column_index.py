"""Paths that only large inputs take, forced on small cases: the hashed column index (used
for depths beyond the dense per-depth tables, above 12; PSR_COLUMN_INDEX=hash) and the base
relaxation with x in global memory (base levels too large for shared memory;
PSR_BASE_RELAX=global) or with x but not the operator rows in shared memory (base levels
above ~790 rows; PSR_BASE_RELAX=shared).  Reconstructions, field evaluation and the reverse
pass agree with the default paths."""
import numpy as np
import pytest
import torch

from test_gpu_adjoint import CASES, QUERIES, SEED, cloud

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["input", "mixed"])
def test_reconstruction_with_hashed_columns_is_identical(monkeypatch, precision):
    from warp_psr_b200 import reconstruct
    p0, m0 = cloud()
    q = torch.tensor(QUERIES, device="cuda", dtype=torch.float64)
    runs = []
    for mode in (None, "hash"):
        if mode:
            monkeypatch.setenv("PSR_COLUMN_INDEX", mode)
        r = reconstruct(torch.tensor(p0, device="cuda"), torch.tensor(m0, device="cuda"), depth=6, full_depth=3,
                        point_weight=2.0, precision=precision)
        v, g, ok = r.evaluate(q)
        runs.append((r.field.coefficients.cpu().numpy(), r.iso_value, v.cpu().numpy(), g.cpu().numpy()))
    for a, b in zip(runs[0], runs[1]):
        np.testing.assert_array_equal(a, b)


def test_reverse_pass_with_hashed_columns_agrees(monkeypatch):
    from warp_psr_b200 import reconstruct_differentiable
    p0, m0 = cloud()
    q = torch.tensor(QUERIES, device="cuda", dtype=torch.float64)
    seed = torch.tensor(SEED, device="cuda", dtype=torch.float64)
    grads = []
    for mode in (None, "hash"):
        if mode:
            monkeypatch.setenv("PSR_COLUMN_INDEX", mode)
        P = torch.tensor(p0, device="cuda", requires_grad=True)
        N = torch.tensor(m0, device="cuda", requires_grad=True)
        res = reconstruct_differentiable(P, N, **CASES["sliced_levels_screened"])
        v, _, _ = res.evaluate(q, centered=True)
        (v * seed).sum().backward()
        grads.append(torch.cat([P.grad.flatten(), N.grad.flatten()]))
    # equal up to the summation order of atomic accumulations
    torch.testing.assert_close(grads[1], grads[0], rtol=1e-10, atol=1e-13)


@pytest.mark.parametrize("forced", ["global", "shared"])
@pytest.mark.parametrize("case", ["spsr_base1_depth4", "psr_base0_constant_mode"])
def test_base_relaxation_in_global_memory_is_identical(monkeypatch, case, forced):
    """PSR_BASE_RELAX=global (x in global memory) and =shared (x in shared memory, operator
    rows from global memory): the base levels' colour relaxation gives the default path's
    result (x and the operator rows staged in shared memory) bit for bit."""
    from warp_psr_b200 import reconstruct
    p0, m0 = cloud()
    opts = {k: v for k, v in CASES[case].items()}
    runs = []
    for mode in (None, forced):
        if mode:
            monkeypatch.setenv("PSR_BASE_RELAX", mode)
        r = reconstruct(torch.tensor(p0, device="cuda"), torch.tensor(m0, device="cuda"), **opts)
        runs.append((r.field.coefficients.cpu().numpy(), r.iso_value))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]


@pytest.mark.parametrize("forced", ["global", "shared"])
def test_reverse_base_relaxation_in_global_memory_agrees(monkeypatch, forced):
    from warp_psr_b200 import reconstruct_differentiable
    p0, m0 = cloud()
    q = torch.tensor(QUERIES, device="cuda", dtype=torch.float64)
    seed = torch.tensor(SEED, device="cuda", dtype=torch.float64)
    grads = []
    for mode in (None, forced):
        if mode:
            monkeypatch.setenv("PSR_BASE_RELAX", mode)
        P = torch.tensor(p0, device="cuda", requires_grad=True)
        N = torch.tensor(m0, device="cuda", requires_grad=True)
        res = reconstruct_differentiable(P, N, **CASES["spsr_base1_depth4"])
        v, _, _ = res.evaluate(q, centered=True)
        (v * seed).sum().backward()
        grads.append(torch.cat([P.grad.flatten(), N.grad.flatten()]))
    torch.testing.assert_close(grads[1], grads[0], rtol=1e-10, atol=1e-13)
