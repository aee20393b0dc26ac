"""Adjoint of the reconstruction (warp-psr reconstruction_adjoint.py) against central finite
differences of the public forward, with the discrete assignments checked fixed — the
reference's tests/test_reconstruction_adjoint.py cases (base 0 / PSR with the constant mode,
base 1 SPSR, a finer depth, repeated base cycles with an early solve depth, exact
interpolation) plus direct-screening levels, repeated and combined backwards and degenerate
groups."""
import numpy as np
import pytest
import torch

from warp_psr_b200 import reconstruct, reconstruct_differentiable

pytestmark = pytest.mark.gpu

QUERIES = [[.1, .1, .1], [-.1, -.1, -.1], [.4, .7, .3], [.05, .3, -.2], [.9, 0., .1], [0., -.95, .2]]
SEED = [.7, -.5, .9, .3, -.4, .6]


def cloud(n=3000, seed=2026, jitter=.01):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    p = d * (1 + .1 * np.sin(3 * d[:, 0])[:, None]) + jitter * rng.normal(size=(n, 3))
    m = d + .05 * rng.normal(size=(n, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    return p, m


CASES = {
    "psr_base0_constant_mode": dict(depth=3, full_depth=0, base_depth=0, point_weight=0.0, iters=2,
                                    samples_per_node=.05),
    "spsr_base1": dict(depth=3, full_depth=1, base_depth=1, point_weight=2.0, iters=2, samples_per_node=.05),
    "spsr_base1_depth4": dict(depth=4, full_depth=1, base_depth=1, point_weight=2.0, iters=2, samples_per_node=.05),
    "cycles2_solve_depth2": dict(depth=3, full_depth=1, base_depth=1, point_weight=2.0, iters=2, samples_per_node=.05,
                                 base_v_cycles=2, solve_depth=2),
    "exact_interpolation": dict(depth=3, full_depth=1, base_depth=1, point_weight=2.0, iters=2, samples_per_node=.05,
                                exact_interpolation=True),
    "sliced_levels_screened": dict(depth=5, full_depth=3, point_weight=2.0, iters=3),
    "sliced_levels_psr": dict(depth=5, full_depth=3, point_weight=0.0, iters=3),
    "spsr_base0": dict(depth=4, full_depth=0, base_depth=0, point_weight=2.0, iters=2, samples_per_node=.5),
    # the default 8 sweeps take the unrolled reverse kernels
    "sliced_levels_8_sweeps": dict(depth=5, full_depth=3, point_weight=2.0, iters=8),
}


def fd_check(options, loss_kind, eps=1e-6, rtol=3e-5, atol=2e-7):
    p0, m0 = cloud()
    P = torch.tensor(p0, device="cuda", requires_grad=True)
    N = torch.tensor(m0, device="cuda", requires_grad=True)
    q = torch.tensor(QUERIES, device="cuda", dtype=torch.float64)
    seed = torch.tensor(SEED, device="cuda", dtype=torch.float64)
    res = reconstruct_differentiable(P, N, **options)
    if loss_kind == "value":
        v, _, valid = res.evaluate(q, centered=True)
        assert bool(valid.all())
        loss = (v * seed).sum()
    elif loss_kind == "gradient":
        _, g, _ = res.evaluate(q)
        loss = (g * torch.stack([seed, -seed, .5 * seed], 1)).sum()
    else:
        loss = res.iso_value
    loss.backward()
    reference = reconstruct(torch.tensor(p0, device="cuda"), torch.tensor(m0, device="cuda"), **options)
    keys = reference.field.keys.cpu().numpy()
    rng = np.random.default_rng(283)
    for array, grad in ((p0, P.grad), (m0, N.grad)):
        grad = grad.cpu().numpy()
        assert np.isfinite(grad).all()
        direction = rng.normal(size=array.shape)
        losses = []
        for sign in (1, -1):
            moved = array + sign * eps * direction
            pp, mm = (moved, m0) if array is p0 else (p0, moved)
            r = reconstruct(torch.tensor(pp, device="cuda"), torch.tensor(mm, device="cuda"), **options)
            np.testing.assert_array_equal(r.field.keys.cpu().numpy(), keys)  # tree unchanged
            if loss_kind == "value":
                v, _, _ = r.evaluate(q)
                losses.append(float(((v - r.iso_value) * seed).sum()))
            elif loss_kind == "gradient":
                _, g, _ = r.evaluate(q)
                losses.append(float((g * torch.stack([seed, -seed, .5 * seed], 1)).sum()))
            else:
                losses.append(r.iso_value)
        fd = (losses[0] - losses[1]) / (2 * eps)
        np.testing.assert_allclose(float((grad * direction).sum()), fd, rtol=rtol, atol=atol)


@pytest.mark.parametrize("case", sorted(CASES))
def test_point_and_normal_vjp_value_loss(case):
    fd_check(CASES[case], "value")


@pytest.mark.parametrize("case", ["spsr_base1", "sliced_levels_screened", "psr_base0_constant_mode"])
def test_point_and_normal_vjp_spatial_gradient_loss(case):
    fd_check(CASES[case], "gradient")


@pytest.mark.parametrize("case", ["spsr_base1", "sliced_levels_screened", "cycles2_solve_depth2"])
def test_point_and_normal_vjp_isovalue(case):
    # isovalue derivatives are small; their FD noise floor sets the absolute budget
    fd_check(CASES[case], "iso", atol=1e-6)


def test_float32_matches_float64_gradient():
    """float32 inputs: the float32 reverse pass agrees with the float64 one (FD in float32
    would move samples across bins, so the float64 gradient is the check)."""
    p0, m0 = cloud()
    q = torch.tensor(QUERIES, device="cuda")
    seed = torch.tensor(SEED, device="cuda")
    grads = {}
    for dtype in (torch.float32, torch.float64):
        P = torch.tensor(p0, device="cuda", dtype=dtype, requires_grad=True)
        N = torch.tensor(m0, device="cuda", dtype=dtype, requires_grad=True)
        res = reconstruct_differentiable(P, N, **CASES["spsr_base1_depth4"])
        v, _, _ = res.evaluate(q.to(dtype), centered=True)
        (v * seed.to(dtype)).sum().backward()
        grads[dtype] = (P.grad.double().cpu().numpy(), N.grad.double().cpu().numpy())
    rng = np.random.default_rng(5)
    for a32, a64 in zip(grads[torch.float32], grads[torch.float64]):
        d = rng.normal(size=a64.shape)
        np.testing.assert_allclose((a32 * d).sum(), (a64 * d).sum(), rtol=2e-2, atol=2e-3)


def test_mixed_precision_gradient_matches_float64():
    p0, m0 = cloud()
    q = torch.tensor(QUERIES, device="cuda", dtype=torch.float64)
    seed = torch.tensor(SEED, device="cuda", dtype=torch.float64)
    out = []
    for precision in ("input", "mixed"):
        P = torch.tensor(p0, device="cuda", requires_grad=True)
        N = torch.tensor(m0, device="cuda", requires_grad=True)
        res = reconstruct_differentiable(P, N, precision=precision, **CASES["sliced_levels_screened"])
        v, _, _ = res.evaluate(q, centered=True)
        (v * seed).sum().backward()
        out.append(torch.cat([P.grad.flatten(), N.grad.flatten()]))
    scale = out[0].abs().max()
    assert float((out[1] - out[0]).abs().max() / scale) < 1e-5


def test_repeated_and_combined_backward():
    p0, m0 = cloud()
    P = torch.tensor(p0, device="cuda", requires_grad=True)
    N = torch.tensor(m0, device="cuda", requires_grad=True)
    q = torch.tensor([[.1, .1, .1]], device="cuda", dtype=torch.float64)
    a = reconstruct_differentiable(P, N, depth=3, full_depth=1, samples_per_node=.05, iters=2)
    b = reconstruct_differentiable(P, N, depth=3, full_depth=1, samples_per_node=.05, iters=3)
    va, _, _ = a.evaluate(q, centered=True)
    vb, _, _ = b.evaluate(q, centered=True)
    ga = torch.autograd.grad(va.sum(), (P, N), retain_graph=True)
    gb = torch.autograd.grad(vb.sum(), (P, N), retain_graph=True)
    gab = torch.autograd.grad(va.sum() + vb.sum(), (P, N), retain_graph=True)
    again = torch.autograd.grad(va.sum() + vb.sum(), (P, N), retain_graph=True)
    for x, y, z, w in zip(ga, gb, gab, again):
        torch.testing.assert_close(z, x + y, rtol=1e-10, atol=1e-11)
        # repeatable up to the summation order of atomic accumulations
        torch.testing.assert_close(w, z, rtol=1e-10, atol=1e-11)
    np.testing.assert_array_equal(P.detach().cpu().numpy(), p0)


def test_omitted_nan_normal_and_positions_only():
    p0, m0 = cloud()
    m0 = m0.copy()
    m0[0] = np.nan
    P = torch.tensor(p0, device="cuda", requires_grad=True)
    N = torch.tensor(m0, device="cuda", requires_grad=True)
    res = reconstruct_differentiable(P, N, depth=3, full_depth=1, iters=2)
    v, _, _ = res.evaluate(torch.tensor([[.1, .1, .1]], device="cuda", dtype=torch.float64), centered=True)
    v.sum().backward()
    assert torch.isfinite(P.grad).all() and torch.isfinite(N.grad).all()
    assert torch.equal(N.grad[0], torch.zeros(3, device="cuda", dtype=torch.float64))
    P2 = torch.tensor(p0, device="cuda", requires_grad=True)
    N2 = torch.tensor(m0, device="cuda")
    res = reconstruct_differentiable(P2, N2, depth=3, full_depth=1, iters=2)
    v, _, _ = res.evaluate(torch.tensor([[.1, .1, .1]], device="cuda", dtype=torch.float64), centered=True)
    v.sum().backward()
    assert torch.isfinite(P2.grad).all() and N2.grad is None


def test_reconstruct_many_single_process():
    from warp_psr_b200 import replicas
    p0, m0 = cloud()
    clouds = [(torch.tensor(p0, device="cuda"), torch.tensor(m0, device="cuda"))] * 2
    out = replicas.reconstruct_many(clouds, depth=4, full_depth=2)
    assert [o[0] for o in out] == [0, 1] and out[0][1] == out[1][1]
