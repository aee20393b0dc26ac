"""Paths of the ordered relaxation that only very large levels take, forced on small cases
through test overrides and compared bit for bit with the oracle's sequential order and with
the default path:

* PSR_RELAX_ROW_CAP=0 -- tasks whose operator rows do not fit shared memory read them from
  global memory (unstaged);
* PSR_RELAX_FOOTPRINT_LIMIT -- a strip whose footprint exceeds the 16-bit index range makes
  the launch narrow its strips (doubling their count) until every footprint fits.  On the
  torus fixture's depth-6 level the default 4 strips have a 912-entry footprint, 8 strips
  740, 16 strips 596 and 32 strips 504, so a limit of 600 narrows the strips 4 -> 16 (or 32);
* PSR_RELAX_KERNEL=pipeline -- the cluster pipelines (one 8-CTA cluster per visit), which the
  library leaves off by default (slower than the dynamic scheduler on the benchmark level).
"""
import numpy as np
import pytest
import torch

import oracle
from kat_util import BY_NAME, inputs, options
from relax_cases import local_system
from test_gpu_relaxation import gpu_relax

pytestmark = pytest.mark.gpu

OVERRIDES = [("PSR_RELAX_ROW_CAP", "0"), ("PSR_RELAX_FOOTPRINT_LIMIT", "600"), ("PSR_RELAX_KERNEL", "pipeline"),
             ("PSR_RELAX_FOOTPRINT_LIMIT", "1")]
FORCED = OVERRIDES[:3]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("name,value", FORCED)
@pytest.mark.parametrize("pattern,size,depth,iters", [("full", 9, 3, 3), ("random", 33, 5, 8)])
def test_forced_relaxation_paths_match_oracle(monkeypatch, dtype, name, value, pattern, size, depth, iters):
    monkeypatch.setenv(name, value)
    keys, offsets, columns, values, b, x = local_system(pattern, size=size, depth=depth, dtype=dtype, seed=3)
    expected = oracle.relax_sliced(keys, depth, offsets, columns, values, b, x, iters)
    np.testing.assert_array_equal(gpu_relax(keys, offsets, columns, values, b, x, depth, iters), expected)


def test_footprint_beyond_every_strip_count_is_an_error(monkeypatch):
    """A footprint that no strip count brings under the limit raises (never a wrong answer)."""
    from warp_psr_b200 import _lib
    monkeypatch.setenv(*OVERRIDES[3])
    keys, offsets, columns, values, b, x = local_system("full", dtype=np.float64)
    with pytest.raises(_lib.PSRError, match="16-bit index range"):
        gpu_relax(keys, offsets, columns, values, b, x, 3, 2)


@pytest.mark.parametrize("precision", ["double", "float", "mixed"])
@pytest.mark.parametrize("name,value", FORCED)
def test_forced_paths_reconstruct_identically(monkeypatch, precision, name, value):
    from warp_psr_b200 import reconstruct
    kat = BY_NAME["torus"]
    p, n = inputs(kat)
    dt = np.float64 if precision == "double" else np.float32
    opts = dict(options(kat["params"]), precision="mixed" if precision == "mixed" else "input")
    P, N = torch.from_numpy(p.astype(dt)).cuda(), torch.from_numpy(n.astype(dt)).cuda()
    default = reconstruct(P, N, **opts)
    monkeypatch.setenv(name, value)
    forced = reconstruct(P, N, **opts)
    np.testing.assert_array_equal(forced.field.coefficients.cpu().numpy(), default.field.coefficients.cpu().numpy())
    assert forced.iso_value == default.iso_value
    if precision != "mixed":
        ref = oracle.OracleResult(p.astype(dt), n.astype(dt), **options(kat["params"]))
        np.testing.assert_array_equal(forced.field.keys.cpu().numpy(), ref.keys)
        np.testing.assert_array_equal(forced.field.coefficients.cpu().numpy(), ref.coefficients)


@pytest.mark.parametrize("precision", ["input", "mixed"])
def test_window_reverse_normal_stencils_match_generic(monkeypatch, precision):
    """The reverse normal-load stencils for same-depth and one-coarser test functions (lock-step
    window kernels) give the generic kernel's gradients (PSR_NORMAL_REVERSE=generic forces the
    generic kernel for every window).  The comparison is to rounding, not bitwise: other
    stages of the reverse pass add with float64 atomics (the cross-term adjoint), so two
    passes over the same inputs already differ in the last bits."""
    from warp_psr_b200 import clouds, reconstruct_differentiable
    p0, n0 = clouds.sphere(20000)
    q = torch.tensor(p0[::97], dtype=torch.float64, device="cuda")
    grads = []
    for mode in (None, "generic"):
        if mode:
            monkeypatch.setenv("PSR_NORMAL_REVERSE", mode)
        P = torch.tensor(p0, dtype=torch.float64, device="cuda", requires_grad=True)
        N = torch.tensor(n0, dtype=torch.float64, device="cuda", requires_grad=True)
        res = reconstruct_differentiable(P, N, depth=7, full_depth=4, point_weight=2.0, precision=precision)
        v, _, _ = res.evaluate(q, centered=True)
        torch.nan_to_num(v).square().sum().backward()
        grads.append((P.grad.cpu().numpy(), N.grad.cpu().numpy()))
    for a, b in zip(grads[0], grads[1]):
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-12 * np.abs(b).max())
