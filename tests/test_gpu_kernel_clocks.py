"""Kernel clocks (psr_kernel_clocks): the per-kernel device times and algorithmic bytes that
the benchmark's per-kernel roofline reads.  Off by default; on for launches issued while
PSR_KERNEL_CLOCKS=1, and reading them clears the totals.  The byte models are checked
against the launch's own sizes: one row visit of the mixed-precision ordered relaxation is
27 float32 operator values, b and x read and x written in float64, a 4-byte row id and a
float64 visit record (144 B with the record the differentiable forward keeps).
"""
import pytest
import torch

from warp_psr_b200 import _lib, clouds, reconstruct, reconstruct_differentiable

pytestmark = pytest.mark.gpu

OPTS = dict(depth=7, full_depth=4, point_weight=2.0)


def cloud():
    p, n = clouds.sphere(20000)
    return torch.tensor(p, dtype=torch.float32, device="cuda"), torch.tensor(n, dtype=torch.float32, device="cuda")


def test_clocks_are_off_by_default(monkeypatch):
    monkeypatch.delenv("PSR_KERNEL_CLOCKS", raising=False)
    _lib.kernel_clocks()
    p, n = cloud()
    reconstruct(p, n, precision="mixed", **OPTS)
    torch.cuda.synchronize()
    assert _lib.kernel_clocks() == []


def test_clocks_cover_forward_and_reverse(monkeypatch):
    monkeypatch.setenv("PSR_KERNEL_CLOCKS", "1")
    _lib.kernel_clocks()
    p, n = cloud()
    P = p.clone().requires_grad_(True)
    res = reconstruct_differentiable(P, n, precision="mixed", **OPTS)
    v, _, _ = res.evaluate(p[:64].double(), centered=True)
    torch.nan_to_num(v).sum().backward()
    torch.cuda.synchronize()
    clocks = {c["kernel"]: c for c in _lib.kernel_clocks()}
    for name in ("assemble_sliced_kernel", "cross_apply_kernel", "normal_stencil_dense_kernel",
                 "relax_colors_shared_kernel", "strip_gs_kernel (forward)", "strip_gs_kernel (reverse)",
                 "normal_stencil_reverse_kernel", "level_rows_reverse_kernel", "screening_points_reverse_kernel"):
        assert name in clocks, name
        c = clocks[name]
        assert c["launches"] > 0 and c["ms"] > 0 and c["bytes"] > 0 and c["units"] > 0, c
    fwd = clocks["strip_gs_kernel (forward)"]
    r = res.result
    # the sliced levels' row visits: rows x 8 sweeps, as the result's diagnostics count them
    assert fwd["units"] == r.diagnostics["relax_row_visits"]
    assert fwd["bytes"] == pytest.approx(fwd["units"] * (27 * 4 + 3 * 8 + 4 + 8))
    assert fwd["launches"] == r.diagnostics["relax_launches"]
    assert _lib.kernel_clocks() == []  # read once, then cleared
