"""Full CUDA reconstruction vs the CPU oracle and the reference's known answers.

Integer results (tree keys, group keys, normal record keys) must be identical.  Floating
point stages follow the same arithmetic in the same order on both sides: float32 runs must
be bitwise equal; float64 runs may differ by a few ulps, because two library transcendentals
(the normal scale's pow, samples.py:75-79, and the splat depths' log, density.py:32-35) can
differ in their last bit between CUDA and glibc.
"""
import numpy as np
import pytest
import torch

import oracle
from kat_util import KATS, inputs, iso_tolerance, options, sha

pytestmark = pytest.mark.gpu

# Relative tolerances of floating-point stage parity (oracle vs CUDA, same precision).
STAGE_RTOL = {"float": 0.0, "double": 1e-13}


def _close(a, b, rtol, what):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if not a.size:
        return
    scale = max(np.abs(b).max(), 1e-30)
    err = np.abs(a - b).max()
    assert err <= rtol * scale, f"{what}: max |diff| {err:.3e} > {rtol:.1e} * {scale:.3e}"


def run_gpu(kat, **extra):
    from warp_psr_b200 import reconstruct
    p, n = inputs(kat)
    return p, n, reconstruct(torch.from_numpy(p).cuda(), torch.from_numpy(n).cuda(), keep_stages=True,
                             **options(kat["params"]), **extra)


@pytest.mark.parametrize("kat", KATS, ids=[k["name"] for k in KATS])
def test_reconstruction_matches_oracle_and_fixture(kat):
    p, n, g = run_gpu(kat)
    prec = kat["params"]["precision"]
    ref = oracle.OracleResult(p, n, **options(kat["params"]))
    rtol = STAGE_RTOL[prec]
    stage = g.diagnostics["stage"]
    fdt = torch.float64 if prec == "double" else torch.float32
    # A1 groups: keys and first indices exact, sums in the same order
    assert np.array_equal(stage("group_keys", torch.int64).cpu().numpy(), ref.stage("group_keys", np.int64))
    assert np.array_equal(stage("group_first", torch.int32).cpu().numpy(), ref.stage("group_first", np.int32))
    npdt = np.float64 if prec == "double" else np.float32
    for name in ("group_sums", "group_normal_sums", "group_weights", "transform"):
        _close(stage(name, fdt).cpu().numpy(), ref.stage(name, npdt), rtol, name)
    # A2 splat depths, A3 normal records
    _close(stage("depths_and_weights", fdt).cpu().numpy(), ref.stage("depths_and_weights", npdt), rtol, "dw")
    assert np.array_equal(stage("normal_keys", torch.int64).cpu().numpy(), ref.stage("normal_keys", np.int64))
    _close(stage("normal_values", fdt).cpu().numpy(), ref.stage("normal_values", npdt), rtol, "normals")
    _close(stage("normal_average", fdt).cpu().numpy(), ref.stage("normal_average", npdt), rtol, "average")
    # A4 tree: exact keys and the reference's hashes
    for level in kat["levels"]:
        d = level["depth"]
        support = g.diagnostics["support_keys"][d].cpu().numpy()
        assert sha(support) == level["support_sha256"], f"support keys differ at depth {d}"
        assert np.array_equal(support, ref.support(d))
    keys = g.field.keys.cpu().numpy()
    assert np.array_equal(keys, ref.keys)
    offs = g.diagnostics["level_offsets"]
    for level in kat["levels"]:
        d = level["depth"]
        assert sha(keys[offs[d]:offs[d + 1]]) == level["active_sha256"], f"active keys differ at depth {d}"
    # A6/A7 loads and right-hand sides per solved level
    prm = ref.options
    for d in range(prm["base_depth"], prm["solve_depth"] + 1):
        try:
            ref.stage(f"rhs_{d}", npdt)
        except KeyError:  # the cascadic loop stops at the first empty level (solver.py:361-362)
            assert stage(f"rhs_{d}", fdt) is None
            break
        _close(stage(f"normal_load_{d}", torch.float64).cpu().numpy(), ref.stage(f"normal_load_{d}", np.float64),
               1e-12, f"load {d}")
        _close(stage(f"rhs_{d}", fdt).cpu().numpy(), ref.stage(f"rhs_{d}", npdt), 4 * rtol, f"rhs {d}")
    # A8-A11 coefficients, cumulative, centroid values, isovalue
    _close(g.field.coefficients.cpu().numpy(), ref.coefficients, 8 * rtol, "coefficients")
    _close(g.field.cumulative.cpu().numpy(), ref.cumulative, 8 * rtol, "cumulative")
    _close(stage("centroid_values", fdt).cpu().numpy(), ref.stage("centroid_values", npdt), 8 * rtol, "centroids")
    assert abs(g.iso_value - ref.iso_value) <= 8 * rtol * max(abs(ref.iso_value), 1e-3)
    atol, rtol_iso = iso_tolerance(prec)
    pr = kat["reference_iso_value"]
    assert abs(g.iso_value - pr) <= atol + rtol_iso * abs(pr)
    # A12 evaluation at model-space queries (inside, on and outside the cube)
    rng = np.random.default_rng(7)
    lo, hi = p.min(0), p.max(0)
    q = (lo + (hi - lo) * rng.uniform(-0.1, 1.1, size=(2000, 3))).astype(p.dtype)
    q = np.concatenate([q, p[:200]]).astype(p.dtype)
    v, gr, ok = g.evaluate(torch.from_numpy(q).cuda())
    rv, rg, rok = ref.evaluate(q)
    assert np.array_equal(ok.cpu().numpy(), rok)
    m = rok.astype(bool)
    _close(v.cpu().numpy()[m], rv[m], 8 * rtol, "values")
    _close(gr.cpu().numpy()[m], rg[m], 64 * rtol, "gradients")
    assert np.isnan(v.cpu().numpy()[~m]).all()
