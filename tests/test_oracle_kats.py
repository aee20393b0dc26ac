"""The CPU oracle against every reference known-answer fixture (no GPU).

Pins the oracle: per-level active/support key SHA-256 must match the reference exactly and
the isovalue must agree with PoissonRecon 262b0f5's within the design budget.
"""
import pytest

import oracle
from kat_util import KATS, inputs, iso_tolerance, options, sha
from kat_inputs import input_sha256


@pytest.mark.parametrize("kat", KATS, ids=[k["name"] for k in KATS])
def test_oracle_matches_reference_fixture(kat):
    p, n = inputs(kat)
    assert input_sha256(p, n) == kat["input_sha256"]
    r = oracle.OracleResult(p, n, **options(kat["params"]))
    for level in kat["levels"]:
        d = level["depth"]
        assert len(r.support(d)) == level["support_count"]
        assert len(r.basis(d)) == level["active_count"]
        assert sha(r.support(d)) == level["support_sha256"], f"support keys differ at depth {d}"
        assert sha(r.basis(d)) == level["active_sha256"], f"active keys differ at depth {d}"
    atol, rtol = iso_tolerance(kat["params"]["precision"])
    ref = kat["reference_iso_value"]
    assert abs(r.iso_value - ref) <= atol + rtol * abs(ref)
    assert abs(r.iso_value - kat["iso_value"]) <= atol + rtol * abs(kat["iso_value"])
