"""Failure paths, without faulting the GPU (warp-psr samples.py:253-257,278-279 for the
degenerate inputs; the bounded waits of the ordered relaxation for the timeout).

* Degenerate inputs -- a nonfinite position, zero extent, coordinates that overflow the
  bounding cube, or no sample with a finite nonzero normal -- raise ValueError with the
  reference's messages (PSR_EDATA through the C ABI) and leave the device usable.
* PSR_RELAX_STALL_TEST=1 makes every wait of the relaxation on its newest slice wait for a
  count that no task publishes, with a 4096-poll limit: the launch ends with PSR_ETIMEOUT,
  the host raises, and the next reconstruction succeeds.
"""
import numpy as np
import pytest
import torch

from warp_psr_b200 import _lib, clouds, reconstruct

pytestmark = pytest.mark.gpu

OPTS = dict(depth=5, full_depth=3, point_weight=2.0)


def good_cloud(dtype=torch.float64):
    p, n = clouds.sphere(5000)
    return torch.tensor(p, dtype=dtype, device="cuda"), torch.tensor(n, dtype=dtype, device="cuda")


def assert_usable(expected_iso):
    p, n = good_cloud()
    assert reconstruct(p, n, **OPTS).iso_value == expected_iso


@pytest.fixture(scope="module")
def clean_iso():
    p, n = good_cloud()
    return reconstruct(p, n, **OPTS).iso_value


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("case", ["nan_position", "inf_position", "zero_extent", "overflowing_cube",
                                  "zero_normals", "nan_normals"])
def test_degenerate_inputs_raise_value_error(clean_iso, dtype, case):
    p, n = good_cloud(dtype)
    if case == "nan_position":
        p[17, 1] = float("nan")
        message = "Nonfinite positions"
    elif case == "inf_position":
        p[3, 0] = float("inf")
        message = "Nonfinite positions"
    elif case == "zero_extent":
        p[:] = torch.tensor([0.25, -0.5, 1.0], dtype=dtype)
        message = "degenerate"
    elif case == "overflowing_cube":
        big = 3e38 if dtype == torch.float32 else 1.7e308
        p[0] = big
        p[1] = -big
        message = "overflowing"
    elif case == "zero_normals":
        n.zero_()
        message = "No accepted samples"
    else:
        n[:] = float("nan")
        message = "No accepted samples"
    with pytest.raises(ValueError, match=message):
        reconstruct(p, n, **OPTS)
    assert_usable(clean_iso)


@pytest.mark.parametrize("precision", ["input", "mixed"])
def test_relaxation_wait_timeout_raises_and_device_stays_usable(monkeypatch, clean_iso, precision):
    p, n = good_cloud()
    monkeypatch.setenv("PSR_RELAX_STALL_TEST", "1")
    with pytest.raises(_lib.PSRError, match="timed out") as info:
        reconstruct(p, n, precision=precision, **OPTS)
    assert info.value.code == _lib.PSR_ETIMEOUT
    monkeypatch.delenv("PSR_RELAX_STALL_TEST")
    assert_usable(clean_iso)
