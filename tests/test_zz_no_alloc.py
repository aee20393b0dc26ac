"""The allocation-free isovalue entry point (psr_isovalue_static) through the C ABI.

It serves callers that cannot allocate device memory while they run (embedded in a
framework whose pool already owns the device memory, or in a loop that must not
allocate).  Its results must equal the allocating entry point's, call after call, since
both run the same kernels in the same order; only the scratch differs (a fixed array in
the library instead of an allocation).  Collected last so an earlier failure stops a
run first.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _call_static(values, weights, out):
    from warp_psr_b200 import _lib
    code = _lib.PSR_FLOAT64 if values.dtype == torch.float64 else _lib.PSR_FLOAT32
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return _lib.load().psr_isovalue_static(code, values.data_ptr(), weights.data_ptr(), values.numel(),
                                           out.data_ptr(), stream)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("count", [1, 1025, 65537, 4_194_304])
def test_static_scratch_matches_allocating_entry_point(dtype, count):
    from warp_psr_b200 import ops
    gen = torch.Generator(device="cuda").manual_seed(count)
    values = torch.randn(count, dtype=dtype, device="cuda", generator=gen)
    weights = torch.rand(count, dtype=dtype, device="cuda", generator=gen) * 4
    expected = ops.isovalue(values, weights).cpu().numpy()
    for _ in range(2):  # two calls in a row share (and overwrite) the static scratch
        out = torch.full((1,), float("nan"), dtype=dtype, device="cuda")
        assert _call_static(values, weights, out) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), expected)


def test_static_scratch_rejects_more_than_its_capacity():
    from warp_psr_b200 import _lib
    values = torch.ones(4_194_305, dtype=torch.float32, device="cuda")
    out = torch.empty(1, dtype=torch.float32, device="cuda")
    assert _call_static(values, values, out) == _lib.PSR_EINVAL
    assert "4,194,304" in _lib.last_error()
