"""The allocation-free isovalue entry point (psr_isovalue_static) through the C ABI.

It serves callers that cannot allocate device memory while they run (embedded in a
framework whose pool already owns the device memory, or in a loop that must not
allocate).  Its results must equal the allocating entry point's, call after call, since
both run the same kernels in the same order; only the scratch differs (a fixed array in
the library instead of an allocation).  Collected last so an earlier failure stops a
run first.
"""
import ctypes
import subprocess
import sys
import textwrap
from pathlib import Path

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


def _cudart():
    from warp_psr_b200 import _lib
    _lib.load()  # brings the CUDA runtime the library links against into the process
    rt = ctypes.CDLL("libcudart.so.12")
    return rt


def test_static_scratch_allocates_no_device_memory():
    """The default stream-ordered pool (every buffer of the library comes from it) sees no
    allocation during a warm call, and the device's free memory does not move."""
    rt = _cudart()
    values = torch.rand(3_000_000, dtype=torch.float64, device="cuda")
    weights = torch.rand(3_000_000, dtype=torch.float64, device="cuda")
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    assert _call_static(values, weights, out) == 0  # first call: loads the module
    torch.cuda.synchronize()
    pool = ctypes.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), torch.cuda.current_device()) == 0
    used_high = 8  # cudaMemPoolAttrUsedMemHigh
    zero = ctypes.c_uint64(0)
    assert rt.cudaMemPoolSetAttribute(pool, used_high, ctypes.byref(zero)) == 0
    before_high = ctypes.c_uint64()
    assert rt.cudaMemPoolGetAttribute(pool, used_high, ctypes.byref(before_high)) == 0
    free0, free1, total = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
    assert rt.cudaMemGetInfo(ctypes.byref(free0), ctypes.byref(total)) == 0
    for _ in range(3):
        assert _call_static(values, weights, out) == 0
    torch.cuda.synchronize()
    assert rt.cudaMemGetInfo(ctypes.byref(free1), ctypes.byref(total)) == 0
    after_high = ctypes.c_uint64()
    assert rt.cudaMemPoolGetAttribute(pool, used_high, ctypes.byref(after_high)) == 0
    assert after_high.value <= before_high.value
    assert free1.value == free0.value
    # the allocating entry point does use the pool, so the probe would have seen it
    from warp_psr_b200 import ops
    ops.isovalue(values, weights)
    torch.cuda.synchronize()
    assert rt.cudaMemPoolGetAttribute(pool, used_high, ctypes.byref(after_high)) == 0
    assert after_high.value > before_high.value


_RESET_CHILD = textwrap.dedent("""
    import ctypes, sys
    import numpy as np
    lib = ctypes.CDLL(sys.argv[1])
    rt = ctypes.CDLL("libcudart.so.12")
    vp = ctypes.c_void_p
    rt.cudaMalloc.argtypes = [ctypes.POINTER(vp), ctypes.c_size_t]
    rt.cudaMemcpy.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_int]
    rt.cudaFree.argtypes = [vp]
    lib.psr_isovalue_static.argtypes = [ctypes.c_int32, vp, vp, ctypes.c_int64, vp, vp]
    lib.psr_isovalue.argtypes = [ctypes.c_int32, vp, vp, ctypes.c_int64, vp, vp]
    rng = np.random.default_rng(5)
    v = rng.normal(size=300_000)
    w = rng.uniform(0, 4, size=300_000)

    def run(entry):
        ptrs = [ctypes.c_void_p() for _ in range(3)]
        for p, size in zip(ptrs, (v.nbytes, w.nbytes, 8)):
            assert rt.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(size)) == 0
        assert rt.cudaMemcpy(ptrs[0], v.ctypes.data, ctypes.c_size_t(v.nbytes), 1) == 0
        assert rt.cudaMemcpy(ptrs[1], w.ctypes.data, ctypes.c_size_t(w.nbytes), 1) == 0
        assert entry(1, ptrs[0], ptrs[1], len(v), ptrs[2], None) == 0
        assert rt.cudaDeviceSynchronize() == 0
        out = np.zeros(1)
        assert rt.cudaMemcpy(out.ctypes.data, ptrs[2], ctypes.c_size_t(8), 2) == 0
        for p in ptrs:
            assert rt.cudaFree(p) == 0
        return out[0]

    expected = run(lib.psr_isovalue)
    assert run(lib.psr_isovalue_static) == expected
    assert rt.cudaDeviceReset() == 0  # a new context: the scratch array has a new address
    assert run(lib.psr_isovalue_static) == expected
    assert run(lib.psr_isovalue_static) == expected
    print("reset ok", expected)
""")


def test_static_scratch_after_device_reset():
    """Calls before and after cudaDeviceReset (which reloads the library's module in a new
    context) agree; run in a child process that never touches torch's allocator."""
    from warp_psr_b200 import _lib
    res = subprocess.run([sys.executable, "-c", _RESET_CHILD, str(_lib.LIB_PATH)], capture_output=True, text=True,
                         timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "reset ok" in res.stdout


def test_static_scratch_rejects_more_than_its_capacity():
    from warp_psr_b200 import _lib
    values = torch.ones(4_194_305, dtype=torch.float32, device="cuda")
    out = torch.empty(1, dtype=torch.float32, device="cuda")
    assert _call_static(values, values, out) == _lib.PSR_EINVAL
    assert "4,194,304" in _lib.last_error()
