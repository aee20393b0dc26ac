"""The C-ABI library loads and exports every entry point its header declares (no GPU calls)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared():
    text = (ROOT / "include" / "psr_b200.h").read_text()
    return sorted(set(re.findall(r"^int (psr_\w+)\(", text, flags=re.M)))


def test_header_declares_the_reference_entry_points():
    names = declared()
    for required in ("psr_reconstruct", "psr_evaluate", "psr_device_field", "psr_free", "psr_last_error",
                     "psr_relax_sliced", "psr_isovalue", "psr_result_info", "psr_result_arrays"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from warp_psr_b200 import _lib
    lib = _lib.load()
    for name in declared():
        assert hasattr(lib, name), name
        assert ctypes.cast(getattr(lib, name), ctypes.c_void_p).value


def test_python_binding_covers_the_header():
    from warp_psr_b200 import _lib
    assert set(declared()) <= set(_lib.EXPORTS)


def test_last_error_is_callable_without_a_device():
    from warp_psr_b200 import _lib
    assert isinstance(_lib.last_error(), str)


@pytest.mark.parametrize("kwargs,message", [
    (dict(depth=0), "depth >= 1"),
    (dict(depth=4, full_depth=5), "base_depth <= full_depth"),
    (dict(depth=16, full_depth=3), "depth <= 15"),
    (dict(iters=0), "positive integers"),
    (dict(point_weight=-1.0), "nonnegative point_weight"),
    (dict(cg_accuracy=0.0), "positive cg_accuracy"),
    (dict(scale=1.0), "scale > 1"),
    (dict(samples_per_node=float("nan")), "samples_per_node"),
    (dict(depth=4.0), "integers"),
])
def test_invalid_arguments_raise_before_any_allocation(kwargs, message):
    import torch
    from warp_psr_b200 import reconstruct
    p = torch.zeros((4, 3))
    with pytest.raises(ValueError, match=message):
        reconstruct(p, p, **kwargs)


def test_cpu_tensors_are_rejected():
    import torch
    from warp_psr_b200 import reconstruct
    p = torch.rand((16, 3))
    with pytest.raises(ValueError, match="CUDA device"):
        reconstruct(p, p, depth=4, full_depth=2)


def test_kernel_clocks_without_pending_launches_need_no_device():
    """With no clocked launch pending, psr_kernel_clocks reports no kernels and makes no CUDA
    call; the struct it fills matches the header's field order."""
    from warp_psr_b200 import _lib
    assert _lib.kernel_clocks() == []
    names = [f[0] for f in _lib.KernelClock._fields_]
    header = (ROOT / "include" / "psr_b200.h").read_text()
    body = header[header.index("typedef struct psr_kernel_clock {"):header.index("} psr_kernel_clock;")]
    assert names == re.findall(r"\b(\w+);", body)
