"""Stage-level entry points on torch CUDA tensors (through the C ABI).

``relax_sliced`` mirrors warp-psr ``relaxation.relax_sliced`` (relaxation.py:189-210) on an
explicit CSR level; ``isovalue`` mirrors ``reconstruction._compute_isovalue``
(reconstruction.py:101-116).
"""
import ctypes

import torch

from . import _lib


def _dtype_code(t):
    if t.dtype == torch.float64:
        return _lib.PSR_FLOAT64
    if t.dtype == torch.float32:
        return _lib.PSR_FLOAT32
    raise ValueError("float32 or float64 tensors required")


def relax_sliced(keys, depth, offsets, columns, values, b, x, iters):
    """In-place ordered sliced Gauss-Seidel of ``x`` (rows = basis keys of ``depth``)."""
    for t in (keys, offsets, columns, values, b, x):
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError("contiguous CUDA tensors required")
    if keys.dtype != torch.int64 or offsets.dtype != torch.int32 or columns.dtype != torch.int32:
        raise ValueError("keys int64, offsets/columns int32 required")
    if not (values.dtype == b.dtype == x.dtype):
        raise ValueError("values, b and x must share a precision")
    with torch.cuda.device(x.device):
        stream = ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)
        _lib.check(_lib.load().psr_relax_sliced(_dtype_code(x), keys.data_ptr(), keys.numel(), depth,
                                                offsets.data_ptr(), columns.data_ptr(), values.data_ptr(),
                                                b.data_ptr(), x.data_ptr(), iters, stream))
    return x


def isovalue(values, weights):
    """sum(v*w)/sum(w) with input-precision products and float64 accumulation."""
    if values.dtype != weights.dtype or values.numel() != weights.numel() or not values.numel():
        raise ValueError("values and weights must match and be nonempty")
    out = torch.empty(1, dtype=values.dtype, device=values.device)
    v, w = values.contiguous(), weights.contiguous()
    with torch.cuda.device(v.device):
        stream = ctypes.c_void_p(torch.cuda.current_stream(v.device).cuda_stream)
        _lib.check(_lib.load().psr_isovalue(_dtype_code(v), v.data_ptr(), w.data_ptr(), v.numel(), out.data_ptr(),
                                            stream))
    return out
