"""ctypes binding of ``libpsr_b200.so`` (the C ABI in ``include/psr_b200.h``).

The library is the only compute path: there is no CPU or PyTorch fallback, and a missing
or unloadable library raises at first use.
"""
import ctypes
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpsr_b200.so"

PSR_OK, PSR_EINVAL, PSR_ECUDA, PSR_EDATA, PSR_ETIMEOUT, PSR_ENOMEM = range(6)
PSR_FLOAT32, PSR_FLOAT64 = 0, 1
PSR_PRECISION_INPUT, PSR_PRECISION_MIXED = 0, 1


class Params(ctypes.Structure):
    _fields_ = [
        ("depth", ctypes.c_int32), ("full_depth", ctypes.c_int32), ("base_depth", ctypes.c_int32),
        ("solve_depth", ctypes.c_int32), ("kernel_depth", ctypes.c_int32),
        ("samples_per_node", ctypes.c_double), ("scale", ctypes.c_double),
        ("point_weight", ctypes.c_double), ("cg_accuracy", ctypes.c_double),
        ("exact_interpolation", ctypes.c_int32), ("iters", ctypes.c_int32), ("base_v_cycles", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("keep_stages", ctypes.c_int32), ("differentiable", ctypes.c_int32),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int32), ("depth", ctypes.c_int32), ("total", ctypes.c_int64), ("groups", ctypes.c_int64),
        ("basis_counts", ctypes.c_int64 * 16), ("support_counts", ctypes.c_int64 * 16),
        ("iso_value", ctypes.c_double), ("cube_to_model", ctypes.c_double * 16),
        ("model_to_cube", ctypes.c_double * 16), ("stage_ms", ctypes.c_double * 8),
        ("relax_ms", ctypes.c_double), ("relax_row_visits", ctypes.c_int64), ("relax_launches", ctypes.c_int64),
        ("relax_finest_ms", ctypes.c_double), ("relax_finest_row_visits", ctypes.c_int64),
        ("normalization", ctypes.c_double * 5), ("backward_ms", ctypes.c_double * 8),
    ]


class Arrays(ctypes.Structure):
    _fields_ = [
        ("keys", ctypes.c_void_p), ("coefficients", ctypes.c_void_p), ("cumulative", ctypes.c_void_p),
        ("level_offsets", ctypes.POINTER(ctypes.c_int64)), ("support_keys", ctypes.c_void_p * 16),
    ]


class FieldHandle(ctypes.Structure):
    """Mirror of ``psr_field_handle`` (warp-psr DeviceField, device_field.py:19-28)."""
    _fields_ = [
        ("keys", ctypes.c_void_p), ("coefficients", ctypes.c_void_p), ("cumulative", ctypes.c_void_p),
        ("count", ctypes.c_int64), ("linear", ctypes.c_double * 9), ("translation", ctypes.c_double * 3),
        ("depth", ctypes.c_int32), ("dtype", ctypes.c_int32), ("iso_value", ctypes.c_double),
        ("hash_slots", ctypes.c_void_p), ("hash_mask", ctypes.c_uint64),
    ]


class KernelClock(ctypes.Structure):
    """Mirror of ``psr_kernel_clock``: one kernel's launches, device ms and algorithmic bytes."""
    _fields_ = [
        ("kernel", ctypes.c_char_p), ("unit", ctypes.c_char_p), ("launches", ctypes.c_int64),
        ("ms", ctypes.c_double), ("bytes", ctypes.c_double), ("units", ctypes.c_double),
    ]


EXPORTS = ("psr_reconstruct", "psr_result_info", "psr_result_arrays", "psr_evaluate", "psr_device_field",
           "psr_free", "psr_last_error", "psr_relax_sliced", "psr_isovalue", "psr_result_stage",
           "psr_kernel_launches", "psr_isovalue_static", "psr_backward", "psr_evaluate_backward",
           "psr_mc_points", "psr_mc_mark", "psr_mc_cells", "psr_mc_triangulate", "psr_extract_mesh",
           "psr_mesh_info", "psr_mesh_arrays", "psr_mesh_free", "psr_kernel_clocks")

_lib = None


class PSRError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


def load():
    """Load and type the library; raises if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH.name} is not built; run `python -m warp_psr_b200.build`")
    L = ctypes.CDLL(str(LIB_PATH))
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
    L.psr_reconstruct.argtypes = [vp, vp, i64, i32, ctypes.POINTER(Params), vp, ctypes.POINTER(vp)]
    L.psr_result_info.argtypes = [vp, ctypes.POINTER(Info)]
    L.psr_result_arrays.argtypes = [vp, ctypes.POINTER(Arrays)]
    L.psr_evaluate.argtypes = [vp, vp, i64, vp, vp, vp, vp]
    L.psr_device_field.argtypes = [vp, ctypes.POINTER(FieldHandle)]
    L.psr_free.argtypes = [vp]
    L.psr_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.psr_relax_sliced.argtypes = [i32, vp, i64, i32, vp, vp, vp, vp, vp, i32, vp]
    L.psr_isovalue.argtypes = [i32, vp, vp, i64, vp, vp]
    L.psr_result_stage.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(vp), ctypes.POINTER(i64), ctypes.POINTER(i32)]
    L.psr_kernel_launches.argtypes = [ctypes.POINTER(i64)]
    L.psr_isovalue_static.argtypes = [i32, vp, vp, i64, vp, vp]
    L.psr_backward.argtypes = [vp, vp, vp, i64, i32, vp, vp, vp, vp, vp, vp, vp]
    L.psr_evaluate_backward.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp, vp, vp]
    shape3, real3 = ctypes.POINTER(i64), ctypes.POINTER(ctypes.c_double)
    L.psr_mc_points.argtypes = [i32, shape3, real3, real3, vp, i64, i64, vp, vp]
    L.psr_mc_mark.argtypes = [i32, vp, shape3, i64, i64, vp, vp, vp]
    L.psr_mc_cells.argtypes = [vp, i64, vp, i64, ctypes.POINTER(i64), vp]
    L.psr_mc_triangulate.argtypes = [i32, shape3, real3, real3, vp, vp, i64, ctypes.POINTER(vp), vp]
    L.psr_extract_mesh.argtypes = [vp, shape3, real3, real3, ctypes.c_double, i64, ctypes.POINTER(i64),
                                   ctypes.POINTER(vp), vp]
    L.psr_mesh_info.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i64), ctypes.POINTER(i64),
                                ctypes.POINTER(i64)]
    L.psr_mesh_arrays.argtypes = [vp] + [ctypes.POINTER(vp)] * 5
    L.psr_mesh_free.argtypes = [vp]
    L.psr_kernel_clocks.argtypes = [ctypes.POINTER(KernelClock), i32, ctypes.POINTER(i32)]
    for name in EXPORTS:
        getattr(L, name).restype = i32
    _lib = L
    return L


def last_error():
    buf = ctypes.create_string_buffer(1024)
    load().psr_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def kernel_launches():
    count = ctypes.c_int64()
    check(load().psr_kernel_launches(ctypes.byref(count)))
    return count.value


def kernel_clocks():
    """Totals of the kernel clocks (launches made while PSR_KERNEL_CLOCKS=1) since the last
    call: a list of dicts (kernel, unit, launches, ms, bytes, units); clears the totals."""
    L = load()
    count = ctypes.c_int32()
    out = (KernelClock * 32)()
    check(L.psr_kernel_clocks(out, 32, ctypes.byref(count)))
    return [{"kernel": c.kernel.decode(), "unit": c.unit.decode(), "launches": int(c.launches), "ms": c.ms,
             "bytes": c.bytes, "units": c.units} for c in out[:min(count.value, 32)]]


def check(code):
    if code != PSR_OK:
        message = last_error()
        if code in (PSR_EINVAL, PSR_EDATA):
            raise ValueError(message)
        raise PSRError(code, message)
