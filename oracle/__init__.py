"""ctypes binding of the CPU oracle (``oracle/psr_oracle.cpp``).

TEST INFRASTRUCTURE ONLY.  The oracle is the checker for the CUDA path: only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` load it.  The
product package never imports this module.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libpsr_oracle.so"


class _Params(ctypes.Structure):
    _fields_ = [
        ("depth", ctypes.c_int32), ("full_depth", ctypes.c_int32), ("base_depth", ctypes.c_int32),
        ("solve_depth", ctypes.c_int32), ("kernel_depth", ctypes.c_int32),
        ("samples_per_node", ctypes.c_double), ("scale", ctypes.c_double),
        ("point_weight", ctypes.c_double), ("cg_accuracy", ctypes.c_double),
        ("exact", ctypes.c_int32), ("iters", ctypes.c_int32), ("base_v_cycles", ctypes.c_int32),
    ]


def build():
    """Compile the oracle library (make), returning its path."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
        L.oracle_reconstruct.restype = vp
        L.oracle_reconstruct.argtypes = [vp, vp, i64, i32, ctypes.POINTER(_Params)]
        L.oracle_tree.restype = vp
        L.oracle_tree.argtypes = [vp, vp, i64, i32, ctypes.POINTER(_Params)]
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_free.argtypes = [vp]
        L.oracle_level_count.restype = i64
        L.oracle_level_count.argtypes = [vp, i32, i32]
        L.oracle_level_keys.restype = ctypes.POINTER(ctypes.c_int64)
        L.oracle_level_keys.argtypes = [vp, i32, i32]
        L.oracle_total.restype = i64
        L.oracle_total.argtypes = [vp]
        L.oracle_keys.restype = ctypes.POINTER(ctypes.c_int64)
        L.oracle_keys.argtypes = [vp]
        L.oracle_coefficients.restype = vp
        L.oracle_coefficients.argtypes = [vp]
        L.oracle_cumulative.restype = vp
        L.oracle_cumulative.argtypes = [vp]
        L.oracle_iso.restype = ctypes.c_double
        L.oracle_iso.argtypes = [vp]
        L.oracle_transforms.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.oracle_stage.restype = vp
        L.oracle_stage.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(i64), ctypes.POINTER(i32)]
        L.oracle_evaluate.argtypes = [vp, vp, i64, vp, vp, vp]
        L.oracle_relax_sliced.restype = i32
        L.oracle_relax_sliced.argtypes = [i32, vp, i64, i32, vp, vp, vp, vp, vp, i32]
        L.oracle_threads.restype = i32
        _lib = L
    return _lib


def params(depth=6, full_depth=3, base_depth=None, solve_depth=None, kernel_depth=None,
           samples_per_node=1.5, scale=1.1, point_weight=2.0, exact_interpolation=False, iters=8,
           base_v_cycles=1, cg_accuracy=1e-3):
    base_depth = full_depth if base_depth is None else base_depth
    solve_depth = depth if solve_depth is None else solve_depth
    kernel_depth = max(depth - 2, 0) if kernel_depth is None else kernel_depth
    return dict(depth=depth, full_depth=full_depth, base_depth=base_depth, solve_depth=solve_depth,
                kernel_depth=kernel_depth, samples_per_node=samples_per_node, scale=scale,
                point_weight=point_weight, exact=int(bool(exact_interpolation)), iters=iters,
                base_v_cycles=base_v_cycles, cg_accuracy=cg_accuracy)


class OracleResult:
    """Owns one oracle reconstruction; arrays are copied out as numpy."""

    def __init__(self, positions, normals, tree_only=False, **options):
        positions = np.ascontiguousarray(positions)
        normals = np.ascontiguousarray(normals, dtype=positions.dtype)
        if positions.dtype not in (np.float32, np.float64):
            raise ValueError("oracle takes float32/float64 positions")
        self.dtype = positions.dtype
        p = params(**options)
        self.options = p
        self._p = _Params(**p)
        L = lib()
        # tree_only: the stages up to the tree (keys and their stages), no solve
        run = L.oracle_tree if tree_only else L.oracle_reconstruct
        self._h = run(positions.ctypes.data, normals.ctypes.data, len(positions), int(self.dtype == np.float64),
                      ctypes.byref(self._p))
        if not self._h:
            raise ValueError(L.oracle_last_error().decode())
        self.depth = p["depth"]

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_free(self._h)
            self._h = None

    def basis(self, d):
        n = lib().oracle_level_count(self._h, d, 0)
        return np.ctypeslib.as_array(lib().oracle_level_keys(self._h, d, 0), (n,)).copy() if n else np.zeros(0, np.int64)

    def support(self, d):
        n = lib().oracle_level_count(self._h, d, 1)
        return np.ctypeslib.as_array(lib().oracle_level_keys(self._h, d, 1), (n,)).copy() if n else np.zeros(0, np.int64)

    @property
    def keys(self):
        n = lib().oracle_total(self._h)
        return np.ctypeslib.as_array(lib().oracle_keys(self._h), (n,)).copy()

    def _scalars(self, ptr):
        n = lib().oracle_total(self._h)
        ctype = ctypes.c_double if self.dtype == np.float64 else ctypes.c_float
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctype)), (n,)).copy()

    @property
    def coefficients(self):
        return self._scalars(lib().oracle_coefficients(self._h))

    @property
    def cumulative(self):
        return self._scalars(lib().oracle_cumulative(self._h))

    @property
    def iso_value(self):
        return lib().oracle_iso(self._h)

    @property
    def transforms(self):
        out = (ctypes.c_double * 32)()
        lib().oracle_transforms(self._h, out)
        return np.array(out).reshape(2, 4, 4)

    def stage(self, name, dtype):
        count, elem = ctypes.c_int64(), ctypes.c_int32()
        ptr = lib().oracle_stage(self._h, name.encode(), ctypes.byref(count), ctypes.byref(elem))
        if count.value < 0:
            raise KeyError(name)
        dtype = np.dtype(dtype)
        assert dtype.itemsize == elem.value or count.value == 0, (name, dtype, elem.value)
        if count.value == 0:
            return np.zeros(0, dtype)
        buf = (ctypes.c_char * (count.value * elem.value)).from_address(ptr)
        return np.frombuffer(bytes(buf), dtype=dtype)

    def evaluate(self, queries):
        q = np.ascontiguousarray(queries, dtype=self.dtype).reshape(-1, 3)
        values = np.empty(len(q), self.dtype)
        grads = np.empty((len(q), 3), self.dtype)
        valid = np.empty(len(q), np.int32)
        lib().oracle_evaluate(self._h, q.ctypes.data, len(q), values.ctypes.data, grads.ctypes.data,
                              valid.ctypes.data)
        return values, grads, valid


def relax_sliced(keys, depth, offsets, columns, values, b, x, iters):
    """Sequential sliced Gauss-Seidel on an explicit CSR level; returns the new x."""
    dtype = np.asarray(values).dtype
    keys = np.ascontiguousarray(keys, np.int64)
    offsets = np.ascontiguousarray(offsets, np.int32)
    columns = np.ascontiguousarray(columns, np.int32)
    values = np.ascontiguousarray(values, dtype)
    b = np.ascontiguousarray(b, dtype)
    x = np.array(x, dtype=dtype, copy=True)
    lib().oracle_relax_sliced(int(dtype == np.float64), keys.ctypes.data, len(keys), depth, offsets.ctypes.data,
                              columns.ctypes.data, values.ctypes.data, b.ctypes.data, x.ctypes.data, iters)
    return x


def threads():
    return lib().oracle_threads()
