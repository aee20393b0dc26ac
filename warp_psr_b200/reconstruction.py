"""Drop-in host API of warp-psr's reconstruction path, backed by ``libpsr_b200``.

Mirrors ``warp_psr.reconstruct`` (warp-psr src/warp_psr/reconstruction.py:137-349): the same
keyword arguments, defaults, validation messages (ValueError before any allocation), and
result object with ``iso_value``, ``evaluate(queries)``, ``device_field()``, ``metadata``
and ``diagnostics``.  Inputs are CUDA tensors of shape (N, 3) — torch tensors, or any
object exposing ``__cuda_array_interface__`` (Warp vec3 arrays, CuPy arrays) — in float32
or float64.  Work runs on the current torch stream of the input's device.
"""
import ctypes
import math
from dataclasses import dataclass

import torch

from . import _lib


def _as_vec3(array, name):
    if not isinstance(array, torch.Tensor):
        if hasattr(array, "__cuda_array_interface__"):
            array = torch.as_tensor(array, device="cuda")
        else:
            raise ValueError("Reconstruction requires matching float32/float64 3D vectors on the same CUDA device")
    if array.dim() == 1 and array.numel() % 3 == 0:
        array = array.view(-1, 3)
    if array.dim() != 2 or array.shape[1] != 3:
        raise ValueError("points and normals must have equal nonempty 1D shapes")
    return array


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class _DeviceArray:
    """Zero-copy view of a result-owned device buffer (keeps the result alive)."""

    def __init__(self, ptr, shape, typestr, owner):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr or 0), False),
                                         "version": 3, "strides": None}
        self._owner = owner


class _Handle:
    """Owns one ``psr_result``; freed with ``psr_free`` when the last view is gone."""

    def __init__(self, ptr):
        self.ptr = ptr
        self._free = _lib.load().psr_free  # held so interpreter shutdown can still free

    def __del__(self):
        if self.ptr and self._free is not None:
            self._free(self.ptr)
            self.ptr = None


@dataclass
class LevelField:
    """Sparse per-level degree-1 field (warp-psr field.py:122-184)."""

    keys: torch.Tensor
    coefficients: torch.Tensor
    linear: tuple
    translation: tuple
    depth: int
    iso_value: float
    cumulative: torch.Tensor = None
    _handle: object = None

    def evaluate(self, queries):
        """Values, model-space gradients and int32 validity; outside the cube = NaN, valid 0."""
        dtype = self.coefficients.dtype
        q = _as_vec3(queries, "queries")
        if q.dtype != dtype or q.device != self.coefficients.device:
            raise ValueError("Query precision/device must match coefficients")
        q = q.contiguous()
        n = q.shape[0]
        values = torch.empty(n, dtype=dtype, device=q.device)
        gradients = torch.empty((n, 3), dtype=dtype, device=q.device)
        valid = torch.empty(n, dtype=torch.int32, device=q.device)
        with torch.cuda.device(q.device):
            _lib.check(_lib.load().psr_evaluate(self._handle.ptr, q.data_ptr(), n, values.data_ptr(),
                                                gradients.data_ptr(), valid.data_ptr(), _stream(q.device)))
        return values, gradients, valid

    def device_field(self):
        return DeviceField(self)


class DeviceField:
    """Zero-copy field handle (warp-psr device_field.py:19-28,115-142).

    ``handle`` is the ``psr_field_handle`` POD of device pointers to pass to CUDA kernels
    that include ``include/psr_field.cuh``; the arrays stay valid while this object lives
    and must not be modified.
    """

    def __init__(self, field):
        self.field = field
        self.handle = _lib.FieldHandle()
        _lib.check(_lib.load().psr_device_field(field._handle.ptr, ctypes.byref(self.handle)))
        self.keys = field.keys
        self.coefficients = field.coefficients
        self.cumulative = field.cumulative
        self.depth = field.depth
        self.linear = field.linear
        self.translation = field.translation
        self.reference = True


@dataclass
class Reconstruction:
    field: LevelField
    metadata: dict
    diagnostics: dict

    @property
    def iso_value(self):
        return self.field.iso_value

    def evaluate(self, queries):
        return self.field.evaluate(queries)

    def device_field(self):
        """Return a zero-copy handle for field evaluation inside CUDA kernels."""
        return self.field.device_field()


def _validate(depth, full_depth, base_depth, solve_depth, kernel_depth, samples_per_node, scale, point_weight,
              iters, base_v_cycles, cg_accuracy):
    # warp-psr reconstruction.py:160-203 (the Warp-Nanogrid limit depth - full_depth <= 7
    # does not apply: this implementation assembles every level with stencils).
    depths = (depth, full_depth, base_depth, solve_depth, kernel_depth)
    if any(not isinstance(v, int) or isinstance(v, bool) for v in depths):
        raise ValueError("Depth parameters must be integers")
    if (not 0 <= base_depth <= full_depth <= solve_depth <= depth <= 15 or depth < 1
            or not 0 <= kernel_depth <= depth):
        raise ValueError("Require 0 <= base_depth <= full_depth <= solve_depth <= depth <= 15, depth >= 1, "
                         "and 0 <= kernel_depth <= depth")
    if (not isinstance(iters, int) or iters < 1 or not isinstance(base_v_cycles, int) or base_v_cycles < 1):
        raise ValueError("iters and base_v_cycles must be positive integers")
    if (not math.isfinite(point_weight) or point_weight < 0 or not math.isfinite(cg_accuracy) or cg_accuracy <= 0):
        raise ValueError("Require finite nonnegative point_weight and positive cg_accuracy")
    if not math.isfinite(samples_per_node) or samples_per_node <= 0 or not math.isfinite(scale) or scale <= 1:
        raise ValueError("Require finite positive samples_per_node and scale > 1")


STAGES = ("samples", "density", "normal_field", "tree", "assembly_and_solve", "field", "isovalue")


def reconstruct(positions, normals, *, depth=6, full_depth=3, base_depth=None, solve_depth=None, kernel_depth=None,
                samples_per_node=1.5, scale=1.1, point_weight=2.0, exact_interpolation=False, iters=8,
                base_v_cycles=1, cg_accuracy=1e-3, precision="input", keep_stages=False, error_vs_fp64=False,
                _differentiable=False):
    """Reconstruct oriented CUDA float32/float64 vectors; point_weight=0 selects PSR.

    Degree one, Neumann boundaries, confidence disabled.  The return value evaluates the
    implicit function and its model-space gradient; the surface is
    ``value == result.iso_value``.  ``precision="input"`` solves in the input precision
    exactly like the reference; ``precision="mixed"`` solves in float64 with float32
    storage of the relaxation operators (float64 coefficients).  ``error_vs_fp64=True``
    also runs the float64 path on the same inputs and records in
    ``metadata["error_vs_fp64"]`` the field's error against it (see ``field_error``).
    """
    if base_depth is None:
        base_depth = full_depth
    if solve_depth is None:
        solve_depth = depth
    if kernel_depth is None:
        kernel_depth = max(depth - 2, 0)
    _validate(depth, full_depth, base_depth, solve_depth, kernel_depth, samples_per_node, scale, point_weight, iters,
              base_v_cycles, cg_accuracy)
    if precision not in ("input", "mixed"):
        raise ValueError("precision must be 'input' or 'mixed'")
    p = _as_vec3(positions, "positions")
    n = _as_vec3(normals, "normals")
    if (p.dtype not in (torch.float32, torch.float64) or n.dtype != p.dtype or not p.is_cuda
            or n.device != p.device):
        raise ValueError("Reconstruction requires matching float32/float64 3D vectors on the same CUDA device")
    if p.shape != n.shape or not p.shape[0]:
        raise ValueError("points and normals must have equal nonempty 1D shapes")
    p = p.contiguous()
    n = n.contiguous()
    params = _lib.Params(depth, full_depth, base_depth, solve_depth, kernel_depth, float(samples_per_node),
                         float(scale), float(point_weight), float(cg_accuracy), int(bool(exact_interpolation)), iters,
                         base_v_cycles, _lib.PSR_PRECISION_MIXED if precision == "mixed" else _lib.PSR_PRECISION_INPUT,
                         int(bool(keep_stages)), int(bool(_differentiable)))
    L = _lib.load()
    out = ctypes.c_void_p()
    dtype_code = _lib.PSR_FLOAT64 if p.dtype == torch.float64 else _lib.PSR_FLOAT32
    with torch.cuda.device(p.device):
        _lib.check(L.psr_reconstruct(p.data_ptr(), n.data_ptr(), p.shape[0], dtype_code, ctypes.byref(params),
                                     _stream(p.device), ctypes.byref(out)))
    handle = _Handle(out.value)
    info = _lib.Info()
    _lib.check(L.psr_result_info(handle.ptr, ctypes.byref(info)))
    arrays = _lib.Arrays()
    _lib.check(L.psr_result_arrays(handle.ptr, ctypes.byref(arrays)))
    out_dtype = torch.float64 if info.dtype == _lib.PSR_FLOAT64 else torch.float32
    typestr = "<f8" if out_dtype == torch.float64 else "<f4"
    total = info.total

    def view(ptr, shape, ts):
        return torch.as_tensor(_DeviceArray(ptr, shape, ts, handle), device=p.device)

    keys = view(arrays.keys, (total,), "<i8")
    coefficients = view(arrays.coefficients, (total,), typestr)
    cumulative = view(arrays.cumulative, (total,), typestr)
    m2c = list(info.model_to_cube)
    linear = tuple(m2c[4 * r + c] for r in range(3) for c in range(3))
    translation = tuple(m2c[4 * r + 3] for r in range(3))
    field = LevelField(keys, coefficients, linear, translation, depth, float(info.iso_value), cumulative, handle)
    basis_counts = [int(info.basis_counts[d]) for d in range(depth + 1)]
    support = [view(arrays.support_keys[d], (int(info.support_counts[d]),), "<i8") for d in range(depth + 1)]
    c2m = list(info.cube_to_model)
    metadata = {
        "precision": "float64" if out_dtype == torch.float64 else "float32",
        "solve_precision": precision,
        "device": str(p.device),
        "basis_counts": basis_counts,
        "timings_seconds": {name: info.stage_ms[i] / 1000.0 for i, name in enumerate(STAGES)},
        "stage_timing_scope": "CUDA stream elapsed time between stage boundaries (count reads included)",
        "exact_interpolation_behavior": "empty constraints in pinned reference (issue #16)"
        if exact_interpolation else "level-clustered approximate constraints",
        "cube_to_model": [c2m[4 * r:4 * r + 4] for r in range(4)],
        "parameters": {"depth": depth, "full_depth": full_depth, "base_depth": base_depth,
                       "solve_depth": solve_depth, "kernel_depth": kernel_depth,
                       "samples_per_node": samples_per_node, "scale": scale, "point_weight": point_weight,
                       "exact_interpolation": exact_interpolation, "iters": iters,
                       "base_v_cycles": base_v_cycles, "cg_accuracy": cg_accuracy},
        "profile": "pinned cascadic degree-1 Neumann",
        "constant_mode": "reference root mean term" if base_depth == 0 and point_weight == 0
        else "reference solve without an added mean term",
    }
    def stage(name, dtype):
        """Copy of an intermediate array kept with keep_stages=True (None if absent)."""
        data, count, elem = ctypes.c_void_p(), ctypes.c_int64(), ctypes.c_int32()
        _lib.check(L.psr_result_stage(handle.ptr, name.encode(), ctypes.byref(data), ctypes.byref(count),
                                      ctypes.byref(elem)))
        if count.value < 0:
            return None
        ts = {torch.int64: "<i8", torch.int32: "<i4", torch.float32: "<f4", torch.float64: "<f8"}[dtype]
        return view(data.value, (count.value,), ts).clone()

    diagnostics = {"groups": int(info.groups), "support_keys": support, "stage": stage,
                   "level_offsets": [int(arrays.level_offsets[d]) for d in range(depth + 2)],
                   "total_seconds": info.stage_ms[7] / 1000.0,
                   "relax_seconds": info.relax_ms / 1000.0, "relax_row_visits": int(info.relax_row_visits),
                   "relax_launches": int(info.relax_launches),
                   "relax_finest_seconds": info.relax_finest_ms / 1000.0,
                   "relax_finest_row_visits": int(info.relax_finest_row_visits),
                   "normalization": tuple(info.normalization)}
    result = Reconstruction(field, metadata, diagnostics)
    if error_vs_fp64:
        options = dict(depth=depth, full_depth=full_depth, base_depth=base_depth, solve_depth=solve_depth,
                       kernel_depth=kernel_depth, samples_per_node=samples_per_node, scale=scale,
                       point_weight=point_weight, exact_interpolation=exact_interpolation, iters=iters,
                       base_v_cycles=base_v_cycles, cg_accuracy=cg_accuracy)
        if out_dtype == torch.float64 and p.dtype == torch.float64 and precision == "input":
            reference = result
        else:
            reference = reconstruct(p.double(), n.double(), **options)
        metadata["error_vs_fp64"] = field_error(result, reference, p)
    return result


def field_error(result, reference, points, extra=20_000, seed=2027):
    """Error of ``result``'s field against ``reference`` (a float64 reconstruction of the same
    inputs), both evaluated in float64 at the input points and at ``extra`` points uniform
    in their bounding box: max |f - f64|, that maximum normalised by max |f64|, the
    isovalue difference, and the number of valid queries."""
    pts = points.detach().to(torch.float64).reshape(-1, 3)
    lo, hi = pts.min(0).values, pts.max(0).values
    gen = torch.Generator(device=pts.device).manual_seed(seed)
    box = lo + (hi - lo) * torch.rand((extra, 3), dtype=torch.float64, device=pts.device, generator=gen)
    q = torch.cat([pts, box])
    ref_v, _, ok = reference.evaluate(q)
    dtype = result.field.coefficients.dtype
    v, _, _ = result.evaluate(q.to(dtype))
    m = ok.bool()
    diff = (v.double()[m] - ref_v[m]).abs().max().item()
    scale = ref_v[m].abs().max().item()
    return {"max_abs": diff, "normalised": diff / scale if scale > 0 else diff,
            "iso_abs": abs(result.iso_value - reference.iso_value), "queries": int(m.sum().item()),
            "reference": "float64 path, same inputs"}


# ---------------------------------------------------------------- differentiable reconstruction
BACKWARD_STAGES = ("field", "mirrored_operators", "reverse_sweeps", "operator_adjoints", "base_multigrid",
                   "point_constraints", "normal_loads", "splats_density_samples")

class _BackwardStats(dict):
    """Holds the forward's result and, once a reverse pass ran, ``"backward_ms"``: the device
    ms per stage of the last pass (BACKWARD_STAGES), read from the library on first access so
    the pass itself needs no host synchronisation."""

    def __init__(self):
        super().__init__()
        self._pending = None

    def reverse_pass_done(self, result):
        self._pending = result

    def _settle(self):
        if self._pending is not None:
            result, self._pending = self._pending, None
            info = _lib.Info()
            _lib.check(_lib.load().psr_result_info(result.field._handle.ptr, ctypes.byref(info)))
            super().__setitem__("backward_ms", dict(zip(BACKWARD_STAGES, (float(v) for v in info.backward_ms))))

    def __getitem__(self, key):
        self._settle()
        return super().__getitem__(key)

    def get(self, key, default=None):
        self._settle()
        return super().get(key, default)

    def __contains__(self, key):
        self._settle()
        return super().__contains__(key)


class _ReconstructFunction(torch.autograd.Function):
    """Forward: a differentiable reconstruction.  Outputs the per-level coefficients, the
    cumulative coefficients, the isovalue and the 5-value sample normalisation; backward is
    the library's reverse pass (psr_backward) onto positions and normals."""

    @staticmethod
    def forward(ctx, positions, normals, box, options):
        result = reconstruct(positions.detach(), normals.detach(), _differentiable=True, **options)
        field = result.field
        dtype, device = field.coefficients.dtype, field.coefficients.device
        box["result"] = result
        ctx.box = box
        ctx.save_for_backward(positions, normals)
        iso = torch.tensor(field.iso_value, dtype=dtype, device=device)
        normalization = torch.tensor(result.diagnostics["normalization"], dtype=dtype, device=device)
        return field.coefficients.clone(), field.cumulative.clone(), iso, normalization

    @staticmethod
    def backward(ctx, g_coef, g_cum, g_iso, g_norm):
        positions, normals = ctx.saved_tensors
        result = ctx.box["result"]
        p = positions.detach().contiguous()
        n = normals.detach().contiguous()
        dtype = result.field.coefficients.dtype
        g_p = torch.empty_like(p)
        g_n = torch.empty_like(n)

        def ptr(t):
            return 0 if t is None else t.to(dtype).contiguous().data_ptr()

        keep = [t.to(dtype).contiguous() if t is not None else None for t in (g_coef, g_cum, g_norm, g_iso)]
        dtype_code = _lib.PSR_FLOAT64 if p.dtype == torch.float64 else _lib.PSR_FLOAT32
        with torch.cuda.device(p.device):
            _lib.check(_lib.load().psr_backward(
                result.field._handle.ptr, p.data_ptr(), n.data_ptr(), p.shape[0], dtype_code,
                ptr(keep[0]), ptr(keep[1]), ptr(keep[3]), ptr(keep[2]),
                g_p.data_ptr(), g_n.data_ptr(), _stream(p.device)))
        ctx.box.reverse_pass_done(result)
        return (g_p if ctx.needs_input_grad[0] else None), (g_n if ctx.needs_input_grad[1] else None), None, None


class _EvaluateFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coefficients, cumulative, iso, normalization, queries, result, centered):
        values, gradients, valid = result.field.evaluate(queries.detach())
        ctx.result = result
        ctx.centered = centered
        ctx.save_for_backward(queries)
        ctx.mark_non_differentiable(valid)
        if centered:
            values = values - iso.detach()
        return values, gradients, valid

    @staticmethod
    def backward(ctx, g_values, g_gradients, _g_valid):
        (queries,) = ctx.saved_tensors
        result = ctx.result
        field = result.field
        dtype = field.coefficients.dtype
        q = queries.detach().contiguous()
        g_coef = torch.zeros_like(field.coefficients)
        g_cum = torch.zeros_like(field.cumulative)
        g_q = torch.zeros_like(q)
        g_norm = torch.zeros(5, dtype=dtype, device=q.device)
        gv = g_values.to(dtype).contiguous() if g_values is not None else None
        gg = g_gradients.to(dtype).contiguous() if g_gradients is not None else None
        with torch.cuda.device(q.device):
            _lib.check(_lib.load().psr_evaluate_backward(
                field._handle.ptr, q.data_ptr(), q.shape[0], gv.data_ptr() if gv is not None else 0,
                gg.data_ptr() if gg is not None else 0, g_coef.data_ptr(), g_cum.data_ptr(), g_q.data_ptr(),
                g_norm.data_ptr(), _stream(q.device)))
        g_iso = None
        if ctx.centered and gv is not None:
            # masked sum without boolean indexing (which would wait for the device)
            g_iso = -torch.where(torch.isfinite(gv), gv, torch.zeros_like(gv)).sum()
        return g_coef, g_cum, g_iso, g_norm, g_q, None, None


class DifferentiableReconstruction:
    """Result of reconstruct_differentiable (warp-psr reconstruction_adjoint.py:45-58).

    ``evaluate(queries, centered=False)`` returns (values, model-space gradients, valid) as
    torch tensors connected to the autograd graph of the input positions and normals;
    ``iso_value`` is a 0-d tensor on the same graph.
    """

    def __init__(self, coefficients, cumulative, iso, normalization, result):
        self.coefficients = coefficients
        self.cumulative = cumulative
        self.iso_value = iso
        self.normalization = normalization
        self.result = result
        self.metadata = dict(result.metadata)
        self.metadata["differentiability"] = {
            "mode": "finite_algorithm_fixed_assignments", "inputs": ["positions", "normals"],
            "constant_options": ["point_weight", "scale", "samples_per_node", "cg_accuracy", "depths", "iterations"],
            "first_order_only": True}
        self.diagnostics = result.diagnostics

    def evaluate(self, queries, *, centered=False):
        q = _as_vec3(queries, "queries")
        dtype = self.result.field.coefficients.dtype
        if q.dtype != dtype or q.device != self.coefficients.device:
            raise ValueError("queries must match field precision and device")
        return _EvaluateFunction.apply(self.coefficients, self.cumulative, self.iso_value, self.normalization, q,
                                       self.result, bool(centered))


def reconstruct_differentiable(positions, normals, **options):
    """Differentiable reconstruction (warp-psr reconstruction_adjoint.py:61-185).

    Same options as ``reconstruct``.  Positions and/or normals must require gradients; the
    VJP is that of the finite algorithm with its discrete choices (groups, tree, bins,
    schedules, CG stopping points) fixed, first order.  Inputs must stay unchanged until
    backward has run.
    """
    if not isinstance(positions, torch.Tensor) or not isinstance(normals, torch.Tensor):
        raise TypeError("positions and normals must be torch tensors")
    if not positions.requires_grad and not normals.requires_grad:
        raise ValueError("track positions and/or normals with requires_grad=True")
    for name, value in options.items():
        if isinstance(value, torch.Tensor):
            raise ValueError(f"{name} must be a constant scalar; only positions and normals support gradients")
    if options.get("keep_stages"):
        raise ValueError("keep_stages is not available for differentiable reconstructions")
    box = _BackwardStats()
    coefficients, cumulative, iso, normalization = _ReconstructFunction.apply(positions, normals, box, options)
    out = DifferentiableReconstruction(coefficients, cumulative, iso, normalization, box["result"])
    out.backward_stats = box  # box["backward_ms"]: device ms per stage of the last reverse pass
    return out
