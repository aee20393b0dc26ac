"""Marching-cubes extraction of the reconstructed surface (warp-psr meshing.py:150-346) on the
library's CUDA kernels (``psr_mc_*``, ``psr_extract_mesh`` in include/psr_b200.h).

The grid, the inside test (centred value >= 0) and the cell selection follow the reference;
the triangulation is this library's own case table (built from the cube faces, crack-free
across cells, normals pointing from inside to outside) with one shared vertex per crossing
grid edge at pa + t (pb - pa), t = fa / (fa - fb).  Cell selection and connectivity carry no
derivative; vertex positions do: when the field values at the kept corners are tracked by
autograd (a callback that returns tracked tensors, or ``extract_mesh(...,
differentiable=True)`` of a ``reconstruct_differentiable`` result) the vertices are recomputed
from them with torch operations in the same order as the kernel, so mesh-vertex losses reach
the isovalue, the coefficients and, through the reconstruction's reverse pass, the input
positions and normals.
"""
import ctypes
import math
import operator
from dataclasses import dataclass

import torch

from . import _lib
from .reconstruction import DifferentiableReconstruction, Reconstruction, _DeviceArray, _stream


@dataclass
class Mesh:
    vertices: torch.Tensor  # (V, 3) model positions, the field's precision
    indices: torch.Tensor   # (3T,) int32, flat triangle vertex indices
    metadata: dict


def _grid(resolution, bounds):
    """(shape, lower, upper) with the reference's checks and messages (meshing.py:121-148)."""
    if isinstance(resolution, int) and not isinstance(resolution, bool):
        resolution = (resolution,) * 3
    try:
        shape = tuple(operator.index(v) for v in resolution)
    except (TypeError, ValueError):
        raise ValueError("resolution must be an integer or three integers >= 2") from None
    if len(shape) != 3 or any(isinstance(v, bool) for v in resolution) or min(shape) < 2:
        raise ValueError("resolution must be an integer or three integers >= 2")
    try:
        lo, hi = (tuple(float(v) for v in row) for row in bounds)
    except (TypeError, ValueError):
        raise ValueError("bounds must contain two finite 3D corners") from None
    if (len(lo) != 3 or len(hi) != 3 or not all(math.isfinite(v) for v in (*lo, *hi))
            or any(a >= b for a, b in zip(lo, hi))):
        raise ValueError("bounds must be finite with lower < upper on every axis")
    if math.prod(n - 1 for n in shape) > 2**31 - 1:
        raise ValueError("extraction cell count exceeds int32 indexing")
    if math.prod(shape) > 2**31 - 1:
        raise ValueError("grid node count exceeds int32 sampling indices")
    return shape, lo, hi


def _c(shape, lo, hi):
    return ((ctypes.c_int64 * 3)(*shape), (ctypes.c_double * 3)(*lo), (ctypes.c_double * 3)(*hi))


def _code(dtype):
    if dtype == torch.float64:
        return _lib.PSR_FLOAT64
    if dtype == torch.float32:
        return _lib.PSR_FLOAT32
    raise ValueError("field values must be float32 or float64")


def _points(shape, lo, hi, dtype, device, *, cells=None, start=0, count):
    out = torch.empty((count, 3), dtype=dtype, device=device)
    s, l, h = _c(shape, lo, hi)
    with torch.cuda.device(device):
        _lib.check(_lib.load().psr_mc_points(_code(dtype), s, l, h, cells.data_ptr() if cells is not None else None,
                                             start, count, out.data_ptr() if count else None, _stream(device)))
    return out


def _take_mesh(ptr, device):
    """Copies a psr_mesh's arrays into torch tensors (stream-ordered) and frees the mesh."""
    L = _lib.load()
    try:
        dt, nv, nt, nc = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _lib.check(L.psr_mesh_info(ptr, ctypes.byref(dt), ctypes.byref(nv), ctypes.byref(nt), ctypes.byref(nc)))
        arrays = [ctypes.c_void_p() for _ in range(5)]
        _lib.check(L.psr_mesh_arrays(ptr, *(ctypes.byref(a) for a in arrays)))
        dtype = torch.float64 if dt.value == _lib.PSR_FLOAT64 else torch.float32

        def copy(addr, count, tdtype, typestr):
            if not count:
                return torch.empty(0, dtype=tdtype, device=device)
            return torch.as_tensor(_DeviceArray(addr.value, (count,), typestr, None), device=device).clone()

        vertices = copy(arrays[0], 3 * nv.value, dtype, "<f8" if dtype == torch.float64 else "<f4").reshape(-1, 3)
        indices = copy(arrays[1], 3 * nt.value, torch.int32, "<i4")
        ends = copy(arrays[3], 2 * nv.value, torch.int64, "<i8").reshape(-1, 2)
        edges = copy(arrays[2], nv.value, torch.int64, "<i8")
        cells = copy(arrays[4], nc.value, torch.int64, "<i8")
        torch.cuda.current_stream(device).synchronize()  # the copies are done before the mesh is freed
        return vertices, indices, ends, cells, edges
    finally:
        L.psr_mesh_free(ptr)


def _triangulate(shape, lo, hi, cells, values, device):
    ptr = ctypes.c_void_p()
    s, l, h = _c(shape, lo, hi)
    vals = values.detach().contiguous()
    with torch.cuda.device(device):
        _lib.check(_lib.load().psr_mc_triangulate(_code(vals.dtype), s, l, h, cells.data_ptr() if len(cells) else None,
                                                  vals.data_ptr() if len(cells) else None, len(cells),
                                                  ctypes.byref(ptr), _stream(device)))
    return _take_mesh(ptr, device)


def _tracked_vertices(points, values, ends):
    """pa + t (pb - pa), t = fa / (fa - fb): the kernel's vertex arithmetic as torch operations
    (no fused multiply-add in either), carrying the corner values' autograd graph."""
    fa, fb = values[ends[:, 0]], values[ends[:, 1]]
    pa, pb = points[ends[:, 0]], points[ends[:, 1]]
    t = fa / (fa - fb)
    return pa + t[:, None] * (pb - pa)


def extract_isosurface(field, *, resolution, bounds, backend="sparse", device=None, slab_size=16,
                       lipschitz_bound=None, classification_field=None, dtype=torch.float32):
    """Zero set of a batched field callback ``field(points) -> values`` (meshing.py:150-281).

    ``points`` are (N, 3) model positions of ``dtype`` on ``device``; the callback returns N
    contiguous values of the same dtype there (subtract the isovalue in the callback).
    ``sparse`` classifies the grid in slabs of ``slab_size`` x-planes into a one-bit-per-cell
    mask and evaluates only the kept cells' corners; ``dense`` classifies the whole grid at
    once (same mesh); ``lipschitz`` needs a caller-proven global bound L in model units and
    skips blocks of 8^3 cells whose centre value exceeds L times their half-diagonal (same
    mesh when the bound holds).  ``classification_field`` (sparse only) may classify without
    recording gradients; it must agree with ``field`` at every grid node.
    """
    if backend not in ("dense", "sparse", "lipschitz"):
        raise ValueError("backend must be dense, sparse, or lipschitz")
    if classification_field is not None and backend != "sparse":
        raise ValueError("classification_field is only used by the sparse backend")
    shape, lo, hi = _grid(resolution, bounds)
    if not isinstance(slab_size, int) or isinstance(slab_size, bool) or slab_size < 1:
        raise ValueError("slab_size must be a positive integer")
    if backend == "lipschitz":
        if lipschitz_bound is None or not math.isfinite(lipschitz_bound) or lipschitz_bound <= 0:
            raise ValueError("lipschitz backend requires a finite positive proven lipschitz_bound")
    elif lipschitz_bound is not None:
        raise ValueError("lipschitz_bound is only used by the lipschitz backend")
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if dtype not in (torch.float32, torch.float64):
        raise ValueError("dtype must be torch.float32 or torch.float64")
    samples = 0

    def sample(points, classification=False):
        nonlocal samples
        callback = classification_field if classification and classification_field is not None else field
        values = callback(points)
        if (not isinstance(values, torch.Tensor) or values.dtype != dtype or values.shape != (len(points),)
                or values.device != device or not values.is_contiguous()):
            raise ValueError("field must return contiguous values of the points' dtype, one per point, on the "
                             "query device")
        samples += len(points)
        return values

    nx, ny, nz = shape
    metadata = {"backend": backend, "resolution": shape, "bounds": (lo, hi),
                "precision": "float64" if dtype == torch.float64 else "float32",
                "cell_selection": "fixed for backward"}
    L = _lib.load()
    s, l, h = _c(shape, lo, hi)
    if backend == "lipschitz":
        cells = _lipschitz_cells(sample, shape, lo, hi, lipschitz_bound, dtype, device, metadata)
    else:
        slab = slab_size if backend == "sparse" else nx - 1
        words = ((nx - 1) * (ny - 1) * (nz - 1) + 31) // 32
        mask = torch.zeros(words, dtype=torch.int32, device=device)
        status = torch.zeros(1, dtype=torch.int32, device=device)
        for start in range(0, nx - 1, slab):
            width = min(slab, nx - 1 - start)
            pts = _points(shape, lo, hi, dtype, device, start=start, count=(width + 1) * ny * nz)
            values = sample(pts, classification=True)
            with torch.cuda.device(device):
                _lib.check(L.psr_mc_mark(_code(dtype), values.detach().data_ptr(), s, start, width, mask.data_ptr(),
                                         status.data_ptr(), _stream(device)))
        count = ctypes.c_int64()
        with torch.cuda.device(device):
            _lib.check(L.psr_mc_cells(mask.data_ptr(), words, None, 0, ctypes.byref(count), _stream(device)))
        if int(status.item()):
            raise ValueError("field returned nonfinite values inside extraction bounds")
        cells = torch.empty(count.value, dtype=torch.int64, device=device)
        if count.value:
            with torch.cuda.device(device):
                _lib.check(L.psr_mc_cells(mask.data_ptr(), words, cells.data_ptr(), count.value, ctypes.byref(count),
                                          _stream(device)))
        metadata.update(retained_cells=count.value, slab_size=slab, selection_bytes=words * 12)
    pts = _points(shape, lo, hi, dtype, device, cells=cells, count=8 * len(cells))
    values = sample(pts) if len(cells) else torch.empty(0, dtype=dtype, device=device)
    vertices, indices, ends, _, edges = _triangulate(shape, lo, hi, cells, values, device)
    if values.requires_grad:
        vertices = _tracked_vertices(pts, values, ends)
    metadata.update(field_evaluations=samples, vertices=len(vertices), triangles=len(indices) // 3,
                    vertex_edges=edges)
    return Mesh(vertices, indices, metadata)


def _lipschitz_cells(sample, shape, lo, hi, bound, dtype, device, metadata, block=8):
    """Cells of the 8^3-cell blocks that the bound cannot exclude: |f(centre)| <= L * r."""
    nx, ny, nz = shape
    step = [(float(torch.tensor(h, dtype=torch.float32)) - float(torch.tensor(l, dtype=torch.float32))) / (n - 1)
            for l, h, n in zip(lo, hi, shape)]
    nb = [(n - 2) // block + 1 for n in shape]
    bi = torch.stack(torch.meshgrid(*(torch.arange(k, device=device) for k in nb), indexing="ij"), -1).reshape(-1, 3)
    c0 = bi * block
    c1 = torch.minimum(c0 + block, torch.tensor([nx - 1, ny - 1, nz - 1], device=device))
    lower = torch.tensor(lo, dtype=torch.float64, device=device)
    st = torch.tensor(step, dtype=torch.float64, device=device)
    centre = lower + st * (c0 + c1).double() * 0.5
    radius = 0.5 * torch.linalg.norm(st * (c1 - c0).double(), dim=1)
    with torch.no_grad():
        v = sample(centre.to(dtype).contiguous()).double()
    keep = v.abs() <= bound * radius
    if not bool(torch.isfinite(v).all()):
        raise ValueError("field returned nonfinite values inside extraction bounds")
    kept = bi[keep]
    offs = torch.stack(torch.meshgrid(*(torch.arange(block, device=device),) * 3, indexing="ij"), -1).reshape(-1, 3)
    c = (kept[:, None, :] * block + offs[None]).reshape(-1, 3)
    c = c[(c[:, 0] < nx - 1) & (c[:, 1] < ny - 1) & (c[:, 2] < nz - 1)]
    cells = ((c[:, 0] * (ny - 1) + c[:, 1]) * (nz - 1) + c[:, 2]).sort().values.contiguous()
    metadata.update(retained_cells=len(cells), lipschitz_bound=bound, blocks=int(len(bi)), kept_blocks=int(len(kept)))
    return cells


def extract_mesh(reconstruction, *, resolution, bounds, iso_value=None, differentiable=False, **options):
    """Mesh of a reconstruction's isosurface (meshing.py:284-346).

    ``reconstruction``: a ``Reconstruction`` (plain) or, with ``differentiable=True``, a
    ``reconstruct_differentiable`` result, whose mesh vertices then carry gradients to the
    input positions and normals and to the isovalue.  ``iso_value`` defaults to the
    reconstruction's; a one-element tensor keeps its own gradient.  The plain sparse path runs
    the whole extraction in the library (psr_extract_mesh: slabs evaluated and classified on
    the device, kept corners evaluated and triangulated); other options go through
    ``extract_isosurface``.  Selection, bounds and connectivity stay fixed.
    """
    if isinstance(reconstruction, DifferentiableReconstruction):
        if not differentiable:
            raise ValueError("a differentiable reconstruction requires differentiable=True for meshing")
        result = reconstruction.result
    elif isinstance(reconstruction, Reconstruction):
        if differentiable:
            raise ValueError("differentiable meshing requires a reconstruct_differentiable result")
        result = reconstruction
    else:
        raise TypeError("expected a Reconstruction or a differentiable reconstruction")
    field = result.field
    device = field.coefficients.device
    dtype = field.coefficients.dtype
    if "device" in options and torch.device(options["device"]) != device:
        raise ValueError("mesh device must match the field device")
    options.pop("device", None)
    if iso_value is None:
        iso = reconstruction.iso_value if differentiable else torch.tensor(field.iso_value, dtype=dtype, device=device)
    elif isinstance(iso_value, torch.Tensor):
        if iso_value.numel() != 1 or iso_value.device != device:
            raise ValueError("iso_value must be one value on the field device")
        if iso_value.requires_grad and not differentiable:
            raise ValueError("tracked iso_value requires differentiable=True")
        iso = iso_value.reshape(()).to(dtype)
    else:
        if not math.isfinite(iso_value):
            raise ValueError("iso_value must be finite")
        iso = torch.tensor(float(iso_value), dtype=dtype, device=device)
    backend = options.get("backend", "sparse")
    fused = backend == "sparse" and not options.get("lipschitz_bound") and not options.get("classification_field")
    if fused:
        slab = options.get("slab_size", 16)
        if not isinstance(slab, int) or isinstance(slab, bool) or slab < 1:
            raise ValueError("slab_size must be a positive integer")
        shape, lo, hi = _grid(resolution, bounds)
        s, l, h = _c(shape, lo, hi)
        ptr, retained = ctypes.c_void_p(), ctypes.c_int64()
        with torch.cuda.device(device):
            _lib.check(_lib.load().psr_extract_mesh(field._handle.ptr, s, l, h, float(iso.detach()), slab,
                                                    ctypes.byref(retained), ctypes.byref(ptr), _stream(device)))
        vertices, indices, ends, cells, edges = _take_mesh(ptr, device)
        metadata = {"backend": "sparse", "resolution": shape, "bounds": (lo, hi),
                    "precision": "float64" if dtype == torch.float64 else "float32",
                    "cell_selection": "fixed for backward", "retained_cells": retained.value, "slab_size": slab,
                    "field_evaluations": int(math.prod(shape) + ((shape[0] - 2) // slab) * shape[1] * shape[2]
                                             + 8 * retained.value)}
        if differentiable and len(cells):
            pts = _points(shape, lo, hi, dtype, device, cells=cells, count=8 * len(cells))
            values, _, _ = reconstruction.evaluate(pts)
            vertices = _tracked_vertices(pts, values - iso, ends)
        elif differentiable:
            vertices = vertices.requires_grad_(True)
        metadata.update(vertices=len(vertices), triangles=len(indices) // 3, vertex_edges=edges)
        return Mesh(vertices, indices, metadata)

    def sample(points):
        if differentiable:
            values, _, _ = reconstruction.evaluate(points)
            return (values - iso).contiguous()
        values, _, _ = field.evaluate(points)
        return (values - iso).contiguous()

    if differentiable and backend == "sparse":
        def classify(points):
            with torch.no_grad():
                values, _, _ = field.evaluate(points)
                return (values - iso.detach()).contiguous()
        options.setdefault("classification_field", classify)
    mesh = extract_isosurface(sample, resolution=resolution, bounds=bounds, device=device, dtype=dtype, **options)
    if differentiable and not len(mesh.vertices):
        mesh.vertices.requires_grad_(True)
    return mesh
