"""Marching cubes on the GPU (warp-psr meshing.py:150-346): bit-for-bit against the CPU
restatement (oracle/marching_cubes.py) on the same node values for every backend and both
precisions; the reconstruction's fused extraction (psr_extract_mesh) against the callback
path; closed, outward-oriented surfaces; and mesh-vertex losses differentiated through the
reconstruction, checked by central differences with the cell selection held fixed."""
import math

import numpy as np
import pytest
import torch

from oracle import marching_cubes as omc
from warp_psr_b200 import reconstruct, reconstruct_differentiable
from warp_psr_b200.meshing import extract_isosurface, extract_mesh

pytestmark = pytest.mark.gpu

LO, HI = (-1.2, -1.1, -1.3), (1.25, 1.2, 1.1)


def _bumpy(points):
    x, y, z = points[:, 0], points[:, 1], points[:, 2]
    r = torch.sqrt((x * x + y * y) + z * z)
    return (0.9 + 0.1 * torch.sin(3.0 * x) * torch.cos(2.0 * y)) - r


def _node_values(field, shape, dtype):
    axes = omc.grid(shape, LO, HI, {torch.float32: np.float32, torch.float64: np.float64}[dtype])
    g = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    return field(torch.from_numpy(g).cuda()).cpu().numpy().reshape(shape)


def _check(mesh, values, shape):
    verts, indices, edges, kept = omc.extract(values, shape, LO, HI)
    assert np.array_equal(mesh.metadata["vertex_edges"].cpu().numpy(), edges)
    assert np.array_equal(mesh.indices.cpu().numpy(), indices)
    assert np.array_equal(mesh.vertices.detach().cpu().numpy(), verts)
    return verts, indices


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("backend", ["sparse", "dense", "lipschitz"])
def test_callback_mesh_matches_restatement(dtype, backend):
    shape = (41, 37, 45)
    opts = dict(lipschitz_bound=2.0) if backend == "lipschitz" else dict(slab_size=7)
    mesh = extract_isosurface(_bumpy, resolution=shape, bounds=(LO, HI), backend=backend, dtype=dtype, **opts)
    verts, indices = _check(mesh, _node_values(_bumpy, shape, dtype), shape)
    assert mesh.metadata["triangles"] == len(indices) // 3 > 1000
    # closed (every directed edge has its opposite) and oriented outward (positive volume)
    tri = indices.reshape(-1, 3).astype(np.int64)
    directed = set(map(tuple, np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]]).tolist()))
    assert all((b, a) in directed for a, b in directed)
    v = verts.astype(np.float64)[tri]
    assert np.einsum("ij,ij->i", v[:, 0], np.cross(v[:, 1], v[:, 2])).sum() / 6 > 2.0


def test_empty_and_nonfinite_fields():
    mesh = extract_isosurface(lambda p: torch.ones(len(p), device=p.device), resolution=9, bounds=(LO, HI))
    assert len(mesh.vertices) == 0 and len(mesh.indices) == 0
    with pytest.raises(ValueError, match="nonfinite"):
        extract_isosurface(lambda p: torch.full((len(p),), float("nan"), device=p.device), resolution=9,
                           bounds=(LO, HI))
    with pytest.raises(ValueError, match="resolution"):
        extract_isosurface(_bumpy, resolution=1, bounds=(LO, HI))


def _inner_bounds(points, margin=1.04):
    """The points' bounding box grown by 4% about its centre: inside the reconstruction cube
    (the box grown by the scale 1.1), so every grid node has a finite field value."""
    p = points.double().cpu().numpy()
    c, h = (p.max(0) + p.min(0)) / 2, (p.max(0) - p.min(0)) / 2 * margin
    return tuple(map(float, c - h)), tuple(map(float, c + h))


def _sphere_cloud(count, dtype, seed=2026):
    rng = np.random.default_rng(seed)
    n = rng.normal(size=(count, 3))
    n /= np.linalg.norm(n, axis=1)[:, None]
    p = n * (1 + 0.05 * n[:, :1])
    return torch.from_numpy(p.astype(dtype)).cuda(), torch.from_numpy(n.astype(dtype)).cuda()


@pytest.mark.parametrize("dtype,precision", [(np.float32, "input"), (np.float32, "mixed"), (np.float64, "input")])
def test_reconstruction_mesh_fused_matches_callback(dtype, precision):
    P, N = _sphere_cloud(20000, dtype)
    res = reconstruct(P, N, depth=6, full_depth=3, precision=precision)
    shape = (48, 50, 46)
    bounds = _inner_bounds(P)
    fused = extract_mesh(res, resolution=shape, bounds=bounds)
    fdt = res.field.coefficients.dtype
    iso = res.iso_value

    def field(points):
        v, _, _ = res.evaluate(points)
        return (v - torch.tensor(iso, dtype=fdt, device=v.device)).contiguous()

    generic = extract_isosurface(field, resolution=shape, bounds=bounds, dtype=fdt, slab_size=5)
    assert torch.equal(fused.indices, generic.indices)
    assert torch.equal(fused.vertices, generic.vertices)
    assert fused.metadata["retained_cells"] == generic.metadata["retained_cells"]
    # vertices lie near the isosurface (linear interpolation of a sharp indicator on a coarse grid)
    v, _, ok = res.evaluate(fused.vertices)
    assert bool(ok.all())
    err = (v.double() - iso).abs()
    assert float(err.median()) < 0.01 and float(err.max()) < 0.1, (float(err.median()), float(err.max()))
    assert len(fused.vertices) == fused.metadata["vertices"]


def test_mesh_vertex_loss_reaches_inputs():
    """loss = sum |v|^2 over the mesh vertices; its gradient on positions and normals against
    central differences (float64, h = 1e-6), with the cell selection and connectivity checked
    unchanged at both perturbed points."""
    P, N = _sphere_cloud(3000, np.float64, seed=7)
    opts = dict(depth=4, full_depth=2, iters=3)
    shape, bounds = (20, 20, 20), _inner_bounds(P)
    p = P.clone().requires_grad_(True)
    n = N.clone().requires_grad_(True)
    res = reconstruct_differentiable(p, n, **opts)
    mesh = extract_mesh(res, resolution=shape, bounds=bounds, differentiable=True)
    loss = (mesh.vertices * mesh.vertices).sum()
    loss.backward()
    rng = np.random.default_rng(11)
    dp = torch.from_numpy(rng.normal(size=P.shape)).cuda()
    dn = torch.from_numpy(rng.normal(size=N.shape)).cuda()
    eps = 1e-6
    values = []
    for sign in (1.0, -1.0):
        r = reconstruct(P + sign * eps * dp, N + sign * eps * dn, **opts)
        m = extract_mesh(r, resolution=shape, bounds=bounds)
        assert torch.equal(m.indices, mesh.indices), "cell selection changed under the perturbation"
        values.append(float((m.vertices * m.vertices).sum()))
    fd = (values[0] - values[1]) / (2 * eps)
    an = float((p.grad * dp).sum() + (n.grad * dn).sum())
    assert math.isfinite(an) and abs(an - fd) <= 1e-4 * abs(fd) + 1e-6, (an, fd)
