"""The marching-cubes restatement (oracle/marching_cubes.py, the CUDA kernels' checker):
its case table closes every surface it cuts and orients it away from the inside."""
import math

import numpy as np

from oracle import marching_cubes as mc


def _edge_uses(indices):
    uses = {}
    for tri in indices.reshape(-1, 3).tolist():
        for k in range(3):
            a, b = tri[k], tri[(k + 1) % 3]
            uses.setdefault((a, b), 0)
            uses[(a, b)] += 1
    return uses


def test_case_table_sizes():
    table = mc.case_table()
    assert table[0] == [] and table[255] == []
    assert all(len(table[code]) >= 1 for code in range(1, 255))
    assert max(len(t) for t in table.values()) <= 8
    assert len(table[1]) == 1 and len(table[3]) == 2


def test_random_fields_give_closed_oriented_surfaces():
    rng = np.random.default_rng(5)
    shape = (9, 8, 7)
    for dtype in (np.float32, np.float64):
        values = rng.normal(size=shape).astype(dtype)
        # no surface reaches the grid's outer faces: every edge is shared by two triangles
        values[0], values[-1], values[:, 0], values[:, -1], values[:, :, 0], values[:, :, -1] = (-1,) * 6
        verts, indices, edges, kept = mc.extract(values, shape, (0, 0, 0), (1, 1, 1))
        uses = _edge_uses(indices)
        assert uses and all(count == 1 for count in uses.values())
        assert all((b, a) in uses for a, b in uses), "every directed edge has its opposite"
        assert len(np.unique(edges)) == len(edges) == len(verts)


def test_sphere_is_closed_with_outward_normals():
    n = 33
    lo, hi = (-1.2,) * 3, (1.2,) * 3
    axes = mc.grid((n, n, n), lo, hi, np.float64)
    x, y, z = np.meshgrid(*axes, indexing="ij")
    values = 1.0 - np.sqrt(x * x + y * y + z * z)  # inside positive
    verts, indices, _, _ = mc.extract(values, (n, n, n), lo, hi)
    tris = verts[indices.reshape(-1, 3).astype(np.int64)]
    volume = np.einsum("ij,ij->i", tris[:, 0], np.cross(tris[:, 1], tris[:, 2])).sum() / 6
    assert abs(volume - 4 / 3 * math.pi) < 0.02 * 4 / 3 * math.pi
    assert len(verts) - len(_edge_uses(indices)) // 2 + len(indices) // 3 == 2  # Euler characteristic
    assert np.abs(np.linalg.norm(verts, axis=1) - 1).max() < 0.01
