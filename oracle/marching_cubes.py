"""CPU restatement of the sparse marching-cubes extraction (test infrastructure only).

Follows warp-psr's grid, inside test and cell selection (meshing.py:38-85,121-148: nodes at
clamp(lower + step * index), step computed in float32, a node inside when its centred value is
>= 0, a cell kept when its corners are mixed) and the library's triangulation: the case table
built from the cube faces (every maximal run of inside corners on a face, walked
counter-clockwise from outside, gives one segment from the edge entering the run to the edge
leaving it; segments chain into loops; each loop is a fan, oriented away from the inside),
one vertex per crossing grid edge at pa + t (pb - pa), t = fa / (fa - fb), vertices numbered
by ascending edge id ((lower node index) * 3 + axis), triangles in ascending cell order.
Warp's own table (the reference's) is not installable here; this restatement is what the
CUDA kernels are checked against, bit for bit.
"""
import numpy as np

CORNER = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
EDGE = [(0, 1), (3, 2), (0, 3), (1, 2), (4, 5), (7, 6), (4, 7), (5, 6), (0, 4), (1, 5), (3, 7), (2, 6)]
FACE = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]


def _edge(a, b):
    for e, (p, q) in enumerate(EDGE):
        if {p, q} == {a, b}:
            return e
    raise ValueError((a, b))


def _loops(code):
    inside = [(code >> c) & 1 for c in range(8)]
    segments = []
    for face in FACE:
        for i in range(4):
            c, prev = face[i], face[i - 1]
            if not inside[c] or inside[prev]:
                continue
            j = i
            while inside[face[(j + 1) % 4]]:
                j = (j + 1) % 4
            segments.append((_edge(prev, c), _edge(face[j], face[(j + 1) % 4])))
    loops, used = [], [False] * len(segments)
    for s in range(len(segments)):
        if used[s]:
            continue
        loop, cur = [segments[s][0]], s
        while True:
            used[cur] = True
            e = segments[cur][1]
            if e == loop[0]:
                break
            loop.append(e)
            cur = next(t for t in range(len(segments)) if not used[t] and segments[t][0] == e)
        loops.append(loop)
    return loops


def case_table():
    """{code: [(e0, e1, e2), ...]} oriented with normals pointing away from the inside."""
    def mid(e):
        a, b = EDGE[e]
        return 0.5 * (np.array(CORNER[a], float) + np.array(CORNER[b], float))

    loop = _loops(1)[0]
    n = np.cross(mid(loop[1]) - mid(loop[0]), mid(loop[2]) - mid(loop[0]))
    flip = n.sum() < 0
    table = {}
    for code in range(256):
        tris = []
        for loop in _loops(code):
            for k in range(1, len(loop) - 1):
                tris.append((loop[0], loop[k + 1], loop[k]) if flip else (loop[0], loop[k], loop[k + 1]))
        table[code] = tris
    return table


def grid(shape, lower, upper, dtype):
    """float32 step (meshing.py:145-147) and the node coordinate arrays per axis in dtype."""
    lo32 = np.array(lower, np.float32)
    hi32 = np.array(upper, np.float32)
    step32 = (hi32 - lo32) / np.array([n - 1 for n in shape], np.float32)
    axes = []
    for a in range(3):
        lo, hi, st = dtype(lo32[a]), dtype(hi32[a]), dtype(step32[a])
        v = lo + st * np.arange(shape[a]).astype(dtype)
        axes.append(np.minimum(np.maximum(v, lo), hi).astype(dtype))
    return axes


def extract(values, shape, lower, upper):
    """Mesh of centred node values (nx, ny, nz): (vertices (V, 3), indices (3T,) int32,
    vertex edge ids (V,), kept cells (C,))."""
    values = np.asarray(values)
    dtype = values.dtype.type
    nx, ny, nz = shape
    axes = grid(shape, lower, upper, dtype)
    inside = values >= 0
    codes = np.zeros((nx - 1, ny - 1, nz - 1), np.int64)
    for c, (dx, dy, dz) in enumerate(CORNER):
        codes |= inside[dx:nx - 1 + dx, dy:ny - 1 + dy, dz:nz - 1 + dz].astype(np.int64) << c
    kept = np.nonzero(((codes != 0) & (codes != 255)).reshape(-1))[0]
    table = case_table()
    corner_edges = []
    for cell in kept.tolist():
        x, rem = divmod(cell, (ny - 1) * (nz - 1))
        y, z = divmod(rem, nz - 1)
        for tri in table[int(codes[x, y, z])]:
            for e in tri:
                a, b = EDGE[e]
                axis = next(k for k in range(3) if CORNER[a][k] != CORNER[b][k])
                node = ((x + CORNER[a][0]) * ny + y + CORNER[a][1]) * nz + z + CORNER[a][2]
                corner_edges.append(node * 3 + axis)
    corner_edges = np.array(corner_edges, np.int64)
    edges, indices = np.unique(corner_edges, return_inverse=True)
    verts = np.zeros((len(edges), 3), dtype)
    for v, edge in enumerate(edges.tolist()):
        node, axis = divmod(edge, 3)
        i, rem = divmod(node, ny * nz)
        j, k = divmod(rem, nz)
        c = [i, j, k]
        d = list(c)
        d[axis] += 1
        pa = np.array([axes[0][c[0]], axes[1][c[1]], axes[2][c[2]]], dtype)
        pb = np.array([axes[0][d[0]], axes[1][d[1]], axes[2][d[2]]], dtype)
        fa, fb = values[c[0], c[1], c[2]], values[d[0], d[1], d[2]]
        t = dtype(fa / (fa - fb))
        verts[v] = pa + t * (pb - pa)
    return verts, indices.astype(np.int32), edges, kept
