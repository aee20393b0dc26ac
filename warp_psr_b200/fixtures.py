"""Reference fixture files: read and write the text formats of warp-psr's offline oracle
(reference/README.md:27-64) and check a reconstruction against a fixture directory.

A fixture directory made by a PoissonRecon 262b0f5 build (tools/make_fixture.py in the
reference) holds these files; ``check_fixture`` is this library's counterpart of the
reference's tools/check_reconstruction.py:16-60, so that the build can be checked against
PoissonRecon whenever such a fixture is provisioned.  Every file is plain text, one record
per line, values separated by blanks and written with 17 significant digits:

* ``input.pts``: ``x y z nx ny nz`` per input point, in input order
  (tools/make_fixture.py:88);
* ``queries.txt``: ``x y z`` per model-space query point;
* ``oracle.txt``: tagged rows -- ``iso v``; ``transform`` and the 16 entries of the
  cube-to-model matrix in PoissonRecon's column-first order; ``q value gx gy gz`` per query
  (value and model-space gradient); ``node d x y z flags ghost index coefficient`` per tree
  node (oracle_instrumented.txt: flags bit 1 marks an active basis function, ghost 1 a node
  outside the non-ghost support, coefficient the per-level correction); thread-pool rows
  (reference/oracle.cpp:54-81,114-116);
* ``stages.txt``: tagged rows -- ``effective`` and the resolved depth, full depth, base
  depth, solve depth, kernel depth, scale, samples per node, point weight, exact
  interpolation, iterations and CG accuracy; ``density_scale w0 w1``; ``sample d x y z px py
  pz weight`` (leaf cell, position sum, weight); ``normal d x y z nx ny nz``; ``density d x
  y z v``; ``load d x y z v`` (unscreened FEM load) (tools/build_reference.py:36-67);
* ``inputs.txt``: ``input id status depth x y z`` per input (reference/README.md:31-36);
* ``manifest.json``: name, precision ("double" or "float") and reconstruction parameters.

Depth and coordinates in the tagged rows are canonical: a basis function or cell of depth d
at integer (x, y, z), the reference's key ``d<<48 | x<<32 | y<<16 | z``.
"""
import json
from pathlib import Path

import numpy as np

# Field budgets of the reference's design (check_reconstruction.py:23): (absolute, relative).
FIELD_TOLERANCE = {"double": (1e-8, 1e-6), "float": (1e-5, 1e-4)}
_SUPPORT_BIAS = 524288  # non-ghost support keys: (x + 2^19) << 40 | (y + 2^19) << 20 | (z + 2^19)


def read_tagged(path):
    """Rows of a tagged text file grouped by their first word: {tag: float64 array (rows x
    values)} (the reference reads these files the same way, tools/make_fixture.py:23-26)."""
    rows = {}
    for line in Path(path).read_text().splitlines():
        parts = line.split()
        if parts:
            rows.setdefault(parts[0], []).append([float(v) for v in parts[1:]])
    return {tag: np.array(values, dtype=np.float64) for tag, values in rows.items()}


def _value(v):
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return format(float(v), ".17g")


def write_tagged(path, rows):
    """Writes (tag, values) rows; integers as integers, reals with 17 significant digits."""
    with open(path, "w") as f:
        for tag, values in rows:
            f.write(" ".join([tag, *(_value(v) for v in values)]) + "\n")


def write_input_pts(path, positions, normals):
    positions = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    normals = np.asarray(normals, dtype=np.float64).reshape(-1, 3)
    if len(positions) != len(normals):
        raise ValueError("positions and normals must have the same length")
    np.savetxt(path, np.column_stack([positions, normals]), fmt="%.17g")


def read_input_pts(path, dtype=np.float64):
    """(positions, normals) of an input.pts file as (n, 3) arrays of `dtype`."""
    data = np.loadtxt(path, ndmin=2)
    if data.shape[1] != 6:
        raise ValueError(f"{path}: expected 6 values per line, found {data.shape[1]}")
    data = data.astype(dtype)
    return np.ascontiguousarray(data[:, :3]), np.ascontiguousarray(data[:, 3:])


def write_queries(path, queries):
    np.savetxt(path, np.asarray(queries, dtype=np.float64).reshape(-1, 3), fmt="%.17g")


def read_queries(path, dtype=np.float64):
    data = np.loadtxt(path, ndmin=2)
    if data.shape[1] != 3:
        raise ValueError(f"{path}: expected 3 values per line, found {data.shape[1]}")
    return np.ascontiguousarray(data.astype(dtype))


def key_coords(keys):
    """(depth, x, y, z) int64 columns of basis keys d<<48 | x<<32 | y<<16 | z."""
    keys = np.asarray(keys, dtype=np.int64)
    return np.stack([keys >> 48, (keys >> 32) & 65535, (keys >> 16) & 65535, keys & 65535], axis=1)


def support_coords(keys):
    """(x, y, z) int64 columns of non-ghost support keys (signed, biased by 2^19)."""
    keys = np.asarray(keys, dtype=np.int64)
    mask = (1 << 20) - 1
    return np.stack([(keys >> 40) - _SUPPORT_BIAS, ((keys >> 20) & mask) - _SUPPORT_BIAS,
                     (keys & mask) - _SUPPORT_BIAS], axis=1)


def node_rows(basis_keys, coefficients, support_keys):
    """``node`` rows of a tree: the union per depth of the active basis functions (flags 2,
    their index and coefficient) and the non-ghost support nodes (ghost 0).

    basis_keys / coefficients: all levels' keys (sorted) and per-level coefficients;
    support_keys: one array of non-ghost support keys per depth."""
    basis_keys = np.asarray(basis_keys, dtype=np.int64)
    coefficients = np.asarray(coefficients, dtype=np.float64)
    bc = key_coords(basis_keys)
    rows = []
    for d, sup in enumerate(support_keys):
        sc = support_coords(sup)
        sel = np.nonzero(bc[:, 0] == d)[0]
        nodes = {}
        for x, y, z in sc.tolist():
            nodes[(x, y, z)] = [0, 0, -1, 0.0]  # flags, ghost, index, coefficient
        for i in sel.tolist():
            xyz = tuple(bc[i, 1:].tolist())
            entry = nodes.setdefault(xyz, [0, 1, -1, 0.0])
            entry[0] |= 2
            entry[2] = i
            entry[3] = float(coefficients[i])
        for (x, y, z), (flags, ghost, index, coefficient) in sorted(nodes.items()):
            rows.append((d, x, y, z, flags, ghost, index, coefficient))
    return rows


def write_oracle(path, *, iso, cube_to_model, values=None, gradients=None, nodes=(), threads=1):
    """oracle.txt: thread-pool rows, iso, transform (column-first), q rows, node rows."""
    m = np.asarray(cube_to_model, dtype=np.float64).reshape(4, 4)
    rows = [("parallel_async", [0]), ("threads", [int(threads)]), ("schedule", [0]), ("chunk_size", [0]),
            ("openmp_effective_threads", [0]), ("iso", [float(iso)]), ("transform", list(m.T.reshape(-1)))]
    if values is not None:
        values = np.asarray(values, dtype=np.float64).reshape(-1)
        gradients = np.asarray(gradients, dtype=np.float64).reshape(-1, 3)
        rows += [("q", [v, *g]) for v, g in zip(values.tolist(), gradients.tolist())]
    rows += [("node", [int(d), int(x), int(y), int(z), int(f), int(gh), int(ix), float(c)])
             for d, x, y, z, f, gh, ix, c in nodes]
    write_tagged(path, rows)


def write_stages(path, *, effective, density_scale=None, samples=None, normals=None, densities=None, loads=None):
    """stages.txt.  effective: the 11 resolved settings (depth, full_depth, base_depth,
    solve_depth, kernel_depth, scale, samples_per_node, point_weight, exact_interpolation,
    iters, cg_accuracy); samples: (keys, position sums (g, 3), weights); normals: (keys,
    values (m, 3)); densities and loads: (keys, values), all keys d<<48 | x<<32 | y<<16 | z."""
    ints = (0, 1, 2, 3, 4, 8, 9)
    rows = [("effective", [int(v) if i in ints else float(v) for i, v in enumerate(effective)])]
    if density_scale is not None:
        rows.append(("density_scale", [float(v) for v in density_scale]))
    if samples is not None:
        keys, sums, weights = samples
        sums = np.asarray(sums, dtype=np.float64).reshape(-1, 3)
        for kc, s, w in zip(key_coords(keys).tolist(), sums.tolist(), np.asarray(weights, np.float64).tolist()):
            rows.append(("sample", [*kc, *s, w]))
    if normals is not None:
        keys, values = normals
        values = np.asarray(values, dtype=np.float64).reshape(-1, 3)
        rows += [("normal", [*kc, *v]) for kc, v in zip(key_coords(keys).tolist(), values.tolist())]
    for tag, block in (("density", densities), ("load", loads)):
        if block is not None:
            keys, values = block
            rows += [(tag, [*kc, float(v)]) for kc, v in zip(key_coords(keys).tolist(),
                                                               np.asarray(values, np.float64).reshape(-1).tolist())]
    write_tagged(path, rows)


def tree_from_nodes(nodes, depth):
    """Per depth (support keys, active basis keys), both sorted, from ``node`` rows
    (tools/check_tree.py:6-22): support = non-ghost nodes in the biased signed encoding,
    active = nodes whose flags have bit 1."""
    nodes = np.asarray(nodes)
    out = []
    for d in range(depth + 1):
        at = nodes[:, 0] == d
        s = nodes[at & (nodes[:, 5] == 0), 1:4].astype(np.int64) + _SUPPORT_BIAS
        support = np.sort((s[:, 0] << 40) | (s[:, 1] << 20) | s[:, 2])
        a = nodes[at & ((nodes[:, 4].astype(np.int64) & 2) != 0), 1:4].astype(np.int64)
        active = np.sort((np.int64(d) << 48) | (a[:, 0] << 32) | (a[:, 1] << 16) | a[:, 2])
        out.append((support, active))
    return out


def refined_cells(nodes, normals, depth):
    """Cells refined below each depth, as sets of (x, y, z): the canonical integration
    partition the reference builds from its exported supports (reference/cells.py:5-30)."""
    required = [set() for _ in range(depth + 1)]
    for row in np.asarray(nodes):
        d = int(row[0])
        if d < 0 or d > depth or not (int(row[4]) & 2):
            continue
        x, y, z = (int(v) for v in row[1:4])
        n = 1 << d
        for a in (0, 1):
            for b in (0, 1):
                for c in (0, 1):
                    q = (x - a, y - b, z - c)
                    if min(q) >= 0 and max(q) < n:
                        required[d].add(q)
    for row in np.asarray(normals):
        d = int(row[0])
        if d < 0 or d > depth:
            continue
        x, y, z = (int(v) for v in row[1:4])
        n = 1 << d
        for a in (-1, 0, 1):
            for b in (-1, 0, 1):
                for c in (-1, 0, 1):
                    q = (x + a, y + b, z + c)
                    if min(q) >= 0 and max(q) < n:
                        required[d].add(q)
    refined = [set() for _ in range(depth + 1)]
    for d in range(depth - 1, -1, -1):
        refined[d] = {(x // 2, y // 2, z // 2) for x, y, z in required[d + 1]}
        required[d].update(refined[d])
    return refined


def query_cell_widths(nodes, normals, cube_queries, depth):
    """Width of the finest refined cell holding each unit-cube query (reference/cells.py:33-48):
    the scale of the reference's gradient budget."""
    refined = refined_cells(nodes, normals, depth)
    cube_queries = np.asarray(cube_queries, dtype=np.float64)
    widths = np.ones(len(cube_queries))
    for d in range(len(refined) - 1):
        keys = np.array(sorted((x << 32) | (y << 16) | z for x, y, z in refined[d]), dtype=np.int64)
        if not len(keys):
            continue
        coord = np.minimum(np.floor(cube_queries * (1 << d)).astype(np.int64), (1 << d) - 1)
        q = (coord[:, 0] << 32) | (coord[:, 1] << 16) | coord[:, 2]
        index = np.searchsorted(keys, q)
        valid = index < len(keys)
        valid[valid] &= keys[index[valid]] == q[valid]
        widths[valid] = 1.0 / (1 << (d + 1))
    return widths


def reconstruct_options(parameters):
    """reconstruct() keywords from a manifest's ``parameters`` (the reference's names)."""
    p = parameters
    return dict(depth=int(p["depth"]), full_depth=int(p["full_depth"]), base_depth=p.get("base_depth"),
                solve_depth=p.get("solve_depth"), kernel_depth=p.get("kernel_depth"), scale=float(p["scale"]),
                samples_per_node=float(p["samples_per_node"]), point_weight=float(p["weight"]),
                exact_interpolation=bool(p.get("exact", False)), iters=int(p.get("iters", 8)),
                base_v_cycles=int(p.get("base_v_cycles", 1)), cg_accuracy=float(p.get("cg_accuracy", 1e-3)))


def check_fixture(directory, device="cuda"):
    """Reconstructs a fixture's input.pts with its manifest's parameters and checks the result
    against its oracle files the way the reference's tools/check_reconstruction.py:16-60 does:
    values and isovalue-centred values at queries.txt, cell-width-scaled cube-frame
    gradients (widths from the node rows and the stages.txt normal rows), the isovalue, and
    the exact non-ghost support and active basis keys of every depth.  Raises AssertionError
    on a difference beyond the design budgets; returns a report of the errors."""
    import torch
    from .reconstruction import reconstruct

    directory = Path(directory)
    manifest = json.loads((directory / "manifest.json").read_text())
    double = manifest["precision"] == "double"
    dtype = np.float64 if double else np.float32
    atol, rtol = FIELD_TOLERANCE["double" if double else "float"]
    options = reconstruct_options(manifest["parameters"])
    positions, normals = read_input_pts(directory / "input.pts", dtype)
    queries = read_queries(directory / "queries.txt", dtype)
    tdev = torch.device(device)
    result = reconstruct(torch.from_numpy(positions).to(tdev), torch.from_numpy(normals).to(tdev), **options)
    v, g, valid = result.evaluate(torch.from_numpy(queries).to(tdev))
    if not bool(valid.all()):
        raise AssertionError("a fixture query lies outside the reconstruction cube")
    actual = np.column_stack([v.double().cpu().numpy(), g.double().cpu().numpy()])
    expected = read_tagged(directory / "oracle.txt")
    q = expected["q"]
    instrumented = directory / "oracle_instrumented.txt"
    nodes = read_tagged(instrumented if instrumented.exists() else directory / "oracle.txt").get("node")
    linear = np.array(result.field.linear, dtype=np.float64).reshape(3, 3)
    inverse = np.linalg.inv(linear)
    cube_grad, ref_grad = actual[:, 1:] @ inverse, q[:, 1:] @ inverse
    np.testing.assert_allclose(actual[:, 0], q[:, 0], atol=atol, rtol=rtol, err_msg="field values")
    centred, ref_centred = actual[:, 0] - result.iso_value, q[:, 0] - expected["iso"][0, 0]
    np.testing.assert_allclose(centred, ref_centred, atol=atol, rtol=rtol, err_msg="centred field values")
    widths = np.ones(len(queries))
    stages = directory / "stages.txt"
    if nodes is not None and stages.exists():
        cube = queries.astype(np.float64) @ linear.T + np.array(result.field.translation)
        widths = query_cell_widths(nodes, read_tagged(stages).get("normal", np.zeros((0, 7))), cube,
                                   options["depth"])
    np.testing.assert_allclose(cube_grad * widths[:, None], ref_grad * widths[:, None], atol=atol, rtol=rtol,
                               err_msg="cell-width-scaled cube gradients")
    np.testing.assert_allclose(result.iso_value, expected["iso"][0, 0], atol=atol, rtol=rtol, err_msg="isovalue")
    tree = None
    if nodes is not None:
        keys = result.field.keys.cpu().numpy()
        offsets = result.diagnostics["level_offsets"]
        tree = []
        for d, (support, active) in enumerate(tree_from_nodes(nodes, options["depth"])):
            mine = result.diagnostics["support_keys"][d].cpu().numpy()
            np.testing.assert_array_equal(mine, support, err_msg=f"non-ghost support keys differ at depth {d}")
            np.testing.assert_array_equal(keys[offsets[d]:offsets[d + 1]], active,
                                          err_msg=f"active basis keys differ at depth {d}")
            tree.append({"depth": d, "support_count": len(support), "active_count": len(active)})
    delta = actual[:, 0] - q[:, 0]
    return {"fixture": manifest.get("name", directory.name), "precision": manifest["precision"],
            "queries": len(queries), "max_abs_value_error": float(np.abs(delta).max()),
            "max_abs_centred_value_error": float(np.abs(centred - ref_centred).max()),
            "max_abs_cube_gradient_error": float(np.abs(cube_grad - ref_grad).max()),
            "iso_value": result.iso_value, "reference_iso_value": float(expected["iso"][0, 0]), "tree": tree}
