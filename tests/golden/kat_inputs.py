"""Seeded oriented clouds of the reference's known-answer fixtures.

Restates the shape generator of warp-psr ``tools/make_fixture.py:51-80`` and the
scale/translation/precision steps of ``tools/make_fixture.py:107-110``.  The result
is checked against the ``input.pts`` SHA-256 recorded for every fixture (the file
the reference wrote with ``np.savetxt(fmt="%.17g")``), so the inputs are pinned
byte-for-byte.
"""
import hashlib
import io

import numpy as np


def shape_points(shape, count, seed):
    rng = np.random.default_rng(seed)
    if shape in ("plane", "sheets"):
        p = rng.uniform(-1, 1, (count, 3))
        p[:, 2] = 0
        n = np.zeros_like(p)
        n[:, 2] = 1
        if shape == "sheets":
            sign = np.where(np.arange(count) % 2, 1.0, -1.0)
            p[:, 2] = 0.035 * sign
            n[:, 2] = sign
        return p, n
    if shape in ("sphere", "cluster", "disconnected"):
        n = rng.normal(size=(count, 3))
        if shape == "cluster":
            m = 9 * count // 10
            n[:m] = rng.normal(scale=0.12, size=(m, 3)) + [0, 0, 1]
        n /= np.linalg.norm(n, axis=1)[:, None]
        if shape == "disconnected":
            p = 0.25 * n
            p[:, 0] += np.where(np.arange(count) % 2, 0.65, -0.65)
            return p, n
        return n, n.copy()
    if shape == "torus":
        u, v = rng.uniform(0, 2 * np.pi, size=(2, count))
        p = np.array([(0.7 + 0.26 * np.cos(v)) * np.cos(u),
                      (0.7 + 0.26 * np.cos(v)) * np.sin(u), 0.26 * np.sin(v)]).T
        n = np.array([np.cos(v) * np.cos(u), np.cos(v) * np.sin(u), np.sin(v)]).T
        return p, n
    raise ValueError(f"unknown fixture shape {shape}")


def fixture_input(params):
    """(positions, normals) in the fixture precision, exactly as the reference saved them."""
    p, n = shape_points(params["shape"], params["count"], params["seed"])
    p = p * params["input_scale"] + np.asarray(params["translation"])
    dtype = np.float32 if params["precision"] == "float" else np.float64
    return p.astype(dtype), n.astype(dtype)


def input_sha256(p, n):
    buf = io.BytesIO()
    np.savetxt(buf, np.column_stack([p, n]), fmt="%.17g")
    return hashlib.sha256(buf.getvalue()).hexdigest()
