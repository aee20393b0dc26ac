"""Random local operators for ordered-relaxation parity (warp-psr tests/test_relaxation.py:110-147)."""
import itertools

import numpy as np


def local_system(pattern, size=9, depth=3, dtype=np.float64, seed=None):
    xyz = list(itertools.product(range(size), repeat=3))
    if pattern == "sparse":
        xyz = [c for i, c in enumerate(xyz) if i % 3 != 0]
    elif pattern == "empty_slices":
        xyz = [c for c in xyz if c[2] not in (2, 5)]
    elif pattern == "random":
        rng = np.random.default_rng(seed)
        keep = rng.uniform(size=len(xyz)) < 0.6
        xyz = [c for c, k in zip(xyz, keep) if k]
    index = {c: i for i, c in enumerate(xyz)}
    rows = []
    for c, i in index.items():
        entries = []
        total = 2.0
        for delta in itertools.product((-1, 0, 1), repeat=3):
            j = index.get(tuple(a + b for a, b in zip(c, delta)))
            if j is None or j == i:
                continue
            value = np.cos(123 * i + 7 * j)
            entries.append((j, value))
            total += abs(value)
        entries.append((i, total))
        entries.sort()
        rows.append(entries)
    offsets = np.zeros(len(rows) + 1, np.int32)
    offsets[1:] = np.cumsum([len(r) for r in rows])
    columns = np.array([j for r in rows for j, _ in r], np.int32)
    values = np.array([v for r in rows for _, v in r], dtype)
    keys = np.array([(depth << 48) | (x << 32) | (y << 16) | z for x, y, z in xyz], np.int64)
    b = np.sin(np.arange(len(xyz))).astype(dtype)
    x = np.cos(np.arange(len(xyz))).astype(dtype)
    return keys, offsets, columns, values, b, x
