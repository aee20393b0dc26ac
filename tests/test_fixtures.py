"""Reference fixture formats (reference/README.md:27-64): readers and writers round trip,
and a fixture written from the CPU oracle reads back to the oracle's own arrays."""
import json

import numpy as np
import pytest

from warp_psr_b200 import fixtures
from fixture_util import write_oracle_fixture


def test_tagged_rows_round_trip_exactly(tmp_path):
    rng = np.random.default_rng(1)
    vals = rng.normal(size=(5, 4)) * 10.0 ** rng.integers(-30, 30, size=(5, 1))
    fixtures.write_tagged(tmp_path / "t.txt", [("q", list(v)) for v in vals] + [("iso", [0.1 + 0.2])])
    back = fixtures.read_tagged(tmp_path / "t.txt")
    assert np.array_equal(back["q"], vals)
    assert back["iso"][0, 0] == 0.1 + 0.2


def test_input_and_queries_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    p, n = rng.normal(size=(50, 3)), rng.normal(size=(50, 3))
    fixtures.write_input_pts(tmp_path / "input.pts", p, n)
    p2, n2 = fixtures.read_input_pts(tmp_path / "input.pts")
    assert np.array_equal(p, p2) and np.array_equal(n, n2)
    p32, _ = fixtures.read_input_pts(tmp_path / "input.pts", np.float32)
    assert p32.dtype == np.float32 and np.array_equal(p32, p.astype(np.float32))
    fixtures.write_queries(tmp_path / "queries.txt", p)
    assert np.array_equal(fixtures.read_queries(tmp_path / "queries.txt"), p)
    (tmp_path / "bad.pts").write_text("1 2 3\n")
    with pytest.raises(ValueError):
        fixtures.read_input_pts(tmp_path / "bad.pts")


def test_node_rows_round_trip_to_tree_keys():
    d = 2
    basis = np.array(sorted((d << 48) | (x << 32) | (y << 16) | z for x, y, z in [(0, 0, 0), (1, 2, 3), (4, 4, 4)]),
                     np.int64)
    coeff = np.array([0.5, -1.0, 2.0])
    bias = 524288
    sup = np.array(sorted(((x + bias) << 40) | ((y + bias) << 20) | (z + bias)
                          for x, y, z in [(-1, 0, 0), (0, 0, 0), (1, 2, 3)]), np.int64)
    rows = fixtures.node_rows(basis, coeff, [np.zeros(0, np.int64), np.zeros(0, np.int64), sup])
    nodes = np.array(rows, dtype=np.float64)
    assert len(nodes) == 4  # (4, 4, 4) is active but outside the non-ghost support
    tree = fixtures.tree_from_nodes(nodes, d)
    assert np.array_equal(tree[d][0], sup) and np.array_equal(tree[d][1], basis)
    ghost = nodes[(nodes[:, 1] == 4)]
    assert ghost[0, 4] == 2 and ghost[0, 5] == 1 and ghost[0, 7] == 2.0


@pytest.mark.parametrize("precision", ["double", "float"])
def test_oracle_fixture_reads_back(tmp_path, precision):
    ref, q = write_oracle_fixture(tmp_path, precision)
    out = fixtures.read_tagged(tmp_path / "oracle.txt")
    assert out["iso"][0, 0] == ref.iso_value
    assert np.array_equal(out["transform"].reshape(4, 4).T, ref.transforms[0])
    v, g, _ = ref.evaluate(q)
    assert np.array_equal(out["q"][:, 0], v.astype(np.float64))
    assert np.array_equal(out["q"][:, 1:], g.astype(np.float64))
    depth = json.loads((tmp_path / "manifest.json").read_text())["parameters"]["depth"]
    for d, (support, active) in enumerate(fixtures.tree_from_nodes(out["node"], depth)):
        assert np.array_equal(support, ref.support(d))
        assert np.array_equal(active, ref.basis(d))
    stages = fixtures.read_tagged(tmp_path / "stages.txt")
    assert stages["effective"].shape == (1, 11)
    assert len(stages["sample"]) == len(ref.stage("group_keys", np.int64))
    assert len(stages["normal"]) == len(ref.stage("normal_keys", np.int64))
    widths = fixtures.query_cell_widths(out["node"], stages["normal"], np.full((1, 3), 0.5), depth)
    assert widths.shape == (1,) and 0 < widths[0] <= 1
