"""check_fixture (the counterpart of the reference's tools/check_reconstruction.py) on
fixture directories written from the CPU oracle: a GPU reconstruction of the fixture's
input.pts meets the design budgets against its oracle.txt, and a planted mistake in the
oracle's files is caught."""
import numpy as np
import pytest

from warp_psr_b200 import fixtures
from fixture_util import write_oracle_fixture

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["double", "float"])
def test_gpu_reconstruction_passes_oracle_fixture(tmp_path, precision):
    write_oracle_fixture(tmp_path, precision)
    report = fixtures.check_fixture(tmp_path)
    atol, rtol = fixtures.FIELD_TOLERANCE[precision]
    assert report["max_abs_value_error"] <= atol + rtol * 2.0
    assert report["tree"] and all(level["active_count"] > 0 for level in report["tree"][2:])


def test_planted_mistake_in_the_oracle_file_is_caught(tmp_path):
    write_oracle_fixture(tmp_path, "double")
    rows = fixtures.read_tagged(tmp_path / "oracle.txt")
    rows["iso"][0, 0] += 1e-4  # the oracle's isovalue, off by far more than the budget
    order = ["parallel_async", "threads", "schedule", "chunk_size", "openmp_effective_threads", "iso", "transform",
             "q", "node"]
    fixtures.write_tagged(tmp_path / "oracle.txt",
                          [(tag, [int(v) if tag == "node" and i < 7 else float(v) for i, v in enumerate(row)])
                           for tag in order for row in rows[tag]])
    with pytest.raises(AssertionError):
        fixtures.check_fixture(tmp_path)
    # a node missing from the tree export
    write_oracle_fixture(tmp_path, "double")
    lines = (tmp_path / "oracle.txt").read_text().splitlines()
    node_lines = [i for i, line in enumerate(lines) if line.startswith("node 3 ")]
    del lines[node_lines[len(node_lines) // 2]]
    (tmp_path / "oracle.txt").write_text("\n".join(lines) + "\n")
    with pytest.raises(AssertionError):
        fixtures.check_fixture(tmp_path)
