"""Extract known-answer records for the screened-Poisson path from the reference's
published result files (warp-psr ``docs/results/*.json``).

Each record keeps what pins the path without PoissonRecon or Warp being runnable:

* the fixture parameters (shape, count, seed, depths, weights, precision),
* the SHA-256 of the ``input.pts`` file the reference generated (``tools/make_fixture.py:86-110``),
* per-level counts and SHA-256 of the canonical active basis keys and non-ghost
  support keys (``tools/check_tree.py:6-22``),
* the Warp reconstruction's isovalue and the PoissonRecon 262b0f5 isovalue,
* the per-level basis counts.

Only fixtures whose inputs are regenerable from a seeded shape are kept
(``external`` inputs are dropped).  Usage::

    python tests/golden/make_kats.py <warp-psr checkout>/docs/results > tests/golden/kats.json
"""
import json
import sys
from pathlib import Path

SOURCES = ("validation.json", "profiles.json", "geometry-profiles.json",
           "solver-traces.json", "tree-metadata.json", "thresholds.json")
PARAMS = ("shape", "count", "seed", "input_scale", "translation", "variant", "depth",
          "full_depth", "base_depth", "solve_depth", "kernel_depth", "scale",
          "samples_per_node", "cg_accuracy", "base_v_cycles", "weight", "exact", "iters",
          "precision")


def records(root):
    out = []
    for source in SOURCES:
        data = json.loads((root / source).read_text())
        items = data.get("fixtures") or data.get("profiles")
        for item in items:
            manifest = item["manifest"]
            params = manifest["parameters"]
            if params.get("shape") in (None, "external") or params.get("dataset"):
                continue
            rec = item["reconstruction"]
            out.append({
                "name": item["fixture"],
                "source": source,
                "params": {k: params.get(k) for k in PARAMS},
                "input_sha256": manifest["input_sha256"],
                "levels": rec["tree"]["levels"],
                "iso_value": rec["iso_value"],
                "reference_iso_value": rec["reference_iso_value"],
                "basis_counts": rec["metadata"]["basis_counts"],
            })
    return out


if __name__ == "__main__":
    root = Path(sys.argv[1])
    json.dump(records(root), sys.stdout, indent=1)
    sys.stdout.write("\n")
