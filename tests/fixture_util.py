"""Fixture directories in the reference's offline-oracle format written from the CPU oracle
(test infrastructure): what a PoissonRecon run would leave, with this repository's own
restatement standing in for PoissonRecon."""
import json

import numpy as np

import oracle
from warp_psr_b200 import fixtures

PARAMS = {"depth": 5, "full_depth": 2, "base_depth": None, "solve_depth": None, "kernel_depth": None, "scale": 1.1,
          "samples_per_node": 1.5, "weight": 2.0, "exact": False, "iters": 8, "base_v_cycles": 1,
          "cg_accuracy": 1e-3}


def cloud(count=3000, seed=2026):
    rng = np.random.default_rng(seed)
    n = rng.normal(size=(count, 3))
    n /= np.linalg.norm(n, axis=1)[:, None]
    return n * (1 + 0.1 * n[:, :1]), n


def write_oracle_fixture(directory, precision="double", params=PARAMS, count=3000, queries=400, seed=2026):
    """input.pts, queries.txt, oracle.txt (iso, transform, q and node rows), stages.txt
    (effective, samples, normals, loads) and manifest.json of the oracle's reconstruction."""
    dtype = np.float64 if precision == "double" else np.float32
    p, n = cloud(count, seed)
    fixtures.write_input_pts(directory / "input.pts", p, n)
    p, n = fixtures.read_input_pts(directory / "input.pts", dtype)
    rng = np.random.default_rng(seed + 1)
    q = p[rng.choice(len(p), queries // 2, replace=False)]
    lo, hi = p.min(0), p.max(0)
    q = np.concatenate([q, lo + (hi - lo) * rng.uniform(size=(queries - len(q), 3))])
    fixtures.write_queries(directory / "queries.txt", q)
    q = fixtures.read_queries(directory / "queries.txt", dtype)
    opts = fixtures.reconstruct_options(params)
    ref = oracle.OracleResult(p, n, **opts)
    v, g, ok = ref.evaluate(q)
    assert ok.all()
    depth = opts["depth"]
    nodes = fixtures.node_rows(ref.keys, ref.coefficients, [ref.support(d) for d in range(depth + 1)])
    fixtures.write_oracle(directory / "oracle.txt", iso=ref.iso_value, cube_to_model=ref.transforms[0], values=v,
                          gradients=g, nodes=nodes)
    prm = ref.options
    effective = [prm["depth"], prm["full_depth"], prm["base_depth"], prm["solve_depth"], prm["kernel_depth"],
                 prm["scale"], prm["samples_per_node"], prm["point_weight"], int(prm["exact"]),
                 prm["iters"], prm["cg_accuracy"]]
    normals = ref.stage("normal_values", dtype).reshape(-1, 4)[:, :3]
    load_keys, load_values = [], []
    keys = ref.keys
    kd = keys >> 48
    for d in range(prm["base_depth"], prm["solve_depth"] + 1):
        try:
            values = ref.stage(f"normal_load_{d}", np.float64)
        except KeyError:
            continue
        load_keys.append(keys[kd == d])
        load_values.append(values)
    fixtures.write_stages(
        directory / "stages.txt", effective=effective,
        samples=(ref.stage("group_keys", np.int64), ref.stage("group_sums", dtype), ref.stage("group_weights", dtype)),
        normals=(ref.stage("normal_keys", np.int64), normals),
        loads=(np.concatenate(load_keys), np.concatenate(load_values)) if load_keys else None)
    (directory / "manifest.json").write_text(json.dumps({"name": f"oracle-{precision}", "precision": precision,
                                                         "parameters": params}))
    return ref, q
