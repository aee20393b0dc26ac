"""Shared helpers for the known-answer fixtures (tests/golden/kats.json)."""
import hashlib
import json
from pathlib import Path

import numpy as np

from kat_inputs import fixture_input

KATS = json.loads((Path(__file__).resolve().parent / "golden" / "kats.json").read_text())
BY_NAME = {k["name"]: k for k in KATS}


def options(params):
    return dict(depth=params["depth"], full_depth=params["full_depth"], base_depth=params["base_depth"],
                solve_depth=params["solve_depth"], kernel_depth=params["kernel_depth"],
                samples_per_node=params["samples_per_node"], scale=params["scale"], point_weight=params["weight"],
                exact_interpolation=params["exact"], iters=params["iters"], base_v_cycles=params["base_v_cycles"],
                cg_accuracy=params["cg_accuracy"])


def sha(keys):
    return hashlib.sha256(np.asarray(keys).astype("<i8").tobytes()).hexdigest()


def iso_tolerance(precision):
    """Design-document budgets (warp-psr design doc :243-248)."""
    return (1e-8, 1e-6) if precision == "double" else (1e-5, 1e-4)


def inputs(kat):
    return fixture_input(kat["params"])
