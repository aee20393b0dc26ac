"""The benchmark's reference arm (the oracle on the host cores) prints one JSON line with every
key of the bench contract; checked on a small cloud so it runs in seconds on the CPU.  Ranks
other than 0 of a multi-process launch print nothing and exit 0."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"}


def run_bench(*args, env=None):
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, capture_output=True, text=True,
                          timeout=300, env=env)


def test_reference_arm_prints_the_contract_line():
    out = run_bench("--impl", "reference", "--steps", "1", "--warmup", "1", "--depth", "5", "--points", "20000")
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [line for line in out.stdout.splitlines() if line.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert KEYS <= set(line), KEYS - set(line)
    assert line["impl"] == "reference" and line["higher_is_better"] is False and line["unit"] == "ms"
    assert line["value"] > 0 and line["ms_per_step"] == line["value"] and line["steps"] == 1
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_stay_silent():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0", "--depth", "4", "--points", "5000",
                    env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
