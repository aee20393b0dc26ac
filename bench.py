#!/usr/bin/env python
"""Depth-9 screened-Poisson benchmark (synthetic stand-in for the eagle scan, 800k points).

One step = one solve+adjoint: a differentiable reconstruction (sample grouping, density and
normal splats, tree, operator assembly, cascadic ordered Gauss-Seidel solve, field and
isovalue) of an 800k-point bumpy sphere at depth 9, full depth 4, point weight 2, a loss on
32 isovalue-centred field values, and the reverse pass onto positions and normals; in the
mixed precision the metric names (float64 solve, float32 relaxation operators).  Multi-GPU runs are independent replicas
(weak scaling): the ordered solve does not shard.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  ``--impl reference`` times the CPU restatement of the
reference algorithm (the oracle) on the host cores instead.
"""
import argparse
import ctypes
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "depth-9 SPSR solve+adjoint ms, FP32/FP64-refined vs FP64, at ≤1e-6 field error"
CONFIG = dict(depth=9, full_depth=4, point_weight=2.0, samples_per_node=1.5, scale=1.1, iters=8)
POINTS = 800_000
WORKLOAD = "bumpy sphere {points} points (SH l<=8, 10x density variation)"
# --config 5: the scale workload (three tori, 3.5M points with 1% outliers and 2% flipped
# normals, depth 10, full depth 5, point weight 4), forward plus adjoint in the mixed precision.
SCALE = dict(metric="depth-10 three-tori SPSR solve+adjoint ms (scale configuration), mixed precision vs FP64",
             config=dict(depth=10, full_depth=5, point_weight=4.0, samples_per_node=1.5, scale=1.1, iters=8),
             points=3_500_000, workload="three tori {points} points (1% outliers, 2% flipped normals)")


def peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cloud():
    from warp_psr_b200 import clouds
    p, n = clouds.three_tori(POINTS) if WORKLOAD.startswith("three tori") else clouds.bumpy_sphere(POINTS)
    return p.astype(np.float32), n.astype(np.float32)


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.first = 0  # samples before this index precede the timed region

    def start_timing(self):
        self.first = len(self.lines)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines[self.first:]:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, flag in zip(names, parts[3:7]):
                if flag.lower() in ("active", "1", "yes"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


class Pool:
    """The device's default stream-ordered memory pool, from which the library takes every
    buffer (cudaMallocAsync): bytes in use now and the high-water mark since a reset."""

    USED_CURRENT, USED_HIGH = 7, 8  # cudaMemPoolAttrUsedMemCurrent / UsedMemHigh

    def __init__(self, device_index):
        from warp_psr_b200 import _lib
        _lib.load()  # brings in the CUDA runtime the library links against
        self.rt = ctypes.CDLL("libcudart.so.12")
        self.pool = ctypes.c_void_p()
        assert self.rt.cudaDeviceGetDefaultMemPool(ctypes.byref(self.pool), device_index) == 0

    def _get(self, attr):
        v = ctypes.c_uint64()
        assert self.rt.cudaMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) == 0
        return int(v.value)

    def used(self):
        return self._get(self.USED_CURRENT)

    def high(self):
        return self._get(self.USED_HIGH)

    def reset_high(self):
        zero = ctypes.c_uint64(0)
        assert self.rt.cudaMemPoolSetAttribute(self.pool, self.USED_HIGH, ctypes.byref(zero)) == 0


def field_error(result, reference, queries):
    """Max |f - f64| at the queries, raw and normalised by max |f64| (both evaluated in float64)."""
    import torch
    q = torch.from_numpy(queries.astype(np.float64)).cuda()
    ref_v, _, ok = reference.evaluate(q)
    if result.field.coefficients.dtype == torch.float64:
        v, _, _ = result.evaluate(q)
    else:
        v, _, _ = result.evaluate(q.float())
        v = v.double()
    m = ok.bool()
    err = (v[m] - ref_v[m]).abs().max().item()
    scale = ref_v[m].abs().max().item()
    iso_err = abs(result.iso_value - reference.iso_value)
    return {"max_abs": err, "normalised": err / scale, "iso_abs": iso_err}


def run_ours(args, rank, world):
    import torch
    from warp_psr_b200 import reconstruct, reconstruct_differentiable, _lib, replicas

    device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(device)
    p_host, n_host = cloud()
    p_pin = torch.from_numpy(p_host).pin_memory()
    n_pin = torch.from_numpy(n_host).pin_memory()
    p_dev = p_pin.to(device)
    n_dev = n_pin.to(device)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)  # > 126 MB L2
    stream = torch.cuda.current_stream(device)

    finest = []  # (seconds, row visits) of the finest level's relaxation launch, per timed step
    split = []   # (forward ms, backward ms) per timed step
    bw_stages = []  # device ms per reverse-pass stage, per timed step
    # The loss of the adjoint: sum of seeded, isovalue-centred field values at 32 queries.
    rng = np.random.default_rng(2027)
    lo, hi = p_host.min(0), p_host.max(0)
    q_host = lo + (hi - lo) * rng.uniform(size=(32, 3))
    seed_host = rng.normal(size=32)

    def step(p_in=None, n_in=None, precision=None):
        """One solve+adjoint: differentiable reconstruction, loss, reverse pass onto the inputs."""
        P = (p_dev if p_in is None else p_in).detach().requires_grad_(True)
        N = (n_dev if n_in is None else n_in).detach().requires_grad_(True)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        res = reconstruct_differentiable(P, N, precision=precision or args.precision, **CONFIG)
        dtype = res.result.field.coefficients.dtype
        q = torch.as_tensor(q_host, dtype=dtype, device=device)
        seed = torch.as_tensor(seed_host, dtype=dtype, device=device)
        v, _, _ = res.evaluate(q, centered=True)
        loss = (torch.nan_to_num(v) * seed).sum()
        e[1].record(stream)
        loss.backward()
        e[2].record(stream)
        e[2].synchronize()
        split.append((e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])))
        bw_stages.append(res.backward_stats.get("backward_ms", {}))
        r = res.result
        finest.append((r.diagnostics["relax_finest_seconds"], r.diagnostics["relax_finest_row_visits"]))
        # Keep only a summary: the tape (several GB at depth 9) is released with the result
        # before the next step, as a training loop would.
        summary = {"dtype": dtype, "coefficients": int(r.field.keys.numel()),
                   "basis_counts": r.metadata["basis_counts"], "timings": r.metadata["timings_seconds"],
                   "relax_seconds": r.diagnostics["relax_seconds"], "relax_launches": r.diagnostics["relax_launches"],
                   "relax_row_visits": r.diagnostics["relax_row_visits"]}
        return summary, P.grad, N.grad

    def timed(fn, k):
        # Python's cyclic garbage collector is run before and paused during the timed steps,
        # as timeit does: its pauses are the interpreter's, not the step's work.
        total = 0.0
        last = None
        gc.collect()
        gc.disable()
        try:
            for _ in range(k):
                last = None  # the previous step's outputs are released before the next step
                flush.fill_(1)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                last = fn()
                b.record(stream)
                b.synchronize()
                total += a.elapsed_time(b)
        finally:
            gc.enable()
        return total / k, last

    # The clock sampler (an nvidia-smi process) starts before the warm-up, so that its start
    # does not fall into a timed step; only the samples taken while timing are summarised.
    clocks = Clocks(device.index).__enter__()
    try:
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        replicas.barrier()
        torch.cuda.synchronize()
        launches0 = _lib.kernel_launches()
        finest.clear()
        split.clear()
        bw_stages.clear()
        clocks.start_timing()
        ms, (result, _, _) = timed(step, args.steps)
    finally:
        clocks.__exit__(None, None, None)
    launches = _lib.kernel_launches() - launches0
    bw_stage_ms = {k: round(statistics.mean(b[k] for b in bw_stages), 3) for k in bw_stages[0]} if bw_stages else {}
    bw_stage_sums = [round(sum(b.values()), 2) for b in bw_stages]  # per timed step: host pauses show as gaps
    fwd_ms = statistics.mean(x[0] for x in split)
    bwd_ms = statistics.mean(x[1] for x in split)
    split_steps = list(split)  # (forward, backward) ms of each timed step
    # the finest level's relaxation launch over the timed steps (the roofline's kernel)
    finest_s = statistics.mean(f[0] for f in finest)
    visits = finest[-1][1]
    torch.cuda.synchronize()
    ms = replicas.max_over_ranks(ms, device)
    replicas.barrier()

    # End to end through the public API with host buffers: pinned H2D copy of the cloud, the
    # solve+adjoint step, and the device-to-host read of the position and normal gradients.
    g_host = [torch.empty(p_pin.shape, dtype=p_pin.dtype).pin_memory() for _ in range(2)]

    def e2e_step():
        p = p_pin.to(device, non_blocking=True)
        n = n_pin.to(device, non_blocking=True)
        r, gp, gn = step(p, n)
        g_host[0].copy_(gp, non_blocking=True)
        g_host[1].copy_(gn, non_blocking=True)
        return None

    e2e_ms, _ = timed(e2e_step, args.steps)
    e2e_ms = replicas.max_over_ranks(e2e_ms, device)
    # the forward alone, not differentiable (what reconstruct() costs)
    plain_ms, plain = timed(lambda: reconstruct(p_dev, n_dev, precision=args.precision, **CONFIG),
                            max(1, args.steps // 2))
    plain_relax = {"finest_ms": round(plain.diagnostics["relax_finest_seconds"] * 1e3, 3),
                   "all_levels_ms": round(plain.diagnostics["relax_seconds"] * 1e3, 3)}
    del plain

    # The float64 path's solve+adjoint step on the same workload (the metric's comparison).
    p64, n64 = p_dev.double(), n_dev.double()
    step(p64, n64, precision="input")  # warm-up: first launches of the float64 kernels, pool growth
    torch.cuda.synchronize()
    split.clear()
    finest.clear()
    ms64_step, (res64, _, _) = timed(lambda: step(p64, n64, precision="input"), max(2, args.steps // 4))
    fp64_step = {"ms": round(ms64_step, 3), "forward_differentiable": round(statistics.mean(x[0] for x in split), 3),
                 "backward": round(statistics.mean(x[1] for x in split), 3),
                 "relax_finest_ms": round(statistics.mean(f[0] for f in finest) * 1e3, 3),
                 "precision": "float64 inputs, input precision (the reference's float64 path)"}
    del p64, n64, res64

    # Memory of the step: the pool's high-water mark over one solve+adjoint step, and the
    # reverse-pass tape = pool bytes held by a differentiable forward's result minus those
    # held by a plain forward's result (same inputs).
    pool = Pool(device.index)
    gc.collect()
    torch.cuda.synchronize()
    pool.reset_high()
    base_used = pool.used()
    torch.cuda.reset_peak_memory_stats(device)
    step()
    torch.cuda.synchronize()
    memory = {"pool_peak_bytes": pool.high() - base_used,
              "torch_peak_bytes": int(torch.cuda.max_memory_allocated(device))}
    gc.collect()
    held = {}
    for name, differentiable in (("plain", False), ("differentiable", True)):
        before = pool.used()
        r = reconstruct(p_dev, n_dev, precision=args.precision, _differentiable=differentiable, **CONFIG)
        torch.cuda.synchronize()
        held[name] = pool.used() - before
        del r
        gc.collect()
        torch.cuda.synchronize()
    memory["result_bytes"] = held["plain"]
    memory["tape_bytes"] = held["differentiable"] - held["plain"]

    # Per-kernel roofline: one more solve+adjoint step (after the timed ones) with the
    # library's kernel clocks on -- CUDA events around each launch of its main kernels, each
    # with the launch's algorithmic bytes (what it must read and write once).
    os.environ["PSR_KERNEL_CLOCKS"] = "1"
    try:
        _lib.kernel_clocks()  # clears earlier totals
        step()
        torch.cuda.synchronize()
        kernel_clocks = _lib.kernel_clocks()
    finally:
        os.environ.pop("PSR_KERNEL_CLOCKS", None)

    out_dtype = "f64" if result["dtype"] == torch.float64 else "f32"
    info = result
    peak_k, _ = peaks()
    kernel_rows = [{"kernel": c["kernel"], "launches": c["launches"], "ms": round(c["ms"], 3),
                    "algorithmic_bytes": int(c["bytes"]), "units": int(c["units"]), "unit": c["unit"],
                    "bytes_per_unit": round(c["bytes"] / c["units"], 1) if c["units"] else None,
                    "achieved": round(c["bytes"] / (c["ms"] * 1e-3) / 1e9, 1) if c["ms"] > 0 else None,
                    "frac": round(c["bytes"] / (c["ms"] * 1e-3) / 1e9 / peak_k, 4) if c["ms"] > 0 else None}
                   for c in sorted(kernel_clocks, key=lambda c: -c["ms"])]
    # Roofline of the dominant kernel: the finest level's ordered-relaxation launch
    # (strip_gs_kernel).  Algorithmic bytes per row visit: 27 operator entries (float32 in the
    # mixed path, else the input precision), b read, x read, x write in the vector precision,
    # and a 4-byte row id.  Its duration is the library's CUDA-event time of that launch,
    # averaged over the timed steps.
    vec = 8 if out_dtype == "f64" else 4
    op = 4 if args.precision == "mixed" else vec
    per_visit = 27 * op + 3 * vec + 4
    algorithmic = visits * per_visit
    achieved = algorithmic / finest_s / 1e9 if finest_s > 0 else None
    peak, peak_kind = peaks()
    traffic_file = ROOT / "profiles" / "strip_gs_depth9_traffic.json"
    traffic = None
    if traffic_file.exists():
        rec = json.loads(traffic_file.read_text())
        if rec.get("precision") == args.precision:
            traffic = rec.get("dram_bytes_per_launch")
    all_s = info["relax_seconds"]
    all_visits = info["relax_row_visits"]

    line = {
        "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": out_dtype, "data": "synthetic",
        "config": {"workload": WORKLOAD.format(points=POINTS) + f", depth {CONFIG['depth']}, full depth "
                               f"{CONFIG['full_depth']}, SPSR point weight {CONFIG['point_weight']:g}, 8 GS iterations; "
                               "step = differentiable reconstruction + 32-query centred-value loss + reverse pass onto "
                               "positions and normals",
                   "points": POINTS, "coefficients": result["coefficients"],
                   "basis_counts": result["basis_counts"], "precision": args.precision,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
                   "python_gc": "collected before and paused during the timed steps, as timeit does"},
        "roofline": {"bound": "hbm", "kernel": f"strip_gs_kernel, finest level (ordered relaxation, depth {CONFIG['depth']})",
                     "achieved": round(achieved, 1) if achieved else None, "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4) if achieved else None, "peak_kind": peak_kind,
                     "algorithmic_bytes": int(algorithmic), "bytes_per_row_visit": per_visit, "row_visits": visits,
                     "launch_ms": round(finest_s * 1e3, 3), "traffic": traffic,
                     "note": "latency-bound: each of the 2^d + 2(iters-1) + 1 waves depends on the previous one",
                     "all_levels": {"launches": info["relax_launches"], "row_visits": all_visits,
                                    "ms": round(all_s * 1e3, 3),
                                    "achieved": round(all_visits * per_visit / all_s / 1e9, 1) if all_s > 0 else None},
                     "kernels": kernel_rows,
                     "kernels_note": "one extra solve+adjoint step with CUDA events around each launch of the library's "
                                     "main kernels; algorithmic bytes = what a launch must read and write once "
                                     "(index structures excluded); frac of the measured HBM copy peak"},
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": int(p_pin.numel() * 4 * 2),
                "d2h_bytes_per_step": int(p_pin.numel() * 4 * 2)},
        "split_ms": {"forward_differentiable": round(fwd_ms, 3), "backward": round(bwd_ms, 3),
                     "adjoint_over_forward": round(bwd_ms / fwd_ms, 3), "forward_plain": round(plain_ms, 3),
                     "backward_stages": bw_stage_ms, "backward_stage_sum_per_step": bw_stage_sums,
                     "per_step": [[round(a, 2), round(b, 2)] for a, b in split_steps]},
        "fp64_step": fp64_step,
        "coefficient_sweeps_per_s": {"step": round(all_visits / (ms / 1e3), 1),
                                     "relaxation_kernels": round(all_visits / all_s, 1) if all_s > 0 else None,
                                     "row_visits_per_step": int(all_visits)},
        "memory": memory,
        "gpu_launches": int(launches),
        "stage_ms": {k: round(v * 1e3, 3) for k, v in result["timings"].items()},
        "clocks": clocks.summary(),
    }
    if rank == 0 and not args.no_accuracy:
        fp64 = reconstruct(p_dev.double(), n_dev.double(), **CONFIG)
        rng = np.random.default_rng(2027)
        lo, hi = p_host.min(0), p_host.max(0)
        q = np.concatenate([p_host[rng.choice(len(p_host), 20000, replace=False)],
                            lo + (hi - lo) * rng.uniform(size=(20000, 3))])
        mixed = reconstruct(p_dev, n_dev, precision=args.precision, **CONFIG)
        line["error_vs_fp64"] = field_error(mixed, fp64, q)
        if args.precision != "input":
            f32 = reconstruct(p_dev, n_dev, **CONFIG)
            line["fp32_error_vs_fp64"] = field_error(f32, fp64, q)
            ms32, r32 = timed(lambda: reconstruct(p_dev, n_dev, **CONFIG), max(1, args.steps // 2))
            ms64, r64 = timed(lambda: reconstruct(p_dev.double(), n_dev.double(), **CONFIG), max(1, args.steps // 2))
            line["variants_ms"] = {"fp32": round(ms32, 3), "fp64": round(ms64, 3), args.precision: round(plain_ms, 3),
                                   "scope": "plain forward reconstruction"}
            line["variants_relax_ms"] = {
                "fp32": {"finest_ms": round(r32.diagnostics["relax_finest_seconds"] * 1e3, 3),
                         "all_levels_ms": round(r32.diagnostics["relax_seconds"] * 1e3, 3)},
                "fp64": {"finest_ms": round(r64.diagnostics["relax_finest_seconds"] * 1e3, 3),
                         "all_levels_ms": round(r64.diagnostics["relax_seconds"] * 1e3, 3)},
                args.precision: plain_relax}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p_host, n_host, steps=1)
        # same work on both sides: the CPU restatement has no reverse pass, so set its forward
        # against the GPU's plain forward
        line["cpu_baseline"]["over_gpu_forward_plain"] = round(line["cpu_baseline"]["value"] / plain_ms, 1)
    return line


def cpu_baseline(p, n, steps):
    import oracle
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        oracle.OracleResult(p, n, **CONFIG)
        times.append((time.perf_counter() - t) * 1e3)
    return {"value": round(statistics.mean(times), 1), "unit": "ms", "cores": oracle.threads(), "kind": "port",
            "sample": f"{len(times)} full forward reconstruction(s) of the benchmark workload by the C++ oracle "
                      f"(OpenMP, {oracle.threads()} threads); the CPU restatement has no reverse pass, so this "
                      f"times the forward part of the step only"}


def run_reference(args):
    """The reference's algorithm on the host cores: the oracle (PoissonRecon and Warp are not available)."""
    import oracle
    p, n = cloud()
    # Warm-up steps run a small sample of the workload (thread pool, page cache).
    small = 50_000
    for _ in range(args.warmup):
        oracle.OracleResult(p[:small], n[:small], **CONFIG)
    budget_s = 240.0
    times = []
    start = time.perf_counter()
    for _ in range(args.steps):
        t = time.perf_counter()
        oracle.OracleResult(p, n, **CONFIG)
        times.append((time.perf_counter() - t) * 1e3)
        if time.perf_counter() - start + times[-1] / 1e3 > budget_s:
            break
    ms = statistics.mean(times)
    return {"metric": METRIC, "value": round(ms, 1), "unit": "ms", "n_gpus": 1, "steps": len(times),
            "warmup": args.warmup, "ms_per_step": round(ms, 1), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": "bumpy sphere 800k points, depth 9, full depth 4, SPSR point weight 2; forward "
                                   "reconstruction by the C++ CPU restatement of warp-psr (PoissonRecon 262b0f5 "
                                   "and Warp are not installable offline; the restatement has no reverse pass)",
                       "points": POINTS},
            "cpu_baseline": {"value": round(ms, 1), "unit": "ms", "cores": oracle.threads(), "kind": "port",
                             "sample": f"{len(times)} full reconstruction(s), warm-up on {small}-point prefixes"},
            "e2e": {"value": round(ms, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--precision", choices=("mixed", "input"), default="mixed")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--depth", type=int, default=None,
                    help="smaller cases for profiling only; the metric is quoted at depth 9")
    ap.add_argument("--points", type=int, default=None, help="points of the cloud (profiling cases)")
    ap.add_argument("--config", type=int, choices=(3, 5), default=3,
                    help="3: the metric's workload (default); 5: the scale workload (no CPU baseline: the CPU "
                         "restatement takes minutes per forward at this size)")
    args = ap.parse_args()
    if args.config == 5:
        globals().update(METRIC=SCALE["metric"], POINTS=SCALE["points"], WORKLOAD=SCALE["workload"])
        CONFIG.update(SCALE["config"])
        args.no_cpu_baseline = True
    if args.depth is not None:
        CONFIG["depth"] = args.depth
    if args.points is not None:
        globals()["POINTS"] = args.points
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "ours" and args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # N independent replicas, one process per GPU, started here when no launcher did
        from warp_psr_b200 import replicas
        rc, out, err = replicas.launch(args.gpus, Path(__file__).resolve(), sys.argv[1:])
        sys.stdout.write(out)
        sys.stderr.write(err)
        sys.exit(rc)
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        line = run_ours(args, rank, world)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
