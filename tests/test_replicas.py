"""Replica helpers on two CPU processes over gloo (the multi-GPU mode runs independent
reconstructions per rank; only timings and small results cross ranks)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import json
    import torch.distributed as dist
    from warp_psr_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        items = list(range(7))
        mine = replicas.shard(items)
        slowest = replicas.max_over_ranks(10.0 + rank)
        gathered = replicas.gather({"rank": rank, "items": mine})
        replicas.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"mine": mine, "max": slowest, "gathered": gathered}, f)
    finally:
        dist.destroy_process_group()


def test_shard_max_and_gather_over_two_gloo_ranks(tmp_path):
    import json
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    out = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert out[0]["mine"] == [0, 2, 4, 6] and out[1]["mine"] == [1, 3, 5]
    assert out[0]["max"] == out[1]["max"] == 11.0
    for o in out:
        assert [g["rank"] for g in o["gathered"]] == [0, 1]
        assert sorted(sum((g["items"] for g in o["gathered"]), [])) == list(range(7))


def test_single_process_is_identity():
    from warp_psr_b200 import replicas
    assert replicas.rank_and_size() == (0, 1)
    assert replicas.shard([1, 2, 3]) == [1, 2, 3]
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.gather("x") == ["x"]


def test_launch_runs_every_rank_and_prints_rank_zeros_line():
    """replicas.launch (what ``bench.py --gpus N`` uses when it is not started by torchrun)
    brings up N ranks; rank 0's line reports all of them and the maximum over ranks."""
    import json
    from pathlib import Path
    from warp_psr_b200 import replicas
    probe = Path(__file__).resolve().parent / "replica_probe.py"
    rc, out, err = replicas.launch(3, probe, timeout=240)
    assert rc == 0, err[-3000:]
    lines = [line for line in out.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["n_gpus"] == 3 and line["value"] == 3.0 and line["local_rank"] == 0
