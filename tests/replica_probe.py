"""A rank of tests/test_replicas.py's launch check: joins the gloo group that
torch.distributed.run set up, takes the maximum over ranks and prints one JSON line on
rank 0 (the shape of the benchmark's line)."""
import json
import os
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import torch.distributed as dist  # noqa: E402

from warp_psr_b200 import replicas  # noqa: E402

dist.init_process_group("gloo")
try:
    rank, world = replicas.rank_and_size()
    slowest = replicas.max_over_ranks(1.0 + rank)
    replicas.barrier()
    if rank == 0:
        print(json.dumps({"n_gpus": world, "value": slowest, "local_rank": int(os.environ["LOCAL_RANK"])}))
finally:
    dist.destroy_process_group()
