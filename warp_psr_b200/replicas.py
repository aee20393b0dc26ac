"""Several GPUs: independent reconstructions, one process per GPU.

The ordered solve does not shard: every level is one wavefront over z, with a dependency
between neighbouring slices at every visit, and a level fits one B200.  Several GPUs
therefore run independent reconstructions (different clouds, or the perturbed inputs of a
finite-difference check), one per rank.  No collective is on the data path; ranks meet only
to agree on timings (the maximum over ranks) and to gather small per-reconstruction results.
Works with any torch.distributed backend (nccl on GPUs, gloo on CPUs).
"""
import os
import signal
import socket
import subprocess
import sys

import torch
import torch.distributed as dist


def rank_and_size():
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(items, rank=None, world_size=None):
    """This rank's share of independent work items (round-robin, stable order)."""
    r, w = rank_and_size()
    rank = r if rank is None else rank
    world_size = w if world_size is None else world_size
    return list(items)[rank::world_size]


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (every rank gets it); the identity on one process."""
    _, w = rank_and_size()
    if w == 1:
        return float(value)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    if rank_and_size()[1] > 1:
        dist.barrier()


def gather(obj):
    """Every rank's picklable obj, in rank order, on every rank."""
    _, w = rank_and_size()
    if w == 1:
        return [obj]
    out = [None] * w
    dist.all_gather_object(out, obj)
    return out


def reconstruct_many(clouds, **options):
    """Reconstruct (positions, normals) pairs spread over the ranks; returns, on every rank,
    [(index, iso_value, coefficient count)] for all clouds in input order."""
    from .reconstruction import reconstruct
    mine = shard(list(enumerate(clouds)))
    local = []
    for index, (positions, normals) in mine:
        result = reconstruct(positions, normals, **options)
        local.append((index, result.iso_value, int(result.field.keys.numel())))
    merged = [item for part in gather(local) for item in part]
    return sorted(merged)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch(nprocs, script, args=(), timeout=3600, env=None):
    """Runs ``script`` as ``nprocs`` ranks of one node (torch.distributed.run, rendezvous on
    127.0.0.1; RANK, LOCAL_RANK, WORLD_SIZE and MASTER_* set for each rank) and returns
    (exit code, stdout, stderr).  The launcher's whole process group is killed if it runs
    past ``timeout`` seconds."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={int(nprocs)}",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}", str(script), *map(str, args)]
    proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, start_new_session=True,
                            env=env)
    try:
        out, err = proc.communicate(timeout=timeout)
    except subprocess.TimeoutExpired:
        os.killpg(proc.pid, signal.SIGKILL)
        out, err = proc.communicate()
        return -signal.SIGKILL, out, err + f"\nreplicas.launch: killed after {timeout} s"
    return proc.returncode, out, err
