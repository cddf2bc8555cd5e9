"""Multi-GPU by replicas: one process per GPU, each processing its own share of the image
pairs.  Pairs are independent and the path has no exchange step, so there is no data
collective: torch.distributed carries only the start barrier and the max-over-ranks
time (NCCL on GPUs; gloo works the same for host-side use and the CPU tests).
Launch with torchrun (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_ADDR/PORT in the environment).
"""
from __future__ import annotations

import datetime
import os


def env_rank():
    """(rank, world_size, local_rank) from the torchrun environment (defaults 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items, rank: int, world: int):
    """Round-robin share of `items` for `rank` (the CLI's --shard r/W uses the same rule)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return list(items)[rank::world]


def init(backend: str = "nccl", timeout_s: float = 600.0):
    """Joins the process group when WORLD_SIZE > 1; returns (rank, world, local_rank)."""
    rank, world, local = env_rank()
    if world > 1:
        import torch
        import torch.distributed as dist

        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return rank, world, local


def _tensor(x, world):
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    return torch.tensor([float(x)], dtype=torch.float64, device=dev)


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return float(x)
    import torch.distributed as dist

    t = _tensor(x, world)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return float(x)
    import torch.distributed as dist

    t = _tensor(x, world)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def finish(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def throughput(units_local: int, seconds_local: float, world: int):
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return sum_over_ranks(units_local, world) / max_over_ranks(seconds_local, world)
