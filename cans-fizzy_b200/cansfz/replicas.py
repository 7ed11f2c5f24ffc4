"""Independent replicas over several GPUs (one process per GPU), the only
multi-GPU form of this library: a 1x1 pencil per GPU, no collective on the
data path.  What the ranks share is host-side bookkeeping: a barrier around
timed regions, the maximum of their device times and the sum of the work
they did, and, for an ensemble of independent cases, which rank runs which
case.  NCCL carries these few scalars between GPU ranks; gloo does on CPU
(tests).  Rendezvous uses the torchrun environment (RANK, WORLD_SIZE,
LOCAL_RANK, MASTER_ADDR/PORT).
"""
from __future__ import annotations

import datetime
import os


def setup(backend: str | None = None, timeout_s: float = 300.0):
    """Join the process group when WORLD_SIZE > 1; returns (rank, world, local)."""
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def _device():
    import torch
    import torch.distributed as dist

    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _reduce(x: float, world: int, op) -> float:
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float, world: int) -> float:
    import torch.distributed as dist

    return _reduce(x, world, dist.ReduceOp.MAX if world > 1 else None)


def sum_over_ranks(x: float, world: int) -> float:
    import torch.distributed as dist

    return _reduce(x, world, dist.ReduceOp.SUM if world > 1 else None)


def whole_job_rate(units_local: float, seconds_local: float, world: int) -> float:
    """Units done by all ranks divided by the slowest rank's time."""
    units = sum_over_ranks(units_local, world)
    secs = max_over_ranks(seconds_local, world)
    return units / secs


def assign_cases(costs, world: int):
    """Greedy longest-first assignment of independent cases (cost: cells x
    steps) to ranks; returns one list of case indices per rank (sorted)."""
    order = sorted(range(len(costs)), key=lambda q: (-costs[q], q))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for q in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(q)
        load[r] += costs[q]
    return [sorted(x) for x in out]


def teardown(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
