"""Multi-GPU plumbing of the solver: one process per GPU, torch.distributed for the
few host-side collectives.  The path has no data-path exchange: lattices (or batch
instances) are independent, so ranks only shard the work, synchronise around timed
regions and reduce scalars (the slowest rank's time, totals).

Launch: python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 ...
(RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from the environment).
"""
from __future__ import annotations

import datetime
import os


def env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment (1, 0, 0 alone)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 300) -> None:
    """Process group with a bounded timeout, so that ranks waiting on a missing peer end
    with an error instead of hanging."""
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def shard(items: list, rank: int, world: int) -> list:
    """Round-robin share of independent work items (lattices, batch instances)."""
    return list(items)[rank::world]


def _reduce(x: float, op: str, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, device=None) -> float:
    """The largest value over ranks (the time of the slowest rank)."""
    return _reduce(x, "max", device)


def sum_over_ranks(x: float, device=None) -> float:
    return _reduce(x, "sum", device)


def barrier(device=None) -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        if device is not None and str(device).startswith("cuda"):
            dist.barrier(device_ids=[int(str(device).split(":")[1])])
        else:
            dist.barrier()
