"""Runs of one process per GPU.

Nothing in the hydrodynamic solve exchanges data between GPUs: each rank
holds a whole problem (its fibers, bodies and periphery) and solves it on its
own device.  A run over N ranks is therefore N independent replicas; the only
cross-rank steps are a barrier around the timed region and the reduction of
the timing to the slowest rank, which sets the time of the whole job.

The helpers take the process group of ``torch.distributed`` when one is
initialised (NCCL on GPUs, gloo on CPU) and are identities otherwise.
"""
from __future__ import annotations

import os


def rank_info() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _group_ready() -> bool:
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier() -> None:
    """Barrier over the ranks of the run (none for a single process)."""
    if _group_ready():
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(values, device=None) -> list[float]:
    """Element-wise maximum over the ranks of a few timings (milliseconds).

    Every rank must call it with the same number of values, in the same
    order relative to its other collectives."""
    vals = [float(v) for v in values]
    if not _group_ready():
        return vals
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu().tolist()]


def aggregate_rate(units_per_rank: float, steps: int, world: int, max_total_ms: float) -> float:
    """Whole-job throughput: the units every replica processed over the
    slowest replica's time for the timed steps."""
    if max_total_ms <= 0.0:
        raise ValueError("the timed region must have a positive duration")
    return units_per_rank * steps * world / (max_total_ms * 1e-3)
