"""Multi-GPU use: one process per GPU, each solving its own slice of a batch.

QP instances are independent, so a batch splits over ranks with no
collective on the data path (qpax's vmap axis becomes the rank axis, then
the instance axis inside each rank).  The only collectives are for timing:
a barrier and the maximum of per-rank times.

    lo, hi = shard_bounds(B, rank, world)     # this rank's instances [lo, hi)
    ...solve Q[lo:hi], ... on this rank's GPU...
    t = max_over_ranks(local_ms)              # whole-job time

Works with the NCCL backend (tensors on this rank's GPU) and with gloo
(tensors on the host), so the host logic is testable without GPUs.
"""

from __future__ import annotations

import torch


def shard_bounds(batch: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous, balanced slice [lo, hi) of `batch` instances for `rank` of `world`
    (sizes differ by at most one; every instance belongs to exactly one rank)."""
    if world < 1 or not 0 <= rank < world or batch < 0:
        raise ValueError(f"bad shard request: batch={batch} rank={rank} world={world}")
    return batch * rank // world, batch * (rank + 1) // world


def _device():
    import torch.distributed as dist

    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float) -> float:
    """Maximum of a per-rank scalar over the default process group (the value
    itself without one)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    """Barrier over the default process group (no-op without one)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
